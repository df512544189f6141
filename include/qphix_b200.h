/*
 * qphix_b200.h -- C-ABI of the B200 (sm_100a) dslash library.
 *
 * The library computes the operator family that qphix-codegen emits for CPU
 * ISAs: the Wilson, clover, twisted-mass (TM) and twisted-mass-clover
 * hopping terms, in the plain "dslash" form and in the "achimbdpsi" form
 * (A.chi - b.D.psi), for isign = +1 ("plus") and -1 ("minus", the dagger),
 * with 18-real or 12-real (two stored rows) gauge links and twisted boundary
 * phases, plus the halo (face) pack and unpack kernels.
 *
 * Every field lives in device memory in the QPhiX tile layouts of
 * codegen/include/decl_common.h:9-62 (Types<FT,V,S,compress12>):
 *   spinor  FourSpinorBlock  FT[3 colour][4 spin][2 re/im][S]       per S x-sites
 *   gauge   SU3MatrixBlock   FT[8 dir][2|3 row][3][2][V]            per tile of V sites
 *   clover  CloverBlock      {diag1[6][V]; off_diag1[15][2][V];
 *                             diag2[6][V]; off_diag2[15][2][V]}       per tile
 *   tmclov  FullCloverBlock  {block1[6][6][2][V]; block2[6][6][2][V]} per tile
 * A tile covers V/S consecutive y rows of S x-sites each.  The reference
 * kernels work on one tile per call and leave the lattice loop, neighbour
 * offsets and per-tile boundary coefficients to the caller (QPhiX); here one
 * call covers a whole checkerboard of a (sub-)lattice described by
 * qb200_lattice, and the neighbour addressing is computed on the device.
 *
 * Conventions (all taken from the reference generator):
 *   - dir d = 2*mu + {0 back, 1 forw}, mu = x,y,z,t   (codegen/dslash.cc:232-233)
 *   - stored link matrix G = U^T: forward hop uses sum_k G[k][c] b[k], backward
 *     hop sum_k conj(G[c][k]) b[k]  (codegen/dslash_common.cc:1678-1727)
 *   - 12-real links rebuild G[2][c] = conj(G[0][c+1]G[1][c+2]-G[0][c+2]G[1][c+1])
 *     (codegen/dslash_common.cc:1657-1676)
 *   - "half" storage is IEEE binary16 bits with no scale (decl_common.h:7)
 *
 * Layout of one site (xcb, y, z, t) on checkerboard cb (x = 2*xcb + ((y+z+t+cb)&1)):
 *   nxh = nx/2, nvecs = nxh/S, ngy = V/S
 *   Pxy  = ny*nvecs + pad_xy,  Pxyz = nz*Pxy + pad_xyz
 *   spinor block  = t*Pxyz + z*Pxy + y*nvecs + xcb/S,      lane = xcb%S
 *   gauge/clover tile = ((t*nz + z)*(ny/ngy) + y/ngy)*nvecs + xcb/S,
 *                 lane = (y%ngy)*S + xcb%S
 *   spinor field length = nt*Pxyz blocks; gauge/clover length = nt*nz*(ny/ngy)*nvecs tiles
 *
 * Face (halo) buffers are site-major: FT[n_face_sites][2 spin][3 colour][2 re/im],
 * the half-spinor ordering of codegen/data_types.cc:508-543 with one site per
 * entry (QB200_F16N: 12 halves scaled by the site's norm, then the FP32 norm,
 * 14 halves per site).  Face sites are enumerated in increasing (t, z, y, xcb) order of the
 * sites whose coordinate in the face dimension is 0 (back face) or N-1
 * (forward face).
 *
 * Error convention: every entry point returns QB200_OK (0) or a negative
 * QB200_E* code and never aborts the process (the reference prints and calls
 * exit(1) on a bad dir, codegen/jinja/dslash_spec.h.j2:28-31).
 * qb200_last_error() returns a message for the calling thread's last error.
 *
 * Streams: `stream` is a cudaStream_t passed as void* (NULL = legacy default
 * stream).  Calls are asynchronous with respect to the host; the library
 * allocates no device memory on these paths.
 */
#ifndef QPHIX_B200_H
#define QPHIX_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define QB200_ABI_VERSION 1

/* status codes */
#define QB200_OK 0
#define QB200_EINVAL (-1)   /* bad scalar argument or lattice description */
#define QB200_ENULL (-2)    /* a required pointer is NULL */
#define QB200_ELAYOUT (-3)  /* (ftype, soalen, veclen) combination not built */
#define QB200_EDIR (-4)     /* dir outside 0..7 */
#define QB200_ECUDA (-5)    /* CUDA launch or runtime error */
#define QB200_EALIGN (-6)   /* device pointer not aligned to the block size */
#define QB200_ENODEV (-7)   /* no CUDA device */

/* storage types (FT of the reference templates) */
#define QB200_F32 0
#define QB200_F64 1
#define QB200_F16 2 /* IEEE binary16 bits, unscaled: the reference's `half` */
/* FP16 spinors with a per-site FP32 norm: each FourSpinorBlock is followed by
 * float norm[S] (block = 24*S halves + 2*S halves, values = half * norm);
 * links and clover are plain binary16.  Not in the reference (new format). */
#define QB200_F16N 3
#define QB200_BF16 4 /* bfloat16 storage everywhere; not in the reference */

typedef struct qb200_lattice {
  int nx, ny, nz, nt; /* local lattice extents in full sites; nx even */
  int soalen;         /* S: x-sites per spinor block (1,2,4,8,16) */
  int veclen;         /* V: sites per gauge/clover tile; V % S == 0 */
  int pad_xy;         /* spinor blocks of padding after each xy plane */
  int pad_xyz;        /* spinor blocks of padding after each xyz volume */
  int ftype;          /* QB200_F32 / F64 / F16 / F16N / BF16 (F16N, BF16: soalen >= 4) */
  int compress12;     /* 1: gauge tiles store 2 rows (12 reals), 0: 3 rows */
  /* time boundary: hops that cross the global t edge are multiplied by
   * t_boundary (+1 periodic, -1 antiperiodic).  t_edge_lo / t_edge_hi say
   * whether local t = 0 / t = nt-1 lie on the global edge (1 on one GPU). */
  double t_boundary;
  int t_edge_lo, t_edge_hi;
} qb200_lattice;

/* ---- library information --------------------------------------------- */
int qb200_abi_version(void);
const char *qb200_last_error(void);
/* 1 if the (ftype, soalen) pair has compiled kernels, else 0 */
int qb200_layout_supported(int ftype, int soalen);
/* number of elements (FT units) of one checkerboard field */
long long qb200_spinor_elems(const qb200_lattice *lat);
long long qb200_gauge_elems(const qb200_lattice *lat);
long long qb200_clover_elems(const qb200_lattice *lat);
long long qb200_full_clover_elems(const qb200_lattice *lat);
/* number of sites on face `dir` (0..7) of one checkerboard */
long long qb200_face_sites(const qb200_lattice *lat, int dir);

/*
 * ---- body kernels ------------------------------------------------------
 * Common arguments:
 *   cb          checkerboard of `out` (and chi); psi lives on 1-cb
 *   accumulate  8 flags.  accumulate[d] != 0: every hop in direction d is
 *               added.  accumulate[d] == 0: hops in direction d that leave
 *               the local sub-lattice are skipped; face_*finish_dir adds them
 *               later.  (The reference passes these per tile; QPhiX clears
 *               them only on tiles at a communicated boundary.)  NULL = all on.
 *   coeff_s     hop coefficient for x, y, z;  coeff_t_f / coeff_t_b for
 *               forward / backward t hops (codegen/dslash.cc:79-86)
 *   tbc_mask    bit mu set: twisted boundary phase tbc_phases[mu] multiplies
 *               every forward hop in dim mu, its conjugate every backward hop
 *               (the tbc_x..tbc_t template flags; dslash_common.cc:1491-1524)
 *   tbc_phases  [4][2] (re, im); may be NULL when tbc_mask == 0
 */

/* Wilson: out = D psi.  Replaces QPhiX::dslash_{plus,minus}_vec
 * (codegen/jinja/dslash_decl.h.j2:6-43). */
int qb200_dslash_plus_vec(const qb200_lattice *lat, int cb, const void *psi,
                          void *out, const void *gauge,
                          const unsigned accumulate[8], double coeff_s,
                          double coeff_t_f, double coeff_t_b,
                          unsigned tbc_mask, const double *tbc_phases,
                          void *stream);
int qb200_dslash_minus_vec(const qb200_lattice *lat, int cb, const void *psi,
                           void *out, const void *gauge,
                           const unsigned accumulate[8], double coeff_s,
                           double coeff_t_f, double coeff_t_b,
                           unsigned tbc_mask, const double *tbc_phases,
                           void *stream);

/* Wilson: out = alpha chi - D psi (hops subtracted).  Replaces
 * QPhiX::dslash_achimbdpsi_{plus,minus}_vec (dslash_decl.h.j2:45-88). */
int qb200_dslash_achimbdpsi_plus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, double alpha, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, const unsigned accumulate[8], void *stream);
int qb200_dslash_achimbdpsi_minus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, double alpha, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, const unsigned accumulate[8], void *stream);

/* Clover: out = A (D psi), A a Hermitian CloverBlock field (callers pass
 * A^-1 for the even-odd operator).  Replaces
 * QPhiX::clov_dslash_{plus,minus}_vec (clov_dslash_decl.h.j2:7-46). */
int qb200_clov_dslash_plus_vec(const qb200_lattice *lat, int cb,
                               const void *psi, void *out, const void *gauge,
                               const void *clover,
                               const unsigned accumulate[8], double coeff_s,
                               double coeff_t_f, double coeff_t_b,
                               unsigned tbc_mask, const double *tbc_phases,
                               void *stream);
int qb200_clov_dslash_minus_vec(const qb200_lattice *lat, int cb,
                                const void *psi, void *out,
                                const void *gauge, const void *clover,
                                const unsigned accumulate[8], double coeff_s,
                                double coeff_t_f, double coeff_t_b,
                                unsigned tbc_mask, const double *tbc_phases,
                                void *stream);

/* Clover: out = A chi + i rho g5 chi (sign flips for minus) - D psi.
 * Replaces QPhiX::clov_dslash_achimbdpsi_{plus,minus}_vec
 * (clov_dslash_decl.h.j2:49-94; dslash_common.cc:1830-1932). */
int qb200_clov_dslash_achimbdpsi_plus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, const void *clover, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, const unsigned accumulate[8],
    double prec_mass_rho, void *stream);
int qb200_clov_dslash_achimbdpsi_minus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, const void *clover, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, const unsigned accumulate[8],
    double prec_mass_rho, void *stream);

/* Twisted mass: out = muinv (1 -/+ i mu g5) D psi.  Replaces
 * QPhiX::tm_dslash_{plus,minus}_vec (tm_dslash_decl.h.j2:5-45;
 * inverse_twisted_term, dslash_common.cc:1234-1359). */
int qb200_tm_dslash_plus_vec(const qb200_lattice *lat, int cb,
                             const void *psi, void *out, const void *gauge,
                             const unsigned accumulate[8], double coeff_s,
                             double coeff_t_f, double coeff_t_b,
                             unsigned tbc_mask, const double *tbc_phases,
                             double mu, double muinv, void *stream);
int qb200_tm_dslash_minus_vec(const qb200_lattice *lat, int cb,
                              const void *psi, void *out, const void *gauge,
                              const unsigned accumulate[8], double coeff_s,
                              double coeff_t_f, double coeff_t_b,
                              unsigned tbc_mask, const double *tbc_phases,
                              double mu, double muinv, void *stream);

/* Twisted mass: out = alpha (1 +/- i mu g5) chi - D psi.  Replaces
 * QPhiX::tm_dslash_achimbdpsi_{plus,minus}_vec (tm_dslash_decl.h.j2:47-91;
 * twisted_term, dslash_common.cc:1364-1489). */
int qb200_tm_dslash_achimbdpsi_plus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, double alpha, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, double mu, const unsigned accumulate[8],
    void *stream);
int qb200_tm_dslash_achimbdpsi_minus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, double alpha, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, double mu, const unsigned accumulate[8],
    void *stream);

/* Twisted-mass clover: out = F (D psi), F a dense FullCloverBlock field.
 * Replaces QPhiX::tm_clov_dslash_{plus,minus}_vec
 * (tm_clov_dslash_decl.h.j2:7-46; full_clover_term, dslash_common.cc:1188-1232). */
int qb200_tm_clov_dslash_plus_vec(const qb200_lattice *lat, int cb,
                                  const void *psi, void *out,
                                  const void *gauge, const void *full_clover,
                                  const unsigned accumulate[8],
                                  double coeff_s, double coeff_t_f,
                                  double coeff_t_b, unsigned tbc_mask,
                                  const double *tbc_phases, void *stream);
int qb200_tm_clov_dslash_minus_vec(const qb200_lattice *lat, int cb,
                                   const void *psi, void *out,
                                   const void *gauge, const void *full_clover,
                                   const unsigned accumulate[8],
                                   double coeff_s, double coeff_t_f,
                                   double coeff_t_b, unsigned tbc_mask,
                                   const double *tbc_phases, void *stream);

/* Twisted-mass clover: out = F chi + i rho g5 chi - D psi.  Replaces
 * QPhiX::tm_clov_dslash_achimbdpsi_{plus,minus}_vec
 * (tm_clov_dslash_decl.h.j2:49-94). */
int qb200_tm_clov_dslash_achimbdpsi_plus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, const void *full_clover, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, const unsigned accumulate[8],
    double prec_mass_rho, void *stream);
int qb200_tm_clov_dslash_achimbdpsi_minus_vec(
    const qb200_lattice *lat, int cb, const void *psi, const void *chi,
    void *out, const void *gauge, const void *full_clover, double coeff_s,
    double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
    const double *tbc_phases, const unsigned accumulate[8],
    double prec_mass_rho, void *stream);

/*
 * ---- face (halo) kernels -----------------------------------------------
 * face_proj_dir: project the sites of `psi` (checkerboard psi_cb) that lie on
 * the face towards `dir` with the projector of the opposite direction and
 * write them to outbuf (the neighbour in direction dir needs them).
 * Replaces QPhiX::face_proj_dir_{plus,minus} (dslash_decl.h.j2:90-99;
 * pack_face_vec, dslash.cc:433-458).
 */
int qb200_face_proj_dir_plus(const qb200_lattice *lat, int psi_cb,
                             const void *psi, void *outbuf, int dir,
                             void *stream);
int qb200_face_proj_dir_minus(const qb200_lattice *lat, int psi_cb,
                              const void *psi, void *outbuf, int dir,
                              void *stream);

/*
 * face_*finish_dir: for the output sites (checkerboard cb) on the face of
 * `dir`, multiply the received half spinors by the link of direction dir,
 * reconstruct and accumulate into out (read-modify-write).  Wilson and TM
 * faces subtract beta*hop, clover and TM-clover faces add beta*hop and apply
 * the clover field to it (codegen/dslash_common.cc:1934-1993).  tbc != 0
 * applies tbc_phases[dir/2].  Replaces QPhiX::face_finish_dir_*,
 * face_clov_finish_dir_*, tm_face_finish_dir_*, tm_clov_face_finish_dir_*
 * (dslash_decl.h.j2:101-115, clov_dslash_decl.h.j2:96-113,
 * tm_dslash_decl.h.j2:93-109, tm_clov_dslash_decl.h.j2:97-113).
 */
int qb200_face_finish_dir_plus(const qb200_lattice *lat, int cb,
                               const void *inbuf, const void *gauge,
                               void *out, double beta, int dir, int tbc,
                               const double *tbc_phases, void *stream);
int qb200_face_finish_dir_minus(const qb200_lattice *lat, int cb,
                                const void *inbuf, const void *gauge,
                                void *out, double beta, int dir, int tbc,
                                const double *tbc_phases, void *stream);
int qb200_face_clov_finish_dir_plus(const qb200_lattice *lat, int cb,
                                    const void *inbuf, const void *gauge,
                                    void *out, const void *clover,
                                    double beta, int dir, int tbc,
                                    const double *tbc_phases, void *stream);
int qb200_face_clov_finish_dir_minus(const qb200_lattice *lat, int cb,
                                     const void *inbuf, const void *gauge,
                                     void *out, const void *clover,
                                     double beta, int dir, int tbc,
                                     const double *tbc_phases, void *stream);
int qb200_tm_face_finish_dir_plus(const qb200_lattice *lat, int cb,
                                  const void *inbuf, const void *gauge,
                                  void *out, double beta, double mu,
                                  double muinv, int dir, int tbc,
                                  const double *tbc_phases, void *stream);
int qb200_tm_face_finish_dir_minus(const qb200_lattice *lat, int cb,
                                   const void *inbuf, const void *gauge,
                                   void *out, double beta, double mu,
                                   double muinv, int dir, int tbc,
                                   const double *tbc_phases, void *stream);
int qb200_tm_clov_face_finish_dir_plus(const qb200_lattice *lat, int cb,
                                       const void *inbuf, const void *gauge,
                                       void *out, const void *full_clover,
                                       double beta, int dir, int tbc,
                                       const double *tbc_phases,
                                       void *stream);
int qb200_tm_clov_face_finish_dir_minus(const qb200_lattice *lat, int cb,
                                        const void *inbuf, const void *gauge,
                                        void *out, const void *full_clover,
                                        double beta, int dir, int tbc,
                                        const double *tbc_phases,
                                        void *stream);

/*
 * ---- even-odd operator, BLAS and solvers ---------------------------------
 * Not part of the reference (its caller, QPhiX, builds these from the
 * kernels); provided so that a GPU caller needs no per-iteration host code.
 *
 * The Schur operator on checkerboard o = target_cb (e = 1 - o):
 *   Mhat psi = A_oo psi - D_oe A_ee^-1 D_eo psi   (hops scaled by coeff_*)
 * built as the plain kernel on e (with the inverse diagonal term) followed by
 * the achimbdpsi kernel on o.  Per family:
 *   wilson     A = alpha (the plain hop is scaled by 1/alpha)
 *   clover     clov[o] = A_oo (CloverBlock), clov[e] = A_ee^-1
 *   tm         A = alpha (1 + i mu g5); mu, muinv as in tm_dslash
 *   tm_clover  clov[o] = F_oo, clov[e] = F_ee^-1 (FullCloverBlock);
 *              clov_dag[] = the same blocks conjugate-transposed (dagger)
 * isign = -1 applies Mhat^dag (the minus kernels, D^dag = D(isign=-1)).
 */
typedef struct qb200_operator {
  int family; /* 0 wilson, 1 clover, 2 tm, 3 tm_clover */
  int target_cb;
  const void *gauge[2];     /* packed links of checkerboard 0 and 1 */
  const void *clov[2];      /* see above, indexed by checkerboard */
  const void *clov_dag[2];  /* tm_clover only */
  double coeff_s, coeff_t_f, coeff_t_b;
  double alpha, mu, muinv, rho;
  unsigned tbc_mask;
  double tbc_phases[4][2];
} qb200_operator;

/* out = Mhat in (isign +1) or Mhat^dag in (-1); tmp_other_cb: one spinor */
int qb200_schur_apply(const qb200_lattice *lat, const qb200_operator *op, int isign, const void *in, void *out,
                      void *tmp_other_cb, void *stream);

/* Allocation-free form of qb200_schur_apply, for callers that cannot
 * provide device scratch memory -- for example a host program whose device
 * memory is owned entirely by its own allocator and that may not call
 * cudaMalloc from this code path, or a time-critical loop where an
 * allocation could synchronise the device.  It has no counterpart in the
 * reference.  The intermediate spinor (the other checkerboard) lives in a
 * static device array of QB200_NOALLOC_SCRATCH_BYTES (32 MiB) that every GPU
 * loading the library holds until exit.  A lattice whose one-checkerboard
 * spinor array (padding included) is larger -- beyond about 349,000 sites
 * per checkerboard in FP32, 174,000 in FP64; a 24^3 x 48 FP32 lattice fits --
 * is rejected with QB200_EINVAL.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller.  The array's address is looked up once per device and kept, so do
 * not use this entry point across cudaDeviceReset (or any other teardown of
 * the device's primary context).  The function allocates nothing. */
#define QB200_NOALLOC_SCRATCH_BYTES (32 << 20)
int qb200_schur_apply_noalloc(const qb200_lattice *lat, const qb200_operator *op, int isign, const void *in,
                              void *out, void *stream);

/* BLAS on n storage elements (a whole spinor array, padding included).
 * Reductions accumulate in FP64 and leave the result on the device;
 * `partials` is device scratch of qb200_blas_partials_len() doubles. */
long long qb200_blas_partials_len(void);
int qb200_blas_axpby(int ftype, long long n, double a, const void *x, double b, void *y, void *stream);
int qb200_blas_convert(int ft_out, void *out, int ft_in, const void *in, long long n, double scale,
                       void *stream);
int qb200_blas_dot(int ftype, long long n, const void *x, const void *y, double *result, double *partials,
                   void *stream);
int qb200_blas_cdot(const qb200_lattice *lat, const void *x, const void *y, double *result /* re, im */,
                    double *partials, void *stream);
/* out = scale * in between spinor arrays of two lattices of the same shape
 * and any storage types (the only conversion that handles QB200_F16N, whose
 * per-site norms the element-wise qb200_blas_* calls reject) */
int qb200_spinor_convert(const qb200_lattice *lat_out, void *out, const qb200_lattice *lat_in, const void *in,
                         double scale, void *stream);

/* Solvers for Mhat x = b on the target checkerboard.  Device workspace of
 * the size the *_workspace_bytes function returns is passed by the caller.
 * rel_res returns |b - Mhat x| / |b|.  CG runs on the normal equations. */
long long qb200_cg_workspace_bytes(const qb200_lattice *lat);
long long qb200_bicgstab_workspace_bytes(const qb200_lattice *lat);
int qb200_invert_cg(const qb200_lattice *lat, const qb200_operator *op, const void *b, void *x, double rel_tol,
                    int max_iter, void *workspace, int *iters, double *rel_res, void *stream);
/* CG on the normal operator itself: Mhat^dag Mhat x = b (the solve a
 * pseudofermion action or force needs); workspace of qb200_cg_workspace_bytes;
 * rel_res = |b - Mhat^dag Mhat x| / |b| */
int qb200_invert_cg_normal(const qb200_lattice *lat, const qb200_operator *op, const void *b, void *x,
                           double rel_tol, int max_iter, void *workspace, int *iters, double *rel_res, void *stream);
int qb200_invert_bicgstab(const qb200_lattice *lat, const qb200_operator *op, const void *b, void *x,
                          double rel_tol, int max_iter, void *workspace, int *iters, double *rel_res,
                          void *stream);
/* Mixed precision with defect correction: residuals and the solution in the
 * high-precision lattice (FP64 storage), corrections solved with the
 * low-precision lattice (FP32 or FP16 storage; its operator fields in that
 * type) to inner_tol.  solver 0: CG on the normal equations, 1: BiCGStab.
 * solver 2: one CG on the normal equations in the low precision with FP64
 * reliable updates (no restarts): x accumulates in FP64 and the FP64
 * residual replaces the low-precision one whenever the latter has fallen by
 * the factor inner_tol (0 < inner_tol < 1); max_inner bounds the
 * iterations, max_outer the updates.
 * Returns the high workspace size; *lo_bytes receives the low one. */
long long qb200_mixed_workspace_bytes(const qb200_lattice *lat_hi, const qb200_lattice *lat_lo,
                                      long long *lo_bytes);
int qb200_invert_mixed(const qb200_lattice *lat_hi, const qb200_operator *op_hi, const qb200_lattice *lat_lo,
                       const qb200_operator *op_lo, int solver, const void *b, void *x, double rel_tol,
                       double inner_tol, int max_inner, int max_outer, void *ws_hi, void *ws_lo,
                       int *inner_iters, int *outer_iters, double *rel_res, void *stream);

/*
 * ---- multi-right-hand-side operator -------------------------------------
 * No counterpart in the reference.  A multi-RHS spinor array holds nrhs
 * (1, 2, 4, 8 or 16) fields of one checkerboard with the right-hand side innermost:
 * FT[block][3 colour][4 spin][2 re/im][S][nrhs] (blocks and padding as in the
 * single layout).  Links and clover are shared by all right-hand sides, so
 * their bytes are read once per nrhs solutions.  Built for FP32 and FP16
 * storage, soalen 4, 8, 16.
 */
typedef struct qb200_coeffs {
  double coeff_s, coeff_t_f, coeff_t_b;
  double alpha, mu, muinv, rho;
  unsigned tbc_mask;
  double tbc_phases[4][2];
} qb200_coeffs;

long long qb200_mrhs_spinor_elems(const qb200_lattice *lat, int nrhs);
/* gather nrhs single-layout fields (host array of device pointers) into one
 * multi-RHS array, and scatter back */
int qb200_mrhs_pack(const qb200_lattice *lat, int nrhs, const void *const *fields, void *mrhs, void *stream);
int qb200_mrhs_unpack(const qb200_lattice *lat, int nrhs, const void *mrhs, void *const *fields, void *stream);
/* the body kernels on multi-RHS arrays: family 0..3 (wilson, clover, tm,
 * tm_clover), achimbdpsi 0/1, isign +1/-1; the meaning of every scalar is
 * that of the single-RHS entry points */
int qb200_dslash_mrhs(const qb200_lattice *lat, int nrhs, int family, int achimbdpsi, int isign, int cb,
                      const void *psi, const void *chi, void *out, const void *gauge, const void *clover,
                      const qb200_coeffs *coeffs, const unsigned accumulate[8], void *stream);
int qb200_schur_apply_mrhs(const qb200_lattice *lat, int nrhs, const qb200_operator *op, int isign, const void *in,
                           void *out, void *tmp_other_cb, void *stream);
/* CG on the normal equations for nrhs systems sharing operator applications;
 * rel_res[nrhs] receives |r|/|rhs| of each normal-equation residual */
long long qb200_cg_mrhs_workspace_bytes(const qb200_lattice *lat, int nrhs);
int qb200_invert_cg_mrhs(const qb200_lattice *lat, int nrhs, const qb200_operator *op, const void *b, void *x,
                         double rel_tol, int max_iter, void *workspace, int *iters, double *rel_res, void *stream);
/* nrhs systems Mhat x_i = b_i in FP64 (b, x: host arrays of nrhs device
 * pointers to FP64 single-layout spinors, lat_hi FP64) with the corrections
 * solved together by the multi-RHS low-precision operator (lat_lo FP16 or
 * FP32); rel_res[nrhs] = |b_i - Mhat x_i| / |b_i| */
long long qb200_mixed_mrhs_workspace_bytes(const qb200_lattice *lat_hi, const qb200_lattice *lat_lo, int nrhs,
                                           long long *lo_bytes);
int qb200_invert_mixed_mrhs(const qb200_lattice *lat_hi, const qb200_operator *op_hi, const qb200_lattice *lat_lo,
                            const qb200_operator *op_lo, int nrhs, const void *const *b, void *const *x,
                            double rel_tol, double inner_tol, int max_inner, int max_outer, void *ws_hi, void *ws_lo,
                            int *inner_iters, int *outer_iters, double *rel_res, void *stream);
/* Multi-RHS CG on the normal equations in the low precision with FP64
 * reliable updates, all right-hand sides updated together: x_i accumulate in
 * FP64, and the residuals b_i - Mhat x_i (FP64) replace the iterated ones
 * whenever every unconverged right-hand side's iterated residual has fallen
 * by delta (0 < delta < 1); the recurrence continues (no restart).  Same
 * arguments and workspaces as qb200_invert_mixed_mrhs; *iters: iterations,
 * *updates: FP64 updates. */
int qb200_invert_reliable_mrhs(const qb200_lattice *lat_hi, const qb200_operator *op_hi,
                               const qb200_lattice *lat_lo, const qb200_operator *op_lo, int nrhs,
                               const void *const *b, void *const *x, double rel_tol, double delta, int max_iter,
                               int max_updates, void *ws_hi, void *ws_lo, int *iters, int *updates, double *rel_res,
                               void *stream);

/* ---- layout converters -------------------------------------------------
 * No counterpart in the reference (QPhiX converts on the host).  Canonical
 * site-major complex fields in device memory, (re, im) pairs of ctype =
 * QB200_F64 or QB200_F32:
 *   spinor  [nt][nz][ny][nxh][4 spin][3 colour]            one checkerboard
 *   links   [4 mu][nt_global][nz][ny][nx][3][3] (U)         the whole lattice
 *   clover  [nt][nz][ny][nxh][2 block][6][6]                one checkerboard
 * (site (xcb, y, z, t) of checkerboard cb at x = 2*xcb + ((y+z+t+cb)&1)),
 * to and from the tile layouts of lat (storage type lat->ftype; QB200_F16N
 * spinors get their per-site norm).  Padding blocks of a spinor field are
 * not written: zero the field once.  qb200_pack_gauge packs the links of
 * checkerboard cb of the local slab whose first time slice is global slice
 * t0 (G = U^T, backward links U(x - mu), rows 0-1 when compress12);
 * qb200_pack_clover keeps the diagonal and lower triangle of each Hermitian
 * block, qb200_pack_full_clover the dense blocks. */
int qb200_pack_spinor(const qb200_lattice *lat, int ctype, const void *canon, void *spinor, void *stream);
int qb200_unpack_spinor(const qb200_lattice *lat, int ctype, const void *spinor, void *canon, void *stream);
int qb200_pack_gauge(const qb200_lattice *lat, int cb, int ctype, const void *links, int nt_global, int t0,
                     void *gauge, void *stream);
int qb200_pack_clover(const qb200_lattice *lat, int ctype, const void *blocks, void *clover, void *stream);
int qb200_pack_full_clover(const qb200_lattice *lat, int ctype, const void *blocks, void *clover, void *stream);

/* ---- batched launch and launch tuning -----------------------------------
 * No counterpart in the reference (its kernels cover one tile of one lattice
 * per call).  One launch applies the same operator (family 0..3 as in
 * qb200_operator, achimbdpsi 0/1, isign) to up to QB200_MAX_BATCH independent
 * lattices of possibly different sizes.  All items share ftype, soalen,
 * veclen and compress12 (soalen >= 4 needs veclen == soalen); each has its
 * own fields, checkerboard and coefficients (qb200_coeffs; hops leaving a
 * lattice wrap around it: every accumulate flag is on).  The per-site
 * operator is that of the single-lattice entry points. */
#define QB200_MAX_BATCH 16
typedef struct qb200_batch_item {
  qb200_lattice lat;
  int cb;
  const void *psi, *chi, *gauge, *clov; /* chi: achimbdpsi only; clov: clover families */
  void *out;
  qb200_coeffs coeffs;
} qb200_batch_item;
/* grid = number of blocks (0: one thread per site; smaller grids make the
 * threads stride through the sites: a persistent launch); block = 64 or 128 */
typedef struct qb200_launch_cfg {
  int grid, block;
} qb200_launch_cfg;
/* cfg NULL: the tuned choice for this batch if qb200_tune_batched has seen
 * its key (operator, layout, lattice sizes, device), else one thread per
 * site with blocks of 128 */
int qb200_dslash_batched(int family, int achimbdpsi, int isign, int nitems, const qb200_batch_item *items,
                         const qb200_launch_cfg *cfg, void *stream);
/* times the candidate launch configurations on these fields (each run
 * writes the operator's result to the items' out), remembers the fastest
 * under the batch's key and returns it; a key already tuned returns at once.
 * Synchronises the stream; do not call it during stream capture. */
int qb200_tune_batched(int family, int achimbdpsi, int isign, int nitems, const qb200_batch_item *items,
                       qb200_launch_cfg *best, double *best_ms, void *stream);
/* the process-wide tuning table as text lines "key grid block ms";
 * load returns the number of entries read or a negative status */
int qb200_tune_cache_save(const char *path);
int qb200_tune_cache_load(const char *path);
void qb200_tune_cache_clear(void);

/* ---- backward: link derivative of the hopping term ----------------------
 * No counterpart in the reference (it has no backward kernels).
 *
 * For L = Re <chi, H psi>, H the eight-hop sum of the plain Wilson dslash on
 * checkerboard cb (qb200_dslash_plus_vec / _minus_vec by isign, same
 * coefficients, twisted phases and time boundary; chi on cb, psi on 1 - cb),
 * writes for each site of cb and each of its eight stored links U
 * (direction 2*mu+1: U_mu(x); 2*mu: U_mu(x - mu)):
 *   gauge == NULL:  F = dL/dRe U + i dL/dIm U                  (3 x 3 complex)
 *   gauge != NULL:  P = TA(F U^dag), the traceless anti-Hermitian
 *                   projection, using the links of `gauge` (checkerboard cb,
 *                   18 or 12 reals); dL/deps along U -> exp(eps X) U is
 *                   Re tr(X^dag P).
 * Layout: real component k = ((dir*3 + row)*3 + col)*2 + re/im of the i-th
 * site of cb in (t, z, y, xcb) order at force[k * nsites + i]
 * (qb200_hop_force_elems reals).  FP32 or FP64 storage; the spinor
 * cotangent of L is the dagger dslash (isign flipped) of chi. */
long long qb200_hop_force_elems(const qb200_lattice *lat);
int qb200_hop_force(const qb200_lattice *lat, int cb, int isign, const void *chi, const void *psi,
                    const void *gauge, double coeff_s, double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                    const double *tbc_phases, void *force, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QPHIX_B200_H */
