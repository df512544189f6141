/*
 * qphix_b200_qphix.h -- the per-tile QPhiX kernel interface, served by the
 * B200 library (C++ only).
 *
 * QPhiX (the C++ host library that calls qphix-codegen's kernels; it is not
 * part of qphix-codegen) includes the generated declarations of
 * codegen/jinja/{dslash,clov_dslash,tm_dslash,tm_clov_dslash}_decl.h.j2 and
 * links one ISA's explicit specialisations of these function templates.  The
 * B200 library exports the same specialisations for a "b200" ISA:
 *
 *     FT = float, double or QPhiX::half (IEEE binary16 bits)
 *     veclen = soalen = 4, 8 or 16, compress12 = true or false,
 *     every tbc_x..tbc_t combination (body kernels), tbc = true or false (faces)
 *
 * so QPhiX links against libqphix_b200.so unchanged.  The declarations below
 * restate the reference's (same template parameters, parameter types and
 * order; they have to be alike for the symbol names to match):
 *   dslash_{plus,minus}_vec, dslash_achimbdpsi_*, face_proj_dir_*,
 *   face_finish_dir_*                         codegen/jinja/dslash_decl.h.j2:6-115
 *   clov_dslash_*, clov_dslash_achimbdpsi_*,
 *   face_clov_finish_dir_*                    codegen/jinja/clov_dslash_decl.h.j2:7-113
 *   tm_dslash_*, tm_dslash_achimbdpsi_*,
 *   tm_face_finish_dir_*                      codegen/jinja/tm_dslash_decl.h.j2:7-109
 *   tm_clov_dslash_*, tm_clov_dslash_achimbdpsi_*,
 *   tm_clov_face_finish_dir_*                 codegen/jinja/tm_clov_dslash_decl.h.j2:7-113
 * and Types<> is the layout contract of codegen/include/decl_common.h:9-62.
 *
 * Semantics: each call computes one tile of veclen sites exactly as the
 * reference's kernel of the same name does (neighbour offsets in FT elements
 * relative to the base pointers, SOA split loads for the x hops, accumulate[]
 * as a lane mask for x and y and a flag for z and t, beta / coeff_* as given,
 * scalars of FT = half passed as binary16 bits).  The work runs on the GPU:
 *   - every pointer must be addressable by the current CUDA device (device
 *     memory, cudaMallocManaged memory, mapped pinned host memory, or any
 *     host memory where the device reports pageable memory access);
 *   - the offset and accumulate arrays are read on the host, at the call;
 *   - the call launches one small kernel on the calling thread's per-thread
 *     default stream and waits for it, so the result is in place when the
 *     call returns and calls from several host threads run side by side.
 * This is the drop-in path for an unmodified QPhiX.  One launch per tile
 * costs a few microseconds, so a GPU-aware caller should hand whole
 * checkerboards to the lattice-level entry points of qphix_b200.h instead.
 * gOffs is not read: the gauge and clover tiles are packed per tile
 * (USE_PACKED_GAUGES / USE_PACKED_CLOVER, on in every reference ISA build),
 * so gBase and clBase already point at the tile.  The prefetch arguments
 * (*prefdist, pfyOffs, pfBase*) are accepted and ignored, as in reference
 * builds without prefetching.
 *
 * Errors: the reference prints and exits on a bad dir
 * (codegen/jinja/dslash_spec.h.j2:28-31); these kernels never exit.  A bad
 * argument or a CUDA error skips the call and records the first error, which
 * qb200_qphix_status() / qb200_qphix_last_error() report until
 * qb200_qphix_clear_status() resets them.
 */
#ifndef QPHIX_B200_QPHIX_H
#define QPHIX_B200_QPHIX_H

extern "C" {
/* first error recorded by a per-tile call (QB200_OK if none), its message,
 * and a reset; thread-safe */
int qb200_qphix_status(void);
const char *qb200_qphix_last_error(void);
void qb200_qphix_clear_status(void);
}

namespace QPhiX {

typedef unsigned short half;

template <typename T, int V, int S, bool compressP>
struct Types {
  typedef T FourSpinorBlock[3][4][2][S];
  typedef T TwoSpinorBlock[3][2][2][V];
  typedef T SU3MatrixBlock[8][(compressP ? 2 : 3)][3][2][V];
  struct CloverBlock {
    T diag1[6][V];
    T off_diag1[15][2][V];
    T diag2[6][V];
    T off_diag2[15][2][V];
  };
  struct FullCloverBlock {
    T block1[6][6][2][V];
    T block2[6][6][2][V];
  };
};

#define QB200_QPHIX_SPINOR const typename Types<FT, veclen, soalen, compress12>::FourSpinorBlock
#define QB200_QPHIX_OUT typename Types<FT, veclen, soalen, compress12>::FourSpinorBlock
#define QB200_QPHIX_GAUGE const typename Types<FT, veclen, soalen, compress12>::SU3MatrixBlock
#define QB200_QPHIX_CLOV const typename Types<FT, veclen, soalen, compress12>::CloverBlock
#define QB200_QPHIX_FCLOV const typename Types<FT, veclen, soalen, compress12>::FullCloverBlock
#define QB200_QPHIX_TBC4 bool tbc_x = false, bool tbc_y = false, bool tbc_z = false, bool tbc_t = false

/* plain body kernels: the hopping term (Wilson), A.Dpsi (clover: the caller
 * passes A^-1 for the inverse-clover operator), muinv (1 -/+ i mu g5) Dpsi
 * (twisted mass), F.Dpsi (twisted-mass clover, F a FullCloverBlock) */
#define QB200_QPHIX_PLAIN_HEAD                                                                           \
  QB200_QPHIX_SPINOR *xyBase, QB200_QPHIX_SPINOR *zbBase, QB200_QPHIX_SPINOR *zfBase,                    \
      QB200_QPHIX_SPINOR *tbBase, QB200_QPHIX_SPINOR *tfBase, QB200_QPHIX_OUT *oBase,                    \
      QB200_QPHIX_GAUGE *gBase
#define QB200_QPHIX_ACH_HEAD                                                                             \
  QB200_QPHIX_SPINOR *xyBase, QB200_QPHIX_SPINOR *zbBase, QB200_QPHIX_SPINOR *zfBase,                    \
      QB200_QPHIX_SPINOR *tbBase, QB200_QPHIX_SPINOR *tfBase, QB200_QPHIX_SPINOR *chiBase,               \
      QB200_QPHIX_OUT *oBase, QB200_QPHIX_GAUGE *gBase
#define QB200_QPHIX_OFFS                                                                                 \
  const int xbOffs[veclen], const int xfOffs[veclen], const int ybOffs[veclen], const int yfOffs[veclen], \
      const int offs[veclen], const int gOffs[veclen], const int siprefdist1, const int siprefdist2,     \
      const int siprefdist3, const int siprefdist4
#define QB200_QPHIX_PF                                                                                   \
  const int pfyOffs[veclen], QB200_QPHIX_SPINOR *pfBase2, QB200_QPHIX_SPINOR *pfBase3,                   \
      QB200_QPHIX_SPINOR *pfBase4

/* ---- Wilson (codegen/jinja/dslash_decl.h.j2:6-115) ---- */
#define QB200_QPHIX_DECL_WILSON(isign)                                                                   \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_OFFS, const int gprefdist,               \
                            QB200_QPHIX_PF, const unsigned int accumulate[8], const FT coeff_s,          \
                            const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2]);          \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void dslash_achimbdpsi_##isign##_vec(QB200_QPHIX_ACH_HEAD, QB200_QPHIX_OFFS, const int chiprefdist,    \
                                       const int gprefdist, QB200_QPHIX_PF, QB200_QPHIX_SPINOR *pfBaseChi, \
                                       const FT alpha, const FT coeff_s, const FT coeff_t_f,             \
                                       const FT coeff_t_b, const FT tbc_phases[4][2],                    \
                                       const unsigned int accumulate[8]);                                \
  template <typename FT, int veclen, int soalen, bool compress12>                                        \
  void face_proj_dir_##isign(QB200_QPHIX_SPINOR *xyBase, const int offs[veclen], const int si_prefdist,  \
                             FT *outbuf, const int hsprefdist, unsigned int mask, int dir);              \
  template <typename FT, int veclen, int soalen, bool compress12, bool tbc = false>                      \
  void face_finish_dir_##isign(const FT *inbuf, QB200_QPHIX_GAUGE *gBase, QB200_QPHIX_OUT *oBase,         \
                               const int gOffs[veclen], const int offs[veclen], const int hsprefdist,    \
                               const int gprefdist, const int soprefdist, const FT beta,                 \
                               unsigned int mask, int dir, const FT tbc_phases[4][2]);

/* ---- clover (codegen/jinja/clov_dslash_decl.h.j2:7-113) ---- */
#define QB200_QPHIX_DECL_CLOVER(isign)                                                                   \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void clov_dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_CLOV *clBase, QB200_QPHIX_OFFS,    \
                                 const int gprefdist, const int clprefdist, QB200_QPHIX_PF,              \
                                 const unsigned int accumulate[8], const FT coeff_s, const FT coeff_t_f, \
                                 const FT coeff_t_b, const FT tbc_phases[4][2]);                         \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void clov_dslash_achimbdpsi_##isign##_vec(                                                             \
      QB200_QPHIX_ACH_HEAD, QB200_QPHIX_CLOV *clBase, QB200_QPHIX_OFFS, const int chiprefdist,          \
      const int gprefdist, const int clprefdist, QB200_QPHIX_PF, QB200_QPHIX_SPINOR *pfBaseChi,           \
      const FT coeff_s, const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2],               \
      const unsigned int accumulate[8], const FT prec_mass_rho);                                         \
  template <typename FT, int veclen, int soalen, bool compress12, bool tbc = false>                      \
  void face_clov_finish_dir_##isign(const FT *inbuf, QB200_QPHIX_GAUGE *gBase, QB200_QPHIX_OUT *oBase,   \
                                    QB200_QPHIX_CLOV *clBase, const int gOffs[veclen],                   \
                                    const int offs[veclen], const int hsprefdist, const int gprefdist,   \
                                    const int soprefdist, const int clprefdist, const FT beta,           \
                                    unsigned int mask, int dir, const FT tbc_phases[4][2]);

/* ---- twisted mass (codegen/jinja/tm_dslash_decl.h.j2:7-109) ---- */
#define QB200_QPHIX_DECL_TM(isign)                                                                       \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void tm_dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_OFFS, const int gprefdist,            \
                               QB200_QPHIX_PF, const unsigned int accumulate[8], const FT coeff_s,       \
                               const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2],        \
                               const FT mu, const FT muinv);                                             \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void tm_dslash_achimbdpsi_##isign##_vec(QB200_QPHIX_ACH_HEAD, QB200_QPHIX_OFFS, const int chiprefdist, \
                                          const int gprefdist, QB200_QPHIX_PF,                           \
                                          QB200_QPHIX_SPINOR *pfBaseChi, const FT alpha, const FT coeff_s, \
                                          const FT coeff_t_f, const FT coeff_t_b,                        \
                                          const FT tbc_phases[4][2], const FT mu,                        \
                                          const unsigned int accumulate[8]);                             \
  template <typename FT, int veclen, int soalen, bool compress12, bool tbc = false>                      \
  void tm_face_finish_dir_##isign(const FT *inbuf, QB200_QPHIX_GAUGE *gBase, QB200_QPHIX_OUT *oBase,     \
                                  const int gOffs[veclen], const int offs[veclen], const int hsprefdist, \
                                  const int gprefdist, const int soprefdist, const FT beta,              \
                                  const FT mu, const FT muinv, unsigned int mask, int dir,               \
                                  const FT tbc_phases[4][2]);

/* ---- twisted-mass clover (codegen/jinja/tm_clov_dslash_decl.h.j2:7-113) ---- */
#define QB200_QPHIX_DECL_TMCLOV(isign)                                                                   \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void tm_clov_dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_FCLOV *clBase, QB200_QPHIX_OFFS, \
                                    const int gprefdist, const int clprefdist, QB200_QPHIX_PF,           \
                                    const unsigned int accumulate[8], const FT coeff_s,                  \
                                    const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2]);  \
  template <typename FT, int veclen, int soalen, bool compress12, QB200_QPHIX_TBC4>                      \
  void tm_clov_dslash_achimbdpsi_##isign##_vec(                                                          \
      QB200_QPHIX_ACH_HEAD, QB200_QPHIX_FCLOV *clBase, QB200_QPHIX_OFFS, const int chiprefdist,         \
      const int gprefdist, const int clprefdist, QB200_QPHIX_PF, QB200_QPHIX_SPINOR *pfBaseChi,           \
      const FT coeff_s, const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2],               \
      const unsigned int accumulate[8], const FT prec_mass_rho);                                         \
  template <typename FT, int veclen, int soalen, bool compress12, bool tbc = false>                      \
  void tm_clov_face_finish_dir_##isign(const FT *inbuf, QB200_QPHIX_GAUGE *gBase, QB200_QPHIX_OUT *oBase, \
                                       QB200_QPHIX_FCLOV *clBase, const int gOffs[veclen],               \
                                       const int offs[veclen], const int hsprefdist,                     \
                                       const int gprefdist, const int soprefdist, const int clprefdist,  \
                                       const FT beta, unsigned int mask, int dir,                        \
                                       const FT tbc_phases[4][2]);

QB200_QPHIX_DECL_WILSON(plus)
QB200_QPHIX_DECL_WILSON(minus)
QB200_QPHIX_DECL_CLOVER(plus)
QB200_QPHIX_DECL_CLOVER(minus)
QB200_QPHIX_DECL_TM(plus)
QB200_QPHIX_DECL_TM(minus)
QB200_QPHIX_DECL_TMCLOV(plus)
QB200_QPHIX_DECL_TMCLOV(minus)

} // namespace QPhiX

#endif
