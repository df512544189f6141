// qb200_api.cu -- the C-ABI of include/qphix_b200.h: argument checking,
// lattice description -> device geometry, and dispatch to the kernels of
// (storage type, SOALEN).  No entry point allocates device memory.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "qphix_b200.h"
#include "qb200_internal.h"

using namespace qb200;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_status(cudaError_t e, const char *what)
{
  if (e == cudaSuccess) return QB200_OK;
  return fail(QB200_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

bool soalen_ok(int s) { return s == 1 || s == 2 || s == 4 || s == 8 || s == 16; }

// checks the lattice description and fills the device geometry
int make_geo(const qb200_lattice *l, GeoDev &g)
{
  if (!l) return fail(QB200_ENULL, "lattice description is NULL");
  if (l->nx <= 0 || l->ny <= 0 || l->nz <= 0 || l->nt <= 0)
    return fail(QB200_EINVAL, "lattice extents must be positive (%d %d %d %d)", l->nx, l->ny, l->nz, l->nt);
  if ((l->nx | l->ny | l->nz | l->nt) & 1)
    return fail(QB200_EINVAL, "lattice extents must be even for checkerboarding (%d %d %d %d)", l->nx, l->ny,
                l->nz, l->nt);
  if (!soalen_ok(l->soalen)) return fail(QB200_ELAYOUT, "soalen %d not in {1,2,4,8,16}", l->soalen);
  if (l->veclen <= 0 || l->veclen % l->soalen)
    return fail(QB200_EINVAL, "veclen %d must be a positive multiple of soalen %d", l->veclen, l->soalen);
  if ((l->nx / 2) % l->soalen)
    return fail(QB200_EINVAL, "nx/2 = %d is not a multiple of soalen %d", l->nx / 2, l->soalen);
  const int ngy = l->veclen / l->soalen;
  if (l->ny % ngy) return fail(QB200_EINVAL, "ny = %d is not a multiple of veclen/soalen = %d", l->ny, ngy);
  if (l->pad_xy < 0 || l->pad_xyz < 0) return fail(QB200_EINVAL, "negative padding");
  if (l->ftype != QB200_F32 && l->ftype != QB200_F64 && l->ftype != QB200_F16 && l->ftype != QB200_F16N &&
      l->ftype != QB200_BF16)
    return fail(QB200_ELAYOUT, "unknown storage type %d", l->ftype);
  if ((l->ftype == QB200_F16N || l->ftype == QB200_BF16) && l->soalen < 4)
    return fail(QB200_ELAYOUT, "storage type %d is built for soalen 4, 8 and 16 only", l->ftype);
  const long long nsites = (long long)(l->nx / 2) * l->ny * l->nz * l->nt;
  if (nsites >= (1LL << 31)) return fail(QB200_EINVAL, "checkerboard of %lld sites is too large", nsites);
  g.nx = l->nx;
  g.ny = l->ny;
  g.nz = l->nz;
  g.nt = l->nt;
  g.nxh = l->nx / 2;
  g.nvecs = g.nxh / l->soalen;
  g.ngy = ngy;
  g.nyg = l->ny / ngy;
  g.V = l->veclen;
  g.Pxy = (long long)l->ny * g.nvecs + l->pad_xy;
  g.Pxyz = (long long)l->nz * g.Pxy + l->pad_xyz;
  g.nsites = (int)nsites;
  g.nrhs = 1;
  return QB200_OK;
}

int check_device()
{
  static int ndev = -1;
  if (ndev < 0) {
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) ndev = 0;
  }
  if (ndev <= 0) return fail(QB200_ENODEV, "no CUDA device");
  return QB200_OK;
}

template <typename C>
void fill_op(OpDev<C> &p, const qb200_lattice *l, int isPlus, int cb, bool negate, double coeff_s,
             double coeff_t_f, double coeff_t_b, unsigned tbc_mask, const double *tbc_phases,
             const unsigned *accumulate)
{
  std::memset(&p, 0, sizeof(p));
  const double sg = negate ? -1.0 : 1.0;
  for (int d = 0; d < 6; d++) p.beta[d] = (C)(sg * coeff_s);
  p.beta[6] = (C)(sg * coeff_t_b);
  p.beta[7] = (C)(sg * coeff_t_f);
  p.tbound = (C)l->t_boundary;
  p.t_edge_lo = l->t_edge_lo ? 1 : 0;
  p.t_edge_hi = l->t_edge_hi ? 1 : 0;
  p.tbc_mask = tbc_mask & 15u;
  for (int m = 0; m < 4; m++) {
    p.tbc[m][0] = (C)(tbc_phases ? tbc_phases[2 * m] : 1.0);
    p.tbc[m][1] = (C)(tbc_phases ? tbc_phases[2 * m + 1] : 0.0);
  }
  p.acc_mask = 0;
  for (int d = 0; d < 8; d++)
    if (!accumulate || accumulate[d]) p.acc_mask |= 1u << d;
  p.isPlus = isPlus;
  p.cb = cb;
}

struct Body {
  int fam;
  bool ach;
  int isPlus;
  int cb;
  const void *psi, *chi, *gauge, *clov;
  void *out;
  const unsigned *accumulate;
  double coeff_s, coeff_t_f, coeff_t_b;
  unsigned tbc_mask;
  const double *tbc_phases;
  double alpha, mu, muinv, rho;
};

template <typename FT>
cudaError_t dispatch_body(const qb200_lattice *l, const Body &b, const GeoDev &g, cudaStream_t st)
{
  typedef typename ftraits<FT>::C C;
  OpDev<C> p;
  fill_op<C>(p, l, b.isPlus, b.cb, b.ach, b.coeff_s, b.coeff_t_f, b.coeff_t_b, b.tbc_mask, b.tbc_phases,
             b.accumulate);
  p.alpha = (C)b.alpha;
  p.mu = (C)b.mu;
  p.muinv = (C)b.muinv;
  p.rho = (C)b.rho;
  LaunchSpec ls;
  ls.fam = b.fam;
  ls.ach = b.ach;
  ls.comp12 = l->compress12 != 0;
  typedef elem_t<FT> E;
  const E *psi = (const E *)b.psi, *chi = (const E *)b.chi, *u = (const E *)b.gauge, *cl = (const E *)b.clov;
  E *out = (E *)b.out;
  switch (l->soalen) {
  case 1: return launch_dslash<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 1)>(ls, psi, chi, u, cl, out, g, p, st);
  case 2: return launch_dslash<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 2)>(ls, psi, chi, u, cl, out, g, p, st);
  case 4: return launch_dslash<FT, 4>(ls, psi, chi, u, cl, out, g, p, st);
  case 8: return launch_dslash<FT, 8>(ls, psi, chi, u, cl, out, g, p, st);
  default: return launch_dslash<FT, 16>(ls, psi, chi, u, cl, out, g, p, st);
  }
}

int run_body(const qb200_lattice *l, const Body &b, void *stream)
{
  GeoDev g;
  int rc = make_geo(l, g);
  if (rc) return rc;
  if (b.cb != 0 && b.cb != 1) return fail(QB200_EINVAL, "cb must be 0 or 1 (got %d)", b.cb);
  if (!b.psi || !b.gauge || !b.out) return fail(QB200_ENULL, "psi, gauge and out must be non-NULL");
  if (b.ach && !b.chi) return fail(QB200_ENULL, "achimbdpsi needs chi");
  if ((b.fam == FAM_CLOVER || b.fam == FAM_TMCLOV) && !b.clov)
    return fail(QB200_ENULL, "clover field is NULL");
  if (b.out == b.psi) return fail(QB200_EINVAL, "out must not alias psi");
  if ((b.tbc_mask & 15u) && !b.tbc_phases) return fail(QB200_ENULL, "tbc_mask set but tbc_phases is NULL");
  rc = check_device();
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch (l->ftype) {
  case QB200_F32: e = dispatch_body<float>(l, b, g, st); break;
  case QB200_F64: e = dispatch_body<double>(l, b, g, st); break;
  case QB200_F16: e = dispatch_body<__half>(l, b, g, st); break;
  case QB200_F16N: e = dispatch_body<half_norm>(l, b, g, st); break;
  default: e = dispatch_body<__nv_bfloat16>(l, b, g, st); break;
  }
  return cuda_status(e, "dslash launch");
}

// face geometry of `dir` on checkerboard cb
int face_spec(const GeoDev &g, int dir, int cb, FaceSpec &f)
{
  if (dir < 0 || dir > 7) return fail(QB200_EDIR, "invalid dir %d (must be 0..7)", dir);
  const int L[4] = {g.nx, g.ny, g.nz, g.nt};
  f.dir = dir;
  f.mu = dir / 2;
  f.coord = (dir & 1) ? L[f.mu] - 1 : 0;
  f.par = f.mu == 0 ? (f.coord & 1) : 0;
  f.cb = cb;
  switch (f.mu) {
  case 0: f.nface = g.nt * g.nz * (g.ny / 2); break;
  case 1: f.nface = g.nt * g.nz * g.nxh; break;
  case 2: f.nface = g.nt * g.ny * g.nxh; break;
  default: f.nface = g.nz * g.ny * g.nxh; break;
  }
  return QB200_OK;
}

template <typename FT>
cudaError_t dispatch_pack(const qb200_lattice *l, const void *psi, void *buf, const GeoDev &g,
                          const FaceSpec &f, int isPlus, cudaStream_t st)
{
  typedef elem_t<FT> E;
  const E *p = (const E *)psi;
  E *o = (E *)buf;
  switch (l->soalen) {
  case 1: return launch_face_pack<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 1)>(p, o, g, f, isPlus, st);
  case 2: return launch_face_pack<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 2)>(p, o, g, f, isPlus, st);
  case 4: return launch_face_pack<FT, 4>(p, o, g, f, isPlus, st);
  case 8: return launch_face_pack<FT, 8>(p, o, g, f, isPlus, st);
  default: return launch_face_pack<FT, 16>(p, o, g, f, isPlus, st);
  }
}

int run_pack(const qb200_lattice *l, int isPlus, int psi_cb, const void *psi, void *outbuf, int dir,
             void *stream)
{
  GeoDev g;
  int rc = make_geo(l, g);
  if (rc) return rc;
  if (psi_cb != 0 && psi_cb != 1) return fail(QB200_EINVAL, "cb must be 0 or 1 (got %d)", psi_cb);
  if (!psi || !outbuf) return fail(QB200_ENULL, "psi and outbuf must be non-NULL");
  FaceSpec f;
  rc = face_spec(g, dir, psi_cb, f);
  if (rc) return rc;
  rc = check_device();
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch (l->ftype) {
  case QB200_F32: e = dispatch_pack<float>(l, psi, outbuf, g, f, isPlus, st); break;
  case QB200_F64: e = dispatch_pack<double>(l, psi, outbuf, g, f, isPlus, st); break;
  case QB200_F16: e = dispatch_pack<__half>(l, psi, outbuf, g, f, isPlus, st); break;
  case QB200_F16N: e = dispatch_pack<half_norm>(l, psi, outbuf, g, f, isPlus, st); break;
  default: e = dispatch_pack<__nv_bfloat16>(l, psi, outbuf, g, f, isPlus, st); break;
  }
  return cuda_status(e, "face pack launch");
}

struct Unpack {
  int fam, isPlus, cb;
  const void *inbuf, *gauge, *clov;
  void *out;
  double beta, mu, muinv;
  int dir, tbc;
  const double *tbc_phases;
};

template <typename FT>
cudaError_t dispatch_unpack(const qb200_lattice *l, const Unpack &u, const GeoDev &g, const FaceSpec &f,
                            cudaStream_t st)
{
  typedef typename ftraits<FT>::C C;
  OpDev<C> p;
  const unsigned mask = u.tbc ? (1u << (u.dir / 2)) : 0u;
  fill_op<C>(p, l, u.isPlus, u.cb, false, 0.0, 0.0, 0.0, mask, u.tbc_phases, nullptr);
  p.beta[0] = (C)u.beta;
  p.mu = (C)u.mu;
  p.muinv = (C)u.muinv;
  typedef elem_t<FT> E;
  const E *in = (const E *)u.inbuf, *gg = (const E *)u.gauge, *cl = (const E *)u.clov;
  E *o = (E *)u.out;
  const bool c12 = l->compress12 != 0;
  switch (l->soalen) {
  case 1: return launch_face_unpack<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 1)>(u.fam, c12, in, gg, cl, o, g, f, p, st);
  case 2: return launch_face_unpack<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 2)>(u.fam, c12, in, gg, cl, o, g, f, p, st);
  case 4: return launch_face_unpack<FT, 4>(u.fam, c12, in, gg, cl, o, g, f, p, st);
  case 8: return launch_face_unpack<FT, 8>(u.fam, c12, in, gg, cl, o, g, f, p, st);
  default: return launch_face_unpack<FT, 16>(u.fam, c12, in, gg, cl, o, g, f, p, st);
  }
}

int run_unpack(const qb200_lattice *l, const Unpack &u, void *stream)
{
  GeoDev g;
  int rc = make_geo(l, g);
  if (rc) return rc;
  if (u.cb != 0 && u.cb != 1) return fail(QB200_EINVAL, "cb must be 0 or 1 (got %d)", u.cb);
  if (!u.inbuf || !u.gauge || !u.out) return fail(QB200_ENULL, "inbuf, gauge and out must be non-NULL");
  if ((u.fam == FAM_CLOVER || u.fam == FAM_TMCLOV) && !u.clov)
    return fail(QB200_ENULL, "clover field is NULL");
  if (u.tbc && !u.tbc_phases) return fail(QB200_ENULL, "tbc set but tbc_phases is NULL");
  FaceSpec f;
  rc = face_spec(g, u.dir, u.cb, f);
  if (rc) return rc;
  rc = check_device();
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch (l->ftype) {
  case QB200_F32: e = dispatch_unpack<float>(l, u, g, f, st); break;
  case QB200_F64: e = dispatch_unpack<double>(l, u, g, f, st); break;
  case QB200_F16: e = dispatch_unpack<__half>(l, u, g, f, st); break;
  case QB200_F16N: e = dispatch_unpack<half_norm>(l, u, g, f, st); break;
  default: e = dispatch_unpack<__nv_bfloat16>(l, u, g, f, st); break;
  }
  return cuda_status(e, "face unpack launch");
}

long long elem_count(const qb200_lattice *l, int what)
{
  GeoDev g;
  if (make_geo(l, g)) return -1;
  const long long ntiles = (long long)l->nt * l->nz * g.nyg * g.nvecs;
  switch (what) {
  case 0: return (long long)l->nt * g.Pxyz * (l->ftype == QB200_F16N ? 26 : 24) * l->soalen;
  case 1: return ntiles * 8 * (l->compress12 ? 2 : 3) * 6 * l->veclen;
  case 2: return ntiles * 72 * l->veclen;
  default: return ntiles * 144 * l->veclen;
  }
}

} // namespace

namespace qb200 {
// shared with the solver translation units
int api_fail(int code, const char *msg) { return fail(code, "%s", msg); }
int api_geo(const qb200_lattice *l, GeoDev &g) { return make_geo(l, g); }
int api_check_device() { return check_device(); }
void api_fill_op_f(OpDev<float> &p, const qb200_lattice *l, int isPlus, int cb, bool negate, double cs, double ctf,
                   double ctb, unsigned tbc_mask, const double *ph, const unsigned *acc)
{
  fill_op<float>(p, l, isPlus, cb, negate, cs, ctf, ctb, tbc_mask, ph, acc);
}

void api_fill_op_d(OpDev<double> &p, const qb200_lattice *l, int isPlus, int cb, bool negate, double cs, double ctf,
                   double ctb, unsigned tbc_mask, const double *ph, const unsigned *acc)
{
  fill_op<double>(p, l, isPlus, cb, negate, cs, ctf, ctb, tbc_mask, ph, acc);
}

int api_body(const qb200_lattice *l, int fam, bool ach, int isPlus, int cb, const void *psi, const void *chi,
             const void *gauge, const void *clov, void *out, const unsigned *accumulate, double coeff_s,
             double coeff_t_f, double coeff_t_b, unsigned tbc_mask, const double *tbc_phases, double alpha,
             double mu, double muinv, double rho, void *stream)
{
  Body b;
  std::memset(&b, 0, sizeof(b));
  b.fam = fam;
  b.ach = ach;
  b.isPlus = isPlus;
  b.cb = cb;
  b.psi = psi;
  b.chi = chi;
  b.gauge = gauge;
  b.clov = clov;
  b.out = out;
  b.accumulate = accumulate;
  b.coeff_s = coeff_s;
  b.coeff_t_f = coeff_t_f;
  b.coeff_t_b = coeff_t_b;
  b.tbc_mask = tbc_mask;
  b.tbc_phases = tbc_phases;
  b.alpha = alpha;
  b.mu = mu;
  b.muinv = muinv;
  b.rho = rho;
  return run_body(l, b, stream);
}
} // namespace qb200

extern "C" {

int qb200_abi_version(void) { return QB200_ABI_VERSION; }
const char *qb200_last_error(void) { return g_err.c_str(); }
int qb200_layout_supported(int ftype, int soalen)
{
  if (!soalen_ok(soalen)) return 0;
  if (ftype == QB200_F32 || ftype == QB200_F64 || ftype == QB200_F16) return 1;
  return (ftype == QB200_F16N || ftype == QB200_BF16) && soalen >= 4;
}
long long qb200_spinor_elems(const qb200_lattice *lat) { return elem_count(lat, 0); }
long long qb200_gauge_elems(const qb200_lattice *lat) { return elem_count(lat, 1); }
long long qb200_clover_elems(const qb200_lattice *lat) { return elem_count(lat, 2); }
long long qb200_full_clover_elems(const qb200_lattice *lat) { return elem_count(lat, 3); }
long long qb200_face_sites(const qb200_lattice *lat, int dir)
{
  GeoDev g;
  if (make_geo(lat, g)) return -1;
  FaceSpec f;
  if (face_spec(g, dir, 0, f)) return -1;
  return f.nface;
}

#define QB_BODY(name, FAM, ACH, PLUS, ...)                                                                 \
  {                                                                                                       \
    Body b;                                                                                               \
    std::memset(&b, 0, sizeof(b));                                                                        \
    b.fam = FAM;                                                                                          \
    b.ach = ACH;                                                                                          \
    b.isPlus = PLUS;                                                                                      \
    __VA_ARGS__;                                                                                          \
    return run_body(lat, b, stream);                                                                      \
  }

#define QB_COMMON                                                                                         \
  b.cb = cb;                                                                                              \
  b.psi = psi;                                                                                            \
  b.out = out;                                                                                            \
  b.gauge = gauge;                                                                                        \
  b.accumulate = accumulate;                                                                              \
  b.coeff_s = coeff_s;                                                                                    \
  b.coeff_t_f = coeff_t_f;                                                                                \
  b.coeff_t_b = coeff_t_b;                                                                                \
  b.tbc_mask = tbc_mask;                                                                                  \
  b.tbc_phases = tbc_phases

// ---- Wilson
int qb200_dslash_plus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out, const void *gauge,
                          const unsigned accumulate[8], double coeff_s, double coeff_t_f, double coeff_t_b,
                          unsigned tbc_mask, const double *tbc_phases, void *stream)
QB_BODY(dslash_plus, FAM_WILSON, false, 1, QB_COMMON)
int qb200_dslash_minus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out, const void *gauge,
                           const unsigned accumulate[8], double coeff_s, double coeff_t_f, double coeff_t_b,
                           unsigned tbc_mask, const double *tbc_phases, void *stream)
QB_BODY(dslash_minus, FAM_WILSON, false, 0, QB_COMMON)

int qb200_dslash_achimbdpsi_plus_vec(const qb200_lattice *lat, int cb, const void *psi, const void *chi,
                                     void *out, const void *gauge, double alpha, double coeff_s,
                                     double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                     const double *tbc_phases, const unsigned accumulate[8], void *stream)
QB_BODY(ach_plus, FAM_WILSON, true, 1, QB_COMMON; b.chi = chi; b.alpha = alpha)
int qb200_dslash_achimbdpsi_minus_vec(const qb200_lattice *lat, int cb, const void *psi, const void *chi,
                                      void *out, const void *gauge, double alpha, double coeff_s,
                                      double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                      const double *tbc_phases, const unsigned accumulate[8], void *stream)
QB_BODY(ach_minus, FAM_WILSON, true, 0, QB_COMMON; b.chi = chi; b.alpha = alpha)

// ---- clover
int qb200_clov_dslash_plus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out, const void *gauge,
                               const void *clover, const unsigned accumulate[8], double coeff_s,
                               double coeff_t_f, double coeff_t_b, unsigned tbc_mask, const double *tbc_phases,
                               void *stream)
QB_BODY(clov_plus, FAM_CLOVER, false, 1, QB_COMMON; b.clov = clover)
int qb200_clov_dslash_minus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out, const void *gauge,
                                const void *clover, const unsigned accumulate[8], double coeff_s,
                                double coeff_t_f, double coeff_t_b, unsigned tbc_mask, const double *tbc_phases,
                                void *stream)
QB_BODY(clov_minus, FAM_CLOVER, false, 0, QB_COMMON; b.clov = clover)

int qb200_clov_dslash_achimbdpsi_plus_vec(const qb200_lattice *lat, int cb, const void *psi, const void *chi,
                                          void *out, const void *gauge, const void *clover, double coeff_s,
                                          double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                          const double *tbc_phases, const unsigned accumulate[8],
                                          double prec_mass_rho, void *stream)
QB_BODY(clov_ach_plus, FAM_CLOVER, true, 1, QB_COMMON; b.chi = chi; b.clov = clover; b.rho = prec_mass_rho)
int qb200_clov_dslash_achimbdpsi_minus_vec(const qb200_lattice *lat, int cb, const void *psi, const void *chi,
                                           void *out, const void *gauge, const void *clover, double coeff_s,
                                           double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                           const double *tbc_phases, const unsigned accumulate[8],
                                           double prec_mass_rho, void *stream)
QB_BODY(clov_ach_minus, FAM_CLOVER, true, 0, QB_COMMON; b.chi = chi; b.clov = clover; b.rho = prec_mass_rho)

// ---- twisted mass
int qb200_tm_dslash_plus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out, const void *gauge,
                             const unsigned accumulate[8], double coeff_s, double coeff_t_f, double coeff_t_b,
                             unsigned tbc_mask, const double *tbc_phases, double mu, double muinv, void *stream)
QB_BODY(tm_plus, FAM_TM, false, 1, QB_COMMON; b.mu = mu; b.muinv = muinv)
int qb200_tm_dslash_minus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out, const void *gauge,
                              const unsigned accumulate[8], double coeff_s, double coeff_t_f, double coeff_t_b,
                              unsigned tbc_mask, const double *tbc_phases, double mu, double muinv, void *stream)
QB_BODY(tm_minus, FAM_TM, false, 0, QB_COMMON; b.mu = mu; b.muinv = muinv)

int qb200_tm_dslash_achimbdpsi_plus_vec(const qb200_lattice *lat, int cb, const void *psi, const void *chi,
                                        void *out, const void *gauge, double alpha, double coeff_s,
                                        double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                        const double *tbc_phases, double mu, const unsigned accumulate[8],
                                        void *stream)
QB_BODY(tm_ach_plus, FAM_TM, true, 1, QB_COMMON; b.chi = chi; b.alpha = alpha; b.mu = mu)
int qb200_tm_dslash_achimbdpsi_minus_vec(const qb200_lattice *lat, int cb, const void *psi, const void *chi,
                                         void *out, const void *gauge, double alpha, double coeff_s,
                                         double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                         const double *tbc_phases, double mu, const unsigned accumulate[8],
                                         void *stream)
QB_BODY(tm_ach_minus, FAM_TM, true, 0, QB_COMMON; b.chi = chi; b.alpha = alpha; b.mu = mu)

// ---- twisted-mass clover
int qb200_tm_clov_dslash_plus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out,
                                  const void *gauge, const void *full_clover, const unsigned accumulate[8],
                                  double coeff_s, double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                  const double *tbc_phases, void *stream)
QB_BODY(tmc_plus, FAM_TMCLOV, false, 1, QB_COMMON; b.clov = full_clover)
int qb200_tm_clov_dslash_minus_vec(const qb200_lattice *lat, int cb, const void *psi, void *out,
                                   const void *gauge, const void *full_clover, const unsigned accumulate[8],
                                   double coeff_s, double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                                   const double *tbc_phases, void *stream)
QB_BODY(tmc_minus, FAM_TMCLOV, false, 0, QB_COMMON; b.clov = full_clover)

int qb200_tm_clov_dslash_achimbdpsi_plus_vec(const qb200_lattice *lat, int cb, const void *psi,
                                             const void *chi, void *out, const void *gauge,
                                             const void *full_clover, double coeff_s, double coeff_t_f,
                                             double coeff_t_b, unsigned tbc_mask, const double *tbc_phases,
                                             const unsigned accumulate[8], double prec_mass_rho, void *stream)
QB_BODY(tmc_ach_plus, FAM_TMCLOV, true, 1, QB_COMMON; b.chi = chi; b.clov = full_clover; b.rho = prec_mass_rho)
int qb200_tm_clov_dslash_achimbdpsi_minus_vec(const qb200_lattice *lat, int cb, const void *psi,
                                              const void *chi, void *out, const void *gauge,
                                              const void *full_clover, double coeff_s, double coeff_t_f,
                                              double coeff_t_b, unsigned tbc_mask, const double *tbc_phases,
                                              const unsigned accumulate[8], double prec_mass_rho, void *stream)
QB_BODY(tmc_ach_minus, FAM_TMCLOV, true, 0, QB_COMMON; b.chi = chi; b.clov = full_clover; b.rho = prec_mass_rho)

// ---- faces
int qb200_face_proj_dir_plus(const qb200_lattice *lat, int psi_cb, const void *psi, void *outbuf, int dir,
                             void *stream)
{
  return run_pack(lat, 1, psi_cb, psi, outbuf, dir, stream);
}
int qb200_face_proj_dir_minus(const qb200_lattice *lat, int psi_cb, const void *psi, void *outbuf, int dir,
                              void *stream)
{
  return run_pack(lat, 0, psi_cb, psi, outbuf, dir, stream);
}

#define QB_UNPACK(FAM, PLUS, CLOV, MU, MUINV)                                                              \
  {                                                                                                       \
    Unpack u;                                                                                             \
    std::memset(&u, 0, sizeof(u));                                                                        \
    u.fam = FAM;                                                                                          \
    u.isPlus = PLUS;                                                                                      \
    u.cb = cb;                                                                                            \
    u.inbuf = inbuf;                                                                                      \
    u.gauge = gauge;                                                                                      \
    u.clov = CLOV;                                                                                        \
    u.out = out;                                                                                          \
    u.beta = beta;                                                                                        \
    u.mu = MU;                                                                                            \
    u.muinv = MUINV;                                                                                      \
    u.dir = dir;                                                                                          \
    u.tbc = tbc;                                                                                          \
    u.tbc_phases = tbc_phases;                                                                            \
    return run_unpack(lat, u, stream);                                                                    \
  }

int qb200_face_finish_dir_plus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge, void *out,
                               double beta, int dir, int tbc, const double *tbc_phases, void *stream)
QB_UNPACK(FAM_WILSON, 1, nullptr, 0.0, 0.0)
int qb200_face_finish_dir_minus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge,
                                void *out, double beta, int dir, int tbc, const double *tbc_phases, void *stream)
QB_UNPACK(FAM_WILSON, 0, nullptr, 0.0, 0.0)
int qb200_face_clov_finish_dir_plus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge,
                                    void *out, const void *clover, double beta, int dir, int tbc,
                                    const double *tbc_phases, void *stream)
QB_UNPACK(FAM_CLOVER, 1, clover, 0.0, 0.0)
int qb200_face_clov_finish_dir_minus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge,
                                     void *out, const void *clover, double beta, int dir, int tbc,
                                     const double *tbc_phases, void *stream)
QB_UNPACK(FAM_CLOVER, 0, clover, 0.0, 0.0)
int qb200_tm_face_finish_dir_plus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge,
                                  void *out, double beta, double mu, double muinv, int dir, int tbc,
                                  const double *tbc_phases, void *stream)
QB_UNPACK(FAM_TM, 1, nullptr, mu, muinv)
int qb200_tm_face_finish_dir_minus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge,
                                   void *out, double beta, double mu, double muinv, int dir, int tbc,
                                   const double *tbc_phases, void *stream)
QB_UNPACK(FAM_TM, 0, nullptr, mu, muinv)
int qb200_tm_clov_face_finish_dir_plus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge,
                                       void *out, const void *full_clover, double beta, int dir, int tbc,
                                       const double *tbc_phases, void *stream)
QB_UNPACK(FAM_TMCLOV, 1, full_clover, 0.0, 0.0)
int qb200_tm_clov_face_finish_dir_minus(const qb200_lattice *lat, int cb, const void *inbuf, const void *gauge,
                                        void *out, const void *full_clover, double beta, int dir, int tbc,
                                        const double *tbc_phases, void *stream)
QB_UNPACK(FAM_TMCLOV, 0, full_clover, 0.0, 0.0)

} // extern "C"
