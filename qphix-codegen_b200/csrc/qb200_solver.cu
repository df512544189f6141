// qb200_solver.cu -- spinor BLAS, the even-odd (Schur) operator and the
// Krylov solvers (CG on M^dag M, BiCGStab on M, and FP64-corrected mixed
// precision CG), as host C++ driving the dslash kernels on one stream.
//
// The reference generates only the kernels; the operator and solvers are
// what its caller (QPhiX) builds from them: the achimbdpsi kernel on the
// target checkerboard applied after the plain kernel (with the inverse
// diagonal term) on the other one gives
//   Mhat psi = A_oo psi - beta^2 D_oe A_ee^-1 D_eo psi
// (codegen/dslash_common.cc:1729-1826 and :1830-1932 for the two halves).
// No entry point allocates device memory: the caller passes a workspace.
#include <algorithm>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "qphix_b200.h"
#include "qb200_blas.cuh"
#include "qb200_internal.h"

namespace qb200 {
int api_fail(int code, const char *msg);
int api_body(const qb200_lattice *l, int fam, bool ach, int isPlus, int cb, const void *psi, const void *chi,
             const void *gauge, const void *clov, void *out, const unsigned *accumulate, double coeff_s,
             double coeff_t_f, double coeff_t_b, unsigned tbc_mask, const double *tbc_phases, double alpha,
             double mu, double muinv, double rho, void *stream);
} // namespace qb200

using namespace qb200;

namespace {

int cuda_rc(cudaError_t e, const char *what)
{
  if (e == cudaSuccess) return QB200_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return api_fail(QB200_ECUDA, m.c_str());
}

int ft_bytes(int ft)
{
  return ft == QB200_F64 ? 8 : ft == QB200_F32 ? 4 : (ft == QB200_F16 || ft == QB200_F16N || ft == QB200_BF16) ? 2 : 0;
}

int grid_for(long long nv)
{
  long long b = (nv + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  return (int)(b < 1 ? 1 : b);
}

// ---- typed BLAS launches -------------------------------------------------

template <typename FT>
cudaError_t axpby_t(long long n, ScalarRef a, const void *x, ScalarRef b, void *y, cudaStream_t st)
{
  const long long nv = n / vec16<FT>::n;
  axpby_kernel<FT><<<grid_for(nv), 256, 0, st>>>(nv, a, (const FT *)x, b, (FT *)y);
  return cudaGetLastError();
}

cudaError_t axpby(int ft, long long n, ScalarRef a, const void *x, ScalarRef b, void *y, cudaStream_t st)
{
  switch (ft) {
  case QB200_F32: return axpby_t<float>(n, a, x, b, y, st);
  case QB200_F64: return axpby_t<double>(n, a, x, b, y, st);
  case QB200_BF16: return axpby_t<__nv_bfloat16>(n, a, x, b, y, st);
  default: return axpby_t<__half>(n, a, x, b, y, st);
  }
}

ScalarRef host(double v)
{
  ScalarRef s;
  s.host = v;
  s.num = nullptr;
  s.den = nullptr;
  s.sign = 1.0;
  return s;
}

ScalarRef ratio(const double *num, const double *den, double sign)
{
  ScalarRef s;
  s.host = 0.0;
  s.num = num;
  s.den = den;
  s.sign = sign;
  return s;
}

template <typename FO, typename FI>
cudaError_t convert_t(long long n, double scale, const void *in, void *out, cudaStream_t st)
{
  convert_kernel<FO, FI><<<grid_for(n), 256, 0, st>>>(n, scale, (const FI *)in, (FO *)out);
  return cudaGetLastError();
}

template <typename FO>
cudaError_t convert_from(int ft_in, long long n, double scale, const void *in, void *out, cudaStream_t st)
{
  switch (ft_in) {
  case QB200_F32: return convert_t<FO, float>(n, scale, in, out, st);
  case QB200_F64: return convert_t<FO, double>(n, scale, in, out, st);
  case QB200_BF16: return convert_t<FO, __nv_bfloat16>(n, scale, in, out, st);
  default: return convert_t<FO, __half>(n, scale, in, out, st);
  }
}

cudaError_t convert(int ft_out, void *out, int ft_in, const void *in, long long n, double scale, cudaStream_t st)
{
  switch (ft_out) {
  case QB200_F32: return convert_from<float>(ft_in, n, scale, in, out, st);
  case QB200_F64: return convert_from<double>(ft_in, n, scale, in, out, st);
  case QB200_BF16: return convert_from<__nv_bfloat16>(ft_in, n, scale, in, out, st);
  default: return convert_from<__half>(ft_in, n, scale, in, out, st);
  }
}

template <typename FT>
cudaError_t dot_t(long long n, const void *x, const void *y, double *partials, double *result, cudaStream_t st)
{
  const long long nv = n / vec16<FT>::n;
  dot_partial_kernel<FT><<<kRedBlocks, kRedThreads, 0, st>>>(nv, (const FT *)x, (const FT *)y, partials);
  finish_kernel<<<1, kRedThreads, 0, st>>>(partials, kRedBlocks, 1, result);
  return cudaGetLastError();
}

// real dot (x == y: norm squared) with the result written to result_dev
cudaError_t dot(int ft, long long n, const void *x, const void *y, double *partials, double *result,
                cudaStream_t st)
{
  switch (ft) {
  case QB200_F32: return dot_t<float>(n, x, y, partials, result, st);
  case QB200_F64: return dot_t<double>(n, x, y, partials, result, st);
  case QB200_BF16: return dot_t<__nv_bfloat16>(n, x, y, partials, result, st);
  default: return dot_t<__half>(n, x, y, partials, result, st);
  }
}

template <typename FT, int S>
cudaError_t cdot_ts(long long n, const void *x, const void *y, double *partials, double *result, cudaStream_t st)
{
  cdot_partial_kernel<FT, S><<<kRedBlocks, kRedThreads, 0, st>>>(n / 2, (const FT *)x, (const FT *)y, partials);
  finish_kernel<<<1, kRedThreads, 0, st>>>(partials, kRedBlocks, 2, result);
  return cudaGetLastError();
}

template <typename FT>
cudaError_t cdot_t(int soalen, long long n, const void *x, const void *y, double *partials, double *result,
                   cudaStream_t st)
{
  switch (soalen) {
  case 1: return cdot_ts<FT, 1>(n, x, y, partials, result, st);
  case 2: return cdot_ts<FT, 2>(n, x, y, partials, result, st);
  case 4: return cdot_ts<FT, 4>(n, x, y, partials, result, st);
  case 8: return cdot_ts<FT, 8>(n, x, y, partials, result, st);
  default: return cdot_ts<FT, 16>(n, x, y, partials, result, st);
  }
}

cudaError_t cdot(int ft, int soalen, long long n, const void *x, const void *y, double *partials, double *result,
                 cudaStream_t st)
{
  switch (ft) {
  case QB200_F32: return cdot_t<float>(soalen, n, x, y, partials, result, st);
  case QB200_F64: return cdot_t<double>(soalen, n, x, y, partials, result, st);
  case QB200_BF16: return cdot_t<__nv_bfloat16>(soalen, n, x, y, partials, result, st);
  default: return cdot_t<__half>(soalen, n, x, y, partials, result, st);
  }
}

// complex y = a x + b y on a spinor field (re/im S apart)
template <typename FT, int S>
__global__ void __launch_bounds__(256) caxpby_kernel(long long npairs, double ar, double ai,
                                                     const FT *__restrict__ x, double br, double bi,
                                                     FT *__restrict__ y)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npairs;
       i += (long long)gridDim.x * blockDim.x) {
    const long long g = i / S;
    const long long e = g * 2 * S + (i - g * S);
    const double xr = to_d(x[e]), xi = to_d(x[e + S]);
    const double yr = to_d(y[e]), yi = to_d(y[e + S]);
    y[e] = from_d<FT>(ar * xr - ai * xi + br * yr - bi * yi);
    y[e + S] = from_d<FT>(ar * xi + ai * xr + br * yi + bi * yr);
  }
}

template <typename FT>
cudaError_t caxpby_t(int soalen, long long n, double ar, double ai, const void *x, double br, double bi, void *y,
                     cudaStream_t st)
{
  const long long np = n / 2;
  const int gr = grid_for(np);
  switch (soalen) {
  case 1: caxpby_kernel<FT, 1><<<gr, 256, 0, st>>>(np, ar, ai, (const FT *)x, br, bi, (FT *)y); break;
  case 2: caxpby_kernel<FT, 2><<<gr, 256, 0, st>>>(np, ar, ai, (const FT *)x, br, bi, (FT *)y); break;
  case 4: caxpby_kernel<FT, 4><<<gr, 256, 0, st>>>(np, ar, ai, (const FT *)x, br, bi, (FT *)y); break;
  case 8: caxpby_kernel<FT, 8><<<gr, 256, 0, st>>>(np, ar, ai, (const FT *)x, br, bi, (FT *)y); break;
  default: caxpby_kernel<FT, 16><<<gr, 256, 0, st>>>(np, ar, ai, (const FT *)x, br, bi, (FT *)y); break;
  }
  return cudaGetLastError();
}

cudaError_t caxpby(int ft, int soalen, long long n, double ar, double ai, const void *x, double br, double bi,
                   void *y, cudaStream_t st)
{
  switch (ft) {
  case QB200_F32: return caxpby_t<float>(soalen, n, ar, ai, x, br, bi, y, st);
  case QB200_F64: return caxpby_t<double>(soalen, n, ar, ai, x, br, bi, y, st);
  case QB200_BF16: return caxpby_t<__nv_bfloat16>(soalen, n, ar, ai, x, br, bi, y, st);
  default: return caxpby_t<__half>(soalen, n, ar, ai, x, br, bi, y, st);
  }
}

// ---- vector spaces: a storage type on a lattice ----------------------------
// F16N spinors carry per-site norms, so their BLAS works per site lane and
// needs SOALEN; every other type is handled element-wise.

struct VS {
  int ft, S;
  long long n; // storage elements of one spinor array
  long long site_lanes() const { return n / (26LL * S) * S; }
};

VS vs_of(const qb200_lattice *l)
{
  VS v;
  v.ft = l->ftype;
  v.S = l->soalen;
  v.n = qb200_spinor_elems(l);
  return v;
}

#define QB_F16N_S(S, CALL)                                                                                        \
  switch (S) {                                                                                                    \
  case 4: { constexpr int SS = 4; CALL; } break;                                                                  \
  case 8: { constexpr int SS = 8; CALL; } break;                                                                  \
  default: { constexpr int SS = 16; CALL; } break;                                                                \
  }

cudaError_t axpby(const VS &v, ScalarRef a, const void *x, ScalarRef b, void *y, cudaStream_t st)
{
  if (v.ft != QB200_F16N) return axpby(v.ft, v.n, a, x, b, y, st);
  const long long nsl = v.site_lanes();
  if ((((uintptr_t)x | (uintptr_t)y) % 16) == 0) {
    // warp tiles of 32 sites, 8 per block of 256 threads
    const long long nblk = nsl / v.S, ntile = (nsl + 31) / 32;
    const int grid = (int)std::min<long long>((ntile + 7) / 8, 148LL * 16);
    QB_F16N_S(v.S, (axpby_f16n_tile_kernel<SS><<<grid, 256, 0, st>>>(nblk, a, (const __half *)x, b, (__half *)y)));
    return cudaGetLastError();
  }
  QB_F16N_S(v.S, (axpby_f16n_kernel<SS><<<grid_for(nsl), 256, 0, st>>>(nsl, a, (const __half *)x, b, (__half *)y)));
  return cudaGetLastError();
}

cudaError_t caxpby(const VS &v, double ar, double ai, const void *x, double br, double bi, void *y, cudaStream_t st)
{
  if (v.ft != QB200_F16N) return caxpby(v.ft, v.S, v.n, ar, ai, x, br, bi, y, st);
  const long long nsl = v.site_lanes();
  QB_F16N_S(v.S, (caxpby_f16n_kernel<SS><<<grid_for(nsl), 256, 0, st>>>(nsl, ar, ai, (const __half *)x, br, bi,
                                                                          (__half *)y)));
  return cudaGetLastError();
}

cudaError_t f16n_dot(const VS &v, bool cplx, const void *x, const void *y, double *partials, double *result,
                     cudaStream_t st)
{
  const long long nsl = v.site_lanes();
  if (!cplx && (((uintptr_t)x | (uintptr_t)y) % 16) == 0) {
    QB_F16N_S(v.S, (dot_f16n_tile_kernel<SS><<<kRedBlocks, kRedThreads, 0, st>>>(nsl / v.S, (const __half *)x,
                                                                                  (const __half *)y, partials)));
  } else if (cplx) {
    QB_F16N_S(v.S, (dot_f16n_partial_kernel<SS, true><<<kRedBlocks, kRedThreads, 0, st>>>(
                        nsl, (const __half *)x, (const __half *)y, partials)));
  } else {
    QB_F16N_S(v.S, (dot_f16n_partial_kernel<SS, false><<<kRedBlocks, kRedThreads, 0, st>>>(
                        nsl, (const __half *)x, (const __half *)y, partials)));
  }
  finish_kernel<<<1, kRedThreads, 0, st>>>(partials, kRedBlocks, cplx ? 2 : 1, result);
  return cudaGetLastError();
}

cudaError_t dot(const VS &v, const void *x, const void *y, double *partials, double *result, cudaStream_t st)
{
  if (v.ft != QB200_F16N) return dot(v.ft, v.n, x, y, partials, result, st);
  return f16n_dot(v, false, x, y, partials, result, st);
}

cudaError_t cdot(const VS &v, const void *x, const void *y, double *partials, double *result, cudaStream_t st)
{
  if (v.ft != QB200_F16N) return cdot(v.ft, v.S, v.n, x, y, partials, result, st);
  return f16n_dot(v, true, x, y, partials, result, st);
}

template <int S, bool TO>
cudaError_t conv_f16n(int ft_plain, long long nsl, double scale, const void *in, void *out, cudaStream_t st)
{
  const int gr = grid_for(nsl);
  switch (ft_plain) {
  case QB200_F32: convert_f16n_kernel<S, float, TO><<<gr, 256, 0, st>>>(nsl, scale, in, out); break;
  case QB200_F64: convert_f16n_kernel<S, double, TO><<<gr, 256, 0, st>>>(nsl, scale, in, out); break;
  case QB200_BF16: convert_f16n_kernel<S, __nv_bfloat16, TO><<<gr, 256, 0, st>>>(nsl, scale, in, out); break;
  default: convert_f16n_kernel<S, __half, TO><<<gr, 256, 0, st>>>(nsl, scale, in, out); break;
  }
  return cudaGetLastError();
}

// out = scale * in between two spinor arrays of the same lattice shape
cudaError_t convert(const VS &vo, void *out, const VS &vi, const void *in, double scale, cudaStream_t st)
{
  if (vo.ft != QB200_F16N && vi.ft != QB200_F16N) return convert(vo.ft, out, vi.ft, in, vi.n, scale, st);
  if (vo.ft == QB200_F16N && vi.ft == QB200_F16N) {
    // copy, then rescale per site (decode, scale, re-encode)
    cudaError_t e = cudaMemcpyAsync(out, in, vo.n * 2, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    return axpby(vo, host(0.0), in, host(scale), out, st);
  }
  if (vo.ft == QB200_F16N) {
    const long long nsl = vo.site_lanes();
    QB_F16N_S(vo.S, return (conv_f16n<SS, true>(vi.ft, nsl, scale, in, out, st)));
  } else {
    const long long nsl = vi.site_lanes();
    QB_F16N_S(vi.S, return (conv_f16n<SS, false>(vo.ft, nsl, scale, in, out, st)));
  }
  return cudaErrorInvalidValue;
}

// ---- the Schur operator ----------------------------------------------------

long long spinor_elems(const qb200_lattice *l) { return qb200_spinor_elems(l); }

// out = Mhat in (isPlus) or Mhat^dag in; tmp is a spinor of the other cb
int schur(const qb200_lattice *l, const qb200_operator *op, int isPlus, const void *in, void *out, void *tmp,
          cudaStream_t st)
{
  const int tc = op->target_cb, oc = 1 - tc;
  const double *ph = &op->tbc_phases[0][0];
  const void *clov_o = op->clov[oc], *clov_t = op->clov[tc];
  if (op->family == 3 && !isPlus) {
    clov_o = op->clov_dag[oc];
    clov_t = op->clov_dag[tc];
  }
  // tmp = A_ee^-1 (beta D_eo in); for Wilson the diagonal is alpha: scale beta by 1/alpha
  const double sc = op->family == 0 ? 1.0 / op->alpha : 1.0;
  int rc = api_body(l, op->family, false, isPlus, oc, in, nullptr, op->gauge[oc], clov_o, tmp, nullptr,
                    op->coeff_s * sc, op->coeff_t_f * sc, op->coeff_t_b * sc, op->tbc_mask, ph, op->alpha, op->mu,
                    op->muinv, op->rho, st);
  if (rc) return rc;
  // out = A_oo in - beta D_oe tmp
  return api_body(l, op->family, true, isPlus, tc, tmp, in, op->gauge[tc], clov_t, out, nullptr, op->coeff_s,
                  op->coeff_t_f, op->coeff_t_b, op->tbc_mask, ph, op->alpha, op->mu, op->muinv, op->rho, st);
}

int check_op(const qb200_lattice *l, const qb200_operator *op)
{
  if (!l || !op) return api_fail(QB200_ENULL, "lattice or operator is NULL");
  if (op->family < 0 || op->family > 3) return api_fail(QB200_EINVAL, "operator family must be 0..3");
  if (op->target_cb != 0 && op->target_cb != 1) return api_fail(QB200_EINVAL, "target_cb must be 0 or 1");
  if (!op->gauge[0] || !op->gauge[1]) return api_fail(QB200_ENULL, "both gauge checkerboards are needed");
  if ((op->family == 1 || op->family == 3) && (!op->clov[0] || !op->clov[1]))
    return api_fail(QB200_ENULL, "clover operator needs A (target cb) and A^-1 (other cb)");
  if (op->family == 3 && (!op->clov_dag[0] || !op->clov_dag[1]))
    return api_fail(QB200_ENULL, "twisted-mass clover operator needs the conjugate-transposed blocks for the dagger");
  if (op->family == 0 && op->alpha == 0.0) return api_fail(QB200_EINVAL, "Wilson operator needs alpha != 0");
  if (qb200_spinor_elems(l) < 0) return api_fail(QB200_EINVAL, "invalid lattice");
  return QB200_OK;
}

// workspace carving
struct Work {
  char *p;
  size_t off;
  void *take(size_t bytes)
  {
    off = (off + 255) & ~(size_t)255;
    void *r = p + off;
    off += bytes;
    return r;
  }
};

size_t spinor_bytes(const qb200_lattice *l) { return (size_t)qb200_spinor_elems(l) * ft_bytes(l->ftype); }

// nspin spinors + the reduction scratch + 32 device scalars
size_t ws_bytes(const qb200_lattice *l, int nspin)
{
  if (qb200_spinor_elems(l) < 0) return 0;
  return nspin * (spinor_bytes(l) + 256) + (kRedPartials + 32) * sizeof(double) + 1024;
}

constexpr int kMaxVecs = 12;

struct Vecs {
  void *v[kMaxVecs];
  double *partials, *scal;
};

// nspin <= kMaxVecs spinors, then the reduction scratch and the scalars
Vecs carve(const qb200_lattice *l, void *ws, int nspin)
{
  Work w{(char *)ws, 0};
  Vecs s;
  if (nspin > kMaxVecs) nspin = kMaxVecs;
  for (int i = 0; i < nspin; i++) s.v[i] = w.take(spinor_bytes(l));
  s.partials = (double *)w.take(kRedPartials * sizeof(double));
  s.scal = (double *)w.take(32 * sizeof(double));
  return s;
}

int fetch(double *h, const double *d, int n, cudaStream_t st)
{
  cudaError_t e = cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return cuda_rc(e, "reduction readback");
}

int copy(void *dst, const void *src, size_t bytes, cudaStream_t st)
{
  return cuda_rc(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st), "copy");
}

// A v = Mhat^dag Mhat v
int normal_op(const qb200_lattice *l, const qb200_operator *op, const void *v, void *Av, void *t, void *tmp,
              cudaStream_t st)
{
  int rc = schur(l, op, 1, v, t, tmp, st);
  if (rc) return rc;
  return schur(l, op, 0, t, Av, tmp, st);
}

// CG on A = Mhat^dag Mhat: A x = rhs, x holds the initial guess.
// ws: 5 spinors (r, p, Ap, t, tmp) + scratch.  Scalars stay on the device
// (alpha = rr/pAp and beta = rr_new/rr are formed inside the axpby
// kernels); the host reads |r|^2 once per iteration for the stopping test.
int cg_core(const qb200_lattice *l, const qb200_operator *op, const void *rhs, void *x, double tol, int max_iter,
            const Vecs &s, int *iters, double *rel, cudaStream_t st, bool x_zero = false)
{
  const VS V = vs_of(l);
  void *r = s.v[0], *p = s.v[1], *Ap = s.v[2], *t = s.v[3], *tmp = s.v[4];
  double *rr_d = s.scal + 0, *rrn_d = s.scal + 1, *pAp_d = s.scal + 2, *bb_d = s.scal + 3;
  int rc;
  // r = rhs - A x (just rhs when the caller zeroed x)
  if (!x_zero && (rc = normal_op(l, op, x, Ap, t, tmp, st))) return rc;
  if ((rc = copy(r, rhs, spinor_bytes(l), st))) return rc;
  cudaError_t e = x_zero ? cudaSuccess : axpby(V, host(-1.0), Ap, host(1.0), r, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p, r, spinor_bytes(l), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = dot(V, r, r, s.partials, rr_d, st);
  if (e == cudaSuccess) e = dot(V, rhs, rhs, s.partials, bb_d, st);
  if ((rc = cuda_rc(e, "cg setup"))) return rc;
  double h[4];
  if ((rc = fetch(h, s.scal, 4, st))) return rc;
  const double bb = h[3];
  double rr = h[0];
  const double stop = tol * tol * bb;
  int k = 0;
  while (rr > stop && k < max_iter) {
    if ((rc = normal_op(l, op, p, Ap, t, tmp, st))) return rc;
    e = dot(V, p, Ap, s.partials, pAp_d, st);
    if (e == cudaSuccess) e = axpby(V, ratio(rr_d, pAp_d, 1.0), p, host(1.0), x, st);
    if (e == cudaSuccess) e = axpby(V, ratio(rr_d, pAp_d, -1.0), Ap, host(1.0), r, st);
    if (e == cudaSuccess) e = dot(V, r, r, s.partials, rrn_d, st);
    if (e == cudaSuccess) e = axpby(V, host(1.0), r, ratio(rrn_d, rr_d, 1.0), p, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rr_d, rrn_d, sizeof(double), cudaMemcpyDeviceToDevice, st);
    if ((rc = cuda_rc(e, "cg iteration"))) return rc;
    if ((rc = fetch(&rr, rr_d, 1, st))) return rc;
    k++;
    if (!std::isfinite(rr)) return api_fail(QB200_EINVAL, "cg: residual is not finite");
  }
  *iters = k;
  *rel = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  return QB200_OK;
}

// BiCGStab on Mhat x = b (x holds the initial guess).  ws: 7 spinors
// (r, r0, p, v, s, t, tmp) + scratch; complex scalars are formed on the host.
int bicgstab_core(const qb200_lattice *l, const qb200_operator *op, const void *b, void *x, double tol, int max_iter,
                  const Vecs &w, int *iters, double *rel, cudaStream_t st)
{
  const VS V = vs_of(l);
  void *r = w.v[0], *r0 = w.v[1], *p = w.v[2], *v = w.v[3], *sv = w.v[4], *t = w.v[5], *tmp = w.v[6];
  double *d = w.scal;
  int rc;
  if ((rc = schur(l, op, 1, x, v, tmp, st))) return rc;
  if ((rc = copy(r, b, spinor_bytes(l), st))) return rc;
  cudaError_t e = axpby(V, host(-1.0), v, host(1.0), r, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(r0, r, spinor_bytes(l), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, spinor_bytes(l), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(v, 0, spinor_bytes(l), st);
  if (e == cudaSuccess) e = dot(V, b, b, w.partials, d + 0, st);
  if (e == cudaSuccess) e = dot(V, r, r, w.partials, d + 1, st);
  if ((rc = cuda_rc(e, "bicgstab setup"))) return rc;
  double h[2];
  if ((rc = fetch(h, d, 2, st))) return rc;
  const double bb = h[0];
  double rr = h[1];
  const double stop = tol * tol * bb;
  double rho_r = 1, rho_i = 0, al_r = 1, al_i = 0, om_r = 1, om_i = 0;
  int k = 0;
  while (rr > stop && k < max_iter) {
    // rho_new = <r0, r>
    if ((e = cdot(V, r0, r, w.partials, d + 2, st)) != cudaSuccess) return cuda_rc(e, "bicgstab");
    double c[2];
    if ((rc = fetch(c, d + 2, 2, st))) return rc;
    // beta = (rho_new / rho) (alpha / omega)
    const double den1 = rho_r * rho_r + rho_i * rho_i, den2 = om_r * om_r + om_i * om_i;
    if (den1 == 0 || den2 == 0) return api_fail(QB200_EINVAL, "bicgstab breakdown");
    const double q_r = (c[0] * rho_r + c[1] * rho_i) / den1, q_i = (c[1] * rho_r - c[0] * rho_i) / den1;
    const double a_r = (al_r * om_r + al_i * om_i) / den2, a_i = (al_i * om_r - al_r * om_i) / den2;
    const double be_r = q_r * a_r - q_i * a_i, be_i = q_r * a_i + q_i * a_r;
    rho_r = c[0];
    rho_i = c[1];
    // p = r + beta (p - omega v)
    e = caxpby(V, -om_r, -om_i, v, 1.0, 0.0, p, st);
    if (e == cudaSuccess) e = caxpby(V, 1.0, 0.0, r, be_r, be_i, p, st);
    if ((rc = cuda_rc(e, "bicgstab p"))) return rc;
    if ((rc = schur(l, op, 1, p, v, tmp, st))) return rc;
    if ((e = cdot(V, r0, v, w.partials, d + 4, st)) != cudaSuccess) return cuda_rc(e, "bicgstab");
    if ((rc = fetch(c, d + 4, 2, st))) return rc;
    const double dd = c[0] * c[0] + c[1] * c[1];
    if (dd == 0) return api_fail(QB200_EINVAL, "bicgstab breakdown");
    al_r = (rho_r * c[0] + rho_i * c[1]) / dd;
    al_i = (rho_i * c[0] - rho_r * c[1]) / dd;
    // s = r - alpha v
    if ((rc = copy(sv, r, spinor_bytes(l), st))) return rc;
    if ((e = caxpby(V, -al_r, -al_i, v, 1.0, 0.0, sv, st)) != cudaSuccess) return cuda_rc(e, "bicgstab");
    if ((rc = schur(l, op, 1, sv, t, tmp, st))) return rc;
    // omega = <t, s> / <t, t>
    e = cdot(V, t, sv, w.partials, d + 6, st);
    if (e == cudaSuccess) e = dot(V, t, t, w.partials, d + 8, st);
    if ((rc = cuda_rc(e, "bicgstab omega"))) return rc;
    double o[3];
    if ((rc = fetch(o, d + 6, 3, st))) return rc;
    if (o[2] == 0) {
      om_r = 0;
      om_i = 0;
    } else {
      om_r = o[0] / o[2];
      om_i = o[1] / o[2];
    }
    // x += alpha p + omega s ; r = s - omega t
    e = caxpby(V, al_r, al_i, p, 1.0, 0.0, x, st);
    if (e == cudaSuccess) e = caxpby(V, om_r, om_i, sv, 1.0, 0.0, x, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r, sv, spinor_bytes(l), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = caxpby(V, -om_r, -om_i, t, 1.0, 0.0, r, st);
    if (e == cudaSuccess) e = dot(V, r, r, w.partials, d + 1, st);
    if ((rc = cuda_rc(e, "bicgstab update"))) return rc;
    if ((rc = fetch(&rr, d + 1, 1, st))) return rc;
    k++;
    if (!std::isfinite(rr)) return api_fail(QB200_EINVAL, "bicgstab: residual is not finite");
  }
  *iters = k;
  *rel = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  return QB200_OK;
}

// |b - Mhat x| / |b| in the precision of the lattice; ws needs 3 spinors + scratch
int true_residual(const qb200_lattice *l, const qb200_operator *op, const void *b, const void *x, void *r,
                  void *tmp, double *partials, double *scal, double *rel, cudaStream_t st)
{
  const VS V = vs_of(l);
  int rc = schur(l, op, 1, x, r, tmp, st);
  if (rc) return rc;
  cudaError_t e = axpby(V, host(1.0), b, host(-1.0), r, st);
  if (e == cudaSuccess) e = dot(V, r, r, partials, scal, st);
  if (e == cudaSuccess) e = dot(V, b, b, partials, scal + 1, st);
  if ((rc = cuda_rc(e, "true residual"))) return rc;
  double h[2];
  if ((rc = fetch(h, scal, 2, st))) return rc;
  *rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
  return QB200_OK;
}

// |b - Mhat^dag Mhat x| / |b|; r, t, tmp: scratch spinors
int true_residual_normal(const qb200_lattice *l, const qb200_operator *op, const void *b, const void *x, void *r,
                         void *t, void *tmp, double *partials, double *scal, double *rel, cudaStream_t st)
{
  const VS V = vs_of(l);
  int rc = normal_op(l, op, x, r, t, tmp, st);
  if (rc) return rc;
  cudaError_t e = axpby(V, host(1.0), b, host(-1.0), r, st);
  if (e == cudaSuccess) e = dot(V, r, r, partials, scal, st);
  if (e == cudaSuccess) e = dot(V, b, b, partials, scal + 1, st);
  if ((rc = cuda_rc(e, "true residual"))) return rc;
  double h[2];
  if ((rc = fetch(h, scal, 2, st))) return rc;
  *rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
  return QB200_OK;
}

bool same_shape(const qb200_lattice *a, const qb200_lattice *b)
{
  return a->nx == b->nx && a->ny == b->ny && a->nz == b->nz && a->nt == b->nt && a->soalen == b->soalen &&
         a->veclen == b->veclen && a->pad_xy == b->pad_xy && a->pad_xyz == b->pad_xyz;
}

} // namespace

extern "C" {

long long qb200_blas_partials_len(void) { return kRedPartials; }

int qb200_blas_axpby(int ftype, long long n, double a, const void *x, double b, void *y, void *stream)
{
  if (!ft_bytes(ftype) || ftype == QB200_F16N)
    return api_fail(QB200_ELAYOUT, "unknown storage type (F16N spinors: use the lattice-aware solver entry points)");
  if (!x || !y) return api_fail(QB200_ENULL, "x and y must be non-NULL");
  if (n % 8) return api_fail(QB200_EINVAL, "n must be a multiple of 8");
  return cuda_rc(axpby(ftype, n, host(a), x, host(b), y, (cudaStream_t)stream), "axpby");
}

int qb200_blas_convert(int ft_out, void *out, int ft_in, const void *in, long long n, double scale, void *stream)
{
  if (!ft_bytes(ft_out) || !ft_bytes(ft_in) || ft_out == QB200_F16N || ft_in == QB200_F16N)
    return api_fail(QB200_ELAYOUT, "unknown storage type (F16N spinors: use qb200_spinor_convert)");
  if (!in || !out) return api_fail(QB200_ENULL, "in and out must be non-NULL");
  return cuda_rc(convert(ft_out, out, ft_in, in, n, scale, (cudaStream_t)stream), "convert");
}

int qb200_blas_dot(int ftype, long long n, const void *x, const void *y, double *result, double *partials,
                   void *stream)
{
  if (!ft_bytes(ftype) || ftype == QB200_F16N)
    return api_fail(QB200_ELAYOUT, "unknown storage type (F16N spinors: use the lattice-aware solver entry points)");
  if (!x || !y || !result || !partials) return api_fail(QB200_ENULL, "x, y, result and partials must be non-NULL");
  if (n % 8) return api_fail(QB200_EINVAL, "n must be a multiple of 8");
  return cuda_rc(dot(ftype, n, x, y, partials, result, (cudaStream_t)stream), "dot");
}

int qb200_blas_cdot(const qb200_lattice *lat, const void *x, const void *y, double *result, double *partials,
                    void *stream)
{
  const long long n = qb200_spinor_elems(lat);
  if (n < 0) return api_fail(QB200_EINVAL, "invalid lattice");
  if (!x || !y || !result || !partials) return api_fail(QB200_ENULL, "x, y, result and partials must be non-NULL");
  return cuda_rc(cdot(vs_of(lat), x, y, partials, result, (cudaStream_t)stream), "cdot");
}

int qb200_spinor_convert(const qb200_lattice *lat_out, void *out, const qb200_lattice *lat_in, const void *in,
                         double scale, void *stream)
{
  if (qb200_spinor_elems(lat_out) < 0 || qb200_spinor_elems(lat_in) < 0)
    return api_fail(QB200_EINVAL, "invalid lattice");
  if (!same_shape(lat_out, lat_in)) return api_fail(QB200_EINVAL, "lattices differ in shape");
  if (!in || !out) return api_fail(QB200_ENULL, "in and out must be non-NULL");
  return cuda_rc(convert(vs_of(lat_out), out, vs_of(lat_in), in, scale, (cudaStream_t)stream), "spinor convert");
}

int qb200_schur_apply(const qb200_lattice *lat, const qb200_operator *op, int isign, const void *in, void *out,
                      void *tmp_other_cb, void *stream)
{
  int rc = check_op(lat, op);
  if (rc) return rc;
  if (!in || !out || !tmp_other_cb) return api_fail(QB200_ENULL, "in, out and tmp must be non-NULL");
  if (in == out) return api_fail(QB200_EINVAL, "out must not alias in");
  return schur(lat, op, isign > 0, in, out, tmp_other_cb, (cudaStream_t)stream);
}

// ---- allocation-free operator application -----------------------------
//
// Device scratch of qb200_schur_apply_noalloc: the intermediate spinor on the
// other checkerboard.  It is a module global, so every GPU that loads the
// library holds these bytes until the process exits, and every call shares
// them: calls whose work overlaps on the GPU (different streams, different
// host threads) race on this one buffer.  Nothing in it has to start at zero:
// the first kernel of each call writes every site of the intermediate before
// the second kernel reads it, and padding blocks are never read.
static __device__ __align__(256) unsigned char g_noalloc_scratch[QB200_NOALLOC_SCRATCH_BYTES];

namespace {
// device address of g_noalloc_scratch, looked up once per device (with that
// device current) by the first call made on it.  The address is kept for the
// life of the process: after cudaDeviceReset (or any teardown of the
// device's primary context) it would name freed memory, so the entry point
// must not be used across a device reset.
void *noalloc_scratch(int *rc)
{
  static std::mutex mu;
  static void *addr[128] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 128) {
    *rc = cuda_rc(e == cudaSuccess ? cudaErrorInvalidDevice : e, "no-alloc scratch: current device");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      *rc = cuda_rc(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "no-alloc scratch: cudaGetSymbolAddress");
      return nullptr;
    }
    addr[dev] = p;
  }
  *rc = QB200_OK;
  return addr[dev];
}
} // namespace

int qb200_schur_apply_noalloc(const qb200_lattice *lat, const qb200_operator *op, int isign, const void *in,
                              void *out, void *stream)
{
  int rc = check_op(lat, op);
  if (rc) return rc;
  if (!in || !out) return api_fail(QB200_ENULL, "in and out must be non-NULL");
  if (in == out) return api_fail(QB200_EINVAL, "out must not alias in");
  const size_t need = spinor_bytes(lat);
  if (need > (size_t)QB200_NOALLOC_SCRATCH_BYTES) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "qb200_schur_apply_noalloc: the lattice needs %zu bytes of scratch for one spinor, more than "
                  "the %d bytes built into the library; use qb200_schur_apply with a caller buffer",
                  need, (int)QB200_NOALLOC_SCRATCH_BYTES);
    return api_fail(QB200_EINVAL, msg);
  }
  void *tmp = noalloc_scratch(&rc);
  if (!tmp) return rc;
  return schur(lat, op, isign > 0, in, out, tmp, (cudaStream_t)stream);
}

long long qb200_cg_workspace_bytes(const qb200_lattice *lat) { return (long long)ws_bytes(lat, 6); }
long long qb200_bicgstab_workspace_bytes(const qb200_lattice *lat) { return (long long)ws_bytes(lat, 7); }
long long qb200_mixed_workspace_bytes(const qb200_lattice *lat_hi, const qb200_lattice *lat_lo,
                                      long long *lo_bytes)
{
  if (lo_bytes) *lo_bytes = (long long)ws_bytes(lat_lo, 9);
  return (long long)ws_bytes(lat_hi, 4);
}

int qb200_invert_cg(const qb200_lattice *lat, const qb200_operator *op, const void *b, void *x, double rel_tol,
                    int max_iter, void *workspace, int *iters, double *rel_res, void *stream)
{
  int rc = check_op(lat, op);
  if (rc) return rc;
  if (!b || !x || !workspace) return api_fail(QB200_ENULL, "b, x and workspace must be non-NULL");
  cudaStream_t st = (cudaStream_t)stream;
  Vecs s = carve(lat, workspace, 6);
  void *rhs = s.v[5];
  // normal equations: rhs = Mhat^dag b
  if ((rc = schur(lat, op, 0, b, rhs, s.v[4], st))) return rc;
  int k = 0;
  double rel = 0.0;
  if ((rc = cg_core(lat, op, rhs, x, rel_tol, max_iter, s, &k, &rel, st))) return rc;
  if (iters) *iters = k;
  double tr = 0.0;
  if ((rc = true_residual(lat, op, b, x, s.v[0], s.v[4], s.partials, s.scal + 10, &tr, st))) return rc;
  if (rel_res) *rel_res = tr;
  return QB200_OK;
}

int qb200_invert_cg_normal(const qb200_lattice *lat, const qb200_operator *op, const void *b, void *x,
                           double rel_tol, int max_iter, void *workspace, int *iters, double *rel_res, void *stream)
{
  int rc = check_op(lat, op);
  if (rc) return rc;
  if (!b || !x || !workspace) return api_fail(QB200_ENULL, "b, x and workspace must be non-NULL");
  cudaStream_t st = (cudaStream_t)stream;
  Vecs s = carve(lat, workspace, 6);
  int k = 0;
  double rel = 0.0;
  if ((rc = cg_core(lat, op, b, x, rel_tol, max_iter, s, &k, &rel, st))) return rc;
  if (iters) *iters = k;
  double tr = 0.0;
  if ((rc = true_residual_normal(lat, op, b, x, s.v[0], s.v[3], s.v[4], s.partials, s.scal + 10, &tr, st)))
    return rc;
  if (rel_res) *rel_res = tr;
  return QB200_OK;
}

int qb200_invert_bicgstab(const qb200_lattice *lat, const qb200_operator *op, const void *b, void *x,
                          double rel_tol, int max_iter, void *workspace, int *iters, double *rel_res, void *stream)
{
  int rc = check_op(lat, op);
  if (rc) return rc;
  if (!b || !x || !workspace) return api_fail(QB200_ENULL, "b, x and workspace must be non-NULL");
  cudaStream_t st = (cudaStream_t)stream;
  Vecs s = carve(lat, workspace, 7);
  int k = 0;
  double rel = 0.0;
  if ((rc = bicgstab_core(lat, op, b, x, rel_tol, max_iter, s, &k, &rel, st))) return rc;
  if (iters) *iters = k;
  double tr = 0.0;
  if ((rc = true_residual(lat, op, b, x, s.v[0], s.v[6], s.partials, s.scal + 10, &tr, st))) return rc;
  if (rel_res) *rel_res = tr;
  return QB200_OK;
}

// CG on the normal equations in the low precision with reliable updates:
// one Krylov space for the whole solve (no restarts).  Each segment starts
// from the FP64 residual r = b - Mhat x, its normal form rn = Mhat^dag r,
// scaled to O(1) components and demoted; the low-precision CG then iterates
// r_lo, p_lo and a low-precision increment x_lo.  When |r_lo| has fallen by
// the factor delta since the segment started (or far enough that the
// segment's FP64 residual, scaled by that fall, would meet rel_tol), x_lo is
// promoted and added to x in FP64, the FP64 residual is recomputed and
// replaces r_lo, and p_lo is rescaled to the new segment's units, so the
// search direction survives the update.
static int reliable_cg(const qb200_lattice *lat_hi, const qb200_operator *op_hi, const qb200_lattice *lat_lo,
                       const qb200_operator *op_lo, const void *b, void *x, double rel_tol, double delta,
                       int max_iter, int max_updates, const Vecs &H, const Vecs &L, int *iters, int *updates,
                       double *rel_out, cudaStream_t st)
{
  const VS VH = vs_of(lat_hi), VL = vs_of(lat_lo);
  const double ncomp = (double)VH.n;
  void *r = H.v[0], *rn = H.v[1], *e_hi = H.v[2], *tmp = H.v[3];
  void *rl = L.v[0], *p = L.v[1], *Ap = L.v[2], *t = L.v[3], *tl = L.v[4], *xl = L.v[8];
  double *d = L.scal;
  int rc;
  cudaError_t e;
  double rel = 1.0;
  if ((rc = true_residual(lat_hi, op_hi, b, x, r, tmp, H.partials, H.scal + 2, &rel, st))) return rc;
  int k = 0, nup = 0;
  double scale = 1.0, rr = 0.0, seg_rr = 0.0, seg_rel = rel;
  bool first = true;
  while (rel > rel_tol && k < max_iter) {
    // new segment from the FP64 residual r (x_lo = 0)
    if ((rc = schur(lat_hi, op_hi, 0, r, rn, tmp, st))) return rc;
    double rrh;
    e = dot(VH, rn, rn, H.partials, H.scal + 4, st);
    if ((rc = cuda_rc(e, "reliable cg norm"))) return rc;
    if ((rc = fetch(&rrh, H.scal + 4, 1, st))) return rc;
    const double s_new = std::sqrt(ncomp / (rrh > 0 ? rrh : 1.0));
    e = convert(VL, rl, VH, rn, s_new, st);
    if (e == cudaSuccess) e = first ? cudaMemcpyAsync(p, rl, spinor_bytes(lat_lo), cudaMemcpyDeviceToDevice, st)
                                    : axpby(VL, host(0.0), rl, host(s_new / scale), p, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(xl, 0, spinor_bytes(lat_lo), st);
    if (e == cudaSuccess) e = dot(VL, rl, rl, L.partials, d + 0, st);
    if ((rc = cuda_rc(e, "reliable cg segment"))) return rc;
    double rrs;
    if ((rc = fetch(&rrs, d + 0, 1, st))) return rc;
    if (!first) {
      // continue the recurrence in the new units: p = r + beta p
      const double beta = rrs / (rr * (s_new / scale) * (s_new / scale));
      e = axpby(VL, host(1.0), rl, host(beta), p, st);
      if ((rc = cuda_rc(e, "reliable cg direction"))) return rc;
    }
    scale = s_new;
    rr = seg_rr = rrs;
    seg_rel = rel;
    first = false;
    bool update = false;
    while (!update && k < max_iter) {
      if ((rc = normal_op(lat_lo, op_lo, p, Ap, t, tl, st))) return rc;
      e = dot(VL, p, Ap, L.partials, d + 1, st);
      if ((rc = cuda_rc(e, "reliable cg pAp"))) return rc;
      double pAp;
      if ((rc = fetch(&pAp, d + 1, 1, st))) return rc;
      const double alpha = rr / pAp;
      e = axpby(VL, host(alpha), p, host(1.0), xl, st);
      if (e == cudaSuccess) e = axpby(VL, host(-alpha), Ap, host(1.0), rl, st);
      if (e == cudaSuccess) e = dot(VL, rl, rl, L.partials, d + 2, st);
      if ((rc = cuda_rc(e, "reliable cg iteration"))) return rc;
      double rrn;
      if ((rc = fetch(&rrn, d + 2, 1, st))) return rc;
      k++;
      if (!std::isfinite(rrn) || !std::isfinite(alpha)) return api_fail(QB200_EINVAL, "cg: residual is not finite");
      update = rrn <= delta * delta * seg_rr || seg_rel * std::sqrt(rrn / seg_rr) <= rel_tol || k == max_iter;
      if (!update) {
        e = axpby(VL, host(1.0), rl, host(rrn / rr), p, st);
        if ((rc = cuda_rc(e, "reliable cg direction"))) return rc;
        rr = rrn;
      }
      // on an update rr keeps |r|^2 of the step before: the next direction's
      // beta divides the replaced residual's |r|^2 by it
    }
    // x += x_lo / scale in FP64, then the FP64 residual
    e = convert(VH, e_hi, VL, xl, 1.0 / scale, st);
    if (e == cudaSuccess) e = axpby(VH, host(1.0), e_hi, host(1.0), x, st);
    if ((rc = cuda_rc(e, "reliable cg update"))) return rc;
    if ((rc = true_residual(lat_hi, op_hi, b, x, r, tmp, H.partials, H.scal + 2, &rel, st))) return rc;
    if (++nup >= max_updates) break;
  }
  *iters = k;
  *updates = nup;
  *rel_out = rel;
  return QB200_OK;
}

// Defect correction: the true residual r = b - Mhat x is formed in the high
// precision (FP64 storage), the correction solved in the low precision
// (FP32 or FP16 storage, FP32 arithmetic) to inner_tol, and accumulated in
// high precision, until |r|/|b| <= rel_tol.  solver: 0 CG on the normal
// equations, 1 BiCGStab.  solver 2: CG on the normal equations with reliable
// updates (reliable_cg; inner_tol is the fall of the low-precision residual
// between FP64 updates, max_inner the iterations, max_outer the updates).
int qb200_invert_mixed(const qb200_lattice *lat_hi, const qb200_operator *op_hi, const qb200_lattice *lat_lo,
                       const qb200_operator *op_lo, int solver, const void *b, void *x, double rel_tol,
                       double inner_tol, int max_inner, int max_outer, void *ws_hi, void *ws_lo,
                       int *inner_iters, int *outer_iters, double *rel_res, void *stream)
{
  int rc = check_op(lat_hi, op_hi);
  if (rc) return rc;
  if ((rc = check_op(lat_lo, op_lo))) return rc;
  if (!same_shape(lat_hi, lat_lo)) return api_fail(QB200_EINVAL, "high and low precision lattices differ in shape");
  if (!b || !x || !ws_hi || !ws_lo) return api_fail(QB200_ENULL, "b, x and workspaces must be non-NULL");
  if (solver < 0 || solver > 2)
    return api_fail(QB200_EINVAL, "solver must be 0 (CG), 1 (BiCGStab) or 2 (CG with reliable updates)");
  if (solver == 2 && !(inner_tol > 0.0 && inner_tol < 1.0))
    return api_fail(QB200_EINVAL, "reliable updates need 0 < inner_tol < 1");
  cudaStream_t st = (cudaStream_t)stream;
  const VS VH = vs_of(lat_hi), VL = vs_of(lat_lo);
  const double ncomp = (double)VH.n; // components of one high-precision spinor array
  Vecs H = carve(lat_hi, ws_hi, 4);   // r, rn (normal residual), e, tmp
  Vecs L = carve(lat_lo, ws_lo, 9);   // solver vectors [0..6], rhs_lo [7], e_lo [8]
  void *r = H.v[0], *rn = H.v[1], *e_hi = H.v[2], *tmp = H.v[3];
  void *rhs_lo = L.v[7], *e_lo = L.v[8];
  cudaError_t e = cudaMemsetAsync(x, 0, spinor_bytes(lat_hi), st);
  if ((rc = cuda_rc(e, "mixed init"))) return rc;
  double bb;
  {
    e = dot(VH, b, b, H.partials, H.scal, st);
    if ((rc = cuda_rc(e, "mixed |b|"))) return rc;
    if ((rc = fetch(&bb, H.scal, 1, st))) return rc;
  }
  int tot = 0, outer = 0;
  double rel = 1.0;
  if (solver == 2) {
    if ((rc = reliable_cg(lat_hi, op_hi, lat_lo, op_lo, b, x, rel_tol, inner_tol, max_inner, max_outer, H, L, &tot,
                          &outer, &rel, st)))
      return rc;
    if (inner_iters) *inner_iters = tot;
    if (outer_iters) *outer_iters = outer;
    if (rel_res) *rel_res = rel;
    return QB200_OK;
  }
  while (outer < max_outer) {
    // r = b - Mhat x (high precision)
    if ((rc = true_residual(lat_hi, op_hi, b, x, r, tmp, H.partials, H.scal + 2, &rel, st))) return rc;
    if (rel <= rel_tol) break;
    const void *src = r;
    if (solver == 0) {
      // correction from the normal equations: Mhat^dag Mhat e = Mhat^dag r
      if ((rc = schur(lat_hi, op_hi, 0, r, rn, tmp, st))) return rc;
      src = rn;
    }
    double rr;
    e = dot(VH, src, src, H.partials, H.scal + 4, st);
    if ((rc = cuda_rc(e, "mixed norm"))) return rc;
    if ((rc = fetch(&rr, H.scal + 4, 1, st))) return rc;
    // scale the low-precision right-hand side to O(1) components
    const double scale = std::sqrt(ncomp / (rr > 0 ? rr : 1.0));
    e = convert(VL, rhs_lo, VH, src, scale, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(e_lo, 0, spinor_bytes(lat_lo), st);
    if ((rc = cuda_rc(e, "mixed demote"))) return rc;
    int k = 0;
    double irel = 0.0;
    if (solver == 0) rc = cg_core(lat_lo, op_lo, rhs_lo, e_lo, inner_tol, max_inner, L, &k, &irel, st, true);
    else rc = bicgstab_core(lat_lo, op_lo, rhs_lo, e_lo, inner_tol, max_inner, L, &k, &irel, st);
    if (rc) return rc;
    tot += k;
    // x += e / scale (high precision)
    e = convert(VH, e_hi, VL, e_lo, 1.0 / scale, st);
    if (e == cudaSuccess) e = axpby(VH, host(1.0), e_hi, host(1.0), x, st);
    if ((rc = cuda_rc(e, "mixed promote"))) return rc;
    outer++;
  }
  if (outer == max_outer) {
    if ((rc = true_residual(lat_hi, op_hi, b, x, r, tmp, H.partials, H.scal + 2, &rel, st))) return rc;
  }
  if (inner_iters) *inner_iters = tot;
  if (outer_iters) *outer_iters = outer;
  if (rel_res) *rel_res = rel;
  return QB200_OK;
}

} // extern "C"
