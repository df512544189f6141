// qb200_mrhs.cu -- multi-right-hand-side operator, layout converters and
// solvers.
//
// Layout: a multi-RHS spinor array holds nrhs fields of one checkerboard with
// the right-hand side innermost, FT[block][3][4][2][S][nrhs] (padding blocks
// as in the single layout).  One thread per (site, right-hand side) then reads
// spinors fully coalesced while the nrhs threads of a site share each link and
// clover load, so the gauge and clover bytes are paid once per nrhs solutions.
// The reference has no multi-RHS kernels; this is an addition of the B200
// build.  Storage types: FP32 and plain FP16; SOALEN 4, 8, 16.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "qphix_b200.h"
#include "qb200_blas.cuh"
#include "qb200_internal.h"

namespace qb200 {
int api_fail(int code, const char *msg);
int api_geo(const qb200_lattice *l, GeoDev &g);
int api_check_device();
int api_body(const qb200_lattice *l, int fam, bool ach, int isPlus, int cb, const void *psi, const void *chi,
             const void *gauge, const void *clov, void *out, const unsigned *accumulate, double coeff_s,
             double coeff_t_f, double coeff_t_b, unsigned tbc_mask, const double *tbc_phases, double alpha,
             double mu, double muinv, double rho, void *stream);
} // namespace qb200

using namespace qb200;

namespace {

constexpr int kMaxRhs = 16;

int cuda_rc(cudaError_t e, const char *what)
{
  if (e == cudaSuccess) return QB200_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return api_fail(QB200_ECUDA, m.c_str());
}

int fbytes(int ft) { return ft == QB200_F64 ? 8 : ft == QB200_F32 ? 4 : 2; }

int grid_for(long long n)
{
  long long b = (n + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  return (int)(b < 1 ? 1 : b);
}

int check_mr(const qb200_lattice *l, int nrhs)
{
  if (!l) return api_fail(QB200_ENULL, "lattice is NULL");
  if (nrhs != 1 && nrhs != 2 && nrhs != 4 && nrhs != 8 && nrhs != 16)
    return api_fail(QB200_EINVAL, "nrhs must be 1, 2, 4, 8 or 16");
  if (l->ftype != QB200_F32 && l->ftype != QB200_F16)
    return api_fail(QB200_ELAYOUT, "multi-RHS kernels are built for FP32 and FP16 storage");
  if (l->soalen != 4 && l->soalen != 8 && l->soalen != 16)
    return api_fail(QB200_ELAYOUT, "multi-RHS kernels are built for soalen 4, 8 and 16");
  GeoDev g;
  return api_geo(l, g);
}

// ---- dslash --------------------------------------------------------------

template <typename FT>
cudaError_t mr_body_t(const qb200_lattice *l, GeoDev g, int fam, bool ach, int isPlus, int cb, const void *psi,
                      const void *chi, void *out, const void *gauge, const void *clov, const qb200_coeffs *c,
                      const unsigned *acc, cudaStream_t st)
{
  typedef comp_t<FT> C;
  OpDev<C> p;
  std::memset(&p, 0, sizeof(p));
  const double sg = ach ? -1.0 : 1.0;
  for (int d = 0; d < 6; d++) p.beta[d] = (C)(sg * c->coeff_s);
  p.beta[6] = (C)(sg * c->coeff_t_b);
  p.beta[7] = (C)(sg * c->coeff_t_f);
  p.tbound = (C)l->t_boundary;
  p.t_edge_lo = l->t_edge_lo ? 1 : 0;
  p.t_edge_hi = l->t_edge_hi ? 1 : 0;
  p.tbc_mask = c->tbc_mask & 15u;
  for (int m = 0; m < 4; m++) {
    p.tbc[m][0] = (C)c->tbc_phases[m][0];
    p.tbc[m][1] = (C)c->tbc_phases[m][1];
  }
  for (int d = 0; d < 8; d++)
    if (!acc || acc[d]) p.acc_mask |= 1u << d;
  p.isPlus = isPlus;
  p.cb = cb;
  p.alpha = (C)c->alpha;
  p.mu = (C)c->mu;
  p.muinv = (C)c->muinv;
  p.rho = (C)c->rho;
  LaunchSpec ls;
  ls.fam = fam;
  ls.ach = ach;
  ls.comp12 = l->compress12 != 0;
  typedef elem_t<FT> E;
  const E *ps = (const E *)psi, *ch = (const E *)chi, *u = (const E *)gauge, *cl = (const E *)clov;
  E *o = (E *)out;
  switch (l->soalen) {
  case 4: return launch_dslash_mrhs<FT, 4>(ls, ps, ch, u, cl, o, g, p, st);
  case 8: return launch_dslash_mrhs<FT, 8>(ls, ps, ch, u, cl, o, g, p, st);
  default: return launch_dslash_mrhs<FT, 16>(ls, ps, ch, u, cl, o, g, p, st);
  }
}

int mr_body(const qb200_lattice *l, int nrhs, int fam, bool ach, int isPlus, int cb, const void *psi,
            const void *chi, void *out, const void *gauge, const void *clov, const qb200_coeffs *c,
            const unsigned *acc, cudaStream_t st)
{
  int rc = check_mr(l, nrhs);
  if (rc) return rc;
  if (fam < 0 || fam > 3) return api_fail(QB200_EINVAL, "family must be 0..3");
  if (cb != 0 && cb != 1) return api_fail(QB200_EINVAL, "cb must be 0 or 1");
  if (!psi || !out || !gauge || !c) return api_fail(QB200_ENULL, "psi, out, gauge and coefficients are required");
  if (ach && !chi) return api_fail(QB200_ENULL, "achimbdpsi needs chi");
  if ((fam == 1 || fam == 3) && !clov) return api_fail(QB200_ENULL, "clover field is NULL");
  if (psi == out) return api_fail(QB200_EINVAL, "out must not alias psi");
  if ((rc = api_check_device())) return rc;
  GeoDev g;
  api_geo(l, g);
  g.nrhs = nrhs;
  cudaError_t e = l->ftype == QB200_F32
                      ? mr_body_t<float>(l, g, fam, ach, isPlus, cb, psi, chi, out, gauge, clov, c, acc, st)
                      : mr_body_t<__half>(l, g, fam, ach, isPlus, cb, psi, chi, out, gauge, clov, c, acc, st);
  return cuda_rc(e, "multi-RHS dslash launch");
}

// ---- layout converters ----------------------------------------------------

struct PtrTab {
  const void *p[kMaxRhs];
  double scale[kMaxRhs];
};

// mrhs[blk][k][l][r] <-> field_r[blk][k][l] with conversion and scaling
template <typename FO, typename FI, bool TO_MR>
__global__ void __launch_bounds__(256) mr_convert_kernel(long long n, int S, int nrhs, PtrTab tab, void *mr)
{
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % nrhs);
    const long long j = e / nrhs; // element of one single-RHS field
    if (TO_MR) {
      const FI *src = reinterpret_cast<const FI *>(tab.p[r]);
      reinterpret_cast<FO *>(mr)[e] = from_d<FO>(tab.scale[r] * to_d(src[j]));
    } else {
      FO *dst = reinterpret_cast<FO *>(const_cast<void *>(tab.p[r]));
      dst[j] = from_d<FO>(tab.scale[r] * to_d(reinterpret_cast<const FI *>(mr)[e]));
    }
  }
  (void)S;
}

template <typename FO, typename FI>
cudaError_t mr_convert_t(bool to_mr, long long n, int S, int nrhs, const PtrTab &tab, void *mr, cudaStream_t st)
{
  if (to_mr) mr_convert_kernel<FO, FI, true><<<grid_for(n), 256, 0, st>>>(n, S, nrhs, tab, mr);
  else mr_convert_kernel<FO, FI, false><<<grid_for(n), 256, 0, st>>>(n, S, nrhs, tab, mr);
  return cudaGetLastError();
}

// single-layout fields of type ft_single <-> multi-RHS array of type ft_mr
cudaError_t mr_convert(bool to_mr, int ft_mr, int ft_single, long long n_total, int S, int nrhs, const PtrTab &tab,
                       void *mr, cudaStream_t st)
{
  // to_mr: FO = mr type, FI = single type; else FO = single type, FI = mr type
  const int fo = to_mr ? ft_mr : ft_single, fi = to_mr ? ft_single : ft_mr;
#define QB_CV(A, B) return mr_convert_t<A, B>(to_mr, n_total, S, nrhs, tab, mr, st)
  if (fo == QB200_F32 && fi == QB200_F32) QB_CV(float, float);
  if (fo == QB200_F32 && fi == QB200_F64) QB_CV(float, double);
  if (fo == QB200_F64 && fi == QB200_F32) QB_CV(double, float);
  if (fo == QB200_F16 && fi == QB200_F16) QB_CV(__half, __half);
  if (fo == QB200_F16 && fi == QB200_F64) QB_CV(__half, double);
  if (fo == QB200_F64 && fi == QB200_F16) QB_CV(double, __half);
  if (fo == QB200_F16 && fi == QB200_F32) QB_CV(__half, float);
  if (fo == QB200_F32 && fi == QB200_F16) QB_CV(float, __half);
#undef QB_CV
  return cudaErrorInvalidValue;
}

// one single-layout field <-> slot `slot` of a multi-RHS array, with scaling
template <typename FO, typename FI, bool TO_MR>
__global__ void __launch_bounds__(256) mr_slot_kernel(long long n1, int nrhs, int slot, const void *__restrict__ in,
                                                      double scale, void *__restrict__ out)
{
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n1;
       j += (long long)gridDim.x * blockDim.x) {
    if (TO_MR)
      reinterpret_cast<FO *>(out)[j * nrhs + slot] = from_d<FO>(scale * to_d(reinterpret_cast<const FI *>(in)[j]));
    else
      reinterpret_cast<FO *>(out)[j] = from_d<FO>(scale * to_d(reinterpret_cast<const FI *>(in)[j * nrhs + slot]));
  }
}

// y[j] += scale * slot of a multi-RHS array (FP64 single-layout y)
template <typename FI>
__global__ void __launch_bounds__(256) mr_slot_add_kernel(long long n1, int nrhs, int slot, const FI *__restrict__ in,
                                                          double scale, double *__restrict__ y)
{
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n1;
       j += (long long)gridDim.x * blockDim.x)
    y[j] += scale * to_d(in[j * nrhs + slot]);
}

cudaError_t mr_slot_add(int ft_mr, long long n1, int nrhs, int slot, const void *in, double scale, void *y,
                        cudaStream_t st)
{
  const int gr = grid_for(n1);
  if (ft_mr == QB200_F32)
    mr_slot_add_kernel<float><<<gr, 256, 0, st>>>(n1, nrhs, slot, (const float *)in, scale, (double *)y);
  else mr_slot_add_kernel<__half><<<gr, 256, 0, st>>>(n1, nrhs, slot, (const __half *)in, scale, (double *)y);
  return cudaGetLastError();
}

// FP64 single field -> slot of an FP32/FP16 multi-RHS array (TO_MR), or back
cudaError_t mr_slot(bool to_mr, int ft_mr, long long n1, int nrhs, int slot, const void *in, double scale, void *out,
                    cudaStream_t st)
{
  const int gr = grid_for(n1);
  if (to_mr) {
    if (ft_mr == QB200_F32) mr_slot_kernel<float, double, true><<<gr, 256, 0, st>>>(n1, nrhs, slot, in, scale, out);
    else mr_slot_kernel<__half, double, true><<<gr, 256, 0, st>>>(n1, nrhs, slot, in, scale, out);
  } else {
    if (ft_mr == QB200_F32) mr_slot_kernel<double, float, false><<<gr, 256, 0, st>>>(n1, nrhs, slot, in, scale, out);
    else mr_slot_kernel<double, __half, false><<<gr, 256, 0, st>>>(n1, nrhs, slot, in, scale, out);
  }
  return cudaGetLastError();
}

// ---- per-RHS BLAS on the multi-RHS layout -----------------------------------

// a[r] = sign * num[r] / den[r] (0 when den[r] == 0), or host[r]
struct VecScalar {
  const double *num, *den;
  double sign;
  double host[kMaxRhs];
  __device__ __forceinline__ double get(int r) const
  {
    if (!num) return host[r];
    const double d = den ? den[r] : 1.0;
    return d == 0.0 ? 0.0 : sign * num[r] / d;
  }
};

// Element-wise and reduction kernels stream 16-byte vectors (vec16<FT>::n
// elements).  The right-hand side of element e is e % nrhs; the grid stride,
// a multiple of 256 vectors, is a multiple of nrhs (<= 16) elements, so each
// lane k of a thread's vectors stays on one right-hand side.  Arithmetic is
// FP32 for FP16 / FP32 storage and FP64 for FP64 storage; reductions
// accumulate in FP64.
template <typename FT> struct mr_calc {
  typedef float T;
};
template <> struct mr_calc<double> {
  typedef double T;
};
template <typename FT> __device__ __forceinline__ typename mr_calc<FT>::T mr_ld(FT v)
{
  return (typename mr_calc<FT>::T)to_d(v);
}
template <> __device__ __forceinline__ float mr_ld<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float mr_ld<float>(float v) { return v; }
template <typename FT> __device__ __forceinline__ FT mr_st(typename mr_calc<FT>::T v) { return from_d<FT>(v); }
template <> __device__ __forceinline__ __half mr_st<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ float mr_st<float>(float v) { return v; }

template <typename FT>
__global__ void __launch_bounds__(256) mr_axpby_kernel(long long nv, int nrhs, VecScalar a, const FT *__restrict__ x,
                                                       VecScalar b, FT *__restrict__ y)
{
  typedef typename mr_calc<FT>::T T;
  constexpr int W = vec16<FT>::n;
  const long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  T av[W], bv[W];
#pragma unroll
  for (int k = 0; k < W; k++) {
    const int r = (int)((i0 * W + k) % nrhs);
    av[k] = (T)a.get(r);
    bv[k] = (T)b.get(r);
  }
  for (long long i = i0; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const V16<FT> vx = ld16(x + i * W);
    V16<FT> vy = ld16(y + i * W);
#pragma unroll
    for (int k = 0; k < W; k++) vy.e[k] = mr_st<FT>(av[k] * mr_ld(vx.e[k]) + bv[k] * mr_ld(vy.e[k]));
    st16(y + i * W, vy);
  }
}

// x[i] * y[i] in FP64 (FP16 products are exact in FP32)
template <typename FT> __device__ __forceinline__ double mr_prod(FT a, FT b) { return to_d(a) * to_d(b); }
template <> __device__ __forceinline__ double mr_prod<__half>(__half a, __half b)
{
  return (double)(__half2float(a) * __half2float(b));
}

// partials[r*kRedBlocks + block] = sum over the block's elements of rhs r
template <typename FT>
__global__ void __launch_bounds__(kRedThreads) mr_dot_kernel(long long nv, int nrhs, const FT *__restrict__ x,
                                                             const FT *__restrict__ y, double *__restrict__ partials)
{
  constexpr int W = vec16<FT>::n;
  __shared__ double sh[kMaxRhs];
  if (threadIdx.x < kMaxRhs) sh[threadIdx.x] = 0.0;
  const long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double acc[W];
#pragma unroll
  for (int k = 0; k < W; k++) acc[k] = 0.0;
  for (long long i = i0; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const V16<FT> vx = ld16(x + i * W);
    const V16<FT> vy = ld16(y + i * W);
#pragma unroll
    for (int k = 0; k < W; k++) acc[k] += mr_prod(vx.e[k], vy.e[k]);
  }
  __syncthreads();
  // Lane k of warp lane l holds element offset l*W + k (mod 32*W), i.e. right-
  // hand side (l*W + k) % nrhs.  Lanes l and l^o agree when o*W is a multiple
  // of nrhs, so a butterfly over those o sums each right-hand side's lanes;
  // the lanes below `first` then hold one sum per right-hand side.
  int first = 16;
  for (int o = 1; o <= 16; o <<= 1)
    if (o * W >= nrhs) {
      first = o;
      break;
    }
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < W; k++) {
    double v = acc[k];
    for (int o = 16; o >= first; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane < first) atomicAdd(&sh[(int)((i0 * W + k) % nrhs)], v);
  }
  __syncthreads();
  if (threadIdx.x < nrhs) partials[threadIdx.x * kRedBlocks + blockIdx.x] = sh[threadIdx.x];
}

__global__ void mr_finish_kernel(const double *__restrict__ partials, int nrhs, double *__restrict__ result)
{
  const int r = blockIdx.x;
  double s = 0.0, dummy = 0.0;
  for (int i = threadIdx.x; i < kRedBlocks; i += blockDim.x) s += partials[r * kRedBlocks + i];
  block_sum2(s, dummy);
  if (threadIdx.x == 0) result[r] = s;
  (void)nrhs;
}

VecScalar vhost(double v)
{
  VecScalar s;
  s.num = s.den = nullptr;
  s.sign = 1.0;
  for (int r = 0; r < kMaxRhs; r++) s.host[r] = v;
  return s;
}

VecScalar vratio(const double *num, const double *den, double sign)
{
  VecScalar s = vhost(0.0);
  s.num = num;
  s.den = den;
  s.sign = sign;
  return s;
}

struct MR {
  int ft, nrhs;
  long long n; // total elements
};

cudaError_t mr_axpby(const MR &m, VecScalar a, const void *x, VecScalar b, void *y, cudaStream_t st)
{
  // a grid stride that is a multiple of nrhs keeps each thread on one rhs
  const int blocks = 148 * 4;
  if (m.ft == QB200_F32)
    mr_axpby_kernel<float><<<blocks, 256, 0, st>>>(m.n / 4, m.nrhs, a, (const float *)x, b, (float *)y);
  else if (m.ft == QB200_F64)
    mr_axpby_kernel<double><<<blocks, 256, 0, st>>>(m.n / 2, m.nrhs, a, (const double *)x, b, (double *)y);
  else mr_axpby_kernel<__half><<<blocks, 256, 0, st>>>(m.n / 8, m.nrhs, a, (const __half *)x, b, (__half *)y);
  return cudaGetLastError();
}

cudaError_t mr_dot(const MR &m, const void *x, const void *y, double *partials, double *result, cudaStream_t st)
{
  if (m.ft == QB200_F32)
    mr_dot_kernel<float><<<kRedBlocks, kRedThreads, 0, st>>>(m.n / 4, m.nrhs, (const float *)x, (const float *)y,
                                                              partials);
  else if (m.ft == QB200_F64)
    mr_dot_kernel<double><<<kRedBlocks, kRedThreads, 0, st>>>(m.n / 2, m.nrhs, (const double *)x, (const double *)y,
                                                               partials);
  else
    mr_dot_kernel<__half><<<kRedBlocks, kRedThreads, 0, st>>>(m.n / 8, m.nrhs, (const __half *)x, (const __half *)y,
                                                               partials);
  mr_finish_kernel<<<m.nrhs, kRedThreads, 0, st>>>(partials, m.nrhs, result);
  return cudaGetLastError();
}

// ---- operator and solver ---------------------------------------------------

qb200_coeffs coeffs_of(const qb200_operator *op, double scale)
{
  qb200_coeffs c;
  c.coeff_s = op->coeff_s * scale;
  c.coeff_t_f = op->coeff_t_f * scale;
  c.coeff_t_b = op->coeff_t_b * scale;
  c.alpha = op->alpha;
  c.mu = op->mu;
  c.muinv = op->muinv;
  c.rho = op->rho;
  c.tbc_mask = op->tbc_mask;
  std::memcpy(c.tbc_phases, op->tbc_phases, sizeof(c.tbc_phases));
  return c;
}

int check_op(const qb200_operator *op)
{
  if (!op) return api_fail(QB200_ENULL, "operator is NULL");
  if (op->family < 0 || op->family > 3) return api_fail(QB200_EINVAL, "operator family must be 0..3");
  if (op->target_cb != 0 && op->target_cb != 1) return api_fail(QB200_EINVAL, "target_cb must be 0 or 1");
  if (!op->gauge[0] || !op->gauge[1]) return api_fail(QB200_ENULL, "both gauge checkerboards are needed");
  if ((op->family == 1 || op->family == 3) && (!op->clov[0] || !op->clov[1]))
    return api_fail(QB200_ENULL, "clover operator needs both clover checkerboards");
  if (op->family == 3 && (!op->clov_dag[0] || !op->clov_dag[1]))
    return api_fail(QB200_ENULL, "twisted-mass clover dagger needs clov_dag");
  if (op->family == 0 && op->alpha == 0.0) return api_fail(QB200_EINVAL, "Wilson operator needs alpha != 0");
  return QB200_OK;
}

// out = Mhat in (or Mhat^dag) on nrhs right-hand sides
int mr_schur(const qb200_lattice *l, int nrhs, const qb200_operator *op, int isPlus, const void *in, void *out,
             void *tmp, cudaStream_t st)
{
  const int tc = op->target_cb, oc = 1 - tc;
  const void *clov_o = op->clov[oc], *clov_t = op->clov[tc];
  if (op->family == 3 && !isPlus) {
    clov_o = op->clov_dag[oc];
    clov_t = op->clov_dag[tc];
  }
  const qb200_coeffs c1 = coeffs_of(op, op->family == 0 ? 1.0 / op->alpha : 1.0);
  int rc = mr_body(l, nrhs, op->family, false, isPlus, oc, in, nullptr, tmp, op->gauge[oc], clov_o, &c1, nullptr, st);
  if (rc) return rc;
  const qb200_coeffs c2 = coeffs_of(op, 1.0);
  return mr_body(l, nrhs, op->family, true, isPlus, tc, tmp, in, out, op->gauge[tc], clov_t, &c2, nullptr, st);
}

size_t single_bytes(const qb200_lattice *l) { return (size_t)qb200_spinor_elems(l) * fbytes(l->ftype); }

size_t ws_bytes(const qb200_lattice *l, int nrhs, int nspin)
{
  if (qb200_spinor_elems(l) < 0) return 0;
  return nspin * (single_bytes(l) * nrhs + 256) + (size_t)(kRedBlocks * kMaxRhs + 16 * kMaxRhs) * 8 + 4096;
}

struct Work {
  char *p;
  size_t off;
  void *take(size_t b)
  {
    off = (off + 255) & ~(size_t)255;
    void *r = p + off;
    off += b;
    return r;
  }
};

struct MRVecs {
  void *v[10];
  double *partials, *scal; // scal: 16 slots of kMaxRhs doubles
  double *slot(int k) { return scal + k * kMaxRhs; }
};

MRVecs mr_carve(const qb200_lattice *l, int nrhs, void *ws, int nspin)
{
  Work w{(char *)ws, 0};
  MRVecs m;
  for (int i = 0; i < nspin && i < 10; i++) m.v[i] = w.take(single_bytes(l) * nrhs);
  m.partials = (double *)w.take((size_t)kRedBlocks * kMaxRhs * 8);
  m.scal = (double *)w.take((size_t)16 * kMaxRhs * 8);
  return m;
}

int fetch(double *h, const double *d, int n, cudaStream_t st)
{
  cudaError_t e = cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return cuda_rc(e, "reduction readback");
}

// CG on Mhat^dag Mhat for nrhs systems at once (independent recurrences,
// shared operator applications).  ws vectors: r, p, Ap, t, tmp.
int mr_cg_core(const qb200_lattice *l, int nrhs, const qb200_operator *op, const void *rhs, void *x, double tol,
               int max_iter, MRVecs &s, int *iters, double *rel, cudaStream_t st, bool x_zero = false)
{
  MR m;
  m.ft = l->ftype;
  m.nrhs = nrhs;
  m.n = qb200_spinor_elems(l) * nrhs;
  const size_t bytes = single_bytes(l) * nrhs;
  void *r = s.v[0], *p = s.v[1], *Ap = s.v[2], *t = s.v[3], *tmp = s.v[4];
  double *rr = s.slot(0), *rrn = s.slot(1), *pAp = s.slot(2), *bb = s.slot(3);
  int rc;
  // r = rhs - A x (just rhs when the caller zeroed x)
  if (!x_zero) {
    if ((rc = mr_schur(l, nrhs, op, 1, x, t, tmp, st))) return rc;
    if ((rc = mr_schur(l, nrhs, op, 0, t, Ap, tmp, st))) return rc;
  }
  cudaError_t e = cudaMemcpyAsync(r, rhs, bytes, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && !x_zero) e = mr_axpby(m, vhost(-1.0), Ap, vhost(1.0), r, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p, r, bytes, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = mr_dot(m, r, r, s.partials, rr, st);
  if (e == cudaSuccess) e = mr_dot(m, rhs, rhs, s.partials, bb, st);
  if ((rc = cuda_rc(e, "multi-RHS cg setup"))) return rc;
  double h_rr[kMaxRhs], h_bb[kMaxRhs];
  if ((rc = fetch(h_bb, bb, nrhs, st))) return rc;
  if ((rc = fetch(h_rr, rr, nrhs, st))) return rc;
  auto done = [&]() {
    for (int i = 0; i < nrhs; i++)
      if (h_rr[i] > tol * tol * h_bb[i]) return false;
    return true;
  };
  int k = 0;
  while (!done() && k < max_iter) {
    if ((rc = mr_schur(l, nrhs, op, 1, p, t, tmp, st))) return rc;
    if ((rc = mr_schur(l, nrhs, op, 0, t, Ap, tmp, st))) return rc;
    e = mr_dot(m, p, Ap, s.partials, pAp, st);
    if (e == cudaSuccess) e = mr_axpby(m, vratio(rr, pAp, 1.0), p, vhost(1.0), x, st);
    if (e == cudaSuccess) e = mr_axpby(m, vratio(rr, pAp, -1.0), Ap, vhost(1.0), r, st);
    if (e == cudaSuccess) e = mr_dot(m, r, r, s.partials, rrn, st);
    if (e == cudaSuccess) e = mr_axpby(m, vhost(1.0), r, vratio(rrn, rr, 1.0), p, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rr, rrn, nrhs * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if ((rc = cuda_rc(e, "multi-RHS cg iteration"))) return rc;
    if ((rc = fetch(h_rr, rr, nrhs, st))) return rc;
    k++;
    for (int i = 0; i < nrhs; i++)
      if (!std::isfinite(h_rr[i])) return api_fail(QB200_EINVAL, "multi-RHS cg: residual is not finite");
  }
  *iters = k;
  for (int i = 0; i < nrhs; i++) rel[i] = h_bb[i] > 0 ? std::sqrt(h_rr[i] / h_bb[i]) : 0.0;
  return QB200_OK;
}

// Multi-RHS CG on the normal equations in the low precision with FP64
// reliable updates, all right-hand sides updated together: each segment
// starts from the FP64 residuals r_i = b_i - Mhat x_i, scaled to unit rms and
// packed, their normal form Mhat^dag r (low precision, all right-hand sides
// in one application) replaces the iterated residual, and p is rescaled to
// the new units, so the recurrence continues (no restart).  A segment ends
// when every unconverged right-hand side's iterated residual has fallen by
// delta, or far enough that its FP64 residual would meet rel_tol; then
// x_i += x_lo_i / scale_i in FP64.
int mr_reliable(const qb200_lattice *lat_hi, const qb200_operator *op_hi, const qb200_lattice *lat_lo,
                const qb200_operator *op_lo, int nrhs, const void *const *b, void *const *x, double rel_tol,
                double delta, int max_iter, int max_updates, void *r, void *tmp, double *partials, double *scal,
                MRVecs &L, const double *bnorm, int *iters, int *updates, double *rel, cudaStream_t st)
{
  MR m;
  m.ft = lat_lo->ftype;
  m.nrhs = nrhs;
  m.n = qb200_spinor_elems(lat_lo) * nrhs;
  const long long n1 = qb200_spinor_elems(lat_hi);
  const size_t bytes = single_bytes(lat_lo) * nrhs;
  void *rl = L.v[0], *p = L.v[1], *Ap = L.v[2], *t = L.v[3], *tl = L.v[4], *r_lo = L.v[5], *xl = L.v[7];
  double *rr_d = L.slot(0), *rrn_d = L.slot(1), *pAp_d = L.slot(2);
  double scale[kMaxRhs], rr[kMaxRhs], seg_rr[kMaxRhs], seg_rel[kMaxRhs], s_new[kMaxRhs], h[kMaxRhs];
  int k = 0, nup = 0, rc;
  bool first = true;
  cudaError_t e;
  while (true) {
    bool all = true;
    for (int i = 0; i < nrhs; i++) {
      if ((rc = qb200_schur_apply(lat_hi, op_hi, 1, x[i], r, tmp, st))) return rc;
      if ((rc = qb200_blas_axpby(QB200_F64, n1, 1.0, b[i], -1.0, r, st))) return rc;
      double rrh;
      if ((rc = qb200_blas_dot(QB200_F64, n1, r, r, scal, partials, st))) return rc;
      if ((rc = fetch(&rrh, scal, 1, st))) return rc;
      rel[i] = bnorm[i] > 0 ? std::sqrt(rrh / bnorm[i]) : 0.0;
      if (rel[i] > rel_tol) all = false;
      s_new[i] = std::sqrt((double)n1 / (rrh > 0 ? rrh : 1.0));
      if ((rc = cuda_rc(mr_slot(true, m.ft, n1, nrhs, i, r, s_new[i], r_lo, st), "multi-RHS pack slot"))) return rc;
    }
    if (all || k >= max_iter || nup >= max_updates) break;
    if ((rc = mr_schur(lat_lo, nrhs, op_lo, 0, r_lo, rl, tl, st))) return rc;
    VecScalar ratio = vhost(0.0);
    for (int i = 0; i < nrhs; i++) ratio.host[i] = first ? 1.0 : s_new[i] / scale[i];
    e = first ? cudaMemcpyAsync(p, rl, bytes, cudaMemcpyDeviceToDevice, st)
              : mr_axpby(m, vhost(0.0), rl, ratio, p, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(xl, 0, bytes, st);
    if (e == cudaSuccess) e = mr_dot(m, rl, rl, L.partials, rr_d, st);
    if ((rc = cuda_rc(e, "multi-RHS reliable segment"))) return rc;
    if ((rc = fetch(h, rr_d, nrhs, st))) return rc;
    if (!first) {
      // continue the recurrence in the new units: p = r + beta p
      VecScalar beta = vhost(0.0);
      // a right-hand side whose residual is exactly zero (a zero source, or
      // one already solved exactly) keeps a zero direction instead of 0/0
      for (int i = 0; i < nrhs; i++) {
        const double den = rr[i] * ratio.host[i] * ratio.host[i];
        beta.host[i] = den > 0 ? h[i] / den : 0.0;
      }
      if ((rc = cuda_rc(mr_axpby(m, vhost(1.0), rl, beta, p, st), "multi-RHS reliable direction"))) return rc;
    }
    for (int i = 0; i < nrhs; i++) {
      scale[i] = s_new[i];
      rr[i] = seg_rr[i] = h[i];
      seg_rel[i] = rel[i];
    }
    first = false;
    bool update = false;
    while (!update && k < max_iter) {
      if ((rc = mr_schur(lat_lo, nrhs, op_lo, 1, p, t, tl, st))) return rc;
      if ((rc = mr_schur(lat_lo, nrhs, op_lo, 0, t, Ap, tl, st))) return rc;
      e = mr_dot(m, p, Ap, L.partials, pAp_d, st);
      if (e == cudaSuccess) e = mr_axpby(m, vratio(rr_d, pAp_d, 1.0), p, vhost(1.0), xl, st);
      if (e == cudaSuccess) e = mr_axpby(m, vratio(rr_d, pAp_d, -1.0), Ap, vhost(1.0), rl, st);
      if (e == cudaSuccess) e = mr_dot(m, rl, rl, L.partials, rrn_d, st);
      if ((rc = cuda_rc(e, "multi-RHS reliable iteration"))) return rc;
      if ((rc = fetch(h, rrn_d, nrhs, st))) return rc;
      k++;
      update = true;
      for (int i = 0; i < nrhs; i++) {
        if (!std::isfinite(h[i])) return api_fail(QB200_EINVAL, "multi-RHS cg: residual is not finite");
        const bool fell = h[i] <= delta * delta * seg_rr[i] || seg_rel[i] * std::sqrt(h[i] / seg_rr[i]) <= rel_tol;
        if (seg_rel[i] > rel_tol && !fell) update = false;
      }
      if (k == max_iter) update = true;
      if (!update) {
        e = mr_axpby(m, vhost(1.0), rl, vratio(rrn_d, rr_d, 1.0), p, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(rr_d, rrn_d, nrhs * sizeof(double), cudaMemcpyDeviceToDevice, st);
        if ((rc = cuda_rc(e, "multi-RHS reliable direction"))) return rc;
        for (int i = 0; i < nrhs; i++) rr[i] = h[i];
      }
      // on an update rr keeps |r|^2 of the step before, for the next beta
    }
    for (int i = 0; i < nrhs; i++)
      if ((rc = cuda_rc(mr_slot_add(m.ft, n1, nrhs, i, xl, 1.0 / scale[i], x[i], st), "multi-RHS update")))
        return rc;
    nup++;
  }
  *iters = k;
  *updates = nup;
  return QB200_OK;
}

} // namespace

extern "C" {

long long qb200_mrhs_spinor_elems(const qb200_lattice *lat, int nrhs)
{
  const long long n = qb200_spinor_elems(lat);
  return n < 0 || nrhs < 1 ? -1 : n * nrhs;
}

int qb200_mrhs_pack(const qb200_lattice *lat, int nrhs, const void *const *fields, void *mrhs, void *stream)
{
  int rc = check_mr(lat, nrhs);
  if (rc) return rc;
  if (!fields || !mrhs) return api_fail(QB200_ENULL, "fields and mrhs must be non-NULL");
  PtrTab tab;
  for (int r = 0; r < nrhs; r++) {
    if (!fields[r]) return api_fail(QB200_ENULL, "a field pointer is NULL");
    tab.p[r] = fields[r];
    tab.scale[r] = 1.0;
  }
  const long long n = qb200_spinor_elems(lat) * nrhs;
  return cuda_rc(mr_convert(true, lat->ftype, lat->ftype, n, lat->soalen, nrhs, tab, mrhs, (cudaStream_t)stream),
                 "multi-RHS pack");
}

int qb200_mrhs_unpack(const qb200_lattice *lat, int nrhs, const void *mrhs, void *const *fields, void *stream)
{
  int rc = check_mr(lat, nrhs);
  if (rc) return rc;
  if (!fields || !mrhs) return api_fail(QB200_ENULL, "fields and mrhs must be non-NULL");
  PtrTab tab;
  for (int r = 0; r < nrhs; r++) {
    if (!fields[r]) return api_fail(QB200_ENULL, "a field pointer is NULL");
    tab.p[r] = fields[r];
    tab.scale[r] = 1.0;
  }
  const long long n = qb200_spinor_elems(lat) * nrhs;
  return cuda_rc(mr_convert(false, lat->ftype, lat->ftype, n, lat->soalen, nrhs, tab, const_cast<void *>(mrhs),
                            (cudaStream_t)stream),
                 "multi-RHS unpack");
}

int qb200_dslash_mrhs(const qb200_lattice *lat, int nrhs, int family, int achimbdpsi, int isign, int cb,
                      const void *psi, const void *chi, void *out, const void *gauge, const void *clover,
                      const qb200_coeffs *coeffs, const unsigned accumulate[8], void *stream)
{
  return mr_body(lat, nrhs, family, achimbdpsi != 0, isign > 0, cb, psi, chi, out, gauge, clover, coeffs,
                 accumulate, (cudaStream_t)stream);
}

int qb200_schur_apply_mrhs(const qb200_lattice *lat, int nrhs, const qb200_operator *op, int isign, const void *in,
                           void *out, void *tmp_other_cb, void *stream)
{
  int rc = check_mr(lat, nrhs);
  if (rc) return rc;
  if ((rc = check_op(op))) return rc;
  if (!in || !out || !tmp_other_cb) return api_fail(QB200_ENULL, "in, out and tmp must be non-NULL");
  return mr_schur(lat, nrhs, op, isign > 0, in, out, tmp_other_cb, (cudaStream_t)stream);
}

long long qb200_cg_mrhs_workspace_bytes(const qb200_lattice *lat, int nrhs) { return (long long)ws_bytes(lat, nrhs, 6); }

int qb200_invert_cg_mrhs(const qb200_lattice *lat, int nrhs, const qb200_operator *op, const void *b, void *x,
                         double rel_tol, int max_iter, void *workspace, int *iters, double *rel_res, void *stream)
{
  int rc = check_mr(lat, nrhs);
  if (rc) return rc;
  if ((rc = check_op(op))) return rc;
  if (!b || !x || !workspace || !rel_res) return api_fail(QB200_ENULL, "b, x, workspace and rel_res are required");
  cudaStream_t st = (cudaStream_t)stream;
  MRVecs s = mr_carve(lat, nrhs, workspace, 6);
  void *rhs = s.v[5];
  if ((rc = mr_schur(lat, nrhs, op, 0, b, rhs, s.v[4], st))) return rc;
  int k = 0;
  if ((rc = mr_cg_core(lat, nrhs, op, rhs, x, rel_tol, max_iter, s, &k, rel_res, st))) return rc;
  if (iters) *iters = k;
  return QB200_OK;
}

long long qb200_mixed_mrhs_workspace_bytes(const qb200_lattice *lat_hi, const qb200_lattice *lat_lo, int nrhs,
                                           long long *lo_bytes)
{
  if (lo_bytes) *lo_bytes = (long long)ws_bytes(lat_lo, nrhs, 8);
  return (long long)ws_bytes(lat_hi, 1, 2);
}

// Defect correction for nrhs systems: per right-hand side the true residual
// b_i - Mhat x_i is formed with the single-RHS FP64 operator (op_hi) and
// packed, scaled to unit rms, into one multi-RHS array of the low precision;
// the normal equations Mhat^dag Mhat e = Mhat^dag r of all right-hand sides
// are solved together with the multi-RHS low precision operator (op_lo, FP16
// or FP32 storage) to inner_tol, and the corrections are accumulated into x
// in FP64.  b and x: host arrays of nrhs device
// pointers to FP64 single-layout spinors.
static int mixed_mrhs(const qb200_lattice *lat_hi, const qb200_operator *op_hi, const qb200_lattice *lat_lo,
                      const qb200_operator *op_lo, int nrhs, const void *const *b, void *const *x, double rel_tol,
                      double inner_tol, int max_inner, int max_outer, void *ws_hi, void *ws_lo, int *inner_iters,
                      int *outer_iters, double *rel_res, void *stream, bool reliable)
{
  int rc = check_mr(lat_lo, nrhs);
  if (rc) return rc;
  if ((rc = check_op(op_hi)) || (rc = check_op(op_lo))) return rc;
  if (!lat_hi || lat_hi->ftype != QB200_F64) return api_fail(QB200_EINVAL, "the high precision lattice must be FP64");
  if (!b || !x || !ws_hi || !ws_lo || !rel_res) return api_fail(QB200_ENULL, "missing argument");
  if (qb200_spinor_elems(lat_hi) != qb200_spinor_elems(lat_lo))
    return api_fail(QB200_EINVAL, "high and low precision lattices differ in shape");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n1 = qb200_spinor_elems(lat_hi);
  Work wh{(char *)ws_hi, 0};
  void *r = wh.take(n1 * 8), *tmp = wh.take(n1 * 8);
  double *partials = (double *)wh.take((size_t)kRedBlocks * 2 * 8);
  double *scal = (double *)wh.take(64 * 8);
  MRVecs L = mr_carve(lat_lo, nrhs, ws_lo, 8);
  void *rhs_lo = L.v[6], *e_lo = L.v[7];
  const size_t lo_bytes = single_bytes(lat_lo) * nrhs;
  for (int i = 0; i < nrhs; i++)
    if ((rc = cuda_rc(cudaMemsetAsync(x[i], 0, n1 * 8, st), "mixed init"))) return rc;
  double bnorm[kMaxRhs], scale[kMaxRhs], rel[kMaxRhs];
  for (int i = 0; i < nrhs; i++) {
    if ((rc = qb200_blas_dot(QB200_F64, n1, b[i], b[i], scal, partials, st))) return rc;
    if ((rc = fetch(&bnorm[i], scal, 1, st))) return rc;
  }
  if (reliable) {
    if (!(inner_tol > 0.0 && inner_tol < 1.0)) return api_fail(QB200_EINVAL, "reliable updates need 0 < inner_tol < 1");
    int k = 0, nup = 0;
    if ((rc = mr_reliable(lat_hi, op_hi, lat_lo, op_lo, nrhs, b, x, rel_tol, inner_tol, max_inner, max_outer, r, tmp,
                          partials, scal, L, bnorm, &k, &nup, rel, st)))
      return rc;
    if (inner_iters) *inner_iters = k;
    if (outer_iters) *outer_iters = nup;
    for (int i = 0; i < nrhs; i++) rel_res[i] = rel[i];
    return QB200_OK;
  }
  // r_lo: the scaled true residuals in the low precision; rhs_lo = Mhat^dag r_lo
  void *r_lo = L.v[5];
  int tot = 0, outer = 0;
  while (true) {
    bool all = true;
    for (int i = 0; i < nrhs; i++) {
      // r = b_i - Mhat x_i in FP64
      if ((rc = qb200_schur_apply(lat_hi, op_hi, 1, x[i], r, tmp, st))) return rc;
      if ((rc = qb200_blas_axpby(QB200_F64, n1, 1.0, b[i], -1.0, r, st))) return rc;
      double rr;
      if ((rc = qb200_blas_dot(QB200_F64, n1, r, r, scal, partials, st))) return rc;
      if ((rc = fetch(&rr, scal, 1, st))) return rc;
      rel[i] = bnorm[i] > 0 ? std::sqrt(rr / bnorm[i]) : 0.0;
      if (rel[i] > rel_tol) all = false;
      // slot i of r_lo: r scaled to unit rms per element
      scale[i] = std::sqrt((double)n1 / (rr > 0 ? rr : 1.0));
      if ((rc = cuda_rc(mr_slot(true, lat_lo->ftype, n1, nrhs, i, r, scale[i], r_lo, st), "multi-RHS pack slot")))
        return rc;
    }
    if (all || outer >= max_outer) break;
    // normal-equation right-hand sides in the low precision: its rounding
    // (~1e-3 relative for FP16) is far below the inner tolerance of a correction
    if ((rc = mr_schur(lat_lo, nrhs, op_lo, 0, r_lo, rhs_lo, L.v[4], st))) return rc;
    if ((rc = cuda_rc(cudaMemsetAsync(e_lo, 0, lo_bytes, st), "mixed zero"))) return rc;
    int k = 0;
    double irel[kMaxRhs];
    if ((rc = mr_cg_core(lat_lo, nrhs, op_lo, rhs_lo, e_lo, inner_tol, max_inner, L, &k, irel, st, true)))
      return rc;
    tot += k;
    for (int i = 0; i < nrhs; i++)
      if ((rc = cuda_rc(mr_slot_add(lat_lo->ftype, n1, nrhs, i, e_lo, 1.0 / scale[i], x[i], st),
                        "multi-RHS correction")))
        return rc;
    outer++;
  }
  if (inner_iters) *inner_iters = tot;
  if (outer_iters) *outer_iters = outer;
  for (int i = 0; i < nrhs; i++) rel_res[i] = rel[i];
  return QB200_OK;
}

int qb200_invert_mixed_mrhs(const qb200_lattice *lat_hi, const qb200_operator *op_hi, const qb200_lattice *lat_lo,
                            const qb200_operator *op_lo, int nrhs, const void *const *b, void *const *x,
                            double rel_tol, double inner_tol, int max_inner, int max_outer, void *ws_hi, void *ws_lo,
                            int *inner_iters, int *outer_iters, double *rel_res, void *stream)
{
  return mixed_mrhs(lat_hi, op_hi, lat_lo, op_lo, nrhs, b, x, rel_tol, inner_tol, max_inner, max_outer, ws_hi, ws_lo,
                    inner_iters, outer_iters, rel_res, stream, false);
}

int qb200_invert_reliable_mrhs(const qb200_lattice *lat_hi, const qb200_operator *op_hi,
                               const qb200_lattice *lat_lo, const qb200_operator *op_lo, int nrhs,
                               const void *const *b, void *const *x, double rel_tol, double delta, int max_iter,
                               int max_updates, void *ws_hi, void *ws_lo, int *iters, int *updates, double *rel_res,
                               void *stream)
{
  return mixed_mrhs(lat_hi, op_hi, lat_lo, op_lo, nrhs, b, x, rel_tol, delta, max_iter, max_updates, ws_hi, ws_lo,
                    iters, updates, rel_res, stream, true);
}

} // extern "C"
