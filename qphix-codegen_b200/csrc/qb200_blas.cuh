// qb200_blas.cuh -- level-1 linear algebra on spinor fields for the solvers.
//
// Fields are whole QPhiX spinor arrays (padding included; padding stays zero
// because every operation is linear and the inputs' padding is zero).
// Element-wise operations stream 16-byte vectors; reductions accumulate in
// FP64 per thread, reduce per block, and write one partial per block into a
// scratch array that a one-block finishing kernel sums into a double on the
// device (results stay on the device so that a solver iteration needs no
// host synchronisation).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace qb200 {

// grid of the reduction kernels: 4 blocks of 256 threads per SM of a B200
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 148 * 4;
// doubles of scratch one reduction needs (two components for complex dots)
constexpr int kRedPartials = 2 * kRedBlocks;

// number of storage elements moved per 16-byte vector
template <typename FT> struct vec16;
template <> struct vec16<float> {
  static constexpr int n = 4;
};
template <> struct vec16<double> {
  static constexpr int n = 2;
};
template <> struct vec16<__half> {
  static constexpr int n = 8;
};
template <> struct vec16<__nv_bfloat16> {
  static constexpr int n = 8;
};

template <typename FT> __device__ __forceinline__ double to_d(FT v);
template <> __device__ __forceinline__ double to_d<float>(float v) { return (double)v; }
template <> __device__ __forceinline__ double to_d<double>(double v) { return v; }
template <> __device__ __forceinline__ double to_d<__half>(__half v) { return (double)__half2float(v); }
template <> __device__ __forceinline__ double to_d<__nv_bfloat16>(__nv_bfloat16 v)
{
  return (double)__bfloat162float(v);
}

template <typename FT> __device__ __forceinline__ FT from_d(double v);
template <> __device__ __forceinline__ float from_d<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ double from_d<double>(double v) { return v; }
template <> __device__ __forceinline__ __half from_d<__half>(double v) { return __float2half_rn((float)v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_d<__nv_bfloat16>(double v)
{
  return __float2bfloat16_rn((float)v);
}

template <typename FT> struct V16 {
  FT e[vec16<FT>::n];
};

template <typename FT> __device__ __forceinline__ V16<FT> ld16(const FT *p)
{
  V16<FT> v;
  *reinterpret_cast<uint4 *>(&v) = __ldg(reinterpret_cast<const uint4 *>(p));
  return v;
}

template <typename FT> __device__ __forceinline__ void st16(FT *p, const V16<FT> &v)
{
  *reinterpret_cast<uint4 *>(p) = *reinterpret_cast<const uint4 *>(&v);
}

// ---------------------------------------------------------------------------
// element-wise: y = a*x + b*y, with a and b from the host or from device
// scalars (a_dev/b_dev non-null: a = a_scale * a_dev[0] (or its ratio form))

struct ScalarRef {
  double host;          // used when dev == nullptr
  const double *num;    // device numerator
  const double *den;    // device denominator (nullptr: 1)
  double sign;
  __device__ __forceinline__ double get() const
  {
    if (!num) return host;
    return sign * (den ? num[0] / den[0] : num[0]);
  }
};

template <typename FT>
__global__ void __launch_bounds__(256) axpby_kernel(long long nv, ScalarRef a, const FT *__restrict__ x,
                                                    ScalarRef b, FT *__restrict__ y)
{
  const double av = a.get(), bv = b.get();
  constexpr int W = vec16<FT>::n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    V16<FT> vx = ld16(x + i * W);
    V16<FT> vy = ld16(y + i * W);
#pragma unroll
    for (int k = 0; k < W; k++) vy.e[k] = from_d<FT>(av * to_d(vx.e[k]) + bv * to_d(vy.e[k]));
    st16(y + i * W, vy);
  }
}

// out = scale * in with conversion of the storage type
template <typename FO, typename FI>
__global__ void __launch_bounds__(256) convert_kernel(long long n, double scale, const FI *__restrict__ in,
                                                      FO *__restrict__ out)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = from_d<FO>(scale * to_d(in[i]));
}

// ---------------------------------------------------------------------------
// reductions

static __device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block sum of two values; thread 0 holds the result
static __device__ __forceinline__ void block_sum2(double &a, double &b)
{
  __shared__ double sa[32], sb[32];
  a = warp_sum(a);
  b = warp_sum(b);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    a = l < nw ? sa[l] : 0.0;
    b = l < nw ? sb[l] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
  }
}

// partials[blockIdx.x] = sum x*y (real dot; x == y gives the norm squared)
template <typename FT>
__global__ void __launch_bounds__(kRedThreads) dot_partial_kernel(long long nv, const FT *__restrict__ x,
                                                                  const FT *__restrict__ y,
                                                                  double *__restrict__ partials)
{
  constexpr int W = vec16<FT>::n;
  double s = 0.0, dummy = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
       i += (long long)gridDim.x * blockDim.x) {
    V16<FT> vx = ld16(x + i * W);
    V16<FT> vy = ld16(y + i * W);
#pragma unroll
    for (int k = 0; k < W; k++) s += to_d(vx.e[k]) * to_d(vy.e[k]);
  }
  block_sum2(s, dummy);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// complex dot <x, y> = sum conj(x) y over a QPhiX spinor field: the real and
// imaginary parts of a component are S elements apart within a block
template <typename FT, int S>
__global__ void __launch_bounds__(kRedThreads) cdot_partial_kernel(long long npairs, const FT *__restrict__ x,
                                                                   const FT *__restrict__ y,
                                                                   double *__restrict__ partials)
{
  double re = 0.0, im = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npairs;
       i += (long long)gridDim.x * blockDim.x) {
    // pair i: group g = i / S of 2S elements, lane i % S
    const long long g = i / S;
    const int l = (int)(i - g * S);
    const long long e = g * 2 * S + l;
    const double xr = to_d(x[e]), xi = to_d(x[e + S]);
    const double yr = to_d(y[e]), yi = to_d(y[e + S]);
    re += xr * yr + xi * yi;
    im += xr * yi - xi * yr;
  }
  block_sum2(re, im);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = re;
    partials[kRedBlocks + blockIdx.x] = im;
  }
}

// result[c] = sum of partials[c*kRedBlocks .. +nblocks) for c < ncomp
static __global__ void __launch_bounds__(kRedThreads) finish_kernel(const double *__restrict__ partials, int nblocks,
                                                             int ncomp, double *__restrict__ result)
{
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
    a += partials[i];
    if (ncomp > 1) b += partials[kRedBlocks + i];
  }
  block_sum2(a, b);
  if (threadIdx.x == 0) {
    result[0] = a;
    if (ncomp > 1) result[1] = b;
  }
}

// ---------------------------------------------------------------------------
// FP16 spinors with a per-site norm: blocks of 24*S halves followed by S
// FP32 norms (2*S halves).  These kernels work per site lane: decode the 24
// values, operate in FP64, re-encode with a fresh norm.

template <int S> struct F16NSite {
  static __device__ __forceinline__ void load(const __half *f, long long sl, double (&v)[24])
  {
    const long long blk = sl / S;
    const int l = (int)(sl - blk * S);
    const __half *b = f + blk * 26 * S;
    const double nrm = (double)__ldg(reinterpret_cast<const float *>(b + 24 * S) + l);
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] = (double)__half2float(b[k * S + l]) * nrm;
  }
  static __device__ __forceinline__ void store(__half *f, long long sl, const double (&v)[24])
  {
    const long long blk = sl / S;
    const int l = (int)(sl - blk * S);
    __half *b = f + blk * 26 * S;
    double m = 0.0;
#pragma unroll
    for (int k = 0; k < 24; k++) m = fmax(m, fabs(v[k]));
    const float nrm = m > 0.0 ? (float)m : 1.0f;
    reinterpret_cast<float *>(b + 24 * S)[l] = nrm;
    const double inv = 1.0 / (double)nrm;
#pragma unroll
    for (int k = 0; k < 24; k++) b[k * S + l] = __float2half_rn((float)(v[k] * inv));
  }
};

// The same decode / encode in FP32: the vectors of an FP16 solve carry 11
// significant bits, so the inner BLAS (axpby, and the per-site terms of the
// dots, whose sums over sites are FP64) run in FP32 arithmetic.
template <int S> struct F16NSiteF {
  static __device__ __forceinline__ void load(const __half *f, long long sl, float (&v)[24])
  {
    const long long blk = sl / S;
    const int l = (int)(sl - blk * S);
    const __half *b = f + blk * 26 * S;
    const float nrm = __ldg(reinterpret_cast<const float *>(b + 24 * S) + l);
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] = __half2float(b[k * S + l]) * nrm;
  }
  static __device__ __forceinline__ void store(__half *f, long long sl, const float (&v)[24])
  {
    const long long blk = sl / S;
    const int l = (int)(sl - blk * S);
    __half *b = f + blk * 26 * S;
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 24; k++) m = fmaxf(m, fabsf(v[k]));
    const float nrm = m > 0.f ? m : 1.0f;
    reinterpret_cast<float *>(b + 24 * S)[l] = nrm;
    const float inv = 1.0f / nrm;
#pragma unroll
    for (int k = 0; k < 24; k++) b[k * S + l] = __float2half_rn(v[k] * inv);
  }
};

// Warp tiles of FP16 + norm vectors: a warp moves the 32/S blocks of 32
// sites (52 bytes per site) between global and shared memory in 16-byte
// vectors and each lane decodes / encodes its own site there, so the global
// accesses are whole sectors instead of the 2*S-byte component pieces that
// one site per thread touches.  Same arithmetic as F16NSiteF.
template <int S> struct F16NTile {
  static constexpr int G = 32 / S;  // blocks per tile
  static constexpr int CH = 52 * S / 16;  // 16-byte vectors per block
  static constexpr int N = G * CH;        // vectors per tile (104)
  static constexpr int BYTES = 16 * N;
  // blocks blk0 .. blk0+G-1 (those below nblk) -> sm
  static __device__ __forceinline__ void load(const __half *f, long long blk0, long long nblk, unsigned char *sm,
                                              int ln)
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(f) + blk0 * CH;
    const long long avail = (nblk - blk0) * CH;
#pragma unroll
    for (int r = 0; r < (N + 31) / 32; r++) {
      const int j = ln + 32 * r;
      if (j < N && j < avail) reinterpret_cast<uint4 *>(sm)[j] = __ldg(src + j);
    }
  }
  static __device__ __forceinline__ void store(__half *f, long long blk0, long long nblk, const unsigned char *sm,
                                               int ln)
  {
    uint4 *dst = reinterpret_cast<uint4 *>(f) + blk0 * CH;
    const long long avail = (nblk - blk0) * CH;
#pragma unroll
    for (int r = 0; r < (N + 31) / 32; r++) {
      const int j = ln + 32 * r;
      if (j < N && j < avail) dst[j] = reinterpret_cast<const uint4 *>(sm)[j];
    }
  }
  // lane ln's site of the tile in sm
  static __device__ __forceinline__ void get(const unsigned char *sm, int ln, float (&v)[24])
  {
    const __half *b = reinterpret_cast<const __half *>(sm + (ln / S) * 52 * S);
    const int l = ln % S;
    const float nrm = reinterpret_cast<const float *>(b + 24 * S)[l];
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] = __half2float(b[k * S + l]) * nrm;
  }
  static __device__ __forceinline__ void put(unsigned char *sm, int ln, const float (&v)[24])
  {
    __half *b = reinterpret_cast<__half *>(sm + (ln / S) * 52 * S);
    const int l = ln % S;
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 24; k++) m = fmaxf(m, fabsf(v[k]));
    const float nrm = m > 0.f ? m : 1.0f;
    reinterpret_cast<float *>(b + 24 * S)[l] = nrm;
    const float inv = 1.0f / nrm;
#pragma unroll
    for (int k = 0; k < 24; k++) b[k * S + l] = __float2half_rn(v[k] * inv);
  }
};

// y = a x + b y over nblk blocks (16-byte aligned fields), 256 threads
template <int S>
__global__ void __launch_bounds__(256) axpby_f16n_tile_kernel(long long nblk, ScalarRef a,
                                                              const __half *__restrict__ x, ScalarRef b,
                                                              __half *__restrict__ y)
{
  typedef F16NTile<S> T;
  __shared__ __align__(16) unsigned char sm[8][2][T::BYTES];
  const float av = (float)a.get(), bv = (float)b.get();
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const long long ntile = (nblk + T::G - 1) / T::G;
  for (long long t = blockIdx.x * 8LL + wp; t < ntile; t += gridDim.x * 8LL) {
    const long long blk0 = t * T::G;
    T::load(x, blk0, nblk, sm[wp][0], ln);
    T::load(y, blk0, nblk, sm[wp][1], ln);
    __syncwarp();
    if (blk0 + ln / S < nblk) {
      float vx[24], vy[24];
      T::get(sm[wp][0], ln, vx);
      T::get(sm[wp][1], ln, vy);
#pragma unroll
      for (int k = 0; k < 24; k++) vy[k] = av * vx[k] + bv * vy[k];
      T::put(sm[wp][1], ln, vy);
    }
    __syncwarp();
    T::store(y, blk0, nblk, sm[wp][1], ln);
    __syncwarp();
  }
}

// real dot partials over nblk blocks (16-byte aligned fields); each site's
// 24 terms in FP32, the sites in FP64; kRedThreads threads
template <int S>
__global__ void __launch_bounds__(kRedThreads) dot_f16n_tile_kernel(long long nblk, const __half *__restrict__ x,
                                                                    const __half *__restrict__ y,
                                                                    double *__restrict__ partials)
{
  typedef F16NTile<S> T;
  constexpr int W = kRedThreads / 32;
  __shared__ __align__(16) unsigned char sm[W][2][T::BYTES];
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const long long ntile = (nblk + T::G - 1) / T::G;
  double re = 0.0, im = 0.0;
  for (long long t = blockIdx.x * (long long)W + wp; t < ntile; t += (long long)gridDim.x * W) {
    const long long blk0 = t * T::G;
    T::load(x, blk0, nblk, sm[wp][0], ln);
    T::load(y, blk0, nblk, sm[wp][1], ln);
    __syncwarp();
    if (blk0 + ln / S < nblk) {
      float vx[24], vy[24];
      T::get(sm[wp][0], ln, vx);
      T::get(sm[wp][1], ln, vy);
      float sr = 0.f;
#pragma unroll
      for (int k = 0; k < 24; k++) sr += vx[k] * vy[k];
      re += (double)sr;
    }
    __syncwarp();
  }
  block_sum2(re, im);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = re;
    partials[kRedBlocks + blockIdx.x] = im;
  }
}

// y = a x + b y
template <int S>
__global__ void __launch_bounds__(256) axpby_f16n_kernel(long long nsl, ScalarRef a, const __half *__restrict__ x,
                                                         ScalarRef b, __half *__restrict__ y)
{
  const float av = (float)a.get(), bv = (float)b.get();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsl;
       i += (long long)gridDim.x * blockDim.x) {
    float vx[24], vy[24];
    F16NSiteF<S>::load(x, i, vx);
    F16NSiteF<S>::load(y, i, vy);
#pragma unroll
    for (int k = 0; k < 24; k++) vy[k] = av * vx[k] + bv * vy[k];
    F16NSiteF<S>::store(y, i, vy);
  }
}

// complex y = a x + b y (components 2j, 2j+1 are re, im)
template <int S>
__global__ void __launch_bounds__(256) caxpby_f16n_kernel(long long nsl, double ar, double ai,
                                                          const __half *__restrict__ x, double br, double bi,
                                                          __half *__restrict__ y)
{
  const float fr = (float)ar, fi = (float)ai, gr = (float)br, gi = (float)bi;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsl;
       i += (long long)gridDim.x * blockDim.x) {
    float vx[24], vy[24];
    F16NSiteF<S>::load(x, i, vx);
    F16NSiteF<S>::load(y, i, vy);
#pragma unroll
    for (int j = 0; j < 12; j++) {
      const float xr = vx[2 * j], xi = vx[2 * j + 1], yr = vy[2 * j], yi = vy[2 * j + 1];
      vy[2 * j] = fr * xr - fi * xi + gr * yr - gi * yi;
      vy[2 * j + 1] = fr * xi + fi * xr + gr * yi + gi * yr;
    }
    F16NSiteF<S>::store(y, i, vy);
  }
}

// partials: real dot (CPLX = false) or complex <x, y> (CPLX = true); each
// site's 24 terms are summed in FP32, the sites in FP64
template <int S, bool CPLX>
__global__ void __launch_bounds__(kRedThreads) dot_f16n_partial_kernel(long long nsl, const __half *__restrict__ x,
                                                                       const __half *__restrict__ y,
                                                                       double *__restrict__ partials)
{
  double re = 0.0, im = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsl;
       i += (long long)gridDim.x * blockDim.x) {
    float vx[24], vy[24];
    F16NSiteF<S>::load(x, i, vx);
    F16NSiteF<S>::load(y, i, vy);
    float sr = 0.f, si = 0.f;
    if (CPLX) {
#pragma unroll
      for (int j = 0; j < 12; j++) {
        sr += vx[2 * j] * vy[2 * j] + vx[2 * j + 1] * vy[2 * j + 1];
        si += vx[2 * j] * vy[2 * j + 1] - vx[2 * j + 1] * vy[2 * j];
      }
    } else {
#pragma unroll
      for (int k = 0; k < 24; k++) sr += vx[k] * vy[k];
    }
    re += (double)sr;
    im += (double)si;
  }
  block_sum2(re, im);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = re;
    partials[kRedBlocks + blockIdx.x] = im;
  }
}

// between F16N and a plain storage type FP (24*S elements per block)
template <int S, typename FP, bool TO_F16N>
__global__ void __launch_bounds__(256) convert_f16n_kernel(long long nsl, double scale, const void *__restrict__ in,
                                                           void *__restrict__ out)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsl;
       i += (long long)gridDim.x * blockDim.x) {
    const long long blk = i / S;
    const int l = (int)(i - blk * S);
    double v[24];
    if (TO_F16N) {
      const FP *p = reinterpret_cast<const FP *>(in) + blk * 24 * S + l;
#pragma unroll
      for (int k = 0; k < 24; k++) v[k] = scale * to_d(p[k * S]);
      F16NSite<S>::store(reinterpret_cast<__half *>(out), i, v);
    } else {
      F16NSite<S>::load(reinterpret_cast<const __half *>(in), i, v);
      FP *p = reinterpret_cast<FP *>(out) + blk * 24 * S + l;
#pragma unroll
      for (int k = 0; k < 24; k++) p[k * S] = from_d<FP>(scale * v[k]);
    }
  }
}

} // namespace qb200
