// qb200_device.cuh -- device-side building blocks of the dslash kernels.
//
// Per-site algebra of the operator family that qphix-codegen generates
// (codegen/dslash_common.cc), written for one CUDA thread per lattice site
// with FP32 (FP64 for double storage) arithmetic in registers.  The spin
// tables of the reference are folded into compile-time structure plus two
// run-time signs, so that isign = +1 and -1 (and the +beta / -beta forms)
// share one instruction stream:
//   - proj_ops_minus[d] == proj_ops_plus[d^1] == proj_ops_plus[d] with the
//     second operand negated (dslash_common.cc:748-766), so the projection is
//     b = psi[a] + sigma * sgn[d][s] * op(psi[b]), sigma = +1 (plus) / -1;
//   - rec_minus_*beta == rec_plus_*beta with the spin-2/3 terms negated
//     (dslash_common.cc:784-890); the table is rec_plus for (isPlus xor fwd),
//     (dslash_common.cc:1771-1787), tau = +1 / -1 selects it;
//   - *_mbeta == *_pbeta with beta -> -beta, folded into the coefficient.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace qb200 {

// operator families
enum { FAM_WILSON = 0, FAM_CLOVER = 1, FAM_TM = 2, FAM_TMCLOV = 3 };

// ---------------------------------------------------------------------
// storage traits.  FT names the storage format, E the element type in
// memory, C the arithmetic type; SPB is the number of E elements per site
// lane of a spinor block (24, or 26 when two extra halves hold the site's
// FP32 norm) and FACE the elements per face site.  ld reads global memory
// through the read-only path, cv converts an element already loaded (from
// shared memory, say).

// FP16 spinors scaled by a per-site FP32 norm (links and clover plain FP16):
// block = FT[3][4][2][S] halves followed by float norm[S].  WIDE_ONLY types
// are built for SOALEN 4, 8 and 16 only.
struct half_norm {};

template <typename FT> struct ftraits;
template <> struct ftraits<float> {
  typedef float E;
  typedef float C;
  static constexpr int SPB = 24, FACE = 12;
  static constexpr bool WIDE_ONLY = false;
  static __device__ __forceinline__ float ld(const float *p) { return __ldg(p); }
  static __device__ __forceinline__ float cv(float v) { return v; }
  static __device__ __forceinline__ void st(float *p, float v) { *p = v; }
};
template <> struct ftraits<double> {
  typedef double E;
  typedef double C;
  static constexpr int SPB = 24, FACE = 12;
  static constexpr bool WIDE_ONLY = false;
  static __device__ __forceinline__ double ld(const double *p) { return __ldg(p); }
  static __device__ __forceinline__ double cv(double v) { return v; }
  static __device__ __forceinline__ void st(double *p, double v) { *p = v; }
};
template <> struct ftraits<__half> {
  typedef __half E;
  typedef float C;
  static constexpr int SPB = 24, FACE = 12;
  static constexpr bool WIDE_ONLY = false;
  static __device__ __forceinline__ float ld(const __half *p) { return __half2float(__ldg(p)); }
  static __device__ __forceinline__ float cv(__half v) { return __half2float(v); }
  static __device__ __forceinline__ void st(__half *p, float v) { *p = __float2half_rn(v); }
};
template <> struct ftraits<__nv_bfloat16> {
  typedef __nv_bfloat16 E;
  typedef float C;
  static constexpr int SPB = 24, FACE = 12;
  static constexpr bool WIDE_ONLY = true;
  static __device__ __forceinline__ float ld(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }
  static __device__ __forceinline__ float cv(__nv_bfloat16 v) { return __bfloat162float(v); }
  static __device__ __forceinline__ void st(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }
};
template <> struct ftraits<half_norm> {
  typedef __half E;
  typedef float C;
  static constexpr int SPB = 26, FACE = 14;
  static constexpr bool WIDE_ONLY = true;
  static __device__ __forceinline__ float ld(const __half *p) { return __half2float(__ldg(p)); }
  static __device__ __forceinline__ float cv(__half v) { return __half2float(v); }
  static __device__ __forceinline__ void st(__half *p, float v) { *p = __float2half_rn(v); }
};

template <typename FT> using elem_t = typename ftraits<FT>::E;
template <typename FT> using comp_t = typename ftraits<FT>::C;

template <typename C> struct cx {
  C re, im;
};

template <typename C> __device__ __forceinline__ cx<C> mk(C r, C i)
{
  cx<C> z;
  z.re = r;
  z.im = i;
  return z;
}

// ---------------------------------------------------------------------
// lattice geometry (see include/qphix_b200.h for the layout)

struct GeoDev {
  int nx, ny, nz, nt;
  int nxh, nvecs, ngy, nyg, V;
  long long Pxy, Pxyz;
  int nsites; // nxh*ny*nz*nt
  int nrhs;   // right-hand sides interleaved innermost (multi-RHS layout), else 1
};

// run-time operator parameters, arithmetic type C
template <typename C> struct OpDev {
  C beta[8];    // hop coefficient per direction (negated for achimbdpsi)
  C tbound;     // time-boundary factor
  C alpha, mu, muinv, rho;
  C tbc[4][2];  // twisted boundary phases
  unsigned tbc_mask;
  unsigned acc_mask; // bit d: accumulate every hop in d (else skip crossing hops)
  int isPlus;
  int cb;
  int t_edge_lo, t_edge_hi;
};

// ---------------------------------------------------------------------
// compile-time spin tables (isPlus orientation)

// projector spin pairs: x,y use (0,3),(1,2); z,t use (0,2),(1,3)
__host__ __device__ constexpr int proj_b(int d, int s) { return (d < 4) ? (s == 0 ? 3 : 2) : (s == 0 ? 2 : 3); }
// second operand multiplied by i for x and z
__host__ __device__ constexpr bool proj_i(int d) { return d == 0 || d == 1 || d == 4 || d == 5; }
// sign of the second operand, proj_ops_plus (dslash_common.cc:748-756)
__host__ __device__ constexpr int proj_sg(int d, int s)
{
  return (d == 0) ? 1 : (d == 1) ? -1 : (d == 2) ? (s == 0 ? -1 : 1) : (d == 3) ? (s == 0 ? 1 : -1)
       : (d == 4) ? (s == 0 ? 1 : -1) : (d == 5) ? (s == 0 ? -1 : 1) : (d == 6) ? 1 : -1;
}
// reconstruction, rec_plus_pbeta (dslash_common.cc:784-812): half-spinor row
// that feeds spin 2 (the other feeds spin 3), i-type, and signs of F1/F2
__host__ __device__ constexpr int rec_s2(int mu) { return mu < 2 ? 1 : 0; }
__host__ __device__ constexpr bool rec_i(int mu) { return mu == 0 || mu == 2; }
__host__ __device__ constexpr int rec_sg2(int mu) { return (mu == 0 || mu == 2) ? -1 : 1; }
__host__ __device__ constexpr int rec_sg3(int mu) { return (mu == 0 || mu == 1) ? -1 : 1; }

// ---------------------------------------------------------------------
// neighbour coordinates

struct Site {
  int xcb, y, z, t, par;
};

__device__ __forceinline__ Site site_of(const GeoDev &g, int i, int cb)
{
  Site s;
  s.xcb = i % g.nxh;
  int r = i / g.nxh;
  s.y = r % g.ny;
  r /= g.ny;
  s.z = r % g.nz;
  s.t = r / g.nz;
  s.par = (s.y + s.z + s.t + cb) & 1;
  return s;
}

// neighbour of site s in direction D; *cross = the hop leaves the local lattice
template <int D>
__device__ __forceinline__ Site neighbour(const GeoDev &g, const Site &s, bool *cross)
{
  Site n = s;
  if (D == 0) {
    *cross = (s.par == 0) && (s.xcb == 0);
    if (s.par == 0) n.xcb = (s.xcb == 0) ? g.nxh - 1 : s.xcb - 1;
  } else if (D == 1) {
    *cross = (s.par == 1) && (s.xcb == g.nxh - 1);
    if (s.par == 1) n.xcb = (s.xcb == g.nxh - 1) ? 0 : s.xcb + 1;
  } else if (D == 2) {
    *cross = s.y == 0;
    n.y = (s.y == 0) ? g.ny - 1 : s.y - 1;
  } else if (D == 3) {
    *cross = s.y == g.ny - 1;
    n.y = (s.y == g.ny - 1) ? 0 : s.y + 1;
  } else if (D == 4) {
    *cross = s.z == 0;
    n.z = (s.z == 0) ? g.nz - 1 : s.z - 1;
  } else if (D == 5) {
    *cross = s.z == g.nz - 1;
    n.z = (s.z == g.nz - 1) ? 0 : s.z + 1;
  } else if (D == 6) {
    *cross = s.t == 0;
    n.t = (s.t == 0) ? g.nt - 1 : s.t - 1;
  } else {
    *cross = s.t == g.nt - 1;
    n.t = (s.t == g.nt - 1) ? 0 : s.t + 1;
  }
  return n;
}

// element index of component 0 of the site in a spinor field (add
// ((c*4+s)*2+ri)*S for component (c,s,ri))
template <typename FT, int S>
__device__ __forceinline__ long long spinor_base(const GeoDev &g, const Site &s)
{
  long long blk = s.t * g.Pxyz + s.z * g.Pxy + (long long)s.y * g.nvecs + s.xcb / S;
  return blk * (ftraits<FT>::SPB * S) + (s.xcb % S);
}

// tile index and lane of a site in the gauge / clover fields
template <int S>
__device__ __forceinline__ long long tile_of(const GeoDev &g, const Site &s, int *lane)
{
  int yq = s.y / g.ngy;
  *lane = (s.y - yq * g.ngy) * S + (s.xcb % S);
  return ((long long)(s.t * g.nz + s.z) * g.nyg + yq) * g.nvecs + s.xcb / S;
}

// ---------------------------------------------------------------------
// loads

template <typename FT, int S>
__device__ __forceinline__ void load_spinor(const elem_t<FT> *__restrict__ f, long long base,
                                            cx<comp_t<FT>> (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      sp[s][c].re = ftraits<FT>::ld(f + base + ((c * 4 + s) * 2 + 0) * S);
      sp[s][c].im = ftraits<FT>::ld(f + base + ((c * 4 + s) * 2 + 1) * S);
    }
  if (ftraits<FT>::SPB == 26) {
    // the lane's norm: float at half offset block*26S + 24S + 2*lane = base + 24S + lane
    const float nrm = __ldg(reinterpret_cast<const float *>(f + base + 24 * S + (base % S)));
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 4; s++) {
        sp[s][c].re *= nrm;
        sp[s][c].im *= nrm;
      }
  }
}

template <typename FT, int S>
__device__ __forceinline__ void store_spinor(elem_t<FT> *__restrict__ f, long long base,
                                             const cx<comp_t<FT>> (&sp)[4][3])
{
  typedef comp_t<FT> C;
  C scale = (C)1;
  if (ftraits<FT>::SPB == 26) {
    C m = 0;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 4; s++) m = fmax(m, fmax(fabs(sp[s][c].re), fabs(sp[s][c].im)));
    const C nrm = m > (C)0 ? m : (C)1;
    *reinterpret_cast<float *>(f + base + 24 * S + (base % S)) = (float)nrm;
    scale = (C)1 / nrm;
  }
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      ftraits<FT>::st(f + base + ((c * 4 + s) * 2 + 0) * S, sp[s][c].re * scale);
      ftraits<FT>::st(f + base + ((c * 4 + s) * 2 + 1) * S, sp[s][c].im * scale);
    }
}

// multi-RHS layout: block = FT[3][4][2][S][nrhs] (no per-site norms);
// component k of lane l, right-hand side r at blk*24*S*nrhs + k*S*nrhs + l*nrhs + r
template <int S>
__device__ __forceinline__ long long spinor_base_mr(const GeoDev &g, const Site &s, int r)
{
  long long blk = s.t * g.Pxyz + s.z * g.Pxy + (long long)s.y * g.nvecs + s.xcb / S;
  return (blk * (24 * S) + (s.xcb % S)) * g.nrhs + r;
}

template <typename FT>
__device__ __forceinline__ void load_spinor_rs(const elem_t<FT> *__restrict__ f, long long base, int cs,
                                               cx<comp_t<FT>> (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      sp[s][c].re = ftraits<FT>::ld(f + base + (long long)((c * 4 + s) * 2 + 0) * cs);
      sp[s][c].im = ftraits<FT>::ld(f + base + (long long)((c * 4 + s) * 2 + 1) * cs);
    }
}

template <typename FT>
__device__ __forceinline__ void store_spinor_rs(elem_t<FT> *__restrict__ f, long long base, int cs,
                                                const cx<comp_t<FT>> (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      ftraits<FT>::st(f + base + (long long)((c * 4 + s) * 2 + 0) * cs, sp[s][c].re);
      ftraits<FT>::st(f + base + (long long)((c * 4 + s) * 2 + 1) * cs, sp[s][c].im);
    }
}

// third row of a 12-real link: G[2][c] = conj(G[0][c+1] G[1][c+2] -
// G[0][c+2] G[1][c+1]), in a fixed order of fused multiply-adds (every
// kernel uses this order, so all give the same bits)
template <typename C>
__device__ __forceinline__ void recon_row3(cx<C> (&G)[3][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
    C re = G[0][c1].re * G[1][c2].re;
    re = fma(-G[0][c1].im, G[1][c2].im, re);
    re = fma(-G[0][c2].re, G[1][c1].re, re);
    re = fma(G[0][c2].im, G[1][c1].im, re);
    C im = G[0][c1].re * G[1][c2].im;
    im = fma(G[0][c1].im, G[1][c2].re, im);
    im = fma(-G[0][c2].re, G[1][c1].im, im);
    im = fma(-G[0][c2].im, G[1][c1].re, im);
    G[2][c].re = re;
    G[2][c].im = -im;
  }
}

// stored link G (= U^T) of direction D; `base` = tile*(8*R*6*V) + lane
template <typename FT, bool COMP12, int D>
__device__ __forceinline__ void load_link(const elem_t<FT> *__restrict__ u, long long base, int V,
                                          cx<comp_t<FT>> (&G)[3][3])
{
  constexpr int R = COMP12 ? 2 : 3;
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      G[r][c].re = ftraits<FT>::ld(u + base + (long long)(((D * R + r) * 3 + c) * 2 + 0) * V);
      G[r][c].im = ftraits<FT>::ld(u + base + (long long)(((D * R + r) * 3 + c) * 2 + 1) * V);
    }
  if (COMP12) recon_row3(G);
}

// ---------------------------------------------------------------------
// one hop: project the neighbour, multiply by the link, apply the twisted
// boundary phase and reconstruct-accumulate into acc with coefficient beta

template <typename C, int D>
__device__ __forceinline__ void project(const cx<C> (&psi)[4][3], C sigma, cx<C> (&b)[2][3])
{
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const C sg = sigma * (C)proj_sg(D, s);
    const int bb = proj_b(D, s);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (proj_i(D)) { // a + sg*i*b
        b[s][c].re = fma(-sg, psi[bb][c].im, psi[s][c].re);
        b[s][c].im = fma(sg, psi[bb][c].re, psi[s][c].im);
      } else {
        b[s][c].re = fma(sg, psi[bb][c].re, psi[s][c].re);
        b[s][c].im = fma(sg, psi[bb][c].im, psi[s][c].im);
      }
    }
  }
}

template <typename C, bool ADJ>
__device__ __forceinline__ void mult_link(const cx<C> (&G)[3][3], const cx<C> (&b)[2][3], cx<C> (&ub)[2][3])
{
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c1 = 0; c1 < 3; c1++) {
      C re = 0, im = 0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        if (ADJ) { // conj(G[c1][k]) * b[k]
          const cx<C> g = G[c1][k];
          re = fma(g.re, b[s][k].re, re);
          re = fma(g.im, b[s][k].im, re);
          im = fma(g.re, b[s][k].im, im);
          im = fma(-g.im, b[s][k].re, im);
        } else { // G[k][c1] * b[k]
          const cx<C> g = G[k][c1];
          re = fma(g.re, b[s][k].re, re);
          re = fma(-g.im, b[s][k].im, re);
          im = fma(g.re, b[s][k].im, im);
          im = fma(g.im, b[s][k].re, im);
        }
      }
      ub[s][c1].re = re;
      ub[s][c1].im = im;
    }
}

template <typename C>
__device__ __forceinline__ void apply_phase(cx<C> (&ub)[2][3], C pr, C pi)
{
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      // explicit contraction order (the multi-RHS pair kernel repeats it)
      const C re = fma(-pi, ub[s][c].im, pr * ub[s][c].re);
      const C im = fma(pi, ub[s][c].re, pr * ub[s][c].im);
      ub[s][c].re = re;
      ub[s][c].im = im;
    }
}

// acc += beta * recons(ub), table rec_plus scaled by tau
template <typename C, int MU>
__device__ __forceinline__ void recons(const cx<C> (&ub)[2][3], C beta, C tau, cx<C> (&acc)[4][3])
{
  const C b2 = beta * tau * (C)rec_sg2(MU);
  const C b3 = beta * tau * (C)rec_sg3(MU);
  constexpr int s2 = rec_s2(MU), s3 = 1 - rec_s2(MU);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[0][c].re = fma(beta, ub[0][c].re, acc[0][c].re);
    acc[0][c].im = fma(beta, ub[0][c].im, acc[0][c].im);
    acc[1][c].re = fma(beta, ub[1][c].re, acc[1][c].re);
    acc[1][c].im = fma(beta, ub[1][c].im, acc[1][c].im);
    if (rec_i(MU)) { // += b * i * ub
      acc[2][c].re = fma(-b2, ub[s2][c].im, acc[2][c].re);
      acc[2][c].im = fma(b2, ub[s2][c].re, acc[2][c].im);
      acc[3][c].re = fma(-b3, ub[s3][c].im, acc[3][c].re);
      acc[3][c].im = fma(b3, ub[s3][c].re, acc[3][c].im);
    } else {
      acc[2][c].re = fma(b2, ub[s2][c].re, acc[2][c].re);
      acc[2][c].im = fma(b2, ub[s2][c].im, acc[2][c].im);
      acc[3][c].re = fma(b3, ub[s3][c].re, acc[3][c].re);
      acc[3][c].im = fma(b3, ub[s3][c].im, acc[3][c].im);
    }
  }
}

// ---------------------------------------------------------------------
// clover-type terms

// Clover arithmetic, shared by every kernel (the same operations in the same
// order everywhere, so that all kernels give the same bits).
//
// Row r of a 6x6 block is summed in two chains -- for the Hermitian
// CloverBlock the diagonal and lower-triangle terms (c < r) in one and the
// upper-triangle terms (c > r) in the other, for the dense FullCloverBlock
// columns 0-2 and 3-5 -- which are added at the end.  Shorter chains round
// less than one running sum; it matters in A.chi - b.D.psi, where the clover
// term and the hops can cancel to a result several times smaller than both.
// MODE_SET: out = row; MODE_ADD: out = out + row (one more rounding).  RHO:
// the row first gets + i rhob in[r] (the i rho g5 chi term of the
// achimbdpsi form, rhob = +/- rho per block, dslash_common.cc:1873-1906).
enum { MODE_SET = 0, MODE_ADD = 1 };

// the Hermitian block `blk` from its packed elements: dg[6] real diagonal,
// od[r(r-1)/2+c] = A[r][c] for r > c, A[c][r] = conj(A[r][c])
// (dslash_common.cc:1098-1186)
template <typename C, int MODE, bool RHO>
__device__ __forceinline__ void herm_apply(const C (&dg)[6], const cx<C> (&od)[15], int blk, C rhob,
                                           const cx<C> (&in)[4][3], cx<C> (&out)[4][3])
{
#pragma unroll
  for (int r = 0; r < 6; r++) {
    const cx<C> v = in[2 * blk + r / 3][r % 3];
    C re1 = dg[r] * v.re, im1 = dg[r] * v.im;
    C re2 = 0, im2 = 0;
#pragma unroll
    for (int c = 0; c < 6; c++) {
      if (c == r) continue;
      const cx<C> w = in[2 * blk + c / 3][c % 3];
      if (c < r) { // A[r][c] = od[r(r-1)/2+c]
        const cx<C> a = od[r * (r - 1) / 2 + c];
        re1 = fma(a.re, w.re, re1);
        re1 = fma(-a.im, w.im, re1);
        im1 = fma(a.re, w.im, im1);
        im1 = fma(a.im, w.re, im1);
      } else { // A[r][c] = conj(od[c(c-1)/2+r])
        const cx<C> a = od[c * (c - 1) / 2 + r];
        re2 = fma(a.re, w.re, re2);
        re2 = fma(a.im, w.im, re2);
        im2 = fma(a.re, w.im, im2);
        im2 = fma(-a.im, w.re, im2);
      }
    }
    C re = re1 + re2, im = im1 + im2;
    if (RHO) {
      re = fma(-rhob, v.im, re);
      im = fma(rhob, v.re, im);
    }
    cx<C> &o = out[2 * blk + r / 3][r % 3];
    if (MODE == MODE_ADD) {
      o.re = o.re + re;
      o.im = o.im + im;
    } else {
      o.re = re;
      o.im = im;
    }
  }
}

// the dense block `blk`; ld(r, c) returns element (r, c)
// (dslash_common.cc:1188-1232)
template <typename C, int MODE, bool RHO, typename LD>
__device__ __forceinline__ void dense_apply(LD ld, int blk, C rhob, const cx<C> (&in)[4][3], cx<C> (&out)[4][3])
{
#pragma unroll
  for (int r = 0; r < 6; r++) {
    C re1 = 0, im1 = 0, re2 = 0, im2 = 0;
#pragma unroll
    for (int c = 0; c < 6; c++) {
      const cx<C> a = ld(r, c);
      const cx<C> w = in[2 * blk + c / 3][c % 3];
      if (c < 3) {
        re1 = fma(a.re, w.re, re1);
        re1 = fma(-a.im, w.im, re1);
        im1 = fma(a.re, w.im, im1);
        im1 = fma(a.im, w.re, im1);
      } else {
        re2 = fma(a.re, w.re, re2);
        re2 = fma(-a.im, w.im, re2);
        im2 = fma(a.re, w.im, im2);
        im2 = fma(a.im, w.re, im2);
      }
    }
    C re = re1 + re2, im = im1 + im2;
    if (RHO) {
      const cx<C> v = in[2 * blk + r / 3][r % 3];
      re = fma(-rhob, v.im, re);
      im = fma(rhob, v.re, im);
    }
    cx<C> &o = out[2 * blk + r / 3][r % 3];
    if (MODE == MODE_ADD) {
      o.re = o.re + re;
      o.im = o.im + im;
    } else {
      o.re = re;
      o.im = im;
    }
  }
}

// the rho of block blk with its sign: + i rho g5 for plus, - for minus
template <typename C> __device__ __forceinline__ C rho_of_block(int blk, int isPlus, C rho)
{
  return ((isPlus != 0) != (blk == 1)) ? rho : -rho;
}

// out (MODE) A in, A the Hermitian CloverBlock block `blk` read from global
// memory; base = tile*72*V + lane
template <typename FT, int MODE, bool RHO>
__device__ __forceinline__ void clover_block(const elem_t<FT> *__restrict__ cl, long long base, int V, int blk,
                                             typename ftraits<FT>::C rhob,
                                             const cx<typename ftraits<FT>::C> (&in)[4][3],
                                             cx<typename ftraits<FT>::C> (&out)[4][3])
{
  typedef typename ftraits<FT>::C C;
  const elem_t<FT> *p = cl + base + (long long)blk * 36 * V;
  C dg[6];
  cx<C> od[15];
#pragma unroll
  for (int i = 0; i < 6; i++) dg[i] = ftraits<FT>::ld(p + (long long)i * V);
#pragma unroll
  for (int i = 0; i < 15; i++) {
    od[i].re = ftraits<FT>::ld(p + (long long)(6 + 2 * i) * V);
    od[i].im = ftraits<FT>::ld(p + (long long)(7 + 2 * i) * V);
  }
  herm_apply<C, MODE, RHO>(dg, od, blk, rhob, in, out);
}

// out (MODE) F in, F a dense FullCloverBlock block read from global memory;
// base = tile*144*V + lane
template <typename FT, int MODE, bool RHO>
__device__ __forceinline__ void full_clover_block(const elem_t<FT> *__restrict__ cl, long long base, int V, int blk,
                                                  typename ftraits<FT>::C rhob,
                                                  const cx<typename ftraits<FT>::C> (&in)[4][3],
                                                  cx<typename ftraits<FT>::C> (&out)[4][3])
{
  typedef typename ftraits<FT>::C C;
  const elem_t<FT> *p = cl + base + (long long)blk * 72 * V;
  dense_apply<C, MODE, RHO>(
      [&](int r, int c) {
        return mk<C>(ftraits<FT>::ld(p + (long long)((r * 6 + c) * 2 + 0) * V),
                     ftraits<FT>::ld(p + (long long)((r * 6 + c) * 2 + 1) * V));
      },
      blk, rhob, in, out);
}

// res (+)= muinv (1 + sg i mu) in, sg = -1 on the upper spins for plus
// (inverse_twisted_term, dslash_common.cc:1234-1359)
template <typename C, bool ACC>
__device__ __forceinline__ void inv_twisted(const cx<C> (&in)[4][3], int isPlus, C mu, C muinv,
                                            cx<C> (&res)[4][3])
{
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const C sg = ((s < 2) == (isPlus != 0)) ? (C)-1 : (C)1;
    const C m = sg * mu;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const C tre = fma(-m, in[s][c].im, in[s][c].re);
      const C tim = fma(m, in[s][c].re, in[s][c].im);
      if (ACC) {
        res[s][c].re = fma(muinv, tre, res[s][c].re);
        res[s][c].im = fma(muinv, tim, res[s][c].im);
      } else {
        res[s][c].re = muinv * tre;
        res[s][c].im = muinv * tim;
      }
    }
  }
}

} // namespace qb200
