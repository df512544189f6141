// qb200_site2_kernel.cuh -- the single-RHS dslash with two neighbouring
// sites per thread in packed FP32x2 arithmetic.
//
// Sites xcb = 2j and 2j+1 of one row sit in lanes l, l+1 (l even) of the
// same spinor block and of the same link / clover tile, so every field
// element of the pair is one 8-byte (FP32) or 4-byte (16-bit) load, and the
// two sites' arithmetic runs as FFMA2 on (site 2j, site 2j+1) pairs with no
// broadcast operands.  The two sites share y, z, t and parity, hence the
// y / z / t neighbours (a pair at the same lanes), the time-boundary factor,
// the twisted phases and the spin tables; their x neighbours are shifted by
// one lane when the parity says so, and are then read element by element.
// The operations and their order per site are those of site_body.
// FP32, FP16, FP16 + norm and BF16 storage (FP32 arithmetic), SOALEN >= 2.
#pragma once

#include <cuda_bf16.h>

#include "qb200_pair_kernel.cuh"

namespace qb200 {

template <typename FT> struct io2;
template <> struct io2<float> {
  static __device__ __forceinline__ float2 ld(const float *p) { return __ldg(reinterpret_cast<const float2 *>(p)); }
  static __device__ __forceinline__ void st(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
  static __device__ __forceinline__ float ld1(const float *p) { return __ldg(p); }
};
template <> struct io2<__half> {
  static __device__ __forceinline__ float2 ld(const __half *p)
  {
    return __half22float2(__ldg(reinterpret_cast<const __half2 *>(p)));
  }
  static __device__ __forceinline__ void st(__half *p, float2 v)
  {
    *reinterpret_cast<__half2 *>(p) = __float22half2_rn(v);
  }
  static __device__ __forceinline__ float ld1(const __half *p) { return __half2float(__ldg(p)); }
};
template <> struct io2<half_norm> : io2<__half> {};
template <> struct io2<__nv_bfloat16> {
  static __device__ __forceinline__ float2 ld(const __nv_bfloat16 *p)
  {
    return __bfloat1622float2(__ldg(reinterpret_cast<const __nv_bfloat162 *>(p)));
  }
  static __device__ __forceinline__ void st(__nv_bfloat16 *p, float2 v)
  {
    *reinterpret_cast<__nv_bfloat162 *>(p) = __float22bfloat162_rn(v);
  }
  static __device__ __forceinline__ float ld1(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }
};

// spinor of the pair at lanes (l, l+1); base = block*SPB*S + l, l even
template <typename FT, int S>
__device__ __forceinline__ void load_spinor2(const elem_t<FT> *__restrict__ f, long long base, c2 (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      sp[s][c].re = io2<FT>::ld(f + base + ((c * 4 + s) * 2 + 0) * S);
      sp[s][c].im = io2<FT>::ld(f + base + ((c * 4 + s) * 2 + 1) * S);
    }
  if (ftraits<FT>::SPB == 26) {
    const float2 nrm = __ldg(reinterpret_cast<const float2 *>(f + base + 24 * S + (base % S)));
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 4; s++) {
        sp[s][c].re = f2mul(sp[s][c].re, nrm);
        sp[s][c].im = f2mul(sp[s][c].im, nrm);
      }
  }
}

// two sites at arbitrary element bases ea, eb (the shifted x neighbours)
template <typename FT, int S>
__device__ __forceinline__ void load_spinor_split(const elem_t<FT> *__restrict__ f, long long ea, long long eb,
                                                  c2 (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const int kr = ((c * 4 + s) * 2 + 0) * S, ki = ((c * 4 + s) * 2 + 1) * S;
      sp[s][c].re = make_float2(io2<FT>::ld1(f + ea + kr), io2<FT>::ld1(f + eb + kr));
      sp[s][c].im = make_float2(io2<FT>::ld1(f + ea + ki), io2<FT>::ld1(f + eb + ki));
    }
  if (ftraits<FT>::SPB == 26) {
    const float2 nrm = make_float2(__ldg(reinterpret_cast<const float *>(f + ea + 24 * S + (ea % S))),
                                   __ldg(reinterpret_cast<const float *>(f + eb + 24 * S + (eb % S))));
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 4; s++) {
        sp[s][c].re = f2mul(sp[s][c].re, nrm);
        sp[s][c].im = f2mul(sp[s][c].im, nrm);
      }
  }
}

// store_spinor for the pair (per-site norms for FP16 + norm)
template <typename FT, int S>
__device__ __forceinline__ void store_spinor2(elem_t<FT> *__restrict__ f, long long base, const c2 (&sp)[4][3])
{
  float2 scale = make_float2(1.f, 1.f);
  if (ftraits<FT>::SPB == 26) {
    float ma = 0.f, mb = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 4; s++) {
        ma = fmaxf(ma, fmaxf(fabsf(sp[s][c].re.x), fabsf(sp[s][c].im.x)));
        mb = fmaxf(mb, fmaxf(fabsf(sp[s][c].re.y), fabsf(sp[s][c].im.y)));
      }
    const float na = ma > 0.f ? ma : 1.f, nb = mb > 0.f ? mb : 1.f;
    *reinterpret_cast<float2 *>(f + base + 24 * S + (base % S)) = make_float2(na, nb);
    scale = make_float2(1.f / na, 1.f / nb);
  }
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const float2 re = ftraits<FT>::SPB == 26 ? f2mul(sp[s][c].re, scale) : sp[s][c].re;
      const float2 im = ftraits<FT>::SPB == 26 ? f2mul(sp[s][c].im, scale) : sp[s][c].im;
      io2<FT>::st(f + base + ((c * 4 + s) * 2 + 0) * S, re);
      io2<FT>::st(f + base + ((c * 4 + s) * 2 + 1) * S, im);
    }
}

// link pair of direction D (lanes l, l+1 of the tile); recon_row3's order
template <typename FT, bool COMP12, int D>
__device__ __forceinline__ void load_link2(const elem_t<FT> *__restrict__ u, long long base, int V, c2 (&G)[3][3])
{
  constexpr int R = COMP12 ? 2 : 3;
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      G[r][c].re = io2<FT>::ld(u + base + (long long)(((D * R + r) * 3 + c) * 2 + 0) * V);
      G[r][c].im = io2<FT>::ld(u + base + (long long)(((D * R + r) * 3 + c) * 2 + 1) * V);
    }
  if (COMP12) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int c1 = (c + 1) % 3, c2i = (c + 2) % 3;
      const c2 a = G[0][c1], b = G[1][c2i], d = G[0][c2i], e = G[1][c1];
      float2 re = f2mul(a.re, b.re);
      re = f2fma(f2mul(bc(-1.f), a.im), b.im, re);
      re = f2fma(f2mul(bc(-1.f), d.re), e.re, re);
      re = f2fma(d.im, e.im, re);
      float2 im = f2mul(a.re, b.im);
      im = f2fma(a.im, b.re, im);
      im = f2fma(f2mul(bc(-1.f), d.re), e.im, im);
      im = f2fma(f2mul(bc(-1.f), d.im), e.re, im);
      G[2][c].re = re;
      G[2][c].im = f2mul(bc(-1.f), im);
    }
  }
}

// ub = G^T b (forward) or conj(G) b (backward), per site; mult_link's order
template <bool ADJ>
__device__ __forceinline__ void mult2p(const c2 (&G)[3][3], const c2 (&b)[2][3], c2 (&ub)[2][3])
{
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c1 = 0; c1 < 3; c1++) {
      float2 re, im;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const c2 g = ADJ ? G[c1][k] : G[k][c1];
        const float2 gin = f2mul(bc(-1.f), g.im);
        if (k == 0) {
          re = f2mul(g.re, b[s][k].re);
          im = f2mul(g.re, b[s][k].im);
        } else {
          re = f2fma(g.re, b[s][k].re, re);
          im = f2fma(g.re, b[s][k].im, im);
        }
        if (ADJ) { // conj(g) b
          re = f2fma(g.im, b[s][k].im, re);
          im = f2fma(gin, b[s][k].re, im);
        } else { // g b
          re = f2fma(gin, b[s][k].im, re);
          im = f2fma(g.im, b[s][k].re, im);
        }
      }
      ub[s][c1].re = re;
      ub[s][c1].im = im;
    }
}

// CloverBlock block `blk` of the pair (clover_block's operations)
template <typename FT>
__device__ __forceinline__ void clover2p(const elem_t<FT> *__restrict__ cl, long long base, int V, int blk,
                                         const c2 (&in)[4][3], c2 (&res)[4][3])
{
  const elem_t<FT> *p = cl + base + (long long)blk * 36 * V;
  float2 dg[6];
  c2 od[15];
#pragma unroll
  for (int i = 0; i < 6; i++) dg[i] = io2<FT>::ld(p + (long long)i * V);
#pragma unroll
  for (int i = 0; i < 15; i++) {
    od[i].re = io2<FT>::ld(p + (long long)(6 + 2 * i) * V);
    od[i].im = io2<FT>::ld(p + (long long)(7 + 2 * i) * V);
  }
#pragma unroll
  for (int r = 0; r < 6; r++) {
    const c2 v = in[2 * blk + r / 3][r % 3];
    float2 re = f2mul(dg[r], v.re), im = f2mul(dg[r], v.im);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      if (c == r) continue;
      const c2 w = in[2 * blk + c / 3][c % 3];
      const c2 a = r > c ? od[r * (r - 1) / 2 + c] : od[c * (c - 1) / 2 + r];
      const float2 ain = f2mul(bc(-1.f), a.im);
      re = f2fma(a.re, w.re, re);
      re = f2fma(r > c ? ain : a.im, w.im, re);
      im = f2fma(a.re, w.im, im);
      im = f2fma(r > c ? a.im : ain, w.re, im);
    }
    res[2 * blk + r / 3][r % 3].re = re;
    res[2 * blk + r / 3][r % 3].im = im;
  }
}

// FullCloverBlock block `blk` of the pair (full_clover_block's operations)
template <typename FT>
__device__ __forceinline__ void full_clover2p(const elem_t<FT> *__restrict__ cl, long long base, int V, int blk,
                                              const c2 (&in)[4][3], c2 (&res)[4][3])
{
  const elem_t<FT> *p = cl + base + (long long)blk * 72 * V;
#pragma unroll
  for (int r = 0; r < 6; r++) {
    float2 re = bc(0.f), im = bc(0.f);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      const float2 ar = io2<FT>::ld(p + (long long)((r * 6 + c) * 2 + 0) * V);
      const float2 ai = io2<FT>::ld(p + (long long)((r * 6 + c) * 2 + 1) * V);
      const c2 w = in[2 * blk + c / 3][c % 3];
      re = f2fma(ar, w.re, re);
      re = f2fma(f2mul(bc(-1.f), ai), w.im, re);
      im = f2fma(ar, w.im, im);
      im = f2fma(ai, w.re, im);
    }
    res[2 * blk + r / 3][r % 3].re = re;
    res[2 * blk + r / 3][r % 3].im = im;
  }
}

template <typename FT, int S, bool COMP12, int D, int VV>
__device__ __forceinline__ void hop2s(const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p, const Site &s0,
                                      const Site &s1, long long obase, long long gbase, c2 (&acc)[4][3])
{
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  const long long ue = (long long)ftraits<FT>::SPB * S;
  bool cross, cross1;
  const long long na = obase + neighbour_offset<S, D>(g, s0, ue, 1, &cross);
  c2 psi[4][3];
  if (MU == 0) {
    // x: the second site's neighbour separately (one lane over when shifted)
    const long long nb = obase + 1 + neighbour_offset<S, D>(g, s1, ue, 1, &cross1);
    if (nb == na + 1 && (na & 1) == 0) load_spinor2<FT, S>(a.psi, na, psi);
    else load_spinor_split<FT, S>(a.psi, na, nb, psi);
  } else {
    if (cross && !((p.acc_mask >> D) & 1u)) return;
    load_spinor2<FT, S>(a.psi, na, psi);
  }
  float beta = p.beta[D];
  if (D == 6 && s0.t == 0 && p.t_edge_lo) beta *= p.tbound;
  if (D == 7 && s0.t == g.nt - 1 && p.t_edge_hi) beta *= p.tbound;
  c2 b[2][3], ub[2][3], G[3][3];
  project2<D>(psi, p.isPlus ? 1.f : -1.f, b);
  load_link2<FT, COMP12, D>(a.gauge, gbase, vlen<VV>(g), G);
  mult2p<!FWD>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) phase2(ub, p.tbc[MU][0], FWD ? p.tbc[MU][1] : -p.tbc[MU][1]);
  recons2<MU>(ub, beta, ((p.isPlus != 0) != FWD) ? 1.f : -1.f, acc);
}

// Grid: blockIdx.y = the (z, t) plane, x covers the plane's site pairs.
// Needs accumulate on for both x directions (a skipped x hop would differ
// between the two sites) and 8-byte aligned fields.
template <typename FT, int S, bool COMP12, int FAM, bool ACH, int VV>
__global__ void __launch_bounds__(128, 3) site2_dslash_kernel(const KArgs<FT> a, const GeoDev g, const OpDev<float> p)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int hx = g.nxh >> 1;
  if (q >= hx * g.ny) return;
  Site s0;
  s0.z = blockIdx.y % g.nz;
  s0.t = blockIdx.y / g.nz;
  s0.y = q / hx;
  s0.xcb = 2 * (q - s0.y * hx);
  s0.par = (s0.y + s0.z + s0.t + p.cb) & 1;
  Site s1 = s0;
  s1.xcb = s0.xcb + 1;
  int lane;
  const long long tile = tile_of<S>(g, s0, &lane);
  constexpr int R = COMP12 ? 2 : 3;
  const int V = vlen<VV>(g);
  const long long gbase = tile * (8LL * R * 6 * V) + lane;
  const long long obase = spinor_base<FT, S>(g, s0);

  c2 res[4][3];
  if (ACH) {
    c2 ch[4][3];
    load_spinor2<FT, S>(a.chi, obase, ch);
    if (FAM == FAM_WILSON) {
#pragma unroll
      for (int sp = 0; sp < 4; sp++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          res[sp][c].re = f2mul(bc(p.alpha), ch[sp][c].re);
          res[sp][c].im = f2mul(bc(p.alpha), ch[sp][c].im);
        }
    } else if (FAM == FAM_TM) {
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        const float m = (((sp < 2) == (p.isPlus != 0)) ? 1.f : -1.f) * p.mu;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          res[sp][c].re = f2mul(bc(p.alpha), f2fma(bc(-m), ch[sp][c].im, ch[sp][c].re));
          res[sp][c].im = f2mul(bc(p.alpha), f2fma(bc(m), ch[sp][c].re, ch[sp][c].im));
        }
      }
    } else {
      const long long cbase = tile * ((FAM == FAM_CLOVER ? 72LL : 144LL) * V) + lane;
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        if (FAM == FAM_CLOVER) clover2p<FT>(a.clov, cbase, V, blk, ch, res);
        else full_clover2p<FT>(a.clov, cbase, V, blk, ch, res);
      }
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        const float r = (((p.isPlus != 0) != (sp >= 2)) ? 1.f : -1.f) * p.rho;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          res[sp][c].re = f2fma(bc(-r), ch[sp][c].im, res[sp][c].re);
          res[sp][c].im = f2fma(bc(r), ch[sp][c].re, res[sp][c].im);
        }
      }
    }
    hop2s<FT, S, COMP12, 0, VV>(a, g, p, s0, s1, obase, gbase, res);
    hop2s<FT, S, COMP12, 1, VV>(a, g, p, s0, s1, obase, gbase, res);
    hop2s<FT, S, COMP12, 2, VV>(a, g, p, s0, s1, obase, gbase, res);
    hop2s<FT, S, COMP12, 3, VV>(a, g, p, s0, s1, obase, gbase, res);
    hop2s<FT, S, COMP12, 4, VV>(a, g, p, s0, s1, obase, gbase, res);
    hop2s<FT, S, COMP12, 5, VV>(a, g, p, s0, s1, obase, gbase, res);
    hop2s<FT, S, COMP12, 6, VV>(a, g, p, s0, s1, obase, gbase, res);
    hop2s<FT, S, COMP12, 7, VV>(a, g, p, s0, s1, obase, gbase, res);
  } else {
    c2 acc[4][3];
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) acc[sp][c].re = acc[sp][c].im = bc(0.f);
    hop2s<FT, S, COMP12, 0, VV>(a, g, p, s0, s1, obase, gbase, acc);
    hop2s<FT, S, COMP12, 1, VV>(a, g, p, s0, s1, obase, gbase, acc);
    hop2s<FT, S, COMP12, 2, VV>(a, g, p, s0, s1, obase, gbase, acc);
    hop2s<FT, S, COMP12, 3, VV>(a, g, p, s0, s1, obase, gbase, acc);
    hop2s<FT, S, COMP12, 4, VV>(a, g, p, s0, s1, obase, gbase, acc);
    hop2s<FT, S, COMP12, 5, VV>(a, g, p, s0, s1, obase, gbase, acc);
    hop2s<FT, S, COMP12, 6, VV>(a, g, p, s0, s1, obase, gbase, acc);
    hop2s<FT, S, COMP12, 7, VV>(a, g, p, s0, s1, obase, gbase, acc);
    if (FAM == FAM_CLOVER || FAM == FAM_TMCLOV) {
      const long long cbase = tile * ((FAM == FAM_CLOVER ? 72LL : 144LL) * V) + lane;
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        if (FAM == FAM_CLOVER) clover2p<FT>(a.clov, cbase, V, blk, acc, res);
        else full_clover2p<FT>(a.clov, cbase, V, blk, acc, res);
      }
    } else if (FAM == FAM_TM) {
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        const float m = (((sp < 2) == (p.isPlus != 0)) ? -1.f : 1.f) * p.mu;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          res[sp][c].re = f2mul(bc(p.muinv), f2fma(bc(-m), acc[sp][c].im, acc[sp][c].re));
          res[sp][c].im = f2mul(bc(p.muinv), f2fma(bc(m), acc[sp][c].re, acc[sp][c].im));
        }
      }
    } else {
#pragma unroll
      for (int sp = 0; sp < 4; sp++)
#pragma unroll
        for (int c = 0; c < 3; c++) res[sp][c] = acc[sp][c];
    }
  }
  store_spinor2<FT, S>(a.out, obase, res);
}

} // namespace qb200
