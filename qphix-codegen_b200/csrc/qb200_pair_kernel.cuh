// qb200_pair_kernel.cuh -- multi-RHS dslash with two right-hand sides per
// thread in packed FP32x2 arithmetic (the sm_100 FFMA2 / FADD2 / FMUL2
// instructions through __ffma2_rn, __fadd2_rn, __fmul2_rn).
//
// Same operator as site_dslash_kernel (the eight hops of dslash_body,
// codegen/dslash.cc:200-323, then the clover / twisted-mass post-term of
// dslash_plain_body or the A.chi pre-term of dslash_achimbdpsi_body,
// codegen/dslash_common.cc:1729-1932) on the multi-RHS layout
// FT[block][3][4][2][S][nrhs].  Thread (site, pair) handles right-hand sides
// 2*pair and 2*pair + 1, which sit next to each other in memory: a spinor
// component of the pair is one 8-byte (FP32) or 4-byte (FP16) load, each link
// and clover element is loaded and (for 12-real links) reconstructed once
// for both, and every multiply-add of the hop and clover arithmetic is one
// packed instruction for both.  The operations and their order per right-hand
// side are those of site_dslash_kernel, so both give the same bits.
// Arithmetic is FP32 for FP32 and FP16 storage.
#pragma once

#include <cuda_fp16.h>

#include "qb200_site_kernel.cuh"

// minimum resident blocks of 128 threads per SM the register allocation must
// allow: the achimbdpsi form (chi and the clover block live next to the
// accumulators) gains from a cap at 128 registers, the plain form and the
// dense twisted-mass-clover block (which would spill under the cap) do not
#ifndef QB_PAIR_MINB_ACH
#define QB_PAIR_MINB_ACH 4
#endif
#ifndef QB_PAIR_MINB_PLAIN
#define QB_PAIR_MINB_PLAIN 1
#endif

namespace qb200 {

struct c2 {
  float2 re, im;
};

__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }

template <typename FT> struct pair_io;
template <> struct pair_io<float> {
  static __device__ __forceinline__ float2 ld(const float *p) { return __ldg(reinterpret_cast<const float2 *>(p)); }
  static __device__ __forceinline__ void st(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
};
template <> struct pair_io<__half> {
  static __device__ __forceinline__ float2 ld(const __half *p)
  {
    return __half22float2(__ldg(reinterpret_cast<const __half2 *>(p)));
  }
  static __device__ __forceinline__ void st(__half *p, float2 v)
  {
    *reinterpret_cast<__half2 *>(p) = __float22half2_rn(v);
  }
};

// component k = (c*4 + s)*2 + ri of the pair at base + k*cs
template <typename FT>
__device__ __forceinline__ void load_pair(const FT *__restrict__ f, long long base, int cs, c2 (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      sp[s][c].re = pair_io<FT>::ld(f + base + (long long)((c * 4 + s) * 2 + 0) * cs);
      sp[s][c].im = pair_io<FT>::ld(f + base + (long long)((c * 4 + s) * 2 + 1) * cs);
    }
}

template <typename FT>
__device__ __forceinline__ void store_pair(FT *__restrict__ f, long long base, int cs, const c2 (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      pair_io<FT>::st(f + base + (long long)((c * 4 + s) * 2 + 0) * cs, sp[s][c].re);
      pair_io<FT>::st(f + base + (long long)((c * 4 + s) * 2 + 1) * cs, sp[s][c].im);
    }
}

template <int D>
__device__ __forceinline__ void project2(const c2 (&psi)[4][3], float sigma, c2 (&b)[2][3])
{
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const float sg = sigma * (float)proj_sg(D, s);
    const int bb = proj_b(D, s);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (proj_i(D)) { // a + sg*i*b
        b[s][c].re = f2fma(bc(-sg), psi[bb][c].im, psi[s][c].re);
        b[s][c].im = f2fma(bc(sg), psi[bb][c].re, psi[s][c].im);
      } else {
        b[s][c].re = f2fma(bc(sg), psi[bb][c].re, psi[s][c].re);
        b[s][c].im = f2fma(bc(sg), psi[bb][c].im, psi[s][c].im);
      }
    }
  }
}

// ub = G^T b (forward) or conj(G) b (ADJ, backward)
template <bool ADJ>
__device__ __forceinline__ void mult2(const cx<float> (&G)[3][3], const c2 (&b)[2][3], c2 (&ub)[2][3])
{
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c1 = 0; c1 < 3; c1++) {
      float2 re, im;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const cx<float> g = ADJ ? G[c1][k] : G[k][c1];
        const float gi = ADJ ? -g.im : g.im; // conj for the backward hop
        if (k == 0) {
          re = f2mul(bc(g.re), b[s][k].re);
          im = f2mul(bc(g.re), b[s][k].im);
        } else {
          re = f2fma(bc(g.re), b[s][k].re, re);
          im = f2fma(bc(g.re), b[s][k].im, im);
        }
        re = f2fma(bc(-gi), b[s][k].im, re);
        im = f2fma(bc(gi), b[s][k].re, im);
      }
      ub[s][c1].re = re;
      ub[s][c1].im = im;
    }
}

__device__ __forceinline__ void phase2(c2 (&ub)[2][3], float pr, float pi)
{
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 re = f2fma(bc(-pi), ub[s][c].im, f2mul(bc(pr), ub[s][c].re));
      const float2 im = f2fma(bc(pi), ub[s][c].re, f2mul(bc(pr), ub[s][c].im));
      ub[s][c].re = re;
      ub[s][c].im = im;
    }
}

// acc += beta * recons(ub) with the rec_plus table scaled by tau
template <int MU>
__device__ __forceinline__ void recons2(const c2 (&ub)[2][3], float beta, float tau, c2 (&acc)[4][3])
{
  const float b2 = beta * tau * (float)rec_sg2(MU);
  const float b3 = beta * tau * (float)rec_sg3(MU);
  constexpr int s2 = rec_s2(MU), s3 = 1 - rec_s2(MU);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[0][c].re = f2fma(bc(beta), ub[0][c].re, acc[0][c].re);
    acc[0][c].im = f2fma(bc(beta), ub[0][c].im, acc[0][c].im);
    acc[1][c].re = f2fma(bc(beta), ub[1][c].re, acc[1][c].re);
    acc[1][c].im = f2fma(bc(beta), ub[1][c].im, acc[1][c].im);
    if (rec_i(MU)) { // += b * i * ub
      acc[2][c].re = f2fma(bc(-b2), ub[s2][c].im, acc[2][c].re);
      acc[2][c].im = f2fma(bc(b2), ub[s2][c].re, acc[2][c].im);
      acc[3][c].re = f2fma(bc(-b3), ub[s3][c].im, acc[3][c].re);
      acc[3][c].im = f2fma(bc(b3), ub[s3][c].re, acc[3][c].im);
    } else {
      acc[2][c].re = f2fma(bc(b2), ub[s2][c].re, acc[2][c].re);
      acc[2][c].im = f2fma(bc(b2), ub[s2][c].im, acc[2][c].im);
      acc[3][c].re = f2fma(bc(b3), ub[s3][c].re, acc[3][c].re);
      acc[3][c].im = f2fma(bc(b3), ub[s3][c].im, acc[3][c].im);
    }
  }
}

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }

// herm_apply (qb200_device.cuh) for a pair of right-hand sides: the same
// chains, operation for operation
template <int MODE, bool RHO>
__device__ __forceinline__ void herm_apply2(const float (&dg)[6], const cx<float> (&od)[15], int blk, float rhob,
                                            const c2 (&in)[4][3], c2 (&out)[4][3])
{
#pragma unroll
  for (int r = 0; r < 6; r++) {
    const c2 v = in[2 * blk + r / 3][r % 3];
    float2 re1 = f2mul(bc(dg[r]), v.re), im1 = f2mul(bc(dg[r]), v.im);
    float2 re2 = bc(0.f), im2 = bc(0.f);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      if (c == r) continue;
      const c2 w = in[2 * blk + c / 3][c % 3];
      if (c < r) { // A[r][c] = od[r(r-1)/2+c]
        const cx<float> a = od[r * (r - 1) / 2 + c];
        re1 = f2fma(bc(a.re), w.re, re1);
        re1 = f2fma(bc(-a.im), w.im, re1);
        im1 = f2fma(bc(a.re), w.im, im1);
        im1 = f2fma(bc(a.im), w.re, im1);
      } else { // A[r][c] = conj(od[c(c-1)/2+r])
        const cx<float> a = od[c * (c - 1) / 2 + r];
        re2 = f2fma(bc(a.re), w.re, re2);
        re2 = f2fma(bc(a.im), w.im, re2);
        im2 = f2fma(bc(a.re), w.im, im2);
        im2 = f2fma(bc(-a.im), w.re, im2);
      }
    }
    float2 re = f2add(re1, re2), im = f2add(im1, im2);
    if (RHO) {
      re = f2fma(bc(-rhob), v.im, re);
      im = f2fma(bc(rhob), v.re, im);
    }
    c2 &o = out[2 * blk + r / 3][r % 3];
    if (MODE == MODE_ADD) {
      o.re = f2add(o.re, re);
      o.im = f2add(o.im, im);
    } else {
      o.re = re;
      o.im = im;
    }
  }
}

// out (MODE) A in, A the Hermitian CloverBlock block `blk`
// (dslash_common.cc:1098-1186); base = tile*72*V + lane
template <typename FT, int MODE, bool RHO>
__device__ __forceinline__ void clover2(const FT *__restrict__ cl, long long base, int V, int blk, float rhob,
                                        const c2 (&in)[4][3], c2 (&out)[4][3])
{
  const FT *p = cl + base + (long long)blk * 36 * V;
  float dg[6];
  cx<float> od[15];
#pragma unroll
  for (int i = 0; i < 6; i++) dg[i] = ftraits<FT>::ld(p + (long long)i * V);
#pragma unroll
  for (int i = 0; i < 15; i++) {
    od[i].re = ftraits<FT>::ld(p + (long long)(6 + 2 * i) * V);
    od[i].im = ftraits<FT>::ld(p + (long long)(7 + 2 * i) * V);
  }
  herm_apply2<MODE, RHO>(dg, od, blk, rhob, in, out);
}

// out (MODE) F in, F a dense FullCloverBlock block (dslash_common.cc:1188-1232),
// dense_apply's chains; base = tile*144*V + lane
template <typename FT, int MODE, bool RHO>
__device__ __forceinline__ void full_clover2(const FT *__restrict__ cl, long long base, int V, int blk, float rhob,
                                             const c2 (&in)[4][3], c2 (&out)[4][3])
{
  const FT *p = cl + base + (long long)blk * 72 * V;
#pragma unroll
  for (int r = 0; r < 6; r++) {
    float2 re1 = bc(0.f), im1 = bc(0.f), re2 = bc(0.f), im2 = bc(0.f);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      const float ar = ftraits<FT>::ld(p + (long long)((r * 6 + c) * 2 + 0) * V);
      const float ai = ftraits<FT>::ld(p + (long long)((r * 6 + c) * 2 + 1) * V);
      const c2 w = in[2 * blk + c / 3][c % 3];
      if (c < 3) {
        re1 = f2fma(bc(ar), w.re, re1);
        re1 = f2fma(bc(-ai), w.im, re1);
        im1 = f2fma(bc(ar), w.im, im1);
        im1 = f2fma(bc(ai), w.re, im1);
      } else {
        re2 = f2fma(bc(ar), w.re, re2);
        re2 = f2fma(bc(-ai), w.im, re2);
        im2 = f2fma(bc(ar), w.im, im2);
        im2 = f2fma(bc(ai), w.re, im2);
      }
    }
    float2 re = f2add(re1, re2), im = f2add(im1, im2);
    if (RHO) {
      const c2 v = in[2 * blk + r / 3][r % 3];
      re = f2fma(bc(-rhob), v.im, re);
      im = f2fma(bc(rhob), v.re, im);
    }
    c2 &o = out[2 * blk + r / 3][r % 3];
    if (MODE == MODE_ADD) {
      o.re = f2add(o.re, re);
      o.im = f2add(o.im, im);
    } else {
      o.re = re;
      o.im = im;
    }
  }
}

template <typename FT, int S, bool COMP12, int D, int VV>
__device__ __forceinline__ void hop2(const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p, const Site &s,
                                     long long obase, long long ue, int le, int cs, long long gbase, c2 (&acc)[4][3])
{
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  bool cross;
  const long long nbase = obase + neighbour_offset<S, D>(g, s, ue, le, &cross);
  if (cross && !((p.acc_mask >> D) & 1u)) return;
  float beta = p.beta[D];
  if (D == 6 && s.t == 0 && p.t_edge_lo) beta *= p.tbound;
  if (D == 7 && s.t == g.nt - 1 && p.t_edge_hi) beta *= p.tbound;
  c2 psi[4][3], b[2][3], ub[2][3];
  cx<float> G[3][3];
  load_pair<FT>(a.psi, nbase, cs, psi);
  project2<D>(psi, p.isPlus ? 1.f : -1.f, b);
  load_link<FT, COMP12, D>(a.gauge, gbase, vlen<VV>(g), G);
  mult2<!FWD>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) phase2(ub, p.tbc[MU][0], FWD ? p.tbc[MU][1] : -p.tbc[MU][1]);
  recons2<MU>(ub, beta, ((p.isPlus != 0) != FWD) ? 1.f : -1.f, acc);
}

template <typename FT, int S, bool COMP12, int VV>
__device__ __forceinline__ void hops2(const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p, const Site &s,
                                      long long obase, long long ue, int le, int cs, long long gbase,
                                      c2 (&acc)[4][3])
{
  hop2<FT, S, COMP12, 0, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  hop2<FT, S, COMP12, 1, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  hop2<FT, S, COMP12, 2, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  hop2<FT, S, COMP12, 3, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  hop2<FT, S, COMP12, 4, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  hop2<FT, S, COMP12, 5, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  hop2<FT, S, COMP12, 6, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  hop2<FT, S, COMP12, 7, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
}

// Grid: blockIdx.y = the (z, t) plane; x covers the plane's sites times
// nrhs/2 pairs (pair fastest).  Requires an even nrhs.  NR: nrhs fixed at
// compile time (so every spinor component sits at a constant offset from the
// site's base), or 0 for the run-time g.nrhs.
template <typename FT, int S, bool COMP12, int FAM, bool ACH, int VV, int NR>
__global__ void __launch_bounds__(128, (ACH && FAM != FAM_TMCLOV) ? QB_PAIR_MINB_ACH : QB_PAIR_MINB_PLAIN)
    pair_dslash_kernel(const KArgs<FT> a, const GeoDev g, const OpDev<float> p)
{
  const int nr = NR ? NR : g.nrhs;
  const int np = nr >> 1;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.nxh * g.ny * np) return;
  const int sp = q / np;
  const int rp = q - sp * np;
  Site s;
  s.z = blockIdx.y % g.nz;
  s.t = blockIdx.y / g.nz;
  s.y = sp / g.nxh;
  s.xcb = sp - s.y * g.nxh;
  s.par = (s.y + s.z + s.t + p.cb) & 1;
  int lane;
  const long long tile = tile_of<S>(g, s, &lane);
  constexpr int R = COMP12 ? 2 : 3;
  const int V = vlen<VV>(g);
  const long long gbase = tile * (8LL * R * 6 * V) + lane;
  // multi-RHS block FT[3][4][2][S][nrhs]: component k of lane l, rhs r at
  // blk*24*S*nrhs + k*S*nrhs + l*nrhs + r
  const long long blk = s.t * g.Pxyz + s.z * g.Pxy + (long long)s.y * g.nvecs + s.xcb / S;
  const long long obase = (blk * (24 * S) + (s.xcb % S)) * nr + 2 * rp;
  const long long ue = 24LL * S * nr;
  const int le = nr;
  const int cs = S * nr;

  c2 acc[4][3], res[4][3];
#pragma unroll
  for (int sp2 = 0; sp2 < 4; sp2++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[sp2][c].re = acc[sp2][c].im = bc(0.f);
  hops2<FT, S, COMP12, VV>(a, g, p, s, obase, ue, le, cs, gbase, acc);
  if (ACH) {
    // the hops (subtracted: beta arrives negated from the host), then + A.chi
    // (ach_finish's operations)
    c2 ch[4][3];
    load_pair<FT>(a.chi, obase, cs, ch);
    if (FAM == FAM_WILSON) {
#pragma unroll
      for (int sp2 = 0; sp2 < 4; sp2++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          acc[sp2][c].re = f2fma(bc(p.alpha), ch[sp2][c].re, acc[sp2][c].re);
          acc[sp2][c].im = f2fma(bc(p.alpha), ch[sp2][c].im, acc[sp2][c].im);
        }
    } else if (FAM == FAM_TM) {
      // alpha (1 +/- i mu g5) chi, + on the upper spins for plus
#pragma unroll
      for (int sp2 = 0; sp2 < 4; sp2++) {
        const float m = (((sp2 < 2) == (p.isPlus != 0)) ? 1.f : -1.f) * p.mu;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          acc[sp2][c].re = f2fma(bc(p.alpha), f2fma(bc(-m), ch[sp2][c].im, ch[sp2][c].re), acc[sp2][c].re);
          acc[sp2][c].im = f2fma(bc(p.alpha), f2fma(bc(m), ch[sp2][c].re, ch[sp2][c].im), acc[sp2][c].im);
        }
      }
    } else {
      const long long cbase = tile * ((FAM == FAM_CLOVER ? 72LL : 144LL) * V) + lane;
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        const float rb = rho_of_block<float>(blk, p.isPlus, p.rho);
        if (FAM == FAM_CLOVER) clover2<FT, MODE_ADD, true>(a.clov, cbase, V, blk, rb, ch, acc);
        else full_clover2<FT, MODE_ADD, true>(a.clov, cbase, V, blk, rb, ch, acc);
      }
    }
#pragma unroll
    for (int sp2 = 0; sp2 < 4; sp2++)
#pragma unroll
      for (int c = 0; c < 3; c++) res[sp2][c] = acc[sp2][c];
  } else {
    if (FAM == FAM_CLOVER || FAM == FAM_TMCLOV) {
      const long long cbase = tile * ((FAM == FAM_CLOVER ? 72LL : 144LL) * V) + lane;
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        if (FAM == FAM_CLOVER) clover2<FT, MODE_SET, false>(a.clov, cbase, V, blk, 0.f, acc, res);
        else full_clover2<FT, MODE_SET, false>(a.clov, cbase, V, blk, 0.f, acc, res);
      }
    } else if (FAM == FAM_TM) {
      // muinv (1 + sg i mu) acc, sg = -1 on the upper spins for plus
#pragma unroll
      for (int sp2 = 0; sp2 < 4; sp2++) {
        const float m = (((sp2 < 2) == (p.isPlus != 0)) ? -1.f : 1.f) * p.mu;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          res[sp2][c].re = f2mul(bc(p.muinv), f2fma(bc(-m), acc[sp2][c].im, acc[sp2][c].re));
          res[sp2][c].im = f2mul(bc(p.muinv), f2fma(bc(m), acc[sp2][c].re, acc[sp2][c].im));
        }
      }
    } else {
#pragma unroll
      for (int sp2 = 0; sp2 < 4; sp2++)
#pragma unroll
        for (int c = 0; c < 3; c++) res[sp2][c] = acc[sp2][c];
    }
  }
  store_pair<FT>(a.out, obase, cs, res);
}

} // namespace qb200
