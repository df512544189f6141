// qb200_site_kernel.cuh -- thread-per-site dslash kernel, generic over every
// QPhiX tile layout (storage type FT, SOALEN S; VECLEN compile-time when it
// equals S, else run-time).
//
// One thread computes one output site of the checkerboard: the eight hops of
// dslash_body (codegen/dslash.cc:200-323) in registers, followed by the
// clover / twisted-mass post-term of dslash_plain_body or the A.chi pre-term
// of dslash_achimbdpsi_body (codegen/dslash_common.cc:1729-1932).
#pragma once

#include "qb200_device.cuh"

namespace qb200 {

template <typename FT> struct KArgs {
  const elem_t<FT> *psi;
  const elem_t<FT> *chi;
  const elem_t<FT> *gauge;
  const elem_t<FT> *clov;
  elem_t<FT> *out;
};

// element offset from a site's spinor base to the base of its neighbour in
// direction D (periodic wrap inside the local lattice).  ue: elements per
// block, le: elements per lane step (1, or nrhs in the multi-RHS layout).
template <int S, int D>
__device__ __forceinline__ long long neighbour_offset(const GeoDev &g, const Site &s, long long ue, int le,
                                                      bool *cross)
{
  const int lane = s.xcb % S;
  const int xb = s.xcb / S;
  if (D == 0) {
    *cross = (s.par == 0) && (s.xcb == 0);
    if (s.par != 0) return 0;
    if (lane > 0) return -le;
    if (xb > 0) return -ue + (long long)(S - 1) * le;
    return (long long)(g.nvecs - 1) * ue + (long long)(S - 1) * le;
  } else if (D == 1) {
    *cross = (s.par == 1) && (s.xcb == g.nxh - 1);
    if (s.par != 1) return 0;
    if (lane < S - 1) return le;
    if (xb < g.nvecs - 1) return ue - (long long)(S - 1) * le;
    return -(long long)(g.nvecs - 1) * ue - (long long)(S - 1) * le;
  } else if (D == 2) {
    *cross = s.y == 0;
    return (s.y > 0 ? -1LL : (long long)(g.ny - 1)) * g.nvecs * ue;
  } else if (D == 3) {
    *cross = s.y == g.ny - 1;
    return (s.y < g.ny - 1 ? 1LL : -(long long)(g.ny - 1)) * g.nvecs * ue;
  } else if (D == 4) {
    *cross = s.z == 0;
    return (s.z > 0 ? -1LL : (long long)(g.nz - 1)) * g.Pxy * ue;
  } else if (D == 5) {
    *cross = s.z == g.nz - 1;
    return (s.z < g.nz - 1 ? 1LL : -(long long)(g.nz - 1)) * g.Pxy * ue;
  } else if (D == 6) {
    *cross = s.t == 0;
    return (s.t > 0 ? -1LL : (long long)(g.nt - 1)) * g.Pxyz * ue;
  } else {
    *cross = s.t == g.nt - 1;
    return (s.t < g.nt - 1 ? 1LL : -(long long)(g.nt - 1)) * g.Pxyz * ue;
  }
}

// VV: compile-time VECLEN (layouts with V == VV), or 0 for the run-time g.V
template <int VV> __device__ __forceinline__ int vlen(const GeoDev &g) { return VV ? VV : g.V; }

template <typename FT, int S, bool COMP12, int D, bool MR, int VV>
__device__ __forceinline__ void do_hop(const KArgs<FT> &a, const GeoDev &g,
                                       const OpDev<typename ftraits<FT>::C> &p, const Site &s, long long obase,
                                       long long ue, int le, long long gbase,
                                       cx<typename ftraits<FT>::C> (&acc)[4][3])
{
  typedef typename ftraits<FT>::C C;
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  bool cross;
  const long long nbase = obase + neighbour_offset<S, D>(g, s, ue, le, &cross);
  if (cross && !((p.acc_mask >> D) & 1u)) return;
  C beta = p.beta[D];
  if (D == 6 && s.t == 0 && p.t_edge_lo) beta *= p.tbound;
  if (D == 7 && s.t == g.nt - 1 && p.t_edge_hi) beta *= p.tbound;

  cx<C> psi[4][3], b[2][3], ub[2][3], G[3][3];
  if (MR) load_spinor_rs<FT>(a.psi, nbase, S * g.nrhs, psi);
  else load_spinor<FT, S>(a.psi, nbase, psi);
  const C sigma = p.isPlus ? (C)1 : (C)-1;
  project<C, D>(psi, sigma, b);
  load_link<FT, COMP12, D>(a.gauge, gbase, vlen<VV>(g), G);
  mult_link<C, !FWD>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) {
    const C pr = p.tbc[MU][0];
    const C pi = FWD ? p.tbc[MU][1] : -p.tbc[MU][1];
    apply_phase<C>(ub, pr, pi);
  }
  // rec_plus for (isPlus xor fwd)
  const C tau = ((p.isPlus != 0) != FWD) ? (C)1 : (C)-1;
  recons<C, MU>(ub, beta, tau, acc);
}

// acc += A.chi (+ i rho g5 chi): the A.chi term of the achimbdpsi form
// (achiResult, dslash_common.cc:1559-1655; rho term :1873-1906), added to
// the hops already summed in acc (beta negated by the host), one rounding
// per component after the term itself.  Wilson: A = alpha; twisted mass:
// alpha (1 +/- i mu g5), + on the upper spins for plus.
template <typename FT, int FAM>
__device__ __forceinline__ void ach_finish(const KArgs<FT> &a, const OpDev<typename ftraits<FT>::C> &p,
                                           long long tile, int lane, int V,
                                           const cx<typename ftraits<FT>::C> (&ch)[4][3],
                                           cx<typename ftraits<FT>::C> (&acc)[4][3])
{
  typedef typename ftraits<FT>::C C;
  if (FAM == FAM_WILSON) {
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        acc[sp][c].re = fma(p.alpha, ch[sp][c].re, acc[sp][c].re);
        acc[sp][c].im = fma(p.alpha, ch[sp][c].im, acc[sp][c].im);
      }
  } else if (FAM == FAM_TM) {
#pragma unroll
    for (int sp = 0; sp < 4; sp++) {
      const C m = (((sp < 2) == (p.isPlus != 0)) ? (C)1 : (C)-1) * p.mu;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        acc[sp][c].re = fma(p.alpha, fma(-m, ch[sp][c].im, ch[sp][c].re), acc[sp][c].re);
        acc[sp][c].im = fma(p.alpha, fma(m, ch[sp][c].re, ch[sp][c].im), acc[sp][c].im);
      }
    }
  } else {
    const long long cbase = tile * ((FAM == FAM_CLOVER ? 72LL : 144LL) * V) + lane;
#pragma unroll
    for (int blk = 0; blk < 2; blk++) {
      const C rb = rho_of_block<C>(blk, p.isPlus, p.rho);
      if (FAM == FAM_CLOVER) clover_block<FT, MODE_ADD, true>(a.clov, cbase, V, blk, rb, ch, acc);
      else full_clover_block<FT, MODE_ADD, true>(a.clov, cbase, V, blk, rb, ch, acc);
    }
  }
}

// res = post-term(acc): clover / full clover / inverse twisted mass / copy
// (dslash_plain_body, dslash_common.cc:1796-1826)
template <typename FT, int FAM>
__device__ __forceinline__ void plain_post(const KArgs<FT> &a, const OpDev<typename ftraits<FT>::C> &p,
                                           long long tile, int lane, int V,
                                           const cx<typename ftraits<FT>::C> (&acc)[4][3],
                                           cx<typename ftraits<FT>::C> (&res)[4][3])
{
  typedef typename ftraits<FT>::C C;
  if (FAM == FAM_CLOVER || FAM == FAM_TMCLOV) {
    const long long cbase = tile * ((FAM == FAM_CLOVER ? 72LL : 144LL) * V) + lane;
#pragma unroll
    for (int blk = 0; blk < 2; blk++) {
      if (FAM == FAM_CLOVER) clover_block<FT, MODE_SET, false>(a.clov, cbase, V, blk, (C)0, acc, res);
      else full_clover_block<FT, MODE_SET, false>(a.clov, cbase, V, blk, (C)0, acc, res);
    }
  } else if (FAM == FAM_TM) {
    inv_twisted<C, false>(acc, p.isPlus, p.mu, p.muinv, res);
  } else {
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) res[sp][c] = acc[sp][c];
  }
}

template <typename FT, int S, bool COMP12, bool MR, int VV>
__device__ __forceinline__ void all_hops(const KArgs<FT> &a, const GeoDev &g, const OpDev<typename ftraits<FT>::C> &p,
                                         const Site &s, long long obase, long long ue, int le, long long gbase,
                                         cx<typename ftraits<FT>::C> (&acc)[4][3])
{
  do_hop<FT, S, COMP12, 0, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  do_hop<FT, S, COMP12, 1, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  do_hop<FT, S, COMP12, 2, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  do_hop<FT, S, COMP12, 3, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  do_hop<FT, S, COMP12, 4, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  do_hop<FT, S, COMP12, 5, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  do_hop<FT, S, COMP12, 6, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  do_hop<FT, S, COMP12, 7, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
}

// The operator at one output site s (and right-hand side rhs of the
// multi-RHS layout when MR).
template <typename FT, int S, bool COMP12, int FAM, bool ACH, bool MR, int VV>
__device__ __forceinline__ void site_body(const KArgs<FT> &a, const GeoDev &g,
                                          const OpDev<typename ftraits<FT>::C> &p, const Site &s, int rhs)
{
  typedef typename ftraits<FT>::C C;
  const int nr = MR ? g.nrhs : 1;
  int lane;
  const long long tile = tile_of<S>(g, s, &lane);
  constexpr int R = COMP12 ? 2 : 3;
  const int V = vlen<VV>(g);
  const long long gbase = tile * (8LL * R * 6 * V) + lane;
  const long long obase = MR ? spinor_base_mr<S>(g, s, rhs) : spinor_base<FT, S>(g, s);
  const long long ue = MR ? 24LL * S * nr : (long long)ftraits<FT>::SPB * S;
  const int le = nr;
  const int cs = S * nr;

  cx<C> res[4][3], acc[4][3];
#pragma unroll
  for (int sp = 0; sp < 4; sp++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[sp][c] = mk<C>(0, 0);
  all_hops<FT, S, COMP12, MR, VV>(a, g, p, s, obase, ue, le, gbase, acc);
  if (ACH) {
    // the hops (subtracted: beta negated by the host), then + A.chi
    cx<C> ch[4][3];
    if (MR) load_spinor_rs<FT>(a.chi, obase, cs, ch);
    else load_spinor<FT, S>(a.chi, obase, ch);
    ach_finish<FT, FAM>(a, p, tile, lane, V, ch, acc);
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) res[sp][c] = acc[sp][c];
  } else {
    plain_post<FT, FAM>(a, p, tile, lane, V, acc, res);
  }
  if (MR) store_spinor_rs<FT>(a.out, obase, cs, res);
  else store_spinor<FT, S>(a.out, obase, res);
}

// Grid: blockIdx.y = the (z, t) plane, x covers the plane's sites (times the
// right-hand sides).  MR: multi-RHS layout, one thread per (site, right-hand
// side) with the right-hand side fastest, so the nrhs threads of a site share
// each link and clover load.
// minimum resident blocks per SM the register allocation must allow
#ifndef QB_SITE_MINB
#define QB_SITE_MINB 1
#endif

template <typename FT, int S, bool COMP12, int FAM, bool ACH, bool MR, int VV>
__global__ void __launch_bounds__(128, QB_SITE_MINB)
    site_dslash_kernel(const KArgs<FT> a, const GeoDev g, const OpDev<typename ftraits<FT>::C> p)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int nr = MR ? g.nrhs : 1;
  if (q >= g.nxh * g.ny * nr) return;
  const int sp = MR ? q / nr : q;
  const int rhs = MR ? q - sp * nr : 0;
  Site s;
  s.z = blockIdx.y % g.nz;
  s.t = blockIdx.y / g.nz;
  s.y = sp / g.nxh;
  s.xcb = sp - s.y * g.nxh;
  s.par = (s.y + s.z + s.t + p.cb) & 1;
  site_body<FT, S, COMP12, FAM, ACH, MR, VV>(a, g, p, s, rhs);
}

// Several lattices (a batch of independent problems with the same storage
// type and layout) in one launch.  Work unit u of the flattened index space
// is site u - first[k] of item k; with a grid smaller than the work the
// threads stride through it (persistent launch).
constexpr int kMaxBatch = 16;

template <typename FT> struct BatchItem {
  KArgs<FT> a;
  GeoDev g;
  OpDev<typename ftraits<FT>::C> p;
  long long first; // first work unit of the item
};

template <typename FT> struct BatchDev {
  BatchItem<FT> it[kMaxBatch];
  int n;
  long long total;
};

template <typename FT, int S, bool COMP12, int FAM, bool ACH, int VV>
__global__ void __launch_bounds__(128) batch_dslash_kernel(const __grid_constant__ BatchDev<FT> b)
{
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < b.total; u += stride) {
    int k = 0;
    while (k + 1 < b.n && u >= b.it[k + 1].first) k++;
    const BatchItem<FT> &it = b.it[k];
    const Site s = site_of(it.g, (int)(u - it.first), it.p.cb);
    site_body<FT, S, COMP12, FAM, ACH, false, VV>(it.a, it.g, it.p, s, 0);
  }
}

} // namespace qb200
