// qb200_staged_kernel.cuh -- the single-RHS dslash for narrow SOALEN layouts
// (VECLEN == SOALEN, one spinor component of a block shorter than a 32-byte
// sector: FP32 SOALEN 4, FP16 / BF16 / FP16+norm SOALEN 4 and 8) with every
// field access staged through shared memory.
//
// In a FourSpinorBlock FT[3][4][2][S] with S = 4 (FP32) one spinor component
// of a block is a 16-byte piece, and the 32 sites of a warp span 32/S blocks:
// a per-component load of the thread-per-site kernel touches 32/S separate
// 16-byte pieces, half a sector each, and the L1 saturates on the number of
// pieces while DRAM is a third busy (the same holds for the link and clover
// tiles, whose lanes are the same S sites).  Here the warp copies whole
// blocks -- each contiguous -- in 16-byte vectors into shared memory and
// every thread then reads its own site's elements from there:
//   * the y, z and t neighbours of a block's S sites lie in one block at the
//     same lanes: 32/S blocks per hop;
//   * the x neighbours lie in the warp's own blocks of the other
//     checkerboard, one lane over (threads whose neighbour falls outside the
//     warp's blocks, at a row end, read it directly);
//   * links (one direction of a tile per hop), the CloverBlock halves, chi,
//     and the result (written to shared memory and stored in 16-byte vectors).
// The arithmetic is that of site_body, operation for operation.
#pragma once

#include "qb200_site_kernel.cuh"

namespace qb200 {

// staging geometry of one warp: G groups (= blocks / tiles) of S lanes
template <typename FT, int S> struct Stage {
  typedef elem_t<FT> E;
  static constexpr int G = 32 / S;
  static constexpr int W = S * (int)sizeof(E) / 4; // 32-bit words of one component
  // bytes per group of a staged piece with `elems` elements per lane, padded
  // so that the G groups of a warp start on different banks
  static constexpr int stride(int elems) { return elems * S * (int)sizeof(E) + ((W * 4 >= 16) ? W * 4 : 16); }
  static constexpr int SPB = ftraits<FT>::SPB;
  static constexpr int SP = stride(SPB);   // spinor block
  static constexpr int LK18 = stride(18);  // one direction of a tile, 18 reals
  static constexpr int CL = stride(36);    // one CloverBlock half
  static constexpr int BUF = G * (SP > CL ? (SP > LK18 ? SP : LK18) : (CL > LK18 ? CL : LK18));
};

// largest component piece (bytes) that is staged
#ifndef QB_STAGE_MAXPIECE
#define QB_STAGE_MAXPIECE 16
#endif

template <typename FT, int S> constexpr bool staged_layout()
{
  return (S == 4 || S == 8) && S * (int)sizeof(elem_t<FT>) <= QB_STAGE_MAXPIECE;
}

// Copy, for every group of the warp, the BYTES bytes that start at element
// `start` of f (the value held by the group's first lane) to buf + group *
// STRIDE.  All 32 lanes call it together.
template <typename FT, int S, int BYTES, int STRIDE>
__device__ __forceinline__ void stage_in(const elem_t<FT> *__restrict__ f, long long start, unsigned char *buf,
                                         int ln)
{
  static_assert(BYTES % 16 == 0 && STRIDE % 16 == 0, "staged pieces are whole 16-byte vectors");
  constexpr int CH = BYTES / 16, N = CH * Stage<FT, S>::G, ROUNDS = (N + 31) / 32;
  const uint4 *base = reinterpret_cast<const uint4 *>(f);
  // the start in 16-byte units (fields below 32 GiB)
  const unsigned v16 = (unsigned)(start * (long long)sizeof(elem_t<FT>) / 16);
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const int j = ln + 32 * r;
    const int gi = (j < N ? j : 0) / CH;
    const unsigned st = __shfl_sync(0xffffffffu, v16, gi * S);
    if (j < N) {
      const int c = j - gi * CH;
      *reinterpret_cast<uint4 *>(buf + gi * STRIDE + c * 16) = __ldg(base + st + c);
    }
  }
}

// the reverse: buf + group * STRIDE -> f at the group's `start`
template <typename FT, int S, int BYTES, int STRIDE>
__device__ __forceinline__ void stage_out(elem_t<FT> *__restrict__ f, long long start, const unsigned char *buf,
                                          int ln, bool group_active)
{
  constexpr int CH = BYTES / 16, N = CH * Stage<FT, S>::G, ROUNDS = (N + 31) / 32;
  uint4 *base = reinterpret_cast<uint4 *>(f);
  const unsigned v16 = (unsigned)(start * (long long)sizeof(elem_t<FT>) / 16);
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const int j = ln + 32 * r;
    const int gi = (j < N ? j : 0) / CH;
    const unsigned st = __shfl_sync(0xffffffffu, v16, gi * S);
    const bool act = __shfl_sync(0xffffffffu, group_active, gi * S);
    if (j < N && act) {
      const int c = j - gi * CH;
      base[st + c] = *reinterpret_cast<const uint4 *>(buf + gi * STRIDE + c * 16);
    }
  }
}

// element (k, lane) of a staged piece
template <typename FT, int S>
__device__ __forceinline__ comp_t<FT> sm_ld(const unsigned char *grp, int k, int lane)
{
  return ftraits<FT>::cv(reinterpret_cast<const elem_t<FT> *>(grp)[k * S + lane]);
}

template <typename FT, int S>
__device__ __forceinline__ void load_spinor_sm(const unsigned char *grp, int lane, cx<comp_t<FT>> (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      sp[s][c].re = sm_ld<FT, S>(grp, (c * 4 + s) * 2 + 0, lane);
      sp[s][c].im = sm_ld<FT, S>(grp, (c * 4 + s) * 2 + 1, lane);
    }
  if (ftraits<FT>::SPB == 26) {
    const float nrm = reinterpret_cast<const float *>(reinterpret_cast<const elem_t<FT> *>(grp) + 24 * S)[lane];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 4; s++) {
        sp[s][c].re *= nrm;
        sp[s][c].im *= nrm;
      }
  }
}

// load_spinor_sm without the FP16 + norm scaling: the site's norm is
// returned in nrm instead (1 for the other storage types)
template <typename FT, int S>
__device__ __forceinline__ void load_spinor_sm_raw(const unsigned char *grp, int lane, cx<comp_t<FT>> (&sp)[4][3],
                                                   comp_t<FT> &nrm)
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      sp[s][c].re = sm_ld<FT, S>(grp, (c * 4 + s) * 2 + 0, lane);
      sp[s][c].im = sm_ld<FT, S>(grp, (c * 4 + s) * 2 + 1, lane);
    }
  nrm = (comp_t<FT>)1;
  if (ftraits<FT>::SPB == 26)
    nrm = reinterpret_cast<const float *>(reinterpret_cast<const elem_t<FT> *>(grp) + 24 * S)[lane];
}

// the inverse of load_spinor_sm, with the norm of store_spinor
template <typename FT, int S>
__device__ __forceinline__ void store_spinor_sm(unsigned char *grp, int lane, const cx<comp_t<FT>> (&sp)[4][3])
{
  typedef comp_t<FT> C;
  elem_t<FT> *b = reinterpret_cast<elem_t<FT> *>(grp);
  C scale = (C)1;
  if (ftraits<FT>::SPB == 26) {
    C m = 0;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int s = 0; s < 4; s++) m = fmax(m, fmax(fabs(sp[s][c].re), fabs(sp[s][c].im)));
    const C nrm = m > (C)0 ? m : (C)1;
    reinterpret_cast<float *>(b + 24 * S)[lane] = (float)nrm;
    scale = (C)1 / nrm;
  }
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      ftraits<FT>::st(b + ((c * 4 + s) * 2 + 0) * S + lane, sp[s][c].re * scale);
      ftraits<FT>::st(b + ((c * 4 + s) * 2 + 1) * S + lane, sp[s][c].im * scale);
    }
}

// stored link G of one direction from a staged tile slab (load_link's formulas)
template <typename FT, int S, bool COMP12>
__device__ __forceinline__ void load_link_sm(const unsigned char *grp, int lane, cx<comp_t<FT>> (&G)[3][3])
{
  typedef comp_t<FT> C;
  constexpr int R = COMP12 ? 2 : 3;
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      G[r][c].re = sm_ld<FT, S>(grp, (r * 3 + c) * 2 + 0, lane);
      G[r][c].im = sm_ld<FT, S>(grp, (r * 3 + c) * 2 + 1, lane);
    }
  if (COMP12) recon_row3(G);
}

// clover_block from a staged CloverBlock half (the same operations)
template <typename FT, int S, int MODE, bool RHO>
__device__ __forceinline__ void clover_block_sm(const unsigned char *grp, int lane, int blk, comp_t<FT> rhob,
                                                const cx<comp_t<FT>> (&in)[4][3], cx<comp_t<FT>> (&out)[4][3])
{
  typedef comp_t<FT> C;
  C dg[6];
  cx<C> od[15];
#pragma unroll
  for (int i = 0; i < 6; i++) dg[i] = sm_ld<FT, S>(grp, i, lane);
#pragma unroll
  for (int i = 0; i < 15; i++) {
    od[i].re = sm_ld<FT, S>(grp, 6 + 2 * i, lane);
    od[i].im = sm_ld<FT, S>(grp, 7 + 2 * i, lane);
  }
  herm_apply<C, MODE, RHO>(dg, od, blk, rhob, in, out);
}

struct WarpCtx {
  unsigned char *buf;
  int ln;            // lane in the warp
  int lane;          // the site's lane in its block / tile
  long long tile;    // the site's tile (== block index within its plane layout)
  long long own;     // element index of the site's own spinor block
  long long blk;     // the site's spinor block index
  long long blk0;    // spinor block of the warp's first group
  unsigned char *xr; // x region (async kernel, 16-bit storage)
  int xhead;         // x-region slot index of the first row's first block
};

// y/z/t hop (D = 2..7) or x hop (D = 0, 1) with staged spinor and link
template <typename FT, int S, bool COMP12, int D>
__device__ __forceinline__ void staged_hop(const KArgs<FT> &a, const GeoDev &g, const OpDev<comp_t<FT>> &p,
                                           const Site &s, long long obase, const WarpCtx &w,
                                           cx<comp_t<FT>> (&acc)[4][3])
{
  typedef comp_t<FT> C;
  typedef Stage<FT, S> St;
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  constexpr int R = COMP12 ? 2 : 3;
  constexpr int LKB = R * 6 * S * (int)sizeof(elem_t<FT>), LKS = St::stride(R * 6);
  constexpr int SPB = St::SPB * S * (int)sizeof(elem_t<FT>);
  bool cross;
  const long long nbase = obase + neighbour_offset<S, D>(g, s, (long long)St::SPB * S, 1, &cross);
  // spinors: y/z/t the neighbour block; x the warp's own blocks of psi
  stage_in<FT, S, SPB, St::SP>(a.psi, MU == 0 ? w.own : nbase - w.lane, w.buf, w.ln);
  // the direction-D slab of the site's link tile
  unsigned char *lbuf = w.buf + St::G * St::SP;
  stage_in<FT, S, LKB, LKS>(a.gauge, w.tile * (8LL * R * 6 * S) + (long long)D * R * 6 * S, lbuf, w.ln);
  __syncwarp();
  cx<C> psi[4][3], G[3][3];
  if (MU == 0) {
    // neighbour element nbase = block * SPB*S + lane'; its group in the staged range
    const long long nb = nbase / (St::SPB * S);
    const int nl = (int)(nbase - nb * (St::SPB * S));
    const long long gi = nb - w.blk0;
    if (gi >= 0 && gi < St::G) load_spinor_sm<FT, S>(w.buf + gi * St::SP, nl, psi);
    else load_spinor<FT, S>(a.psi, nbase, psi);
  } else {
    load_spinor_sm<FT, S>(w.buf + (w.ln / S) * St::SP, w.lane, psi);
  }
  load_link_sm<FT, S, COMP12>(lbuf + (w.ln / S) * LKS, w.lane, G);
  __syncwarp();
  if (cross && !((p.acc_mask >> D) & 1u)) return;
  C beta = p.beta[D];
  if (D == 6 && s.t == 0 && p.t_edge_lo) beta *= p.tbound;
  if (D == 7 && s.t == g.nt - 1 && p.t_edge_hi) beta *= p.tbound;
  cx<C> b[2][3], ub[2][3];
  const C sigma = p.isPlus ? (C)1 : (C)-1;
  project<C, D>(psi, sigma, b);
  mult_link<C, !FWD>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) {
    const C pr = p.tbc[MU][0];
    const C pi = FWD ? p.tbc[MU][1] : -p.tbc[MU][1];
    apply_phase<C>(ub, pr, pi);
  }
  const C tau = ((p.isPlus != 0) != FWD) ? (C)1 : (C)-1;
  recons<C, MU>(ub, beta, tau, acc);
}

template <typename FT, int S, bool COMP12>
__device__ __forceinline__ void staged_hops(const KArgs<FT> &a, const GeoDev &g, const OpDev<comp_t<FT>> &p,
                                            const Site &s, long long obase, const WarpCtx &w,
                                            cx<comp_t<FT>> (&acc)[4][3])
{
  staged_hop<FT, S, COMP12, 0>(a, g, p, s, obase, w, acc);
  staged_hop<FT, S, COMP12, 1>(a, g, p, s, obase, w, acc);
  staged_hop<FT, S, COMP12, 2>(a, g, p, s, obase, w, acc);
  staged_hop<FT, S, COMP12, 3>(a, g, p, s, obase, w, acc);
  staged_hop<FT, S, COMP12, 4>(a, g, p, s, obase, w, acc);
  staged_hop<FT, S, COMP12, 5>(a, g, p, s, obase, w, acc);
  staged_hop<FT, S, COMP12, 6>(a, g, p, s, obase, w, acc);
  staged_hop<FT, S, COMP12, 7>(a, g, p, s, obase, w, acc);
}

// out (MODE) the CloverBlock of the site's tile applied to in (RHO: with
// the + i rho g5 in term), both halves staged
template <typename FT, int S, int MODE, bool RHO>
__device__ __forceinline__ void staged_clover(const KArgs<FT> &a, const WarpCtx &w, int isPlus, comp_t<FT> rho,
                                              const cx<comp_t<FT>> (&in)[4][3], cx<comp_t<FT>> (&out)[4][3])
{
  typedef Stage<FT, S> St;
  constexpr int CLB = 36 * S * (int)sizeof(elem_t<FT>);
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    stage_in<FT, S, CLB, St::CL>(a.clov, w.tile * (72LL * S) + blk * 36LL * S, w.buf, w.ln);
    __syncwarp();
    clover_block_sm<FT, S, MODE, RHO>(w.buf + (w.ln / S) * St::CL, w.lane, blk,
                                      rho_of_block<comp_t<FT>>(blk, isPlus, rho), in, out);
    __syncwarp();
  }
}

// out (MODE) the FullCloverBlock of the site's tile applied to in (dense 6x6
// complex per half, dense_apply's operation order; RHO: with the + i rho g5
// in term), both halves staged; buf needs Stage::G * Stage::stride(72) bytes
template <typename FT, int S, int MODE, bool RHO>
__device__ __forceinline__ void staged_full_clover(const KArgs<FT> &a, const WarpCtx &w, int isPlus, comp_t<FT> rho,
                                                   const cx<comp_t<FT>> (&in)[4][3], cx<comp_t<FT>> (&out)[4][3])
{
  typedef comp_t<FT> C;
  typedef Stage<FT, S> St;
  constexpr int FCB = 72 * S * (int)sizeof(elem_t<FT>);
  constexpr int FCS = St::stride(72);
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    stage_in<FT, S, FCB, FCS>(a.clov, w.tile * (144LL * S) + blk * 72LL * S, w.buf, w.ln);
    __syncwarp();
    const unsigned char *grp = w.buf + (w.ln / S) * FCS;
    const int lane = w.lane;
    dense_apply<C, MODE, RHO>(
        [&](int r, int c) {
          return mk<C>(sm_ld<FT, S>(grp, (r * 6 + c) * 2 + 0, lane), sm_ld<FT, S>(grp, (r * 6 + c) * 2 + 1, lane));
        },
        blk, rho_of_block<C>(blk, isPlus, rho), in, out);
    __syncwarp();
  }
}

template <typename FT, int S, bool COMP12> struct StagedSmem {
  static constexpr int BYTES = Stage<FT, S>::BUF + Stage<FT, S>::G * Stage<FT, S>::stride((COMP12 ? 2 : 3) * 6);
};

// The operator at site q0 (the warp's lane's site) of plane (z, t); buf is
// the warp's shared-memory area.  Called by all 32 lanes of a warp together.
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__device__ __forceinline__ void staged_body(const KArgs<FT> &a, const GeoDev &g, const OpDev<comp_t<FT>> &p, int z,
                                            int t, int q0, unsigned char *buf)
{
  typedef comp_t<FT> C;
  typedef Stage<FT, S> St;
  const int nplane = g.nxh * g.ny;
  const bool active = q0 < nplane;
  const int q = active ? q0 : nplane - 1;
  Site s;
  s.z = z;
  s.t = t;
  s.y = q / g.nxh;
  s.xcb = q - s.y * g.nxh;
  s.par = (s.y + s.z + s.t + p.cb) & 1;
  WarpCtx w;
  w.buf = buf;
  w.ln = threadIdx.x & 31;
  w.tile = tile_of<S>(g, s, &w.lane);
  const long long obase = spinor_base<FT, S>(g, s);
  w.blk = obase / (St::SPB * S);
  w.own = w.blk * (St::SPB * S);
  w.blk0 = __shfl_sync(0xffffffffu, w.blk, 0);
  constexpr int SPB = St::SPB * S * (int)sizeof(elem_t<FT>);

  cx<C> acc[4][3];
#pragma unroll
  for (int sp = 0; sp < 4; sp++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[sp][c] = mk<C>(0, 0);
  staged_hops<FT, S, COMP12>(a, g, p, s, obase, w, acc);
  if (ACH) {
    // the hops (subtracted: beta negated by the host), then + A.chi
    cx<C> ch[4][3];
    stage_in<FT, S, SPB, St::SP>(a.chi, w.own, w.buf, w.ln);
    __syncwarp();
    load_spinor_sm<FT, S>(w.buf + (w.ln / S) * St::SP, w.lane, ch);
    __syncwarp();
    if (FAM == FAM_CLOVER) staged_clover<FT, S, MODE_ADD, true>(a, w, p.isPlus, p.rho, ch, acc);
    else ach_finish<FT, FAM>(a, p, w.tile, w.lane, S, ch, acc);
  } else {
    cx<C> res[4][3];
    if (FAM == FAM_CLOVER) staged_clover<FT, S, MODE_SET, false>(a, w, p.isPlus, (C)0, acc, res);
    else plain_post<FT, FAM>(a, p, w.tile, w.lane, S, acc, res);
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) acc[sp][c] = res[sp][c];
  }
  // the result through shared memory, out in 16-byte vectors
  store_spinor_sm<FT, S>(w.buf + (w.ln / S) * St::SP, w.lane, acc);
  __syncwarp();
  stage_out<FT, S, SPB, St::SP>(a.out, w.own, w.buf, w.ln, active);
  __syncwarp();
}

// Work unit: one warp's 32 sites of one (z, t) plane, numbered over all
// planes ((nxh*ny + 31)/32 per plane, so that no warp idles when a plane's
// sites do not fill whole blocks); one-dimensional grid of blocks of 128
// threads, at most 128 registers (4 blocks per SM).  Threads past the
// plane's last site take part in the warp's copies (on a clamped site) and
// store nothing.  Needs 16-byte aligned fields smaller than 32 GiB.
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__global__ void __launch_bounds__(128, 4)
    staged_site_kernel(const KArgs<FT> a, const GeoDev g, const OpDev<comp_t<FT>> p)
{
  __shared__ __align__(16) unsigned char smem[4][StagedSmem<FT, S, COMP12>::BYTES];
  const int wpp = (g.nxh * g.ny + 31) >> 5;
  const long long u = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  if (u >= (long long)wpp * g.nz * g.nt) return; // whole warps
  const int plane = (int)(u / wpp);
  const int wi = (int)(u - (long long)plane * wpp);
  staged_body<FT, S, COMP12, FAM, ACH>(a, g, p, plane % g.nz, plane / g.nz, wi * 32 + (threadIdx.x & 31),
                                       smem[threadIdx.x >> 5]);
}

// Batched form: work unit = one warp's 32 sites of one plane of one item;
// b.it[k].first and b.total count such warps (each plane padded to whole
// warps).  The loop is uniform across a warp.  The per-item parameters read
// through the parameter block take registers: 3 blocks per SM keep it from
// spilling.
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__global__ void __launch_bounds__(128, 3) batch_staged_kernel(const __grid_constant__ BatchDev<FT> b)
{
  __shared__ __align__(16) unsigned char smem[4][StagedSmem<FT, S, COMP12>::BYTES];
  const long long stride = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long u = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < b.total; u += stride) {
    int k = 0;
    while (k + 1 < b.n && u >= b.it[k + 1].first) k++;
    const BatchItem<FT> &it = b.it[k];
    const int wpp = (it.g.nxh * it.g.ny + 31) >> 5; // warps per plane
    const long long loc = u - it.first;
    const int plane = (int)(loc / wpp);
    const int wi = (int)(loc - (long long)plane * wpp);
    staged_body<FT, S, COMP12, FAM, ACH>(it.a, it.g, it.p, plane % it.g.nz, plane / it.g.nz,
                                         wi * 32 + (threadIdx.x & 31), smem[threadIdx.x >> 5]);
  }
}

} // namespace qb200
