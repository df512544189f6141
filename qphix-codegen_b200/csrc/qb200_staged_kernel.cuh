// qb200_staged_kernel.cuh -- staging geometry and shared-memory helpers for
// the kernels that move every field through shared memory
// (qb200_async_kernel.cuh, and for the batched launch): whole spinor blocks,
// link-tile slabs and clover blocks are copied in 16-byte vectors and each
// thread reads its own site's elements from there.
//
// In a FourSpinorBlock FT[3][4][2][S] with small S one spinor component of a
// block is a short piece (16 bytes for FP32 SOALEN 4), and a thread-per-site
// load of one component by a warp touches 32/S separate pieces; staging whole
// blocks turns those into contiguous 16-byte copies.  The arithmetic of the
// helpers below (loads, stores, links, clover blocks) is that of the
// register forms in qb200_device.cuh, operation for operation.
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

} // namespace qb200
