// qb200_async_kernel.cuh -- the single-RHS dslash with the neighbour spinors
// and links of the next hop in flight while the current hop computes.
//
// The thread-per-site kernel waits on global loads (long-scoreboard stalls)
// with about 20 warps per SM: each hop's 24 spinor and 12-18 link loads are
// issued only when the hop starts.  Here a warp copies, with cp.async, the
// blocks its 32 sites need for hop D+1 (the neighbour spinor blocks, or its
// own blocks of psi for the x hops, and the direction-(D+1) slab of its link
// tiles) into one of two shared-memory buffers while it computes hop D from
// the other, so the copies cost no registers and overlap the arithmetic.
// The post-hop term's operands follow the same way: chi (or the first
// CloverBlock half of the clover dslash) is copied into hop buffer 0 while
// hop 7 computes, and each further CloverBlock half into a freed hop buffer
// while the previous one computes.
// The per-site reads from shared memory, the x-neighbour handling and the
// clover / chi / result staging are those of qb200_staged_kernel.cuh; the
// arithmetic is that of site_body, operation for operation.
// Layouts with VECLEN == SOALEN in {4, 8, 16}, 32- and 16-bit storage.
#pragma once

#include "qb200_staged_kernel.cuh"

namespace qb200 {

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// stage_in with asynchronous copies (completion: cp_async_wait + __syncwarp)
template <typename FT, int S, int BYTES, int STRIDE>
__device__ __forceinline__ void stage_in_async(const elem_t<FT> *__restrict__ f, long long start, unsigned char *buf,
                                               int ln)
{
  static_assert(BYTES % 16 == 0 && STRIDE % 16 == 0, "staged pieces are whole 16-byte vectors");
  constexpr int CH = BYTES / 16, N = CH * Stage<FT, S>::G, ROUNDS = (N + 31) / 32;
  const uint4 *base = reinterpret_cast<const uint4 *>(f);
  const unsigned v16 = (unsigned)(start * (long long)sizeof(elem_t<FT>) / 16);
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const int j = ln + 32 * r;
    const int gi = (j < N ? j : 0) / CH;
    const unsigned st = __shfl_sync(0xffffffffu, v16, gi * S);
    if (j < N) cp_async16(buf + gi * STRIDE + (j - gi * CH) * 16, base + st + (j - gi * CH));
  }
}

template <typename FT, int S, bool COMP12> struct AsyncCfg {
  typedef Stage<FT, S> St;
  static constexpr int R = COMP12 ? 2 : 3;
  static constexpr int SPB = St::SPB * S * (int)sizeof(elem_t<FT>);  // spinor block bytes
  static constexpr int LKB = R * 6 * S * (int)sizeof(elem_t<FT>);    // link slab bytes
  static constexpr int LKS = St::stride(R * 6);
  static constexpr int HOP = St::G * (St::SP + LKS);                 // one hop's staged bytes
  static constexpr int FCL = St::G * St::stride(72);  // staged FullCloverBlock halves
  static constexpr int XOFF = (2 * HOP > St::G * St::CL) ? (2 * HOP > FCL ? 2 * HOP : FCL)
                                                         : (St::G * St::CL > FCL ? St::G * St::CL : FCL);
  // 16-bit storage: an x region, staged once for both x hops, holds blocks
  // blk0-1 .. blk0+G, the first block of the warp's first row and the last
  // block of its last row -- every x neighbour of the warp's sites, also
  // when a row of the lattice does not start or end with the warp.  (For
  // 32-bit storage it would not fit next to four warps' hop buffers; x
  // neighbours outside the warp's own blocks are then read from global
  // memory.)
  static constexpr bool XREG = sizeof(elem_t<FT>) == 2;
  static constexpr int XS = St::G + 4;
  static constexpr int BUF = XOFF + (XREG ? XS * St::SP : 0);
};

template <typename FT, int S> constexpr bool async_layout()
{
  return (S == 4 || S == 8 || S == 16) && sizeof(elem_t<FT>) <= 4;
}

// copy the x region of psi (AsyncCfg::XS blocks) to w.xr; blocks outside
// the field are skipped (their slots are never read)
template <typename FT, int S, bool COMP12>
__device__ __forceinline__ void stage_xregion(const elem_t<FT> *__restrict__ f, long long blk0, long long head,
                                              long long tail, long long nblocks, unsigned char *xr, int ln)
{
  typedef AsyncCfg<FT, S, COMP12> A;
  typedef Stage<FT, S> St;
  constexpr int CH = A::SPB / 16, N = CH * A::XS, ROUNDS = (N + 31) / 32;
  static_assert(A::SPB % 16 == 0, "staged blocks are whole 16-byte vectors");
  const uint4 *base = reinterpret_cast<const uint4 *>(f);
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const int j = ln + 32 * r;
    const int slot = j / CH, c = j - slot * CH;
    const long long b = slot < St::G + 2 ? blk0 - 1 + slot : (slot == St::G + 2 ? head : tail);
    if (j < N && b >= 0 && b < nblocks) cp_async16(xr + slot * St::SP + c * 16, base + b * CH + c);
  }
}

// x neighbour of site s in direction D (0: back, 1: forward): its block
// within the row and its lane
template <int S, int D>
__device__ __forceinline__ void x_neighbour(const GeoDev &g, const Site &s, int &xb, int &ln)
{
  int x = s.xcb;
  if (D == 0 && s.par == 0) x = x > 0 ? x - 1 : g.nxh - 1;
  if (D == 1 && s.par == 1) x = x < g.nxh - 1 ? x + 1 : 0;
  xb = x / S;
  ln = x % S;
}

// issue the copies of hop D into buf
template <typename FT, int S, bool COMP12, int D>
__device__ __forceinline__ void prefetch_hop(const KArgs<FT> &a, const GeoDev &g, const Site &s, long long obase,
                                             const WarpCtx &w, unsigned char *buf)
{
  typedef AsyncCfg<FT, S, COMP12> A;
  typedef Stage<FT, S> St;
  if (!(A::XREG && D < 2)) {
    bool cross;
    const long long nbase = obase + neighbour_offset<S, D>(g, s, (long long)St::SPB * S, 1, &cross);
    stage_in_async<FT, S, A::SPB, St::SP>(a.psi, D < 2 ? w.own : nbase - w.lane, buf, w.ln);
  }
  stage_in_async<FT, S, A::LKB, A::LKS>(a.gauge, w.tile * (8LL * A::R * 6 * S) + (long long)D * A::R * 6 * S,
                                        buf + St::G * St::SP, w.ln);
}

// hop D from the staged copies in buf (the operations of do_hop)
template <typename FT, int S, bool COMP12, int D>
__device__ __forceinline__ void compute_hop(const KArgs<FT> &a, const GeoDev &g, const OpDev<comp_t<FT>> &p,
                                            const Site &s, long long obase, const WarpCtx &w,
                                            const unsigned char *buf, cx<comp_t<FT>> (&acc)[4][3])
{
  typedef comp_t<FT> C;
  typedef AsyncCfg<FT, S, COMP12> A;
  typedef Stage<FT, S> St;
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  bool cross;
  const long long nbase = obase + neighbour_offset<S, D>(g, s, (long long)St::SPB * S, 1, &cross);
  if (cross && !((p.acc_mask >> D) & 1u)) return;
  cx<C> psi[4][3], G[3][3];
  // FP16 + norm: the neighbour's norm scales the hop's coefficient, not its
  // 24 components (the hop is linear in psi)
  C nrm = (C)1;
  if (MU == 0 && A::XREG) {
    int xb, nl;
    x_neighbour<S, D>(g, s, xb, nl);
    // slot of the row's first block, then of the neighbour's block
    int sl = (int)(w.blk - w.blk0) + 1 - s.xcb / S + xb;
    sl = (sl >= 0 && sl < St::G + 2) ? sl : (sl == w.xhead ? St::G + 2 : St::G + 3);
    load_spinor_sm_raw<FT, S>(w.xr + sl * St::SP, nl, psi, nrm);
  } else if (MU == 0) {
    const long long nb = nbase / (St::SPB * S);
    const int nl = (int)(nbase - nb * (St::SPB * S));
    const long long gi = nb - w.blk0;
    if (gi >= 0 && gi < St::G) load_spinor_sm<FT, S>(buf + gi * St::SP, nl, psi);
    else load_spinor<FT, S>(a.psi, nbase, psi);
  } else {
    load_spinor_sm_raw<FT, S>(buf + (w.ln / S) * St::SP, w.lane, psi, nrm);
  }
  load_link_sm<FT, S, COMP12>(buf + St::G * St::SP + (w.ln / S) * A::LKS, w.lane, G);
  C beta = p.beta[D];
  if (D == 6 && s.t == 0 && p.t_edge_lo) beta *= p.tbound;
  if (D == 7 && s.t == g.nt - 1 && p.t_edge_hi) beta *= p.tbound;
  if (ftraits<FT>::SPB == 26) beta *= nrm;
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

// The first operand of the post-hop term, copied into hop buffer 0 while hop
// 7 computes from buffer 1: chi for the A.chi - b.D.psi forms, else the
// first CloverBlock half of the clover dslash (none for the other forms).
template <typename FT, int FAM, bool ACH> struct AsyncTail {
  static constexpr bool CHI = ACH;
  static constexpr bool CLOVER0 = !ACH && FAM == FAM_CLOVER;
  static constexpr bool ANY = CHI || CLOVER0;
};

template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__device__ __forceinline__ void prefetch_tail(const KArgs<FT> &a, const WarpCtx &w)
{
  typedef Stage<FT, S> St;
  typedef AsyncTail<FT, FAM, ACH> TL;
  if constexpr (TL::CHI) stage_in_async<FT, S, AsyncCfg<FT, S, COMP12>::SPB, St::SP>(a.chi, w.own, w.buf, w.ln);
  if constexpr (TL::CLOVER0)
    stage_in_async<FT, S, 36 * S * (int)sizeof(elem_t<FT>), St::CL>(a.clov, w.tile * (72LL * S), w.buf, w.ln);
}

// one pipeline step: issue hop D+1 (after hop 6: the post-hop term's first
// operand, prefetch_tail), wait for hop D, compute hop D
template <typename FT, int S, bool COMP12, int FAM, bool ACH, int D>
__device__ __forceinline__ void pipe_step(const KArgs<FT> &a, const GeoDev &g, const OpDev<comp_t<FT>> &p,
                                          const Site &s, long long obase, const WarpCtx &w,
                                          cx<comp_t<FT>> (&acc)[4][3])
{
  typedef AsyncCfg<FT, S, COMP12> A;
  if constexpr (D < 7) {
    prefetch_hop<FT, S, COMP12, D + 1>(a, g, s, obase, w, w.buf + ((D + 1) & 1) * A::HOP);
    cp_async_commit();
    cp_async_wait<1>();
  } else if constexpr (AsyncTail<FT, FAM, ACH>::ANY) {
    prefetch_tail<FT, S, COMP12, FAM, ACH>(a, w); // hop buffer 0 is free: hop 6 was the last to read it
    cp_async_commit();
    cp_async_wait<1>();
  } else {
    cp_async_wait<0>();
  }
  __syncwarp();
  compute_hop<FT, S, COMP12, D>(a, g, p, s, obase, w, w.buf + (D & 1) * A::HOP, acc);
  __syncwarp();
}

template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__device__ __forceinline__ void async_hops(const KArgs<FT> &a, const GeoDev &g, const OpDev<comp_t<FT>> &p,
                                           const Site &s, long long obase, const WarpCtx &w,
                                           cx<comp_t<FT>> (&acc)[4][3])
{
  prefetch_hop<FT, S, COMP12, 0>(a, g, s, obase, w, w.buf);
  cp_async_commit();
  pipe_step<FT, S, COMP12, FAM, ACH, 0>(a, g, p, s, obase, w, acc);
  pipe_step<FT, S, COMP12, FAM, ACH, 1>(a, g, p, s, obase, w, acc);
  pipe_step<FT, S, COMP12, FAM, ACH, 2>(a, g, p, s, obase, w, acc);
  pipe_step<FT, S, COMP12, FAM, ACH, 3>(a, g, p, s, obase, w, acc);
  pipe_step<FT, S, COMP12, FAM, ACH, 4>(a, g, p, s, obase, w, acc);
  pipe_step<FT, S, COMP12, FAM, ACH, 5>(a, g, p, s, obase, w, acc);
  pipe_step<FT, S, COMP12, FAM, ACH, 6>(a, g, p, s, obase, w, acc);
  pipe_step<FT, S, COMP12, FAM, ACH, 7>(a, g, p, s, obase, w, acc);
}

// The CloverBlock (both halves) applied to in, MODE into out: half 0 is in
// hop buffer 0 (prefetch_tail's copy, or `issue0` copies it now), half 1 is
// copied into hop buffer 1 here, so that it lands while half 0 computes.
// The operations of staged_clover.
template <typename FT, int S, bool COMP12, int MODE, bool RHO>
__device__ __forceinline__ void async_clover(const KArgs<FT> &a, const WarpCtx &w, int isPlus, comp_t<FT> rho,
                                             bool issue0, const cx<comp_t<FT>> (&in)[4][3],
                                             cx<comp_t<FT>> (&out)[4][3])
{
  typedef Stage<FT, S> St;
  typedef AsyncCfg<FT, S, COMP12> A;
  constexpr int CLB = 36 * S * (int)sizeof(elem_t<FT>);
  static_assert(St::G * St::CL <= A::HOP, "a CloverBlock half fits in a hop buffer");
  if (issue0) {
    stage_in_async<FT, S, CLB, St::CL>(a.clov, w.tile * (72LL * S), w.buf, w.ln);
    cp_async_commit();
  }
  stage_in_async<FT, S, CLB, St::CL>(a.clov, w.tile * (72LL * S) + 36LL * S, w.buf + A::HOP, w.ln);
  cp_async_commit();
  cp_async_wait<1>();
  __syncwarp();
  clover_block_sm<FT, S, MODE, RHO>(w.buf + (w.ln / S) * St::CL, w.lane, 0,
                                    rho_of_block<comp_t<FT>>(0, isPlus, rho), in, out);
  cp_async_wait<0>();
  __syncwarp();
  clover_block_sm<FT, S, MODE, RHO>(w.buf + A::HOP + (w.ln / S) * St::CL, w.lane, 1,
                                    rho_of_block<comp_t<FT>>(1, isPlus, rho), in, out);
  __syncwarp();
}

// The operator at site q0 (this lane's) of plane (z, t), all 32 lanes of a
// warp together; buf is the warp's AsyncCfg::BUF bytes of shared memory.
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__device__ __forceinline__ void async_body(const KArgs<FT> &a, const GeoDev &g, const OpDev<comp_t<FT>> &p, int z,
                                           int t, int q0, unsigned char *buf)
{
  typedef comp_t<FT> C;
  typedef Stage<FT, S> St;
  typedef AsyncCfg<FT, S, COMP12> A;
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
  if (A::XREG) {
    // the x region's copies go out now and complete with hop 0's
    w.xr = buf + A::XOFF;
    w.xhead = 1 - __shfl_sync(0xffffffffu, s.xcb, 0) / S;
    const long long tail = __shfl_sync(0xffffffffu, w.blk, 31) - __shfl_sync(0xffffffffu, s.xcb, 31) / S + g.nvecs - 1;
    stage_xregion<FT, S, COMP12>(a.psi, w.blk0, w.blk0 - 1 + w.xhead, tail, g.Pxyz * g.nt, w.xr, w.ln);
  }

  cx<C> acc[4][3];
#pragma unroll
  for (int sp = 0; sp < 4; sp++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[sp][c] = mk<C>(0, 0);
  async_hops<FT, S, COMP12, FAM, ACH>(a, g, p, s, obase, w, acc);
  cx<C> res[4][3];
  if (ACH) {
    // the hops (subtracted: beta negated by the host), then + A.chi; chi is
    // in hop buffer 0 (copied during hop 7)
    cx<C> ch[4][3];
    if (FAM == FAM_CLOVER) {
      // CloverBlock half 0 into hop buffer 1 while chi is read out
      stage_in_async<FT, S, 36 * S * (int)sizeof(elem_t<FT>), St::CL>(a.clov, w.tile * (72LL * S),
                                                                        w.buf + A::HOP, w.ln);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncwarp();
    load_spinor_sm<FT, S>(w.buf + (w.ln / S) * St::SP, w.lane, ch);
    __syncwarp();
    if (FAM == FAM_CLOVER) {
      // half 1 into hop buffer 0 (chi is in registers), then both halves
      constexpr int CLB = 36 * S * (int)sizeof(elem_t<FT>);
      stage_in_async<FT, S, CLB, St::CL>(a.clov, w.tile * (72LL * S) + 36LL * S, w.buf, w.ln);
      cp_async_commit();
      cp_async_wait<1>();
      __syncwarp();
      clover_block_sm<FT, S, MODE_ADD, true>(w.buf + A::HOP + (w.ln / S) * St::CL, w.lane, 0,
                                             rho_of_block<C>(0, p.isPlus, p.rho), ch, acc);
      cp_async_wait<0>();
      __syncwarp();
      clover_block_sm<FT, S, MODE_ADD, true>(w.buf + (w.ln / S) * St::CL, w.lane, 1,
                                             rho_of_block<C>(1, p.isPlus, p.rho), ch, acc);
      __syncwarp();
    } else if (FAM == FAM_TMCLOV) staged_full_clover<FT, S, MODE_ADD, true>(a, w, p.isPlus, p.rho, ch, acc);
    else ach_finish<FT, FAM>(a, p, w.tile, w.lane, S, ch, acc);
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) res[sp][c] = acc[sp][c];
  } else {
    if (FAM == FAM_CLOVER) async_clover<FT, S, COMP12, MODE_SET, false>(a, w, p.isPlus, (C)0, false, acc, res);
    else if (FAM == FAM_TMCLOV) staged_full_clover<FT, S, MODE_SET, false>(a, w, p.isPlus, (C)0, acc, res);
    else plain_post<FT, FAM>(a, p, w.tile, w.lane, S, acc, res);
  }
  store_spinor_sm<FT, S>(w.buf + (w.ln / S) * St::SP, w.lane, res);
  __syncwarp();
  stage_out<FT, S, A::SPB, St::SP>(a.out, w.own, w.buf, w.ln, active);
  __syncwarp();
}

// Work unit: one warp's 32 sites of one (z, t) plane, numbered over all
// planes (warp_units_per_plane per plane), so that no warp idles when a
// plane's sites do not fill whole blocks of 128 threads; one-dimensional grid
// of warp_blocks(g) blocks of 128 threads.  Threads past the plane's last
// site take part in the warp's copies (on a clamped site) and store nothing.
// Needs 16-byte aligned fields smaller than 32 GiB.
__host__ __device__ __forceinline__ int warp_units_per_plane(const GeoDev &g) { return (g.nxh * g.ny + 31) >> 5; }
__host__ __device__ __forceinline__ long long warp_units(const GeoDev &g)
{
  return (long long)warp_units_per_plane(g) * g.nz * g.nt;
}
inline long long warp_blocks(const GeoDev &g) { return (warp_units(g) + 3) / 4; }

// resident blocks per SM the register allocation must allow: five for the
// 32-bit clover forms (their 38.9 KB of shared memory per block fit five
// times; the others already stay under 102 registers or hold more shared
// memory), four otherwise
#ifndef QB_ASYNC_MINB_CLOVER
#define QB_ASYNC_MINB_CLOVER 5
#endif
template <typename FT, int FAM> constexpr int async_minb()
{
  return (FAM == FAM_CLOVER && sizeof(elem_t<FT>) == 4) ? QB_ASYNC_MINB_CLOVER : 4;
}

template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__global__ void __launch_bounds__(128, async_minb<FT, FAM>())
    async_site_kernel(const KArgs<FT> a, const GeoDev g, const OpDev<comp_t<FT>> p)
{
  __shared__ __align__(16) unsigned char smem[4][AsyncCfg<FT, S, COMP12>::BUF];
  const long long u = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  if (u >= warp_units(g)) return; // whole warps
  const int wpp = warp_units_per_plane(g);
  const int plane = (int)(u / wpp);
  const int wi = (int)(u - (long long)plane * wpp);
  async_body<FT, S, COMP12, FAM, ACH>(a, g, p, plane % g.nz, plane / g.nz, wi * 32 + (threadIdx.x & 31),
                                      smem[threadIdx.x >> 5]);
}

// Batched form: work unit = one warp's 32 sites of one plane of one item;
// b.it[k].first and b.total count such warps (each plane padded to whole
// warps).  The loop is uniform across a warp.
// resident blocks per SM the batched kernel's registers must allow: four
// (128 registers; the per-item parameters cost a 16-byte spill); five would
// spill over a kilobyte
#ifndef QB_BATCH_MINB
#define QB_BATCH_MINB 4
#endif
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__global__ void __launch_bounds__(128, QB_BATCH_MINB) batch_async_kernel(const __grid_constant__ BatchDev<FT> b)
{
  __shared__ __align__(16) unsigned char smem[4][AsyncCfg<FT, S, COMP12>::BUF];
  const long long stride = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long u = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < b.total; u += stride) {
    int k = 0;
    while (k + 1 < b.n && u >= b.it[k + 1].first) k++;
    const BatchItem<FT> &it = b.it[k];
    const int wpp = (it.g.nxh * it.g.ny + 31) >> 5;
    const long long loc = u - it.first;
    const int plane = (int)(loc / wpp);
    const int wi = (int)(loc - (long long)plane * wpp);
    async_body<FT, S, COMP12, FAM, ACH>(it.a, it.g, it.p, plane % it.g.nz, plane / it.g.nz,
                                        wi * 32 + (threadIdx.x & 31), smem[threadIdx.x >> 5]);
  }
}

} // namespace qb200
