// qb200_twin_kernel.cuh -- the single-RHS dslash for 16-bit storage (FP16,
// FP16 + per-site norm, BF16) with two neighbouring sites per thread and
// every field staged through shared memory.
//
// With 16-bit storage a site moves few bytes but still needs the full FP32
// arithmetic, so a thread-per-site kernel is issue-bound: one FFMA per FP32
// operation, one shared-memory load and one conversion per stored element,
// and ~50 address instructions per hop for its 16-byte cp.async rounds.
// Here:
//   * thread t of a warp owns the sites xcb and xcb + 1 (xcb even) of one row,
//     lanes (l, l+1) of one spinor block and of one link / clover tile, so
//     every stored element of the pair is one 32-bit half2 / bfloat162 load
//     and every operation of the site arithmetic is one FFMA2 / FMUL2 / FADD2
//     on (site, site + 1) pairs -- no broadcast operands.  The operations and
//     their order per site are those of site_body, so all kernels give the
//     same bits;
//   * a warp owns 64 consecutive sites of one (z, t) plane: 64 / S blocks and
//     as many link / clover tiles (the "groups"), and the S / 2 threads that
//     own a group's sites copy that group's pieces (the neighbour block of
//     the hop, the hop's link slab, chi, the clover blocks, and the result on
//     the way out) with 16-byte cp.async / vector stores: one base address
//     per thread and piece, fixed offsets per 16 bytes, so a copied 16 bytes
//     costs a few instructions.  (cp.async.bulk from one lane per piece was
//     tried: its operands must be warp-uniform, and with a piece per group
//     the compiler serialises the copies at 10-20 instructions each.)
//   * for SOALEN 8 and 16 the y/z/t neighbour blocks, the link slabs and chi
//     are read from shared memory with ldmatrix, four elements of the
//     thread's two lanes per instruction (tw_ld_elems), a quarter of the
//     32-bit shared loads;
//   * the x neighbours come from an x region staged once (the warp's blocks,
//     one on either side, the first block of the first row and the last
//     block of the last row), which overlays the second spinor buffer; the
//     next hop's copies are in flight while the warp computes the current one
//     (cp.async groups, two spinor and two link buffers).
// Layouts: VECLEN == SOALEN in {4, 8, 16}; fields 16-byte aligned, smaller
// than 32 GiB.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "qb200_async_kernel.cuh"
#include "qb200_pair_kernel.cuh"

namespace qb200 {

// --------------------------------------------------------------------------
// staging geometry of one warp (64 sites, G = 64 / S groups)

template <typename FT, int S, bool COMP12> struct TwinCfg {
  typedef elem_t<FT> E;
  static_assert(sizeof(E) == 2, "the twin kernel serves 16-bit storage");
  static constexpr int G = 64 / S;                                // groups (blocks / tiles) per warp
  static constexpr int TPG = S / 2;                               // threads per group
  static constexpr int SPB = ftraits<FT>::SPB;                    // elements per lane of a spinor block
  static constexpr int SPBB = SPB * S * 2;                        // spinor block bytes
  static constexpr int R = COMP12 ? 2 : 3;
  static constexpr int LKB = R * 6 * S * 2;                       // link slab bytes (one direction of a tile)
  static constexpr int TLB = 8 * LKB;                             // link tile bytes
  static constexpr int SP = Stage<FT, S>::stride(SPB);            // staged spinor block (bank-spread padding)
  static constexpr int LKS = Stage<FT, S>::stride(R * 6);         // staged link slab
  static constexpr int CLB = 72 * S * 2, CS = CLB + 16;           // staged CloverBlock (both halves)
  static constexpr int FCB = 72 * S * 2, FCS = Stage<FT, S>::stride(72); // FullCloverBlock half
  static constexpr int XS = G + 4;                                // x region slots
  // spinor buffer 0 at slot 0; spinor buffer 1 and the x region share the
  // slots from G on (the x region is read by hops 0 and 1 only, buffer 1 is
  // first written for hop 3); link buffers after them; after the hops the
  // clover blocks reuse the space from 0
  static constexpr int X0 = G * SP;                               // x region / spinor buffer 1
  static constexpr int LOFF = X0 + XS * SP;
  static constexpr int mx(int a, int b) { return a > b ? a : b; }
  static constexpr int DOFF = mx(mx(LOFF + 2 * G * LKS, G * CS), G * FCS); // neighbour-block table
  static constexpr int WB0 = DOFF + 8 * 32 * 4;
  static constexpr int WB = (WB0 + 127) / 128 * 128;              // bytes per warp
  static_assert(SPBB % 16 == 0 && LKB % 16 == 0 && CLB % 16 == 0 && FCB % 16 == 0, "copies of 16-byte units");
  static_assert(SP % 16 == 0 && LKS % 16 == 0 && CS % 16 == 0 && FCS % 16 == 0 && X0 % 16 == 0 && LOFF % 16 == 0,
                "16-byte aligned staging slots");
};

constexpr int kTwinWarps = 4; // warps per block
// resident blocks per SM the register allocation must allow: 4 (128
// registers) for the Wilson and twisted-mass forms; the clover forms hold
// chi, the accumulators and the clover elements at once and would spill
// there, so they get 3 (168 registers)
#ifndef QB_TWIN_MINB
#define QB_TWIN_MINB 4
#endif
#ifndef QB_TWIN_MINB_CLOVER
#define QB_TWIN_MINB_CLOVER 3
#endif

template <typename FT, int S> constexpr bool twin_layout()
{
  return (S == 4 || S == 8 || S == 16) && sizeof(elem_t<FT>) == 2;
}

// two adjacent stored elements -> float2
template <typename FT> struct tw_io;
template <> struct tw_io<__half> {
  static __device__ __forceinline__ float2 cv2(const void *p) { return __half22float2(*(const __half2 *)p); }
  static __device__ __forceinline__ void st2(void *p, float2 v) { *(__half2 *)p = __float22half2_rn(v); }
};
template <> struct tw_io<half_norm> : tw_io<__half> {};
template <> struct tw_io<__nv_bfloat16> {
  static __device__ __forceinline__ float2 cv2(const void *p)
  {
    return __bfloat1622float2(*(const __nv_bfloat162 *)p);
  }
  static __device__ __forceinline__ void st2(void *p, float2 v) { *(__nv_bfloat162 *)p = __float22bfloat162_rn(v); }
};

// element k of the lanes (l, l+1) of a staged group
template <typename FT, int S>
__device__ __forceinline__ float2 tw_ld2(const unsigned char *grp, int k, int l)
{
  return tw_io<FT>::cv2(reinterpret_cast<const elem_t<FT> *>(grp) + k * S + l);
}

// two adjacent stored elements held in a 32-bit register -> float2
template <typename FT> __device__ __forceinline__ float2 tw_cvt(unsigned v)
{
  return tw_io<FT>::cv2(&v);
}

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3)
{
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2(unsigned addr, unsigned &r0, unsigned &r1)
{
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(addr));
}

// Elements 0..NE-1 of the thread's lanes (2 tig, 2 tig + 1) in its group's
// staged piece (group r's piece at base + r * GST, element k at + k * 2S
// bytes), as raw 32-bit pairs.  S = 8, 16: ldmatrix, four elements per
// instruction -- matrix m of pass q is element 4q + m of the warp's groups,
// one 16-byte row per group (two for S = 16), and thread t receives bytes
// 4 (t % 4) of row t / 4, which are its own two lanes.  S = 4 (an element
// of a group is 8 bytes, half a row): 32-bit loads.  All 32 lanes call it.
template <typename FT, int S, int GST, int NE>
__device__ __forceinline__ void tw_ld_elems(const unsigned char *base, int ln, unsigned (&v)[NE])
{
  static_assert(NE % 2 == 0, "elements in pairs");
  if constexpr (S >= 8) {
    static_assert(GST % 16 == 0, "16-byte aligned rows");
    constexpr int RPG = S / 8; // 16-byte rows per element of a group
    const int r = ln & 7, m = ln >> 3;
    const unsigned a = (unsigned)__cvta_generic_to_shared(base) + (unsigned)((r / RPG) * GST + m * 2 * S + (r % RPG) * 16);
#pragma unroll
    for (int q = 0; q < NE / 4; q++) ldsm_x4(a + q * 8 * S, v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    if constexpr (NE % 4 == 2) ldsm_x2(a + (NE / 4) * 8 * S, v[NE - 2], v[NE - 1]);
  } else {
    const int gi = ln / (S / 2), tig = ln - gi * (S / 2);
#pragma unroll
    for (int k = 0; k < NE; k++) v[k] = *reinterpret_cast<const unsigned *>(base + gi * GST + k * 2 * S + 4 * tig);
  }
}

__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// recon_row3 on a pair of links, operation for operation
__device__ __forceinline__ void recon_row3_2(c2 (&G)[3][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int c1 = (c + 1) % 3, c2i = (c + 2) % 3;
    float2 re = f2mul(G[0][c1].re, G[1][c2i].re);
    re = f2fma(neg2(G[0][c1].im), G[1][c2i].im, re);
    re = f2fma(neg2(G[0][c2i].re), G[1][c1].re, re);
    re = f2fma(G[0][c2i].im, G[1][c1].im, re);
    float2 im = f2mul(G[0][c1].re, G[1][c2i].im);
    im = f2fma(G[0][c1].im, G[1][c2i].re, im);
    im = f2fma(neg2(G[0][c2i].re), G[1][c1].im, im);
    im = f2fma(neg2(G[0][c2i].im), G[1][c1].re, im);
    G[2][c].re = re;
    G[2][c].im = neg2(im);
  }
}

// mult_link on a pair of links (per-site link elements, no broadcasts)
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
        const float2 gi = ADJ ? neg2(g.im) : g.im; // conj for the backward hop
        if (k == 0) {
          re = f2mul(g.re, b[s][k].re);
          im = f2mul(g.re, b[s][k].im);
        } else {
          re = f2fma(g.re, b[s][k].re, re);
          im = f2fma(g.re, b[s][k].im, im);
        }
        re = f2fma(neg2(gi), b[s][k].im, re);
        im = f2fma(gi, b[s][k].re, im);
      }
      ub[s][c1].re = re;
      ub[s][c1].im = im;
    }
}

// recons with a per-site coefficient pair
template <int MU>
__device__ __forceinline__ void recons2v(const c2 (&ub)[2][3], float2 beta, float tau, c2 (&acc)[4][3])
{
  const float s2 = tau * (float)rec_sg2(MU), s3 = tau * (float)rec_sg3(MU);
  const float2 b2 = make_float2(beta.x * s2, beta.y * s2);
  const float2 b3 = make_float2(beta.x * s3, beta.y * s3);
  constexpr int i2 = rec_s2(MU), i3 = 1 - rec_s2(MU);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[0][c].re = f2fma(beta, ub[0][c].re, acc[0][c].re);
    acc[0][c].im = f2fma(beta, ub[0][c].im, acc[0][c].im);
    acc[1][c].re = f2fma(beta, ub[1][c].re, acc[1][c].re);
    acc[1][c].im = f2fma(beta, ub[1][c].im, acc[1][c].im);
    if (rec_i(MU)) { // += b * i * ub
      acc[2][c].re = f2fma(neg2(b2), ub[i2][c].im, acc[2][c].re);
      acc[2][c].im = f2fma(b2, ub[i2][c].re, acc[2][c].im);
      acc[3][c].re = f2fma(neg2(b3), ub[i3][c].im, acc[3][c].re);
      acc[3][c].im = f2fma(b3, ub[i3][c].re, acc[3][c].im);
    } else {
      acc[2][c].re = f2fma(b2, ub[i2][c].re, acc[2][c].re);
      acc[2][c].im = f2fma(b2, ub[i2][c].im, acc[2][c].im);
      acc[3][c].re = f2fma(b3, ub[i3][c].re, acc[3][c].re);
      acc[3][c].im = f2fma(b3, ub[i3][c].im, acc[3][c].im);
    }
  }
}

// herm_apply on a pair of sites, elements read from a staged CloverBlock
// half (dg: element i, od: elements 6 + 2i, 7 + 2i), operation for operation
template <typename FT, int S, int MODE, bool RHO>
__device__ __forceinline__ void herm_apply_tw(const unsigned char *grp, int l, int blk, float rhob,
                                              const c2 (&in)[4][3], c2 (&out)[4][3])
{
#pragma unroll
  for (int r = 0; r < 6; r++) {
    const c2 v = in[2 * blk + r / 3][r % 3];
    const float2 d = tw_ld2<FT, S>(grp, r, l);
    float2 re1 = f2mul(d, v.re), im1 = f2mul(d, v.im);
    float2 re2 = bc(0.f), im2 = bc(0.f);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      if (c == r) continue;
      const c2 w = in[2 * blk + c / 3][c % 3];
      const int o = c < r ? r * (r - 1) / 2 + c : c * (c - 1) / 2 + r;
      const float2 ar = tw_ld2<FT, S>(grp, 6 + 2 * o, l), ai = tw_ld2<FT, S>(grp, 7 + 2 * o, l);
      if (c < r) { // A[r][c] = od[r(r-1)/2+c]
        re1 = f2fma(ar, w.re, re1);
        re1 = f2fma(neg2(ai), w.im, re1);
        im1 = f2fma(ar, w.im, im1);
        im1 = f2fma(ai, w.re, im1);
      } else { // A[r][c] = conj(od[c(c-1)/2+r])
        re2 = f2fma(ar, w.re, re2);
        re2 = f2fma(ai, w.im, re2);
        im2 = f2fma(ar, w.im, im2);
        im2 = f2fma(neg2(ai), w.re, im2);
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

// dense_apply (a dense FullCloverBlock half on a pair of sites) for rows r0,
// r0 + 1 of block `blk` only, their 24 elements staged at grp (element
// (r - r0) * 12 + 2c + ri); dense_apply's operations per row, so the block
// applied two rows at a time gives the same bits
template <typename FT, int S, int MODE, bool RHO>
__device__ __forceinline__ void dense_rows_tw(const unsigned char *grp, int l, int blk, int r0, float rhob,
                                              const c2 (&in)[4][3], c2 (&out)[4][3])
{
#pragma unroll
  for (int rr = 0; rr < 2; rr++) {
    const int r = r0 + rr;
    float2 re1 = bc(0.f), im1 = bc(0.f), re2 = bc(0.f), im2 = bc(0.f);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      const float2 ar = tw_ld2<FT, S>(grp, (rr * 6 + c) * 2 + 0, l);
      const float2 ai = tw_ld2<FT, S>(grp, (rr * 6 + c) * 2 + 1, l);
      const c2 w = in[2 * blk + c / 3][c % 3];
      if (c < 3) {
        re1 = f2fma(ar, w.re, re1);
        re1 = f2fma(neg2(ai), w.im, re1);
        im1 = f2fma(ar, w.im, im1);
        im1 = f2fma(ai, w.re, im1);
      } else {
        re2 = f2fma(ar, w.re, re2);
        re2 = f2fma(neg2(ai), w.im, re2);
        im2 = f2fma(ar, w.im, im2);
        im2 = f2fma(ai, w.re, im2);
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

// --------------------------------------------------------------------------
// copies

// the group's BYTES from gsrc to sdst, chunk k = tig + TPG c of 16 bytes
// per thread (tig: the thread's index in its group)
template <int BYTES, int TPG>
__device__ __forceinline__ void tw_cp(unsigned char *sdst, const void *gsrc, int tig)
{
  constexpr int CH = BYTES / 16;
  const uint4 *src = reinterpret_cast<const uint4 *>(gsrc);
#pragma unroll
  for (int c = 0; c < (CH + TPG - 1) / TPG; c++) {
    const int k = tig + c * TPG;
    if (CH % TPG == 0 || k < CH) cp_async16(sdst + k * 16, src + k);
  }
}

// the reverse with vector stores (shared -> global)
template <int BYTES, int TPG>
__device__ __forceinline__ void tw_st(void *gdst, const unsigned char *ssrc, int tig)
{
  constexpr int CH = BYTES / 16;
  uint4 *dst = reinterpret_cast<uint4 *>(gdst);
#pragma unroll
  for (int c = 0; c < (CH + TPG - 1) / TPG; c++) {
    const int k = tig + c * TPG;
    if (CH % TPG == 0 || k < CH) dst[k] = *reinterpret_cast<const uint4 *>(ssrc + k * 16);
  }
}

struct TwinCtx {
  unsigned char *buf; // the warp's shared memory
  int ln;             // lane in the warp
  int gi, tig;        // this thread's group and its index in the group
  int lane;           // the pair's first lane in its block (even)
  long long tile;     // the pair's link / clover tile
  long long own;      // element index of the pair's spinor block
  long long blk, blk0;
  int xhead;          // x-region slot of the first row's first block
};

// the neighbour block of hop D (2..7) into spinor buffer (D & 1), slot gi.
// The block offset comes from the thread's table in shared memory (written
// once at the start): computed in place, every hop's 64-bit addresses were
// hoisted to the start and held in registers (226 of them).
template <typename FT, int S, bool COMP12, int D>
__device__ __forceinline__ void tw_issue_spinor(const KArgs<FT> &a, const TwinCtx &w)
{
  typedef TwinCfg<FT, S, COMP12> T;
  const int d = reinterpret_cast<const int *>(w.buf + T::DOFF)[(D - 2) * 32 + w.ln];
  tw_cp<T::SPBB, T::TPG>(w.buf + (D & 1) * T::X0 + w.gi * T::SP, a.psi + w.own + (long long)d * (T::SPB * S), w.tig);
}

// the link slab of direction D of the group's tile into link buffer (D & 1)
template <typename FT, int S, bool COMP12, int D>
__device__ __forceinline__ void tw_issue_link(const KArgs<FT> &a, const TwinCtx &w)
{
  typedef TwinCfg<FT, S, COMP12> T;
  tw_cp<T::LKB, T::TPG>(w.buf + T::LOFF + ((D & 1) * T::G + w.gi) * T::LKS,
                        a.gauge + w.tile * (8LL * T::R * 6 * S) + (long long)D * T::R * 6 * S, w.tig);
}

// x-region slot and lane of the x neighbour at xn of a site in the row whose
// first block is at slot `row0`
template <int S, int G>
__device__ __forceinline__ void tw_xslot(int row0, int xn, int xhead, int &slot, int &lane)
{
  int sl = row0 + xn / S;
  sl = (sl >= 0 && sl < G + 2) ? sl : (sl == xhead ? G + 2 : G + 3);
  slot = sl;
  lane = xn % S;
}

// hop D (x hops from the x region, the others from spinor buffer D & 1;
// the link slab from link buffer D & 1)
template <typename FT, int S, bool COMP12, int D>
__device__ __forceinline__ void tw_compute_hop(const GeoDev &g, const OpDev<float> &p, const Site &s,
                                               const TwinCtx &w, c2 (&acc)[4][3])
{
  typedef TwinCfg<FT, S, COMP12> T;
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  c2 psi[4][3];
  float2 nrm = make_float2(1.f, 1.f);
  bool crossA = false, crossB = false;
  if (MU == 0) {
    // sites xcb (A) and xcb + 1 (B); their x neighbours, one element at a time
    int xa = s.xcb, xb = s.xcb + 1;
    if (D == 0 && s.par == 0) {
      crossA = xa == 0;
      xa = xa > 0 ? xa - 1 : g.nxh - 1;
      xb = xb - 1;
    }
    if (D == 1 && s.par == 1) {
      crossB = xb == g.nxh - 1;
      xa = xa + 1;
      xb = xb < g.nxh - 1 ? xb + 1 : 0;
    }
    const int row0 = (int)(w.blk - w.blk0) + 1 - s.xcb / S;
    int sa, la, sb, lb;
    tw_xslot<S, T::G>(row0, xa, w.xhead, sa, la);
    tw_xslot<S, T::G>(row0, xb, w.xhead, sb, lb);
    const unsigned char *ga = w.buf + T::X0 + sa * T::SP, *gb = w.buf + T::X0 + sb * T::SP;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        const int kr = (c * 4 + sp) * 2, ki = kr + 1;
        psi[sp][c].re = make_float2(sm_ld<FT, S>(ga, kr, la), sm_ld<FT, S>(gb, kr, lb));
        psi[sp][c].im = make_float2(sm_ld<FT, S>(ga, ki, la), sm_ld<FT, S>(gb, ki, lb));
      }
    if (T::SPB == 26)
      nrm = make_float2(reinterpret_cast<const float *>(ga + 48 * S)[la],
                        reinterpret_cast<const float *>(gb + 48 * S)[lb]);
  } else {
    const unsigned char *grp = w.buf + (D & 1) * T::X0 + w.gi * T::SP;
    unsigned v[24];
    tw_ld_elems<FT, S, T::SP, 24>(w.buf + (D & 1) * T::X0, w.ln, v);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        psi[sp][c].re = tw_cvt<FT>(v[(c * 4 + sp) * 2 + 0]);
        psi[sp][c].im = tw_cvt<FT>(v[(c * 4 + sp) * 2 + 1]);
      }
    if (T::SPB == 26) nrm = reinterpret_cast<const float2 *>(grp + 48 * S)[w.lane >> 1];
    bool cross;
    neighbour_offset<S, D>(g, s, 1, 1, &cross);
    crossA = crossB = cross;
  }
  c2 G[3][3];
  {
    unsigned v[T::R * 6];
    tw_ld_elems<FT, S, T::LKS, T::R * 6>(w.buf + T::LOFF + (D & 1) * T::G * T::LKS, w.ln, v);
#pragma unroll
    for (int r = 0; r < T::R; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        G[r][c].re = tw_cvt<FT>(v[(r * 3 + c) * 2 + 0]);
        G[r][c].im = tw_cvt<FT>(v[(r * 3 + c) * 2 + 1]);
      }
    if (COMP12) recon_row3_2(G);
  }
  float beta = p.beta[D];
  if (D == 6 && s.t == 0 && p.t_edge_lo) beta *= p.tbound;
  if (D == 7 && s.t == g.nt - 1 && p.t_edge_hi) beta *= p.tbound;
  // FP16 + norm: the neighbour's norm scales the coefficient; a skipped hop
  // (crossing, accumulate[D] == 0) adds 0 * hop
  float2 b2 = make_float2(beta * nrm.x, beta * nrm.y);
  if (!((p.acc_mask >> D) & 1u)) {
    if (crossA) b2.x = 0.f;
    if (crossB) b2.y = 0.f;
  }
  c2 b[2][3], ub[2][3];
  project2<D>(psi, p.isPlus ? 1.f : -1.f, b);
  mult2p<!FWD>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) phase2(ub, p.tbc[MU][0], FWD ? p.tbc[MU][1] : -p.tbc[MU][1]);
  recons2v<MU>(ub, b2, ((p.isPlus != 0) != FWD) ? 1.f : -1.f, acc);
}

// the group's FullCloverBlock of its tile (tl), taken two rows of a half at a
// time: piece q (0..5) is rows 2 (q % 3), 2 (q % 3) + 1 of half q / 3, 24
// consecutive elements per lane; it goes into spinor buffer b's slot of the
// group (24 elements fit in a spinor block's slot)
template <typename FT, int S, bool COMP12>
__device__ __forceinline__ void tw_issue_fcl_piece(const KArgs<FT> &a, const TwinCtx &w, long long tl, int q, int b)
{
  typedef TwinCfg<FT, S, COMP12> T;
  static_assert(24 <= T::SPB, "a piece fits in a spinor slot");
  tw_cp<24 * S * 2, T::TPG>(w.buf + (b ? T::X0 : 0) + w.gi * T::SP,
                            a.clov + tl * (144LL * S) + (q / 3) * 72LL * S + (q % 3) * 24LL * S, w.tig);
}

// the pair's tile, from the table written at the start
template <typename FT, int S, bool COMP12> __device__ __forceinline__ long long tw_tile(const TwinCtx &w)
{
  typedef TwinCfg<FT, S, COMP12> T;
  return reinterpret_cast<const long long *>(w.buf + T::DOFF + 6 * 32 * 4)[w.ln];
}

// The FullCloverBlock applied to in (MODE into out) in its six pieces, piece
// q read from spinor buffer (q + B0) & 1; piece 0's copy is in flight on
// entry, and each further piece is copied while the one before computes.
template <typename FT, int S, bool COMP12, int MODE, bool RHO, int B0>
__device__ __forceinline__ void tw_full_clover_pieces(const KArgs<FT> &a, const TwinCtx &w, long long tl, int isPlus,
                                                      float rho, const c2 (&in)[4][3], c2 (&out)[4][3])
{
  typedef TwinCfg<FT, S, COMP12> T;
#pragma unroll
  for (int q = 0; q < 6; q++) {
    if (q < 5) {
      tw_issue_fcl_piece<FT, S, COMP12>(a, w, tl, q + 1, (q + 1 + B0) & 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncwarp();
    dense_rows_tw<FT, S, MODE, RHO>(w.buf + (((q + B0) & 1) ? T::X0 : 0) + w.gi * T::SP, w.lane, q / 3, 2 * (q % 3),
                                    rho_of_block<float>(q / 3, isPlus, rho), in, out);
    __syncwarp();
  }
}

// one pipeline step: issue hop D+1's copies (its neighbour block, from hop 2
// on, and its link slab), wait for hop D's, compute hop D.  With hop 7 (spinor
// buffer 0 is free from then on), the post-hop term's first operand: chi for
// the A.chi - b.D.psi forms, else piece 0 of the TM-clover FullCloverBlock.
template <typename FT, int S, bool COMP12, int FAM, bool ACH, int D>
__device__ __forceinline__ void tw_step(const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p, const Site &s,
                                        long long obase, const TwinCtx &w, c2 (&acc)[4][3])
{
  typedef TwinCfg<FT, S, COMP12> T;
  if constexpr (D < 7) {
    if constexpr (D + 1 >= 2) tw_issue_spinor<FT, S, COMP12, D + 1>(a, w);
    tw_issue_link<FT, S, COMP12, D + 1>(a, w);
    cp_async_commit();
    cp_async_wait<1>();
  } else if constexpr (ACH) {
    tw_cp<T::SPBB, T::TPG>(w.buf + w.gi * T::SP, a.chi + w.own, w.tig);
    cp_async_commit();
    cp_async_wait<1>();
  } else if constexpr (FAM == FAM_TMCLOV) {
    tw_issue_fcl_piece<FT, S, COMP12>(a, w, tw_tile<FT, S, COMP12>(w), 0, 0);
    cp_async_commit();
    cp_async_wait<1>();
  } else {
    cp_async_wait<0>();
  }
  __syncwarp();
  tw_compute_hop<FT, S, COMP12, D>(g, p, s, w, acc);
  __syncwarp();
}

// The operator on the warp's 64 sites (chunk `chunk` of plane (z, t)); this
// thread's pair is sites q0, q0 + 1 of the plane.
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__device__ __forceinline__ void twin_body(const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p, int z, int t,
                                          int chunk, unsigned char *buf)
{
  typedef TwinCfg<FT, S, COMP12> T;
  typedef elem_t<FT> E;
  TwinCtx w;
  w.buf = buf;
  w.ln = threadIdx.x & 31;
  w.gi = w.ln / T::TPG;
  w.tig = w.ln - w.gi * T::TPG;
  const int nplane = g.nxh * g.ny;
  const int c0 = chunk * 64;
  const int q0 = c0 + 2 * w.ln;
  const bool active = q0 < nplane;
  const int q = active ? q0 : nplane - 2;
  Site s;
  s.z = z;
  s.t = t;
  s.y = q / g.nxh;
  s.xcb = q - s.y * g.nxh;
  s.par = (s.y + s.z + s.t + p.cb) & 1;
  w.tile = tile_of<S>(g, s, &w.lane);
  const long long obase = spinor_base<FT, S>(g, s);
  const long long ue = (long long)T::SPB * S; // elements per spinor block
  w.blk = obase / ue;
  w.own = w.blk * ue;
  const long long pbase = (long long)t * g.Pxyz + (long long)z * g.Pxy; // the plane's first block
  w.blk0 = pbase + c0 / S;
  w.xhead = 1 - (c0 % g.nxh) / S;
  {
    // block offsets of the y, z, t neighbours (hops 2..7) of the pair's block
    int *dt = reinterpret_cast<int *>(w.buf + T::DOFF);
    bool cross;
    dt[0 * 32 + w.ln] = (int)neighbour_offset<S, 2>(g, s, 1, 0, &cross);
    dt[1 * 32 + w.ln] = (int)neighbour_offset<S, 3>(g, s, 1, 0, &cross);
    dt[2 * 32 + w.ln] = (int)neighbour_offset<S, 4>(g, s, 1, 0, &cross);
    dt[3 * 32 + w.ln] = (int)neighbour_offset<S, 5>(g, s, 1, 0, &cross);
    dt[4 * 32 + w.ln] = (int)neighbour_offset<S, 6>(g, s, 1, 0, &cross);
    dt[5 * 32 + w.ln] = (int)neighbour_offset<S, 7>(g, s, 1, 0, &cross);
    // the pair's tile, read back when the clover blocks are copied
    reinterpret_cast<long long *>(dt + 6 * 32)[w.ln] = w.tile;
  }

  // x region: slot 1 + g holds group g's own block (copied by the group),
  // slots 0 and G + 1 the blocks on either side, G + 2 the first row's first
  // block, G + 3 the last row's last block (all threads; slots outside the
  // field stay unused)
  tw_cp<T::SPBB, T::TPG>(w.buf + T::X0 + (1 + w.gi) * T::SP, a.psi + w.own, w.tig);
  {
    const int nvalid = nplane - c0 < 64 ? nplane - c0 : 64;
    const int ylast = (c0 + nvalid - 1) / g.nxh;
    const long long tail = pbase + (long long)ylast * g.nvecs + g.nvecs - 1;
    const long long nblocks = g.Pxyz * g.nt;
    constexpr int CH = T::SPBB / 16;
#pragma unroll
    for (int c = 0; c < (4 * CH + 31) / 32; c++) {
      const int m = w.ln + 32 * c;
      const int e = m / CH, k = m - e * CH; // extra slot e (0..3), chunk k
      const int slot = e == 0 ? 0 : (e == 1 ? T::G + 1 : (e == 2 ? T::G + 2 : T::G + 3));
      const long long b = e == 0 ? w.blk0 - 1 : (e == 1 ? w.blk0 + T::G : (e == 2 ? w.blk0 - 1 + w.xhead : tail));
      if (m < 4 * CH && b >= 0 && b < nblocks)
        cp_async16(w.buf + T::X0 + slot * T::SP + k * 16, reinterpret_cast<const uint4 *>(a.psi + b * ue) + k);
    }
  }
  tw_issue_link<FT, S, COMP12, 0>(a, w);
  cp_async_commit();

  c2 acc[4][3];
#pragma unroll
  for (int sp = 0; sp < 4; sp++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[sp][c].re = acc[sp][c].im = bc(0.f);
  tw_step<FT, S, COMP12, FAM, ACH, 0>(a, g, p, s, obase, w, acc);
  tw_step<FT, S, COMP12, FAM, ACH, 1>(a, g, p, s, obase, w, acc);
  tw_step<FT, S, COMP12, FAM, ACH, 2>(a, g, p, s, obase, w, acc);
  tw_step<FT, S, COMP12, FAM, ACH, 3>(a, g, p, s, obase, w, acc);
  tw_step<FT, S, COMP12, FAM, ACH, 4>(a, g, p, s, obase, w, acc);
  tw_step<FT, S, COMP12, FAM, ACH, 5>(a, g, p, s, obase, w, acc);
  tw_step<FT, S, COMP12, FAM, ACH, 6>(a, g, p, s, obase, w, acc);
  tw_step<FT, S, COMP12, FAM, ACH, 7>(a, g, p, s, obase, w, acc);

  // the tile from the table: its chunk addresses are formed here, not held
  // in registers across the hops
  const long long tl = reinterpret_cast<const long long *>(w.buf + T::DOFF + 6 * 32 * 4)[w.ln];
  const E *clov_tile = a.clov + tl * (FAM == FAM_CLOVER ? 72LL * S : 144LL * S);
  c2 res[4][3];
  if (ACH) {
    // the hops (subtracted: beta negated by the host), then + A.chi; chi is
    // in spinor buffer 0 (copied with hop 7)
    c2 ch[4][3];
    if (FAM == FAM_TMCLOV) {
      // piece 0 of the FullCloverBlock into spinor buffer 1 while chi is read
      tw_issue_fcl_piece<FT, S, COMP12>(a, w, tl, 0, 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncwarp();
    {
      const unsigned char *grp = w.buf + w.gi * T::SP;
      float2 cn = make_float2(1.f, 1.f);
      if (T::SPB == 26) cn = reinterpret_cast<const float2 *>(grp + 48 * S)[w.lane >> 1];
      unsigned v[24];
      tw_ld_elems<FT, S, T::SP, 24>(w.buf, w.ln, v);
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int sp = 0; sp < 4; sp++) {
          ch[sp][c].re = tw_cvt<FT>(v[(c * 4 + sp) * 2 + 0]);
          ch[sp][c].im = tw_cvt<FT>(v[(c * 4 + sp) * 2 + 1]);
          if (T::SPB == 26) {
            ch[sp][c].re = f2mul(ch[sp][c].re, cn);
            ch[sp][c].im = f2mul(ch[sp][c].im, cn);
          }
        }
    }
    __syncwarp();
    if (FAM == FAM_WILSON) {
#pragma unroll
      for (int sp = 0; sp < 4; sp++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          acc[sp][c].re = f2fma(bc(p.alpha), ch[sp][c].re, acc[sp][c].re);
          acc[sp][c].im = f2fma(bc(p.alpha), ch[sp][c].im, acc[sp][c].im);
        }
    } else if (FAM == FAM_TM) {
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        const float m = (((sp < 2) == (p.isPlus != 0)) ? 1.f : -1.f) * p.mu;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          acc[sp][c].re = f2fma(bc(p.alpha), f2fma(bc(-m), ch[sp][c].im, ch[sp][c].re), acc[sp][c].re);
          acc[sp][c].im = f2fma(bc(p.alpha), f2fma(bc(m), ch[sp][c].re, ch[sp][c].im), acc[sp][c].im);
        }
      }
    } else if (FAM == FAM_CLOVER) {
      // the whole CloverBlock of the tile (both halves)
      tw_cp<T::CLB, T::TPG>(w.buf + w.gi * T::CS, clov_tile, w.tig);
      cp_async_commit();
      cp_async_wait<0>();
      __syncwarp();
#pragma unroll
      for (int blk = 0; blk < 2; blk++)
        herm_apply_tw<FT, S, MODE_ADD, true>(w.buf + w.gi * T::CS + blk * (T::CLB / 2), w.lane, blk,
                                             rho_of_block<float>(blk, p.isPlus, p.rho), ch, acc);
      __syncwarp();
    } else {
      // the FullCloverBlock two rows at a time, piece 0 in spinor buffer 1
      tw_full_clover_pieces<FT, S, COMP12, MODE_ADD, true, 1>(a, w, tl, p.isPlus, p.rho, ch, acc);
    }
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) res[sp][c] = acc[sp][c];
  } else {
    if (FAM == FAM_CLOVER) {
      tw_cp<T::CLB, T::TPG>(w.buf + w.gi * T::CS, clov_tile, w.tig);
      cp_async_commit();
      cp_async_wait<0>();
      __syncwarp();
#pragma unroll
      for (int blk = 0; blk < 2; blk++)
        herm_apply_tw<FT, S, MODE_SET, false>(w.buf + w.gi * T::CS + blk * (T::CLB / 2), w.lane, blk, 0.f, acc,
                                              res);
      __syncwarp();
    } else if (FAM == FAM_TMCLOV) {
      // two rows at a time, piece 0 (copied with hop 7) in spinor buffer 0
      tw_full_clover_pieces<FT, S, COMP12, MODE_SET, false, 0>(a, w, tl, p.isPlus, 0.f, acc, res);
    } else if (FAM == FAM_TM) {
      // muinv (1 + sg i mu) acc, sg = -1 on the upper spins for plus
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

  // the result: pairs to the group's slot (with the per-site norms of FP16 +
  // norm, store_spinor's rule), then the group's threads store the block
  {
    unsigned char *grp = w.buf + w.gi * T::SP;
    float2 scale = make_float2(1.f, 1.f);
    if (T::SPB == 26) {
      float ma = 0.f, mb = 0.f;
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int sp = 0; sp < 4; sp++) {
          ma = fmaxf(ma, fmaxf(fabsf(res[sp][c].re.x), fabsf(res[sp][c].im.x)));
          mb = fmaxf(mb, fmaxf(fabsf(res[sp][c].re.y), fabsf(res[sp][c].im.y)));
        }
      const float na = ma > 0.f ? ma : 1.f, nb = mb > 0.f ? mb : 1.f;
      reinterpret_cast<float2 *>(grp + 48 * S)[w.lane >> 1] = make_float2(na, nb);
      scale = make_float2(1.f / na, 1.f / nb);
    }
    E *e = reinterpret_cast<E *>(grp);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int sp = 0; sp < 4; sp++) {
        tw_io<FT>::st2(e + ((c * 4 + sp) * 2 + 0) * S + w.lane, f2mul(res[sp][c].re, scale));
        tw_io<FT>::st2(e + ((c * 4 + sp) * 2 + 1) * S + w.lane, f2mul(res[sp][c].im, scale));
      }
    __syncwarp();
    if (active) tw_st<T::SPBB, T::TPG>(a.out + w.own, grp, w.tig);
  }
}

// Grid: one warp per chunk of 64 sites of a (z, t) plane; nchunk chunks per
// plane, kTwinWarps warps per block, TwinCfg::WB bytes of dynamic shared
// memory per warp.
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
__global__ void __launch_bounds__(kTwinWarps * 32,
                                  (FAM == FAM_CLOVER || FAM == FAM_TMCLOV) ? QB_TWIN_MINB_CLOVER : QB_TWIN_MINB)
    twin_site_kernel(const KArgs<FT> a, const GeoDev g, const OpDev<float> p, int nchunk)
{
  typedef TwinCfg<FT, S, COMP12> T;
  extern __shared__ __align__(128) unsigned char tw_smem[];
  const int warp = threadIdx.x >> 5;
  const long long wg = (long long)blockIdx.x * kTwinWarps + warp;
  const long long nw = (long long)g.nz * g.nt * nchunk;
  if (wg >= nw) return;
  const int plane = (int)(wg / nchunk);
  const int chunk = (int)(wg - (long long)plane * nchunk);
  twin_body<FT, S, COMP12, FAM, ACH>(a, g, p, plane % g.nz, plane / g.nz, chunk, tw_smem + warp * T::WB);
}

} // namespace qb200
