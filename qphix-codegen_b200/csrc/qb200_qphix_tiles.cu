// qb200_qphix_tiles.cu -- the per-tile QPhiX kernel interface on the GPU.
//
// Defines the function templates declared in include/qphix_b200_qphix.h
// (the signatures of codegen/jinja/*_decl.h.j2) and instantiates them for a
// "b200" ISA: FT = float, double, QPhiX::half; veclen = soalen = 4, 8, 16;
// compress12 true/false; all 16 tbc_x..t combinations of the body kernels
// and tbc true/false of the face kernels.  QPhiX, which calls these once per
// tile of veclen sites, links against this library unchanged.
//
// Each call checks its arguments on the host, copies the offset and
// accumulate arrays into the kernel's parameter block and runs one 32-thread
// block (thread l = lane l of the tile) on the calling thread's per-thread
// default stream, then waits for it.  The per-site arithmetic is the one of
// the lattice-level kernels (qb200_device.cuh), so a tile computed here has
// the same bits as the same sites computed by qb200_dslash; only the
// addressing differs: it follows the reference's per-tile contract
// (codegen/data_types.cc:60-198):
//   - y, z, t and the site itself: row j of the tile reads S contiguous
//     elements at base + offs[j*S] (+ component*S) with base = xyBase for y
//     (ybOffs / yfOffs), zbBase..tfBase for z / t and xyBase / chiBase /
//     oBase (offs) for the site, its chi and its result;
//   - x backward (loadSplitSOAFVec, codegen/inst_sp_vec16.cc:609-636): lane
//     0 of row j reads one element at xyBase + xbOffs[j*S], lanes 1..S-1 read
//     S-1 contiguous elements at xyBase + xbOffs[j*S+1];
//   - x forward: lanes 0..S-2 read S-1 contiguous elements at
//     xyBase + xfOffs[j*S], lane S-1 one element at xyBase + xfOffs[j*S+S-1];
//   - accumulate[d]: lane mask for x and y, flag for z and t
//     (codegen/dslash.cc:109,248-290);
//   - beta per direction: coeff_s for x, y, z, coeff_t_b / coeff_t_f for t
//     back / forward (codegen/dslash.cc:79-86), subtracted in the achimbdpsi
//     form;
//   - faces (codegen/data_types.cc:462-626): component e = (spin*3+colour)*2
//     + re/im of the half spinor at outbuf[e*n + k], n = (veclen/soalen+1)/2
//     for x (k counts the lanes of mask that can lie on the face: lane 0 of a
//     row for dir 0, lane S-1 for dir 1), n = soalen for y when
//     soalen < veclen (row 0 for dir 2, the last row for dir 3), else
//     n = veclen and k = the lane.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "qphix_b200.h"
#include "qphix_b200_qphix.h"
#include "qb200_site_kernel.cuh"

namespace qb200 {
namespace qtile {

constexpr int kMaxLanes = 32;

// one call's parameter block (kernel parameters, under 1 KB)
struct TileDev {
  const void *xy, *zb, *zf, *tb, *tf, *chi, *gauge, *clov;
  void *out;
  const void *inbuf;
  void *outbuf;
  int xb[kMaxLanes], xf[kMaxLanes], yb[kMaxLanes], yf[kMaxLanes], offs[kMaxLanes];
  unsigned acc[8];
  double cs, ctf, ctb, alpha, mu, muinv, rho, beta;
  double tbc[4][2];
  unsigned tbc_mask;
  unsigned mask; // faces: lane mask
  int V, S, isPlus, dir;
};

// ---- device side ------------------------------------------------------

template <typename FT>
__device__ __forceinline__ void ld_site(const elem_t<FT> *p, int S, cx<comp_t<FT>> (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      sp[s][c].re = ftraits<FT>::ld(p + ((c * 4 + s) * 2 + 0) * S);
      sp[s][c].im = ftraits<FT>::ld(p + ((c * 4 + s) * 2 + 1) * S);
    }
}

template <typename FT>
__device__ __forceinline__ void st_site(elem_t<FT> *p, int S, const cx<comp_t<FT>> (&sp)[4][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int s = 0; s < 4; s++) {
      ftraits<FT>::st(p + ((c * 4 + s) * 2 + 0) * S, sp[s][c].re);
      ftraits<FT>::st(p + ((c * 4 + s) * 2 + 1) * S, sp[s][c].im);
    }
}

// first element (component 0) of lane l's neighbour in direction D
template <typename FT, int D>
__device__ __forceinline__ const elem_t<FT> *nb_ptr(const TileDev &a, int l)
{
  typedef elem_t<FT> E;
  const int S = a.S, j = l / S, ls = l - j * S, r0 = j * S;
  const E *xy = (const E *)a.xy;
  if (D == 0) return ls == 0 ? xy + a.xb[r0] : xy + a.xb[r0 + 1] + (ls - 1);
  if (D == 1) return ls < S - 1 ? xy + a.xf[r0] + ls : xy + a.xf[r0 + S - 1];
  if (D == 2) return xy + a.yb[r0] + ls;
  if (D == 3) return xy + a.yf[r0] + ls;
  const E *b = (const E *)(D == 4 ? a.zb : D == 5 ? a.zf : D == 6 ? a.tb : a.tf);
  return b + a.offs[r0] + ls;
}

template <typename FT, bool COMP12, int D>
__device__ __forceinline__ void tile_hop(const TileDev &a, const OpDev<comp_t<FT>> &p, int l,
                                         cx<comp_t<FT>> (&acc)[4][3])
{
  typedef comp_t<FT> C;
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  if (D < 4 ? !((a.acc[D] >> l) & 1u) : a.acc[D] == 0u) return;
  cx<C> psi[4][3], b[2][3], ub[2][3], G[3][3];
  ld_site<FT>(nb_ptr<FT, D>(a, l), a.S, psi);
  project<C, D>(psi, p.isPlus ? (C)1 : (C)-1, b);
  load_link<FT, COMP12, D>((const elem_t<FT> *)a.gauge, l, a.V, G);
  mult_link<C, !FWD>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) apply_phase<C>(ub, p.tbc[MU][0], FWD ? p.tbc[MU][1] : -p.tbc[MU][1]);
  recons<C, MU>(ub, p.beta[D], ((p.isPlus != 0) != FWD) ? (C)1 : (C)-1, acc);
}

template <typename FT>
__device__ __forceinline__ OpDev<comp_t<FT>> op_of(const TileDev &a, bool negate)
{
  typedef comp_t<FT> C;
  OpDev<C> p;
  const double sg = negate ? -1.0 : 1.0;
  for (int d = 0; d < 6; d++) p.beta[d] = (C)(sg * a.cs);
  p.beta[6] = (C)(sg * a.ctb);
  p.beta[7] = (C)(sg * a.ctf);
  p.tbound = (C)1;
  p.alpha = (C)a.alpha;
  p.mu = (C)a.mu;
  p.muinv = (C)a.muinv;
  p.rho = (C)a.rho;
  for (int m = 0; m < 4; m++) {
    p.tbc[m][0] = (C)a.tbc[m][0];
    p.tbc[m][1] = (C)a.tbc[m][1];
  }
  p.tbc_mask = a.tbc_mask;
  p.acc_mask = 0xffu;
  p.isPlus = a.isPlus;
  p.cb = 0;
  p.t_edge_lo = p.t_edge_hi = 0;
  return p;
}

template <typename FT, bool COMP12, int FAM, bool ACH>
__global__ void __launch_bounds__(kMaxLanes) tile_body_kernel(const __grid_constant__ TileDev a)
{
  typedef comp_t<FT> C;
  typedef elem_t<FT> E;
  const int l = threadIdx.x;
  if (l >= a.V) return;
  const OpDev<C> p = op_of<FT>(a, ACH);
  cx<C> acc[4][3], res[4][3];
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[s][c] = mk<C>(0, 0);
  tile_hop<FT, COMP12, 0>(a, p, l, acc);
  tile_hop<FT, COMP12, 1>(a, p, l, acc);
  tile_hop<FT, COMP12, 2>(a, p, l, acc);
  tile_hop<FT, COMP12, 3>(a, p, l, acc);
  tile_hop<FT, COMP12, 4>(a, p, l, acc);
  tile_hop<FT, COMP12, 5>(a, p, l, acc);
  tile_hop<FT, COMP12, 6>(a, p, l, acc);
  tile_hop<FT, COMP12, 7>(a, p, l, acc);
  const int S = a.S, j = l / S, own = a.offs[j * S] + (l - j * S);
  KArgs<FT> k;
  k.psi = k.chi = k.gauge = nullptr;
  k.out = nullptr;
  k.clov = (const E *)a.clov;
  if (ACH) {
    cx<C> ch[4][3];
    ld_site<FT>((const E *)a.chi + own, S, ch);
    ach_finish<FT, FAM>(k, p, 0, l, a.V, ch, acc);
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) res[s][c] = acc[s][c];
  } else {
    plain_post<FT, FAM>(k, p, 0, l, a.V, acc, res);
  }
  st_site<FT>((E *)a.out + own, S, res);
}

// face slot of lane l in direction D: -1 when the lane takes no part; *n =
// lanes per component in the face buffer
template <int D>
__device__ __forceinline__ int face_slot(const TileDev &a, int l, int *n)
{
  const int S = a.S, V = a.V, j = l / S, ls = l - j * S;
  if (D < 2) {
    *n = (V / S + 1) / 2;
    unsigned possible = 0;
    for (int r = 0; r < V; r += S) possible |= 1u << (r + (D == 0 ? 0 : S - 1));
    const unsigned act = a.mask & possible;
    if (!((act >> l) & 1u)) return -1;
    return __popc(act & ((1u << l) - 1u));
  }
  if (D < 4 && S != V) {
    *n = S;
    const int row = D == 2 ? 0 : V / S - 1;
    return j == row ? ls : -1;
  }
  *n = V;
  return l;
}

template <typename FT, int D>
__device__ __forceinline__ void tile_pack_lane(const TileDev &a, int l)
{
  typedef comp_t<FT> C;
  typedef elem_t<FT> E;
  int n;
  const int k = face_slot<D>(a, l, &n);
  if (k < 0) return;
  cx<C> sp[4][3], b[2][3];
  const bool masked = D < 4 && !((a.mask >> l) & 1u); // y lane outside the mask: zero
  if (masked) {
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) sp[s][c] = mk<C>(0, 0);
  } else {
    const int j = l / a.S;
    ld_site<FT>((const E *)a.xy + a.offs[j * a.S] + (l - j * a.S), a.S, sp);
  }
  // the projector of the opposite direction (codegen/dslash.cc:451-454)
  project<C, D>(sp, a.isPlus ? (C)-1 : (C)1, b);
  E *o = (E *)a.outbuf;
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      ftraits<FT>::st(o + ((s * 3 + c) * 2 + 0) * n + k, b[s][c].re);
      ftraits<FT>::st(o + ((s * 3 + c) * 2 + 1) * n + k, b[s][c].im);
    }
}

template <typename FT>
__global__ void __launch_bounds__(kMaxLanes) tile_pack_kernel(const __grid_constant__ TileDev a)
{
  const int l = threadIdx.x;
  if (l >= a.V) return;
  switch (a.dir) {
  case 0: tile_pack_lane<FT, 0>(a, l); break;
  case 1: tile_pack_lane<FT, 1>(a, l); break;
  case 2: tile_pack_lane<FT, 2>(a, l); break;
  case 3: tile_pack_lane<FT, 3>(a, l); break;
  case 4: tile_pack_lane<FT, 4>(a, l); break;
  case 5: tile_pack_lane<FT, 5>(a, l); break;
  case 6: tile_pack_lane<FT, 6>(a, l); break;
  default: tile_pack_lane<FT, 7>(a, l); break;
  }
}

// recons_add_face_vec (codegen/dslash.cc:463-553): +beta for clover faces,
// -beta otherwise (codegen/dslash_common.cc:1975-1981), then the clover /
// full clover / A^-1 term on that contribution
template <typename FT, bool COMP12, int FAM, int D>
__device__ __forceinline__ void tile_unpack_lane(const TileDev &a, int l)
{
  typedef comp_t<FT> C;
  typedef elem_t<FT> E;
  constexpr int MU = D / 2;
  constexpr bool BACK = (D & 1) == 0;
  constexpr bool CLOV = (FAM == FAM_CLOVER || FAM == FAM_TMCLOV);
  constexpr bool TM = (FAM == FAM_TM || FAM == FAM_TMCLOV);
  int n;
  const int k = face_slot<D>(a, l, &n);
  if (k < 0) return;
  if (D < 4 && !((a.mask >> l) & 1u)) return;
  const OpDev<C> p = op_of<FT>(a, false);
  const int S = a.S, j = l / S;
  E *op = (E *)a.out + a.offs[j * S] + (l - j * S);
  const E *in = (const E *)a.inbuf;
  cx<C> o[4][3], b[2][3], ub[2][3], G[3][3];
  ld_site<FT>(op, S, o);
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      b[s][c].re = ftraits<FT>::ld(in + ((s * 3 + c) * 2 + 0) * n + k);
      b[s][c].im = ftraits<FT>::ld(in + ((s * 3 + c) * 2 + 1) * n + k);
    }
  load_link<FT, COMP12, D>((const E *)a.gauge, l, a.V, G);
  mult_link<C, BACK>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) apply_phase<C>(ub, p.tbc[MU][0], BACK ? -p.tbc[MU][1] : p.tbc[MU][1]);
  const C tau = ((p.isPlus != 0) == BACK) ? (C)1 : (C)-1;
  const C beta = CLOV ? (C)a.beta : (C)-a.beta;
  if (CLOV || TM) {
    cx<C> dout[4][3];
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) dout[s][c] = mk<C>(0, 0);
    recons<C, MU>(ub, beta, tau, dout);
    if (CLOV) {
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        if (FAM == FAM_CLOVER)
          clover_block<FT, MODE_ADD, false>((const E *)a.clov, l, a.V, blk, (C)0, dout, o);
        else
          full_clover_block<FT, MODE_ADD, false>((const E *)a.clov, l, a.V, blk, (C)0, dout, o);
      }
    } else {
      inv_twisted<C, true>(dout, p.isPlus, p.mu, p.muinv, o);
    }
  } else {
    recons<C, MU>(ub, beta, tau, o);
  }
  st_site<FT>(op, S, o);
}

template <typename FT, bool COMP12, int FAM>
__global__ void __launch_bounds__(kMaxLanes) tile_unpack_kernel(const __grid_constant__ TileDev a)
{
  const int l = threadIdx.x;
  if (l >= a.V) return;
  switch (a.dir) {
  case 0: tile_unpack_lane<FT, COMP12, FAM, 0>(a, l); break;
  case 1: tile_unpack_lane<FT, COMP12, FAM, 1>(a, l); break;
  case 2: tile_unpack_lane<FT, COMP12, FAM, 2>(a, l); break;
  case 3: tile_unpack_lane<FT, COMP12, FAM, 3>(a, l); break;
  case 4: tile_unpack_lane<FT, COMP12, FAM, 4>(a, l); break;
  case 5: tile_unpack_lane<FT, COMP12, FAM, 5>(a, l); break;
  case 6: tile_unpack_lane<FT, COMP12, FAM, 6>(a, l); break;
  default: tile_unpack_lane<FT, COMP12, FAM, 7>(a, l); break;
  }
}

// ---- host side --------------------------------------------------------

std::atomic<int> g_status{QB200_OK};
std::mutex g_msg_mu;
std::string g_msg;

void record(int code, const char *what)
{
  int expect = QB200_OK;
  if (g_status.compare_exchange_strong(expect, code)) {
    std::lock_guard<std::mutex> lock(g_msg_mu);
    g_msg = what;
  }
  std::fprintf(stderr, "qphix_b200: %s\n", what);
}

// storage type of the library for a QPhiX FT
template <typename T> struct storage;
template <> struct storage<float> { typedef float type; };
template <> struct storage<double> { typedef double type; };
template <> struct storage<unsigned short> { typedef __half type; };

inline double scal(float v) { return v; }
inline double scal(double v) { return v; }
inline double scal(unsigned short v) { return (double)__half2float(__ushort_as_half(v)); }

template <typename T> inline void phases(TileDev &d, const T tbc_phases[4][2], unsigned mask)
{
  d.tbc_mask = mask;
  for (int m = 0; m < 4; m++) {
    d.tbc[m][0] = tbc_phases ? scal(tbc_phases[m][0]) : 1.0;
    d.tbc[m][1] = tbc_phases ? scal(tbc_phases[m][1]) : 0.0;
  }
  if (mask && !tbc_phases) record(QB200_ENULL, "twisted boundary phases requested but tbc_phases is NULL");
}

inline bool shape_ok(int V, int S)
{
  if (V < 1 || V > kMaxLanes || S < 1 || V % S) {
    record(QB200_ELAYOUT, "veclen must be a multiple of soalen and at most 32");
    return false;
  }
  return true;
}

inline void copy_offs(int *dst, const int *src, int V)
{
  if (src) std::memcpy(dst, src, sizeof(int) * V);
}

inline bool run(const void *kernel, const TileDev &d, const char *what)
{
  void *args[] = {const_cast<TileDev *>(&d)};
  cudaError_t e = cudaLaunchKernel(kernel, dim3(1), dim3(kMaxLanes), args, 0, cudaStreamPerThread);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
  if (e != cudaSuccess) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    record(QB200_ECUDA, buf);
    return false;
  }
  return true;
}

template <typename ST, bool C12>
const void *body_kernel(int fam, bool ach)
{
  switch (fam * 2 + (ach ? 1 : 0)) {
  case 0: return (const void *)tile_body_kernel<ST, C12, FAM_WILSON, false>;
  case 1: return (const void *)tile_body_kernel<ST, C12, FAM_WILSON, true>;
  case 2: return (const void *)tile_body_kernel<ST, C12, FAM_CLOVER, false>;
  case 3: return (const void *)tile_body_kernel<ST, C12, FAM_CLOVER, true>;
  case 4: return (const void *)tile_body_kernel<ST, C12, FAM_TM, false>;
  case 5: return (const void *)tile_body_kernel<ST, C12, FAM_TM, true>;
  case 6: return (const void *)tile_body_kernel<ST, C12, FAM_TMCLOV, false>;
  default: return (const void *)tile_body_kernel<ST, C12, FAM_TMCLOV, true>;
  }
}

template <typename ST, bool C12>
const void *unpack_kernel(int fam)
{
  switch (fam) {
  case FAM_WILSON: return (const void *)tile_unpack_kernel<ST, C12, FAM_WILSON>;
  case FAM_CLOVER: return (const void *)tile_unpack_kernel<ST, C12, FAM_CLOVER>;
  case FAM_TM: return (const void *)tile_unpack_kernel<ST, C12, FAM_TM>;
  default: return (const void *)tile_unpack_kernel<ST, C12, FAM_TMCLOV>;
  }
}

// the arguments every body kernel shares
struct BodyCall {
  int fam;
  bool ach;
  int isPlus;
  const void *xy, *zb, *zf, *tb, *tf, *chi, *gauge, *clov;
  void *out;
  const int *xb, *xf, *yb, *yf, *offs;
  const unsigned *acc;
};

template <typename T, int V, int S, bool C12>
void body(const BodyCall &b, unsigned tbc_mask, const T tbc_phases[4][2], T cs, T ctf, T ctb, double alpha,
          double mu, double muinv, double rho)
{
  typedef typename storage<T>::type ST;
  if (!shape_ok(V, S)) return;
  if (!b.xy || !b.out || !b.gauge || !b.offs || !b.acc || (b.ach && !b.chi) ||
      ((b.fam == FAM_CLOVER || b.fam == FAM_TMCLOV) && !b.clov)) {
    record(QB200_ENULL, "dslash tile: a required pointer is NULL");
    return;
  }
  if ((b.acc[0] || b.acc[1]) && (!b.xb || !b.xf)) {
    record(QB200_ENULL, "dslash tile: x offsets are NULL");
    return;
  }
  if ((b.acc[2] || b.acc[3]) && (!b.yb || !b.yf)) {
    record(QB200_ENULL, "dslash tile: y offsets are NULL");
    return;
  }
  TileDev d;
  std::memset(&d, 0, sizeof(d));
  d.xy = b.xy; d.zb = b.zb; d.zf = b.zf; d.tb = b.tb; d.tf = b.tf;
  d.chi = b.chi; d.gauge = b.gauge; d.clov = b.clov; d.out = b.out;
  copy_offs(d.xb, b.xb, V);
  copy_offs(d.xf, b.xf, V);
  copy_offs(d.yb, b.yb, V);
  copy_offs(d.yf, b.yf, V);
  copy_offs(d.offs, b.offs, V);
  for (int k = 0; k < 8; k++) d.acc[k] = b.acc[k];
  const char *znull = nullptr;
  if (d.acc[4] && !b.zb) znull = "zbBase";
  if (d.acc[5] && !b.zf) znull = "zfBase";
  if (d.acc[6] && !b.tb) znull = "tbBase";
  if (d.acc[7] && !b.tf) znull = "tfBase";
  if (znull) {
    std::string m = std::string("dslash tile: ") + znull + " is NULL";
    record(QB200_ENULL, m.c_str());
    return;
  }
  d.cs = scal(cs);
  d.ctf = scal(ctf);
  d.ctb = scal(ctb);
  d.alpha = alpha;
  d.mu = mu;
  d.muinv = muinv;
  d.rho = rho;
  phases(d, tbc_phases, tbc_mask);
  d.V = V;
  d.S = S;
  d.isPlus = b.isPlus;
  run(body_kernel<ST, C12>(b.fam, b.ach), d, "dslash tile launch");
}

template <typename T, int V, int S>
void pack(int isPlus, const void *xy, const int *offs, T *outbuf, unsigned mask, int dir)
{
  typedef typename storage<T>::type ST;
  if (!shape_ok(V, S)) return;
  if (dir < 0 || dir > 7) {
    record(QB200_EDIR, "face_proj_dir: invalid dir (must be 0..7)");
    return;
  }
  if (!xy || !offs || !outbuf) {
    record(QB200_ENULL, "face_proj_dir: a required pointer is NULL");
    return;
  }
  TileDev d;
  std::memset(&d, 0, sizeof(d));
  d.xy = xy;
  d.outbuf = outbuf;
  copy_offs(d.offs, offs, V);
  d.mask = mask;
  d.V = V;
  d.S = S;
  d.isPlus = isPlus;
  d.dir = dir;
  if (dir < 2) { // the packed lanes must fit the (veclen/soalen+1)/2 slots
    unsigned possible = 0;
    for (int r = 0; r < V; r += S) possible |= 1u << (r + (dir == 0 ? 0 : S - 1));
    if (__builtin_popcount(mask & possible) > (V / S + 1) / 2) {
      record(QB200_EINVAL, "face_proj_dir: mask selects more x-face lanes than the buffer holds");
      return;
    }
  }
  run((const void *)tile_pack_kernel<ST>, d, "face pack tile launch");
}

template <typename T, int V, int S, bool C12>
void unpack(int fam, int isPlus, const T *inbuf, const void *gauge, void *out, const void *clov, T beta, double mu,
            double muinv, unsigned mask, int dir, const int *offs, bool tbc, const T tbc_phases[4][2])
{
  typedef typename storage<T>::type ST;
  if (!shape_ok(V, S)) return;
  if (dir < 0 || dir > 7) {
    record(QB200_EDIR, "face finish: invalid dir (must be 0..7)");
    return;
  }
  if (!inbuf || !gauge || !out || !offs || ((fam == FAM_CLOVER || fam == FAM_TMCLOV) && !clov)) {
    record(QB200_ENULL, "face finish: a required pointer is NULL");
    return;
  }
  TileDev d;
  std::memset(&d, 0, sizeof(d));
  d.inbuf = inbuf;
  d.gauge = gauge;
  d.out = out;
  d.clov = clov;
  copy_offs(d.offs, offs, V);
  d.beta = scal(beta);
  d.mu = mu;
  d.muinv = muinv;
  d.mask = mask;
  phases(d, tbc_phases, tbc ? (1u << (dir / 2)) : 0u);
  d.V = V;
  d.S = S;
  d.isPlus = isPlus;
  d.dir = dir;
  if (dir < 2) {
    unsigned possible = 0;
    for (int r = 0; r < V; r += S) possible |= 1u << (r + (dir == 0 ? 0 : S - 1));
    if (__builtin_popcount(mask & possible) > (V / S + 1) / 2) {
      record(QB200_EINVAL, "face finish: mask selects more x-face lanes than the buffer holds");
      return;
    }
  }
  run(unpack_kernel<ST, C12>(fam), d, "face unpack tile launch");
}

} // namespace qtile
} // namespace qb200

extern "C" {
int qb200_qphix_status(void) { return qb200::qtile::g_status.load(); }

const char *qb200_qphix_last_error(void)
{
  static thread_local std::string copy;
  std::lock_guard<std::mutex> lock(qb200::qtile::g_msg_mu);
  copy = qb200::qtile::g_msg;
  return copy.c_str();
}

void qb200_qphix_clear_status(void)
{
  std::lock_guard<std::mutex> lock(qb200::qtile::g_msg_mu);
  qb200::qtile::g_status.store(QB200_OK);
  qb200::qtile::g_msg.clear();
}
}

// ---- the QPhiX templates ----------------------------------------------

namespace QPhiX {

using qb200::FAM_CLOVER;
using qb200::FAM_TM;
using qb200::FAM_TMCLOV;
using qb200::FAM_WILSON;
using qb200::qtile::BodyCall;

#define QB200_TBC_MASK ((tbc_x ? 1u : 0u) | (tbc_y ? 2u : 0u) | (tbc_z ? 4u : 0u) | (tbc_t ? 8u : 0u))
#define QB200_BODY_COMMON(FAMV, ACHV, PLUS, CHI, CLOV)                                                   \
  BodyCall b;                                                                                          \
  b.fam = FAMV;                                                                                        \
  b.ach = ACHV;                                                                                        \
  b.isPlus = PLUS;                                                                                     \
  b.xy = xyBase; b.zb = zbBase; b.zf = zfBase; b.tb = tbBase; b.tf = tfBase;                           \
  b.chi = CHI; b.gauge = gBase; b.clov = CLOV; b.out = oBase;                                          \
  b.xb = xbOffs; b.xf = xfOffs; b.yb = ybOffs; b.yf = yfOffs; b.offs = offs;                           \
  b.acc = accumulate;                                                                                  \
  (void)gOffs; (void)siprefdist1; (void)siprefdist2; (void)siprefdist3; (void)siprefdist4;            \
  (void)pfyOffs; (void)pfBase2; (void)pfBase3; (void)pfBase4

#define QB200_TPL template <typename FT, int veclen, int soalen, bool compress12, bool tbc_x, bool tbc_y, bool tbc_z, bool tbc_t>
#define QB200_FACE_TPL template <typename FT, int veclen, int soalen, bool compress12, bool tbc>
#define QB200_RUN_BODY(...) qb200::qtile::body<FT, veclen, soalen, compress12>(b, QB200_TBC_MASK, tbc_phases, __VA_ARGS__)

#define QB200_DEF_ISIGN(isign, PLUS)                                                                     \
  QB200_TPL void dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_OFFS, const int gprefdist,     \
                                      QB200_QPHIX_PF, const unsigned int accumulate[8], const FT coeff_s, \
                                      const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2]) \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_WILSON, false, PLUS, nullptr, nullptr);                                      \
    (void)gprefdist;                                                                                   \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, 1.0, 0.0, 1.0, 0.0);                                 \
  }                                                                                                    \
  QB200_TPL void dslash_achimbdpsi_##isign##_vec(                                                      \
      QB200_QPHIX_ACH_HEAD, QB200_QPHIX_OFFS, const int chiprefdist, const int gprefdist, QB200_QPHIX_PF, \
      QB200_QPHIX_SPINOR *pfBaseChi, const FT alpha, const FT coeff_s, const FT coeff_t_f,               \
      const FT coeff_t_b, const FT tbc_phases[4][2], const unsigned int accumulate[8])                 \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_WILSON, true, PLUS, chiBase, nullptr);                                       \
    (void)chiprefdist; (void)gprefdist; (void)pfBaseChi;                                               \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, qb200::qtile::scal(alpha), 0.0, 1.0, 0.0);           \
  }                                                                                                    \
  QB200_TPL void clov_dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_CLOV *clBase,           \
                                           QB200_QPHIX_OFFS, const int gprefdist, const int clprefdist, \
                                           QB200_QPHIX_PF, const unsigned int accumulate[8],           \
                                           const FT coeff_s, const FT coeff_t_f, const FT coeff_t_b,   \
                                           const FT tbc_phases[4][2])                                  \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_CLOVER, false, PLUS, nullptr, clBase);                                       \
    (void)gprefdist; (void)clprefdist;                                                                 \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, 1.0, 0.0, 1.0, 0.0);                                 \
  }                                                                                                    \
  QB200_TPL void clov_dslash_achimbdpsi_##isign##_vec(                                                 \
      QB200_QPHIX_ACH_HEAD, QB200_QPHIX_CLOV *clBase, QB200_QPHIX_OFFS, const int chiprefdist,          \
      const int gprefdist, const int clprefdist, QB200_QPHIX_PF, QB200_QPHIX_SPINOR *pfBaseChi,          \
      const FT coeff_s, const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2],               \
      const unsigned int accumulate[8], const FT prec_mass_rho)                                        \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_CLOVER, true, PLUS, chiBase, clBase);                                        \
    (void)chiprefdist; (void)gprefdist; (void)clprefdist; (void)pfBaseChi;                             \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, 1.0, 0.0, 1.0, qb200::qtile::scal(prec_mass_rho));   \
  }                                                                                                    \
  QB200_TPL void tm_dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_OFFS, const int gprefdist,  \
                                         QB200_QPHIX_PF, const unsigned int accumulate[8],             \
                                         const FT coeff_s, const FT coeff_t_f, const FT coeff_t_b,     \
                                         const FT tbc_phases[4][2], const FT mu, const FT muinv)       \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_TM, false, PLUS, nullptr, nullptr);                                          \
    (void)gprefdist;                                                                                   \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, 1.0, qb200::qtile::scal(mu), qb200::qtile::scal(muinv), \
                   0.0);                                                                               \
  }                                                                                                    \
  QB200_TPL void tm_dslash_achimbdpsi_##isign##_vec(                                                   \
      QB200_QPHIX_ACH_HEAD, QB200_QPHIX_OFFS, const int chiprefdist, const int gprefdist, QB200_QPHIX_PF, \
      QB200_QPHIX_SPINOR *pfBaseChi, const FT alpha, const FT coeff_s, const FT coeff_t_f,               \
      const FT coeff_t_b, const FT tbc_phases[4][2], const FT mu, const unsigned int accumulate[8])    \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_TM, true, PLUS, chiBase, nullptr);                                           \
    (void)chiprefdist; (void)gprefdist; (void)pfBaseChi;                                               \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, qb200::qtile::scal(alpha), qb200::qtile::scal(mu), 1.0, \
                   0.0);                                                                               \
  }                                                                                                    \
  QB200_TPL void tm_clov_dslash_##isign##_vec(QB200_QPHIX_PLAIN_HEAD, QB200_QPHIX_FCLOV *clBase,       \
                                              QB200_QPHIX_OFFS, const int gprefdist,                   \
                                              const int clprefdist, QB200_QPHIX_PF,                    \
                                              const unsigned int accumulate[8], const FT coeff_s,      \
                                              const FT coeff_t_f, const FT coeff_t_b,                  \
                                              const FT tbc_phases[4][2])                               \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_TMCLOV, false, PLUS, nullptr, clBase);                                       \
    (void)gprefdist; (void)clprefdist;                                                                 \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, 1.0, 0.0, 1.0, 0.0);                                 \
  }                                                                                                    \
  QB200_TPL void tm_clov_dslash_achimbdpsi_##isign##_vec(                                              \
      QB200_QPHIX_ACH_HEAD, QB200_QPHIX_FCLOV *clBase, QB200_QPHIX_OFFS, const int chiprefdist,         \
      const int gprefdist, const int clprefdist, QB200_QPHIX_PF, QB200_QPHIX_SPINOR *pfBaseChi,          \
      const FT coeff_s, const FT coeff_t_f, const FT coeff_t_b, const FT tbc_phases[4][2],               \
      const unsigned int accumulate[8], const FT prec_mass_rho)                                        \
  {                                                                                                    \
    QB200_BODY_COMMON(FAM_TMCLOV, true, PLUS, chiBase, clBase);                                        \
    (void)chiprefdist; (void)gprefdist; (void)clprefdist; (void)pfBaseChi;                             \
    QB200_RUN_BODY(coeff_s, coeff_t_f, coeff_t_b, 1.0, 0.0, 1.0, qb200::qtile::scal(prec_mass_rho));   \
  }                                                                                                    \
  template <typename FT, int veclen, int soalen, bool compress12>                                      \
  void face_proj_dir_##isign(QB200_QPHIX_SPINOR *xyBase, const int offs[veclen], const int si_prefdist, \
                             FT *outbuf, const int hsprefdist, unsigned int mask, int dir)              \
  {                                                                                                    \
    (void)si_prefdist; (void)hsprefdist;                                                               \
    qb200::qtile::pack<FT, veclen, soalen>(PLUS, xyBase, offs, outbuf, mask, dir);                     \
  }                                                                                                    \
  QB200_FACE_TPL void face_finish_dir_##isign(const FT *inbuf, QB200_QPHIX_GAUGE *gBase,                \
                                              QB200_QPHIX_OUT *oBase, const int gOffs[veclen],         \
                                              const int offs[veclen], const int hsprefdist,            \
                                              const int gprefdist, const int soprefdist, const FT beta, \
                                              unsigned int mask, int dir, const FT tbc_phases[4][2])    \
  {                                                                                                    \
    (void)gOffs; (void)hsprefdist; (void)gprefdist; (void)soprefdist;                                  \
    qb200::qtile::unpack<FT, veclen, soalen, compress12>(FAM_WILSON, PLUS, inbuf, gBase, oBase, nullptr, beta, \
                                                         0.0, 1.0, mask, dir, offs, tbc, tbc_phases);  \
  }                                                                                                    \
  QB200_FACE_TPL void face_clov_finish_dir_##isign(                                                    \
      const FT *inbuf, QB200_QPHIX_GAUGE *gBase, QB200_QPHIX_OUT *oBase, QB200_QPHIX_CLOV *clBase,       \
      const int gOffs[veclen], const int offs[veclen], const int hsprefdist, const int gprefdist,        \
      const int soprefdist, const int clprefdist, const FT beta, unsigned int mask, int dir,            \
      const FT tbc_phases[4][2])                                                                       \
  {                                                                                                    \
    (void)gOffs; (void)hsprefdist; (void)gprefdist; (void)soprefdist; (void)clprefdist;                \
    qb200::qtile::unpack<FT, veclen, soalen, compress12>(FAM_CLOVER, PLUS, inbuf, gBase, oBase, clBase, beta, \
                                                         0.0, 1.0, mask, dir, offs, tbc, tbc_phases);  \
  }                                                                                                    \
  QB200_FACE_TPL void tm_face_finish_dir_##isign(                                                      \
      const FT *inbuf, QB200_QPHIX_GAUGE *gBase, QB200_QPHIX_OUT *oBase, const int gOffs[veclen],        \
      const int offs[veclen], const int hsprefdist, const int gprefdist, const int soprefdist,           \
      const FT beta, const FT mu, const FT muinv, unsigned int mask, int dir, const FT tbc_phases[4][2]) \
  {                                                                                                    \
    (void)gOffs; (void)hsprefdist; (void)gprefdist; (void)soprefdist;                                  \
    qb200::qtile::unpack<FT, veclen, soalen, compress12>(FAM_TM, PLUS, inbuf, gBase, oBase, nullptr, beta,   \
                                                         qb200::qtile::scal(mu), qb200::qtile::scal(muinv), \
                                                         mask, dir, offs, tbc, tbc_phases);            \
  }                                                                                                    \
  QB200_FACE_TPL void tm_clov_face_finish_dir_##isign(                                                 \
      const FT *inbuf, QB200_QPHIX_GAUGE *gBase, QB200_QPHIX_OUT *oBase, QB200_QPHIX_FCLOV *clBase,      \
      const int gOffs[veclen], const int offs[veclen], const int hsprefdist, const int gprefdist,        \
      const int soprefdist, const int clprefdist, const FT beta, unsigned int mask, int dir,            \
      const FT tbc_phases[4][2])                                                                       \
  {                                                                                                    \
    (void)gOffs; (void)hsprefdist; (void)gprefdist; (void)soprefdist; (void)clprefdist;                \
    qb200::qtile::unpack<FT, veclen, soalen, compress12>(FAM_TMCLOV, PLUS, inbuf, gBase, oBase, clBase, beta, \
                                                         0.0, 1.0, mask, dir, offs, tbc, tbc_phases);  \
  }

QB200_DEF_ISIGN(plus, 1)
QB200_DEF_ISIGN(minus, 0)

// ---- explicit instantiations of the b200 ISA --------------------------
//
// Parameter lists in their adjusted form (arrays as pointers, top-level
// const dropped); they name the same functions as the declarations.
#define QI_SP(T, V, C) const Types<T, V, V, C>::FourSpinorBlock *
#define QI_OUT(T, V, C) Types<T, V, V, C>::FourSpinorBlock *
#define QI_G(T, V, C) const Types<T, V, V, C>::SU3MatrixBlock *
#define QI_CL(T, V, C) const Types<T, V, V, C>::CloverBlock *
#define QI_FCL(T, V, C) const Types<T, V, V, C>::FullCloverBlock *
#define QI_OFFS const int *, const int *, const int *, const int *, const int *, const int *, int, int, int, int
#define QI_PF(T, V, C) const int *, QI_SP(T, V, C), QI_SP(T, V, C), QI_SP(T, V, C)
#define QI_PH(T) const T (*)[2]
#define QI_PLAIN(T, V, C) QI_SP(T, V, C), QI_SP(T, V, C), QI_SP(T, V, C), QI_SP(T, V, C), QI_SP(T, V, C), \
                          QI_OUT(T, V, C), QI_G(T, V, C)
#define QI_ACH(T, V, C) QI_SP(T, V, C), QI_SP(T, V, C), QI_SP(T, V, C), QI_SP(T, V, C), QI_SP(T, V, C),   \
                        QI_SP(T, V, C), QI_OUT(T, V, C), QI_G(T, V, C)

#define QI_BODY_ISIGN(isign, T, V, C, X, Y, Z, W)                                                          \
  template void dslash_##isign##_vec<T, V, V, C, X, Y, Z, W>(QI_PLAIN(T, V, C), QI_OFFS, int, QI_PF(T, V, C), \
                                                            const unsigned *, T, T, T, QI_PH(T));           \
  template void dslash_achimbdpsi_##isign##_vec<T, V, V, C, X, Y, Z, W>(                                    \
      QI_ACH(T, V, C), QI_OFFS, int, int, QI_PF(T, V, C), QI_SP(T, V, C), T, T, T, T, QI_PH(T),             \
      const unsigned *);                                                                                    \
  template void clov_dslash_##isign##_vec<T, V, V, C, X, Y, Z, W>(                                          \
      QI_PLAIN(T, V, C), QI_CL(T, V, C), QI_OFFS, int, int, QI_PF(T, V, C), const unsigned *, T, T, T,      \
      QI_PH(T));                                                                                            \
  template void clov_dslash_achimbdpsi_##isign##_vec<T, V, V, C, X, Y, Z, W>(                               \
      QI_ACH(T, V, C), QI_CL(T, V, C), QI_OFFS, int, int, int, QI_PF(T, V, C), QI_SP(T, V, C), T, T, T,      \
      QI_PH(T), const unsigned *, T);                                                                       \
  template void tm_dslash_##isign##_vec<T, V, V, C, X, Y, Z, W>(QI_PLAIN(T, V, C), QI_OFFS, int,           \
                                                               QI_PF(T, V, C), const unsigned *, T, T, T,   \
                                                               QI_PH(T), T, T);                             \
  template void tm_dslash_achimbdpsi_##isign##_vec<T, V, V, C, X, Y, Z, W>(                                 \
      QI_ACH(T, V, C), QI_OFFS, int, int, QI_PF(T, V, C), QI_SP(T, V, C), T, T, T, T, QI_PH(T), T,          \
      const unsigned *);                                                                                    \
  template void tm_clov_dslash_##isign##_vec<T, V, V, C, X, Y, Z, W>(                                       \
      QI_PLAIN(T, V, C), QI_FCL(T, V, C), QI_OFFS, int, int, QI_PF(T, V, C), const unsigned *, T, T, T,     \
      QI_PH(T));                                                                                            \
  template void tm_clov_dslash_achimbdpsi_##isign##_vec<T, V, V, C, X, Y, Z, W>(                            \
      QI_ACH(T, V, C), QI_FCL(T, V, C), QI_OFFS, int, int, int, QI_PF(T, V, C), QI_SP(T, V, C), T, T, T,     \
      QI_PH(T), const unsigned *, T);

#define QI_BODY(T, V, C, X, Y, Z, W) QI_BODY_ISIGN(plus, T, V, C, X, Y, Z, W) QI_BODY_ISIGN(minus, T, V, C, X, Y, Z, W)
#define QI_BODY_T(T, V, C, X, Y, Z) QI_BODY(T, V, C, X, Y, Z, false) QI_BODY(T, V, C, X, Y, Z, true)
#define QI_BODY_Z(T, V, C, X, Y) QI_BODY_T(T, V, C, X, Y, false) QI_BODY_T(T, V, C, X, Y, true)
#define QI_BODY_Y(T, V, C, X) QI_BODY_Z(T, V, C, X, false) QI_BODY_Z(T, V, C, X, true)
#define QI_BODY_X(T, V, C) QI_BODY_Y(T, V, C, false) QI_BODY_Y(T, V, C, true)

#define QI_FACE_ISIGN(isign, T, V, C, B)                                                                   \
  template void face_finish_dir_##isign<T, V, V, C, B>(const T *, QI_G(T, V, C), QI_OUT(T, V, C),            \
                                                      const int *, const int *, int, int, int, T, unsigned, \
                                                      int, QI_PH(T));                                       \
  template void face_clov_finish_dir_##isign<T, V, V, C, B>(const T *, QI_G(T, V, C), QI_OUT(T, V, C),       \
                                                           QI_CL(T, V, C), const int *, const int *, int,   \
                                                           int, int, int, T, unsigned, int, QI_PH(T));      \
  template void tm_face_finish_dir_##isign<T, V, V, C, B>(const T *, QI_G(T, V, C), QI_OUT(T, V, C),         \
                                                         const int *, const int *, int, int, int, T, T, T,  \
                                                         unsigned, int, QI_PH(T));                          \
  template void tm_clov_face_finish_dir_##isign<T, V, V, C, B>(const T *, QI_G(T, V, C), QI_OUT(T, V, C),    \
                                                              QI_FCL(T, V, C), const int *, const int *,    \
                                                              int, int, int, int, T, unsigned, int,         \
                                                              QI_PH(T));
#define QI_PACK_ISIGN(isign, T, V, C)                                                                      \
  template void face_proj_dir_##isign<T, V, V, C>(QI_SP(T, V, C), const int *, int, T *, int, unsigned, int);

#define QI_ALL_C(T, V, C)                                                                                  \
  QI_BODY_X(T, V, C)                                                                                       \
  QI_FACE_ISIGN(plus, T, V, C, false) QI_FACE_ISIGN(plus, T, V, C, true)                                   \
  QI_FACE_ISIGN(minus, T, V, C, false) QI_FACE_ISIGN(minus, T, V, C, true)                                 \
  QI_PACK_ISIGN(plus, T, V, C) QI_PACK_ISIGN(minus, T, V, C)
#define QI_ALL(T, V) QI_ALL_C(T, V, true) QI_ALL_C(T, V, false)

QI_ALL(float, 4)
QI_ALL(float, 8)
QI_ALL(float, 16)
QI_ALL(double, 4)
QI_ALL(double, 8)
QI_ALL(double, 16)
QI_ALL(half, 4)
QI_ALL(half, 8)
QI_ALL(half, 16)

} // namespace QPhiX
