// qb200_force.cu -- backward of the hopping term: the link derivative
// ("fermion force") of L = Re <chi, H(U) psi>, where H is the eight-hop sum
// of the plain dslash (codegen/dslash_common.cc:1729-1826, without the
// clover / twisted post-term) on checkerboard cb.
//
// For hop d of output site x: ub = M_d(G) b with b = proj_d(psi(x+-mu)), and
// the reconstruction adds beta*recons_d(ub).  Writing
//   h = conj(phase_d) * recons_d^dag(beta * chi(x))      (2 x 3 complex)
// the derivative with respect to the stored link G (complex convention
// dL/dRe + i dL/dIm) is
//   forward (ub = G^T b):      dG[k][c] = sum_s h[s][c] conj(b[s][k])
//   backward (ub = G^dag-ish): dG[c][k] = sum_s conj(h[s][c]) b[s][k]
// and is reported for the link matrix U = G^T: forward hops give dU_mu(x),
// backward hops dU_mu(x - mu).  With the gauge field given, the kernel
// returns instead the su(3) projection P = TA(F U^dag) (traceless
// anti-Hermitian part), for which dL/deps along U -> exp(eps X) U equals
// Re tr(X^dag P).  FP32 or FP64 storage, written in the storage type.
// The reference has no backward kernels; this is an addition of the B200
// build.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>

#include "qphix_b200.h"
#include "qb200_async_kernel.cuh"
#include "qb200_internal.h"

namespace qb200 {
int api_fail(int code, const char *msg);
int api_geo(const qb200_lattice *l, GeoDev &g);
int api_check_device();
} // namespace qb200

using namespace qb200;

namespace {

// h += adjoint of recons (rec_plus table scaled by tau) applied to beta*chi
template <typename C, int MU>
__device__ __forceinline__ void recons_adj(const cx<C> (&chi)[4][3], C beta, C tau, cx<C> (&h)[2][3])
{
  const C b2 = beta * tau * (C)rec_sg2(MU);
  const C b3 = beta * tau * (C)rec_sg3(MU);
  constexpr int s2 = rec_s2(MU), s3 = 1 - rec_s2(MU);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    h[0][c] = mk<C>(beta * chi[0][c].re, beta * chi[0][c].im);
    h[1][c] = mk<C>(beta * chi[1][c].re, beta * chi[1][c].im);
    if (rec_i(MU)) { // recons adds b*i*ub -> adjoint adds b*(-i)*chi
      h[s2][c].re += b2 * chi[2][c].im;
      h[s2][c].im -= b2 * chi[2][c].re;
      h[s3][c].re += b3 * chi[3][c].im;
      h[s3][c].im -= b3 * chi[3][c].re;
    } else {
      h[s2][c].re += b2 * chi[2][c].re;
      h[s2][c].im += b2 * chi[2][c].im;
      h[s3][c].re += b3 * chi[3][c].re;
      h[s3][c].im += b3 * chi[3][c].im;
    }
  }
}

// Output layout: component k = ((D*3 + a)*3 + b)*2 + ri of site i (the
// site-th site of cb in (t, z, y, xcb) order) at out[k * nsites + i], so a
// warp's stores are contiguous.
//
// The force of hop D at one site from its neighbour spinor nb, chi, beta and
// (PROJ) the stored link G of the hop.
template <typename FT, bool PROJ, int D>
__device__ __forceinline__ void force_from(const cx<comp_t<FT>> (&nb)[4][3], const cx<comp_t<FT>> (&chi)[4][3],
                                           const cx<comp_t<FT>> (&G)[3][3], comp_t<FT> beta,
                                           const OpDev<comp_t<FT>> &p, elem_t<FT> *__restrict__ o, int ns)
{
  typedef comp_t<FT> C;
  constexpr int MU = D / 2;
  constexpr bool FWD = (D & 1) != 0;
  cx<C> b[2][3], h[2][3];
  project<C, D>(nb, p.isPlus ? (C)1 : (C)-1, b);
  const C tau = ((p.isPlus != 0) != FWD) ? (C)1 : (C)-1;
  recons_adj<C, MU>(chi, beta, tau, h);
  if ((p.tbc_mask >> MU) & 1u) {
    // ub was multiplied by ph = phase (forward) or conj(phase); h <- conj(ph) h
    const C pr = p.tbc[MU][0];
    const C pi = FWD ? -p.tbc[MU][1] : p.tbc[MU][1];
#pragma unroll
    for (int sp = 0; sp < 2; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const C re = pr * h[sp][c].re - pi * h[sp][c].im;
        const C im = pr * h[sp][c].im + pi * h[sp][c].re;
        h[sp][c].re = re;
        h[sp][c].im = im;
      }
  }
  // F[a][bb]: derivative with respect to U = G^T
  cx<C> F[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      C re = 0, im = 0;
#pragma unroll
      for (int sp = 0; sp < 2; sp++) {
        if (FWD) { // F[c1][k] = sum_s h[s][c1] conj(b[s][k]),  a = c1, bb = k
          re += h[sp][a].re * b[sp][bb].re + h[sp][a].im * b[sp][bb].im;
          im += h[sp][a].im * b[sp][bb].re - h[sp][a].re * b[sp][bb].im;
        } else { // F[k][c1] = sum_s conj(h[s][c1]) b[s][k],  a = k, bb = c1
          re += h[sp][bb].re * b[sp][a].re + h[sp][bb].im * b[sp][a].im;
          im += h[sp][bb].re * b[sp][a].im - h[sp][bb].im * b[sp][a].re;
        }
      }
      F[a][bb] = mk<C>(re, im);
    }
  if (PROJ) {
    // P = TA(F U^dag), U^dag[k][bb] = conj(U[bb][k]) = conj(G[k][bb])
    cx<C> M[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int bb = 0; bb < 3; bb++) {
        C re = 0, im = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          re += F[a][k].re * G[k][bb].re + F[a][k].im * G[k][bb].im;
          im += F[a][k].im * G[k][bb].re - F[a][k].re * G[k][bb].im;
        }
        M[a][bb] = mk<C>(re, im);
      }
    const C tr3 = (M[0][0].im + M[1][1].im + M[2][2].im) / (C)3;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int bb = 0; bb < 3; bb++) {
        // (M - M^dag)/2 - i Im(tr M)/3
        F[a][bb].re = (C)0.5 * (M[a][bb].re - M[bb][a].re);
        F[a][bb].im = (C)0.5 * (M[a][bb].im + M[bb][a].im) - (a == bb ? tr3 : (C)0);
      }
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int bb = 0; bb < 3; bb++) {
      ftraits<FT>::st(o + (long long)(((D * 3 + a) * 3 + bb) * 2 + 0) * ns, F[a][bb].re);
      ftraits<FT>::st(o + (long long)(((D * 3 + a) * 3 + bb) * 2 + 1) * ns, F[a][bb].im);
    }
}

// the hop coefficient of direction D at site s (time-boundary factor included)
template <typename C, int D>
__device__ __forceinline__ C force_beta(const GeoDev &g, const OpDev<C> &p, const Site &s)
{
  C beta = p.beta[D];
  if (D == 6 && s.t == 0 && p.t_edge_lo) beta *= p.tbound;
  if (D == 7 && s.t == g.nt - 1 && p.t_edge_hi) beta *= p.tbound;
  return beta;
}

template <typename FT, int S, bool PROJ, bool COMP12, int D>
__device__ __forceinline__ void force_dir(const elem_t<FT> *__restrict__ psi, const elem_t<FT> *__restrict__ gauge,
                                          const GeoDev &g, const OpDev<comp_t<FT>> &p, const Site &s, long long gbase,
                                          const cx<comp_t<FT>> (&chi)[4][3], elem_t<FT> *__restrict__ o, int ns)
{
  typedef comp_t<FT> C;
  bool cross;
  const Site n = neighbour<D>(g, s, &cross);
  cx<C> nb[4][3], G[3][3];
  load_spinor<FT, S>(psi, spinor_base<FT, S>(g, n), nb);
  if (PROJ) load_link<FT, COMP12, D>(gauge, gbase, g.V, G);
  force_from<FT, PROJ, D>(nb, chi, G, force_beta<C, D>(g, p, s), p, o, ns);
}

template <typename FT, int S, bool PROJ, bool COMP12>
__global__ void __launch_bounds__(128)
    force_kernel(const elem_t<FT> *__restrict__ chi, const elem_t<FT> *__restrict__ psi,
                 const elem_t<FT> *__restrict__ gauge, elem_t<FT> *__restrict__ out, const GeoDev g,
                 const OpDev<comp_t<FT>> p)
{
  typedef comp_t<FT> C;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nsites) return;
  const Site s = site_of(g, i, p.cb);
  cx<C> ch[4][3];
  load_spinor<FT, S>(chi, spinor_base<FT, S>(g, s), ch);
  long long gbase = 0;
  if (PROJ) {
    int lane;
    const long long tile = tile_of<S>(g, s, &lane);
    gbase = tile * (8LL * (COMP12 ? 2 : 3) * 6 * g.V) + lane;
  }
  elem_t<FT> *o = out + i;
  const int ns = g.nsites;
  force_dir<FT, S, PROJ, COMP12, 0>(psi, gauge, g, p, s, gbase, ch, o, ns);
  force_dir<FT, S, PROJ, COMP12, 1>(psi, gauge, g, p, s, gbase, ch, o, ns);
  force_dir<FT, S, PROJ, COMP12, 2>(psi, gauge, g, p, s, gbase, ch, o, ns);
  force_dir<FT, S, PROJ, COMP12, 3>(psi, gauge, g, p, s, gbase, ch, o, ns);
  force_dir<FT, S, PROJ, COMP12, 4>(psi, gauge, g, p, s, gbase, ch, o, ns);
  force_dir<FT, S, PROJ, COMP12, 5>(psi, gauge, g, p, s, gbase, ch, o, ns);
  force_dir<FT, S, PROJ, COMP12, 6>(psi, gauge, g, p, s, gbase, ch, o, ns);
  force_dir<FT, S, PROJ, COMP12, 7>(psi, gauge, g, p, s, gbase, ch, o, ns);
}

// ---- staged form: FP32, VECLEN == SOALEN in {4, 8, 16} -------------------
//
// With narrow blocks (SOALEN 4: one spinor component of a block is a
// 16-byte piece) the thread-per-site kernel's neighbour loads touch 32/S
// pieces per warp and component and wait one load latency per direction.
// Here, as in async_site_kernel, a warp owns 32 sites of one (z, t) plane and
// copies with cp.async, in 16-byte vectors, the blocks its sites need for
// direction D+1 (the neighbour blocks and, with the projection, the
// direction's link slab) into one of two shared-memory buffers while it
// computes and stores the force of direction D.  chi and an x region (the
// warp's blocks, one on either side, the first block of its first row and
// the last block of its last row: every x neighbour of its sites) are copied
// with direction 0's link; the x region overlays spinor buffer 1, which
// direction 3 is the first to use, and chi spinor buffer 0, read before
// direction 2's copies go out.  The arithmetic is force_from's; the output is
// written directly (per component, a warp's stores are 32 consecutive sites).
template <typename FT, int S, bool PROJ, bool COMP12> struct ForceCfg {
  typedef Stage<FT, S> St;
  static constexpr int R = COMP12 ? 2 : 3;
  static constexpr int SPB = St::SPB * S * (int)sizeof(elem_t<FT>); // spinor block bytes
  static constexpr int LKB = R * 6 * S * (int)sizeof(elem_t<FT>);   // link slab bytes
  static constexpr int LKS = St::stride(R * 6);
  static constexpr int XS = St::G + 4;                              // x region slots
  static constexpr int S1 = St::G * St::SP;                         // spinor buffer 1 / x region
  static constexpr int L0 = S1 + XS * St::SP;                       // link buffers
  static constexpr int WB = L0 + (PROJ ? 2 * St::G * LKS : 0);      // bytes per warp
  static constexpr int spin(int b) { return b ? S1 : 0; }
  static constexpr int link(int b) { return L0 + b * St::G * LKS; }
};

template <typename FT, int S> constexpr bool force_async_layout()
{
  return (S == 4 || S == 8 || S == 16) && sizeof(elem_t<FT>) == 4;
}

// copies of direction D (D >= 2: the neighbour blocks; x directions read the
// x region) and, projected, its link slab
template <typename FT, int S, bool PROJ, bool COMP12, int D>
__device__ __forceinline__ void force_prefetch(const elem_t<FT> *__restrict__ psi,
                                               const elem_t<FT> *__restrict__ gauge, const GeoDev &g, const Site &s,
                                               long long obase, const WarpCtx &w)
{
  typedef ForceCfg<FT, S, PROJ, COMP12> A;
  typedef Stage<FT, S> St;
  if (D >= 2) {
    bool cross;
    const long long nbase = obase + neighbour_offset<S, D>(g, s, (long long)St::SPB * S, 1, &cross);
    stage_in_async<FT, S, A::SPB, St::SP>(psi, nbase - w.lane, w.buf + A::spin(D & 1), w.ln);
  }
  if (PROJ)
    stage_in_async<FT, S, A::LKB, A::LKS>(gauge, w.tile * (8LL * A::R * 6 * S) + (long long)D * A::R * 6 * S,
                                          w.buf + A::link(D & 1), w.ln);
}

// one pipeline step: issue direction D+1, wait for D, read D's neighbour
// (and link) from shared memory, then compute and store D's force
template <typename FT, int S, bool PROJ, bool COMP12, int D>
__device__ __forceinline__ void force_step(const elem_t<FT> *__restrict__ psi, const elem_t<FT> *__restrict__ gauge,
                                           const GeoDev &g, const OpDev<comp_t<FT>> &p, const Site &s,
                                           long long obase, const WarpCtx &w, const cx<comp_t<FT>> (&chi)[4][3],
                                           elem_t<FT> *__restrict__ o, int ns, bool active)
{
  typedef comp_t<FT> C;
  typedef ForceCfg<FT, S, PROJ, COMP12> A;
  typedef Stage<FT, S> St;
  if (D < 7) {
    force_prefetch<FT, S, PROJ, COMP12, (D < 7 ? D + 1 : 7)>(psi, gauge, g, s, obase, w);
    cp_async_commit();
    cp_async_wait<1>();
  } else {
    cp_async_wait<0>();
  }
  __syncwarp();
  cx<C> nb[4][3], G[3][3];
  if (D < 2) {
    int xb, nl;
    x_neighbour<S, D>(g, s, xb, nl);
    // slot of the row's first block, then of the neighbour's block
    int sl = (int)(w.blk - w.blk0) + 1 - s.xcb / S + xb;
    sl = (sl >= 0 && sl < St::G + 2) ? sl : (sl == w.xhead ? St::G + 2 : St::G + 3);
    load_spinor_sm<FT, S>(w.xr + sl * St::SP, nl, nb);
  } else {
    load_spinor_sm<FT, S>(w.buf + A::spin(D & 1) + (w.ln / S) * St::SP, w.lane, nb);
  }
  if (PROJ) load_link_sm<FT, S, COMP12>(w.buf + A::link(D & 1) + (w.ln / S) * A::LKS, w.lane, G);
  __syncwarp();
  if (active) force_from<FT, PROJ, D>(nb, chi, G, force_beta<C, D>(g, p, s), p, o, ns);
}

// Work unit: one warp's 32 sites of one (z, t) plane, numbered over all
// planes (wpp units per plane), so that no warp idles when a plane's sites
// do not fill whole blocks; lanes past the plane's last site take part in
// the copies (on a clamped site) and store nothing.  ForceCfg::WB bytes of
// dynamic shared memory per warp; fields 16-byte aligned, below 32 GiB.
template <typename FT, int S, bool PROJ, bool COMP12>
__global__ void __launch_bounds__(128, 4)
    async_force_kernel(const elem_t<FT> *__restrict__ chi, const elem_t<FT> *__restrict__ psi,
                       const elem_t<FT> *__restrict__ gauge, elem_t<FT> *__restrict__ out, const GeoDev g,
                       const OpDev<comp_t<FT>> p)
{
  typedef comp_t<FT> C;
  typedef Stage<FT, S> St;
  typedef ForceCfg<FT, S, PROJ, COMP12> A;
  extern __shared__ __align__(128) unsigned char fsmem[];
  const int nplane = g.nxh * g.ny;
  const int wpp = (nplane + 31) >> 5;
  const long long u = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (u >= (long long)wpp * g.nz * g.nt) return; // whole warps
  const int plane = (int)(u / wpp);
  const int q0 = (int)(u - (long long)plane * wpp) * 32 + (threadIdx.x & 31);
  const bool active = q0 < nplane;
  const int q = active ? q0 : nplane - 1;
  Site s;
  s.z = plane % g.nz;
  s.t = plane / g.nz;
  s.y = q / g.nxh;
  s.xcb = q - s.y * g.nxh;
  s.par = (s.y + s.z + s.t + p.cb) & 1;
  WarpCtx w;
  w.buf = fsmem + (threadIdx.x >> 5) * A::WB;
  w.ln = threadIdx.x & 31;
  w.tile = tile_of<S>(g, s, &w.lane);
  const long long obase = spinor_base<FT, S>(g, s);
  w.blk = obase / (St::SPB * S);
  w.own = w.blk * (St::SPB * S);
  w.blk0 = __shfl_sync(0xffffffffu, w.blk, 0);
  w.xr = w.buf + A::S1;
  w.xhead = 1 - __shfl_sync(0xffffffffu, s.xcb, 0) / S;
  const long long tail = __shfl_sync(0xffffffffu, w.blk, 31) - __shfl_sync(0xffffffffu, s.xcb, 31) / S + g.nvecs - 1;
  // chi, the x region and direction 0's link in one group
  stage_in_async<FT, S, A::SPB, St::SP>(chi, w.own, w.buf, w.ln);
  stage_xregion<FT, S, COMP12>(psi, w.blk0, w.blk0 - 1 + w.xhead, tail, g.Pxyz * g.nt, w.xr, w.ln);
  force_prefetch<FT, S, PROJ, COMP12, 0>(psi, gauge, g, s, obase, w);
  cp_async_commit();
  cp_async_wait<0>();
  __syncwarp();
  cx<C> ch[4][3];
  load_spinor_sm<FT, S>(w.buf + (w.ln / S) * St::SP, w.lane, ch);
  __syncwarp();
  elem_t<FT> *o = out + (long long)plane * nplane + q;
  const int ns = g.nsites;
  force_step<FT, S, PROJ, COMP12, 0>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
  force_step<FT, S, PROJ, COMP12, 1>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
  force_step<FT, S, PROJ, COMP12, 2>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
  force_step<FT, S, PROJ, COMP12, 3>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
  force_step<FT, S, PROJ, COMP12, 4>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
  force_step<FT, S, PROJ, COMP12, 5>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
  force_step<FT, S, PROJ, COMP12, 6>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
  force_step<FT, S, PROJ, COMP12, 7>(psi, gauge, g, p, s, obase, w, ch, o, ns, active);
}

template <typename FT, int S, bool PROJ, bool COMP12>
cudaError_t go_async_force(const elem_t<FT> *c, const elem_t<FT> *ps, const elem_t<FT> *u, elem_t<FT> *o,
                           const GeoDev &g, const OpDev<comp_t<FT>> &p, cudaStream_t st)
{
  typedef ForceCfg<FT, S, PROJ, COMP12> A;
  const long long warps = (long long)((g.nxh * g.ny + 31) / 32) * g.nz * g.nt;
  const long long blocks = (warps + 3) / 4;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  const int smem = 4 * A::WB;
  // the dynamic shared-memory limit of this kernel, raised once per device
  static std::atomic<unsigned long long> raised{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!(raised.load() & (1ull << dev))) {
    e = cudaFuncSetAttribute(async_force_kernel<FT, S, PROJ, COMP12>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return e;
    raised.fetch_or(1ull << dev);
  }
  async_force_kernel<FT, S, PROJ, COMP12><<<(unsigned)blocks, 128, smem, st>>>(c, ps, u, o, g, p);
  return cudaGetLastError();
}

template <typename FT, int S>
bool launch_async_s(bool proj, bool comp12, const elem_t<FT> *c, const elem_t<FT> *ps, const elem_t<FT> *u,
                    elem_t<FT> *o, const GeoDev &g, const OpDev<comp_t<FT>> &p, cudaStream_t st, cudaError_t *e)
{
  if constexpr (force_async_layout<FT, S>()) {
    if (!proj) *e = go_async_force<FT, S, false, false>(c, ps, u, o, g, p, st);
    else if (comp12) *e = go_async_force<FT, S, true, true>(c, ps, u, o, g, p, st);
    else *e = go_async_force<FT, S, true, false>(c, ps, u, o, g, p, st);
    return true;
  }
  return false;
}

template <typename FT, int S>
void launch_s(bool proj, bool comp12, int blocks, const elem_t<FT> *c, const elem_t<FT> *ps, const elem_t<FT> *u,
              elem_t<FT> *o, const GeoDev &g, const OpDev<comp_t<FT>> &p, cudaStream_t st)
{
  if (!proj) force_kernel<FT, S, false, false><<<blocks, 128, 0, st>>>(c, ps, u, o, g, p);
  else if (comp12) force_kernel<FT, S, true, true><<<blocks, 128, 0, st>>>(c, ps, u, o, g, p);
  else force_kernel<FT, S, true, false><<<blocks, 128, 0, st>>>(c, ps, u, o, g, p);
}

template <typename FT>
cudaError_t launch_force(int S, bool proj, bool comp12, const void *chi, const void *psi, const void *gauge,
                         void *out, const GeoDev &g, const OpDev<comp_t<FT>> &p, cudaStream_t st)
{
  typedef elem_t<FT> E;
  const int blocks = (g.nsites + 127) / 128;
  const E *c = (const E *)chi, *ps = (const E *)psi, *u = (const E *)gauge;
  E *o = (E *)out;
  const bool aligned = ((uintptr_t)chi % 16 == 0) && ((uintptr_t)psi % 16 == 0) &&
                       (!proj || (uintptr_t)gauge % 16 == 0);
  if (g.V == S && aligned) {
    bool done = false;
    cudaError_t e = cudaSuccess;
    switch (S) {
    case 4: done = launch_async_s<FT, 4>(proj, comp12, c, ps, u, o, g, p, st, &e); break;
    case 8: done = launch_async_s<FT, 8>(proj, comp12, c, ps, u, o, g, p, st, &e); break;
    case 16: done = launch_async_s<FT, 16>(proj, comp12, c, ps, u, o, g, p, st, &e); break;
    default: break;
    }
    if (done) return e;
  }
  switch (S) {
  case 1: launch_s<FT, 1>(proj, comp12, blocks, c, ps, u, o, g, p, st); break;
  case 2: launch_s<FT, 2>(proj, comp12, blocks, c, ps, u, o, g, p, st); break;
  case 4: launch_s<FT, 4>(proj, comp12, blocks, c, ps, u, o, g, p, st); break;
  case 8: launch_s<FT, 8>(proj, comp12, blocks, c, ps, u, o, g, p, st); break;
  default: launch_s<FT, 16>(proj, comp12, blocks, c, ps, u, o, g, p, st); break;
  }
  return cudaGetLastError();
}

template <typename C>
void fill(OpDev<C> &p, const qb200_lattice *l, int isPlus, int cb, double cs, double ctf, double ctb,
          unsigned tbc_mask, const double *ph)
{
  std::memset(&p, 0, sizeof(p));
  for (int d = 0; d < 6; d++) p.beta[d] = (C)cs;
  p.beta[6] = (C)ctb;
  p.beta[7] = (C)ctf;
  p.tbound = (C)l->t_boundary;
  p.t_edge_lo = l->t_edge_lo ? 1 : 0;
  p.t_edge_hi = l->t_edge_hi ? 1 : 0;
  p.tbc_mask = tbc_mask & 15u;
  for (int m = 0; m < 4; m++) {
    p.tbc[m][0] = (C)(ph ? ph[2 * m] : 1.0);
    p.tbc[m][1] = (C)(ph ? ph[2 * m + 1] : 0.0);
  }
  p.acc_mask = 0xffu;
  p.isPlus = isPlus;
  p.cb = cb;
}

} // namespace

extern "C" {

long long qb200_hop_force_elems(const qb200_lattice *lat)
{
  GeoDev g;
  if (!lat || api_geo(lat, g)) return -1;
  return (long long)g.nsites * 8 * 9 * 2;
}

int qb200_hop_force(const qb200_lattice *lat, int cb, int isign, const void *chi, const void *psi,
                    const void *gauge, double coeff_s, double coeff_t_f, double coeff_t_b, unsigned tbc_mask,
                    const double *tbc_phases, void *force, void *stream)
{
  GeoDev g;
  int rc = api_geo(lat, g);
  if (rc) return rc;
  if (lat->ftype != QB200_F32 && lat->ftype != QB200_F64)
    return api_fail(QB200_ELAYOUT, "the force kernel is built for FP32 and FP64 storage");
  if (cb != 0 && cb != 1) return api_fail(QB200_EINVAL, "cb must be 0 or 1");
  if (!chi || !psi || !force) return api_fail(QB200_ENULL, "chi, psi and force must be non-NULL");
  if ((tbc_mask & 15u) && !tbc_phases) return api_fail(QB200_ENULL, "tbc_mask set but tbc_phases is NULL");
  if ((rc = api_check_device())) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const bool proj = gauge != nullptr, c12 = lat->compress12 != 0;
  cudaError_t e;
  if (lat->ftype == QB200_F32) {
    OpDev<float> p;
    fill<float>(p, lat, isign > 0, cb, coeff_s, coeff_t_f, coeff_t_b, tbc_mask, tbc_phases);
    e = launch_force<float>(lat->soalen, proj, c12, chi, psi, gauge, force, g, p, st);
  } else {
    OpDev<double> p;
    fill<double>(p, lat, isign > 0, cb, coeff_s, coeff_t_f, coeff_t_b, tbc_mask, tbc_phases);
    e = launch_force<double>(lat->soalen, proj, c12, chi, psi, gauge, force, g, p, st);
  }
  if (e != cudaSuccess) return api_fail(QB200_ECUDA, cudaGetErrorString(e));
  return QB200_OK;
}

} // extern "C"
