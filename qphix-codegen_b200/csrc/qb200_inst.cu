// qb200_inst.cu -- kernel instantiations and launchers for one storage type
// and SOALEN.  Compiled once per (QB_FT, QB_S) pair by the build so that the
// translation units build in parallel.
#include <atomic>
#include <cstdint>
#include <type_traits>

#include "qb200_face_kernel.cuh"
#include "qb200_internal.h"
#include "qb200_staged_kernel.cuh"
#include "qb200_async_kernel.cuh"
#include "qb200_twin_kernel.cuh"

// the single-RHS operator with the next hop's copies in flight (cp.async)
#ifndef QB_ASYNC
#define QB_ASYNC 1
#endif
// 16-bit storage: two sites per thread, bulk-copy staging (qb200_twin_kernel.cuh)
#ifndef QB_TWIN
#define QB_TWIN 1
#endif

#if QB_MRHS
#include "qb200_pair_kernel.cuh"
#endif

#ifndef QB_FT
#error "QB_FT (float, double, __half) must be defined"
#endif
#ifndef QB_S
#error "QB_S (SOALEN) must be defined"
#endif

namespace qb200 {

namespace {
constexpr int kThreads = 128;

// two sites per thread for 16-bit storage: one warp per 64 sites of a plane
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
cudaError_t go_twin(const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p, cudaStream_t st)
{
  typedef TwinCfg<FT, S, COMP12> T;
  const int nchunk = (g.nxh * g.ny + 63) / 64;
  const long long nw = (long long)g.nz * g.nt * nchunk;
  const long long blocks = (nw + kTwinWarps - 1) / kTwinWarps;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  const int smem = kTwinWarps * T::WB;
  // the dynamic shared-memory limit of this kernel, raised once per device
  static std::atomic<unsigned long long> raised{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!(raised.load() & (1ull << dev))) {
    e = cudaFuncSetAttribute(twin_site_kernel<FT, S, COMP12, FAM, ACH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return e;
    raised.fetch_or(1ull << dev);
  }
  twin_site_kernel<FT, S, COMP12, FAM, ACH><<<(unsigned)blocks, kTwinWarps * 32, smem, st>>>(a, g, p, nchunk);
  return cudaGetLastError();
}

template <typename FT, int S, bool COMP12, int FAM, bool ACH, bool MR>
cudaError_t go(const KArgs<FT> &a, const GeoDev &g, const OpDev<typename ftraits<FT>::C> &p,
               cudaStream_t st)
{
  // one grid row per (z, t) plane
  const long long n = (long long)g.nxh * g.ny * (MR ? g.nrhs : 1);
  const dim3 grid((unsigned)((n + kThreads - 1) / kThreads), (unsigned)(g.nz * g.nt));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  if constexpr (QB_TWIN && !MR && twin_layout<FT, S>()) {
    const bool al = (((uintptr_t)a.psi | (uintptr_t)a.out | (uintptr_t)a.gauge) % 16 == 0) &&
                    (!ACH || (uintptr_t)a.chi % 16 == 0) && ((FAM != FAM_CLOVER && FAM != FAM_TMCLOV) || (uintptr_t)a.clov % 16 == 0);
    if (g.V == S && al) return go_twin<FT, S, COMP12, FAM, ACH>(a, g, p, st);
  }
  if constexpr (QB_ASYNC && !MR && async_layout<FT, S>()) {
    const bool al = (((uintptr_t)a.psi | (uintptr_t)a.out | (uintptr_t)a.gauge) % 16 == 0) &&
                    (!ACH || (uintptr_t)a.chi % 16 == 0) && ((FAM != FAM_CLOVER && FAM != FAM_TMCLOV) || (uintptr_t)a.clov % 16 == 0);
    if (g.V == S && al) {
      const long long nb = warp_blocks(g);
      if (nb > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
      async_site_kernel<FT, S, COMP12, FAM, ACH><<<(unsigned)nb, kThreads, 0, st>>>(a, g, p);
      return cudaGetLastError();
    }
  }
  // VECLEN known at compile time for the V == S layouts
  if (S >= 4 && g.V == S) site_dslash_kernel<FT, S, COMP12, FAM, ACH, MR, (S >= 4 ? S : 0)><<<grid, kThreads, 0, st>>>(a, g, p);
  else site_dslash_kernel<FT, S, COMP12, FAM, ACH, MR, 0><<<grid, kThreads, 0, st>>>(a, g, p);
  return cudaGetLastError();
}

template <typename FT, int S, bool COMP12, bool MR>
cudaError_t go_fam(const LaunchSpec &ls, const KArgs<FT> &a, const GeoDev &g,
                   const OpDev<typename ftraits<FT>::C> &p, cudaStream_t st)
{
  switch (ls.fam * 2 + (ls.ach ? 1 : 0)) {
  case 0: return go<FT, S, COMP12, FAM_WILSON, false, MR>(a, g, p, st);
  case 1: return go<FT, S, COMP12, FAM_WILSON, true, MR>(a, g, p, st);
  case 2: return go<FT, S, COMP12, FAM_CLOVER, false, MR>(a, g, p, st);
  case 3: return go<FT, S, COMP12, FAM_CLOVER, true, MR>(a, g, p, st);
  case 4: return go<FT, S, COMP12, FAM_TM, false, MR>(a, g, p, st);
  case 5: return go<FT, S, COMP12, FAM_TM, true, MR>(a, g, p, st);
  case 6: return go<FT, S, COMP12, FAM_TMCLOV, false, MR>(a, g, p, st);
  case 7: return go<FT, S, COMP12, FAM_TMCLOV, true, MR>(a, g, p, st);
  }
  return cudaErrorInvalidValue;
}

#if QB_MRHS
// two right-hand sides per thread (even nrhs)
template <typename FT, int S, bool COMP12, int FAM, bool ACH>
cudaError_t go_pair(const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p, cudaStream_t st)
{
  const long long n = (long long)g.nxh * g.ny * (g.nrhs / 2);
  const dim3 grid((unsigned)((n + kThreads - 1) / kThreads), (unsigned)(g.nz * g.nt));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  if (g.V != S) pair_dslash_kernel<FT, S, COMP12, FAM, ACH, 0, 0><<<grid, kThreads, 0, st>>>(a, g, p);
  else if (g.nrhs == 2) pair_dslash_kernel<FT, S, COMP12, FAM, ACH, S, 2><<<grid, kThreads, 0, st>>>(a, g, p);
  else if (g.nrhs == 4) pair_dslash_kernel<FT, S, COMP12, FAM, ACH, S, 4><<<grid, kThreads, 0, st>>>(a, g, p);
  else if (g.nrhs == 8) pair_dslash_kernel<FT, S, COMP12, FAM, ACH, S, 8><<<grid, kThreads, 0, st>>>(a, g, p);
  else if (g.nrhs == 16) pair_dslash_kernel<FT, S, COMP12, FAM, ACH, S, 16><<<grid, kThreads, 0, st>>>(a, g, p);
  else pair_dslash_kernel<FT, S, COMP12, FAM, ACH, S, 0><<<grid, kThreads, 0, st>>>(a, g, p);
  return cudaGetLastError();
}

template <typename FT, int S, bool COMP12>
cudaError_t go_pair_fam(const LaunchSpec &ls, const KArgs<FT> &a, const GeoDev &g, const OpDev<float> &p,
                        cudaStream_t st)
{
  switch (ls.fam * 2 + (ls.ach ? 1 : 0)) {
  case 0: return go_pair<FT, S, COMP12, FAM_WILSON, false>(a, g, p, st);
  case 1: return go_pair<FT, S, COMP12, FAM_WILSON, true>(a, g, p, st);
  case 2: return go_pair<FT, S, COMP12, FAM_CLOVER, false>(a, g, p, st);
  case 3: return go_pair<FT, S, COMP12, FAM_CLOVER, true>(a, g, p, st);
  case 4: return go_pair<FT, S, COMP12, FAM_TM, false>(a, g, p, st);
  case 5: return go_pair<FT, S, COMP12, FAM_TM, true>(a, g, p, st);
  case 6: return go_pair<FT, S, COMP12, FAM_TMCLOV, false>(a, g, p, st);
  case 7: return go_pair<FT, S, COMP12, FAM_TMCLOV, true>(a, g, p, st);
  }
  return cudaErrorInvalidValue;
}
#endif

template <typename FT, int S, bool COMP12, int FAM>
cudaError_t go_unpack(const elem_t<FT> *buf, const elem_t<FT> *gauge, const elem_t<FT> *clov, elem_t<FT> *out,
                      const GeoDev &g, const FaceDev &f, const OpDev<comp_t<FT>> &p, cudaStream_t st)
{
  const int blocks = (f.nface + kThreads - 1) / kThreads;
  face_unpack_kernel<FT, S, COMP12, FAM><<<blocks, kThreads, 0, st>>>(buf, gauge, clov, out, g, f, p);
  return cudaGetLastError();
}

template <typename FT, int S, bool COMP12, int FAM, bool ACH>
cudaError_t go_batch(const BatchDev<FT> &b, bool vfixed, int grid, int block, cudaStream_t st)
{
  // async-staged kernel (V == S, S >= 4, 32- or 16-bit), one warp per 32
  // sites of a plane
  if constexpr (QB_ASYNC && async_layout<FT, S>()) {
    bool al = vfixed;
    for (int k = 0; k < b.n && al; k++) {
      const KArgs<FT> &x = b.it[k].a;
      al = (((uintptr_t)x.psi | (uintptr_t)x.out | (uintptr_t)x.gauge) % 16 == 0) &&
           (!ACH || (uintptr_t)x.chi % 16 == 0) && ((FAM != FAM_CLOVER && FAM != FAM_TMCLOV) || (uintptr_t)x.clov % 16 == 0);
    }
    if (al) {
      BatchDev<FT> bw = b;
      long long first = 0;
      for (int k = 0; k < b.n; k++) {
        bw.it[k].first = first;
        first += (long long)b.it[k].g.nz * b.it[k].g.nt * ((b.it[k].g.nxh * b.it[k].g.ny + 31) / 32);
      }
      bw.total = first;
      batch_async_kernel<FT, S, COMP12, FAM, ACH><<<grid, block, 0, st>>>(bw);
      return cudaGetLastError();
    }
  }
  if (S >= 4 && vfixed) batch_dslash_kernel<FT, S, COMP12, FAM, ACH, (S >= 4 ? S : 0)><<<grid, block, 0, st>>>(b);
  else if (S < 4) batch_dslash_kernel<FT, S, COMP12, FAM, ACH, 0><<<grid, block, 0, st>>>(b);
  else return cudaErrorInvalidValue; // SOALEN >= 4 layouts batch only with VECLEN == SOALEN
  return cudaGetLastError();
}

FaceDev to_dev(const FaceSpec &s)
{
  FaceDev f;
  f.dir = s.dir;
  f.mu = s.mu;
  f.coord = s.coord;
  f.par = s.par;
  f.nface = s.nface;
  f.cb = s.cb;
  return f;
}
} // namespace

template <typename FT, int S>
cudaError_t launch_dslash(const LaunchSpec &ls, const elem_t<FT> *psi, const elem_t<FT> *chi,
                          const elem_t<FT> *gauge, const elem_t<FT> *clov, elem_t<FT> *out, const GeoDev &g,
                          const OpDev<comp_t<FT>> &p, cudaStream_t st)
{
  KArgs<FT> a;
  a.psi = psi;
  a.chi = chi;
  a.gauge = gauge;
  a.clov = clov;
  a.out = out;
  if (g.nsites == 0) return cudaSuccess;
  return ls.comp12 ? go_fam<FT, S, true, false>(ls, a, g, p, st) : go_fam<FT, S, false, false>(ls, a, g, p, st);
}

#if QB_MRHS
template <typename FT, int S>
cudaError_t launch_dslash_mrhs(const LaunchSpec &ls, const elem_t<FT> *psi, const elem_t<FT> *chi,
                               const elem_t<FT> *gauge, const elem_t<FT> *clov, elem_t<FT> *out, const GeoDev &g,
                               const OpDev<comp_t<FT>> &p, cudaStream_t st)
{
  KArgs<FT> a;
  a.psi = psi;
  a.chi = chi;
  a.gauge = gauge;
  a.clov = clov;
  a.out = out;
  if (g.nsites == 0) return cudaSuccess;
  if (g.nrhs % 2 == 0)
    return ls.comp12 ? go_pair_fam<FT, S, true>(ls, a, g, p, st) : go_pair_fam<FT, S, false>(ls, a, g, p, st);
  return ls.comp12 ? go_fam<FT, S, true, true>(ls, a, g, p, st) : go_fam<FT, S, false, true>(ls, a, g, p, st);
}
#endif

template <typename FT, int S>
cudaError_t launch_dslash_batched(const LaunchSpec &ls, const BatchDev<FT> &b, bool vfixed, int grid, int block,
                                  cudaStream_t st)
{
  if (b.total == 0) return cudaSuccess;
  switch (ls.fam * 4 + (ls.ach ? 2 : 0) + (ls.comp12 ? 1 : 0)) {
  case 0: return go_batch<FT, S, false, FAM_WILSON, false>(b, vfixed, grid, block, st);
  case 1: return go_batch<FT, S, true, FAM_WILSON, false>(b, vfixed, grid, block, st);
  case 2: return go_batch<FT, S, false, FAM_WILSON, true>(b, vfixed, grid, block, st);
  case 3: return go_batch<FT, S, true, FAM_WILSON, true>(b, vfixed, grid, block, st);
  case 4: return go_batch<FT, S, false, FAM_CLOVER, false>(b, vfixed, grid, block, st);
  case 5: return go_batch<FT, S, true, FAM_CLOVER, false>(b, vfixed, grid, block, st);
  case 6: return go_batch<FT, S, false, FAM_CLOVER, true>(b, vfixed, grid, block, st);
  case 7: return go_batch<FT, S, true, FAM_CLOVER, true>(b, vfixed, grid, block, st);
  case 8: return go_batch<FT, S, false, FAM_TM, false>(b, vfixed, grid, block, st);
  case 9: return go_batch<FT, S, true, FAM_TM, false>(b, vfixed, grid, block, st);
  case 10: return go_batch<FT, S, false, FAM_TM, true>(b, vfixed, grid, block, st);
  case 11: return go_batch<FT, S, true, FAM_TM, true>(b, vfixed, grid, block, st);
  case 12: return go_batch<FT, S, false, FAM_TMCLOV, false>(b, vfixed, grid, block, st);
  case 13: return go_batch<FT, S, true, FAM_TMCLOV, false>(b, vfixed, grid, block, st);
  case 14: return go_batch<FT, S, false, FAM_TMCLOV, true>(b, vfixed, grid, block, st);
  case 15: return go_batch<FT, S, true, FAM_TMCLOV, true>(b, vfixed, grid, block, st);
  }
  return cudaErrorInvalidValue;
}

template <typename FT, int S>
cudaError_t launch_face_pack(const elem_t<FT> *psi, elem_t<FT> *buf, const GeoDev &g, const FaceSpec &fs,
                             int isPlus, cudaStream_t st)
{
  if (fs.nface == 0) return cudaSuccess;
  const FaceDev f = to_dev(fs);
  const int blocks = (f.nface + kThreads - 1) / kThreads;
  face_pack_kernel<FT, S><<<blocks, kThreads, 0, st>>>(psi, buf, g, f, isPlus);
  return cudaGetLastError();
}

template <typename FT, int S>
cudaError_t launch_face_unpack(int fam, bool comp12, const elem_t<FT> *buf, const elem_t<FT> *gauge,
                               const elem_t<FT> *clov, elem_t<FT> *out, const GeoDev &g, const FaceSpec &fs,
                               const OpDev<comp_t<FT>> &p, cudaStream_t st)
{
  if (fs.nface == 0) return cudaSuccess;
  const FaceDev f = to_dev(fs);
  switch (fam * 2 + (comp12 ? 1 : 0)) {
  case 0: return go_unpack<FT, S, false, FAM_WILSON>(buf, gauge, clov, out, g, f, p, st);
  case 1: return go_unpack<FT, S, true, FAM_WILSON>(buf, gauge, clov, out, g, f, p, st);
  case 2: return go_unpack<FT, S, false, FAM_CLOVER>(buf, gauge, clov, out, g, f, p, st);
  case 3: return go_unpack<FT, S, true, FAM_CLOVER>(buf, gauge, clov, out, g, f, p, st);
  case 4: return go_unpack<FT, S, false, FAM_TM>(buf, gauge, clov, out, g, f, p, st);
  case 5: return go_unpack<FT, S, true, FAM_TM>(buf, gauge, clov, out, g, f, p, st);
  case 6: return go_unpack<FT, S, false, FAM_TMCLOV>(buf, gauge, clov, out, g, f, p, st);
  case 7: return go_unpack<FT, S, true, FAM_TMCLOV>(buf, gauge, clov, out, g, f, p, st);
  }
  return cudaErrorInvalidValue;
}

typedef elem_t<QB_FT> QB_E;
template cudaError_t launch_dslash<QB_FT, QB_S>(const LaunchSpec &, const QB_E *, const QB_E *, const QB_E *,
                                                const QB_E *, QB_E *, const GeoDev &, const OpDev<comp_t<QB_FT>> &,
                                                cudaStream_t);
template cudaError_t launch_dslash_batched<QB_FT, QB_S>(const LaunchSpec &, const BatchDev<QB_FT> &, bool, int, int,
                                                        cudaStream_t);
template cudaError_t launch_face_pack<QB_FT, QB_S>(const QB_E *, QB_E *, const GeoDev &, const FaceSpec &, int,
                                                   cudaStream_t);
#if QB_MRHS
template cudaError_t launch_dslash_mrhs<QB_FT, QB_S>(const LaunchSpec &, const QB_E *, const QB_E *, const QB_E *,
                                                     const QB_E *, QB_E *, const GeoDev &,
                                                     const OpDev<comp_t<QB_FT>> &, cudaStream_t);
#endif
template cudaError_t launch_face_unpack<QB_FT, QB_S>(int, bool, const QB_E *, const QB_E *, const QB_E *, QB_E *,
                                                     const GeoDev &, const FaceSpec &, const OpDev<comp_t<QB_FT>> &,
                                                     cudaStream_t);

} // namespace qb200
