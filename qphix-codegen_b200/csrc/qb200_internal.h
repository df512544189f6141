// qb200_internal.h -- host-side declarations shared by the C-ABI layer and
// the per-(storage type, SOALEN) kernel translation units.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "qb200_site_kernel.cuh"

namespace qb200 {

// what one launch computes
struct LaunchSpec {
  int fam;        // FAM_WILSON .. FAM_TMCLOV
  bool ach;       // achimbdpsi form
  bool comp12;    // 12-real links
};

// body kernel launcher, defined in qb200_inst.cu for each (FT, S)
template <typename FT, int S>
cudaError_t launch_dslash(const LaunchSpec &ls, const elem_t<FT> *psi, const elem_t<FT> *chi,
                          const elem_t<FT> *gauge, const elem_t<FT> *clov, elem_t<FT> *out, const GeoDev &g,
                          const OpDev<comp_t<FT>> &p, cudaStream_t st);

// multi-RHS body kernel launcher (g.nrhs right-hand sides interleaved
// innermost), defined in qb200_inst.cu for FT in {float, __half}, S in {4, 8, 16}
template <typename FT, int S>
cudaError_t launch_dslash_mrhs(const LaunchSpec &ls, const elem_t<FT> *psi, const elem_t<FT> *chi,
                               const elem_t<FT> *gauge, const elem_t<FT> *clov, elem_t<FT> *out, const GeoDev &g,
                               const OpDev<comp_t<FT>> &p, cudaStream_t st);

// batched launcher (qb200_site_kernel.cuh: batch_dslash_kernel), defined in
// qb200_inst.cu for each (FT, S); vfixed: every item has VECLEN == SOALEN
// (compile-time VECLEN for S >= 4); block <= 128
template <typename FT, int S>
cudaError_t launch_dslash_batched(const LaunchSpec &ls, const BatchDev<FT> &b, bool vfixed, int grid, int block,
                                  cudaStream_t st);

// face launchers, defined in qb200_inst.cu for each (FT, S)
struct FaceSpec {
  int dir, mu, coord, par, nface, cb;
};
template <typename FT, int S>
cudaError_t launch_face_pack(const elem_t<FT> *psi, elem_t<FT> *buf, const GeoDev &g, const FaceSpec &f,
                             int isPlus, cudaStream_t st);
template <typename FT, int S>
cudaError_t launch_face_unpack(int fam, bool comp12, const elem_t<FT> *buf, const elem_t<FT> *gauge,
                               const elem_t<FT> *clov, elem_t<FT> *out, const GeoDev &g, const FaceSpec &f,
                               const OpDev<comp_t<FT>> &p, cudaStream_t st);

} // namespace qb200
