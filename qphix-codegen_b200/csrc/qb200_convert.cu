// qb200_convert.cu -- layout converters between canonical site-major complex
// fields and the QPhiX tile layouts, on the device.
//
// Canonical formats (complex numbers as (re, im) pairs of FP64 or FP32):
//   spinor  [nt][nz][ny][nxh][4 spin][3 colour]            one checkerboard
//   links   [4 mu][nt_global][nz][ny][nx][3][3] U          the whole lattice
//   clover  [nt][nz][ny][nxh][2 block][6][6]                one checkerboard
// Site (xcb, y, z, t) of checkerboard cb sits at x = 2*xcb + ((y+z+t+cb)&1).
// The tile side follows codegen/include/decl_common.h:9-62: FourSpinorBlock
// FT[3][4][2][S] (+ float norm[S] for QB200_F16N), SU3MatrixBlock
// FT[8][2|3][3][2][V] storing G = U^T with the backward link U(x - mu) at the
// output site (codegen/dslash_common.cc:1678-1727, 12-real: rows 0 and 1 of
// G, :1657-1676), CloverBlock {diag[6], off_diag[15][2]} per block with
// off_diag[r(r-1)/2 + c] = A[r][c], r > c (:1098-1186), FullCloverBlock
// [2][6][6][2].  The reference has no converters (QPhiX's, not part of it,
// run on the host); these are the B200 build's own.
#include <cstdint>

#include "qphix_b200.h"
#include "qb200_internal.h"

namespace qb200 {
int api_fail(int code, const char *msg);
int api_geo(const qb200_lattice *l, GeoDev &g);
int api_check_device();
} // namespace qb200

using namespace qb200;

namespace {

constexpr int kT = 256;

__device__ __forceinline__ void site_coords(const GeoDev &g, long long i, int &xcb, int &y, int &z, int &t)
{
  xcb = (int)(i % g.nxh);
  long long r = i / g.nxh;
  y = (int)(r % g.ny);
  r /= g.ny;
  z = (int)(r % g.nz);
  t = (int)(r / g.nz);
}

__device__ __forceinline__ long long spinor_block(const GeoDev &g, int xcb, int y, int z, int t, int S)
{
  return t * g.Pxyz + z * g.Pxy + (long long)y * g.nvecs + xcb / S;
}

__device__ __forceinline__ long long tile_index(const GeoDev &g, int xcb, int y, int z, int t, int S, int *lane)
{
  const int yq = y / g.ngy;
  *lane = (y - yq * g.ngy) * S + xcb % S;
  return ((long long)(t * g.nz + z) * g.nyg + yq) * g.nvecs + xcb / S;
}

template <typename CT> __device__ __forceinline__ double cd(const CT *p, long long i) { return (double)p[i]; }

template <typename FT>
__device__ __forceinline__ void put(elem_t<FT> *p, long long i, double v)
{
  ftraits<FT>::st(p + i, (comp_t<FT>)v);
}

// one thread per site: 24 reals in, 24 (+ norm) out
template <typename FT, typename CT>
__global__ void __launch_bounds__(kT) pack_spinor_kernel(const GeoDev g, int S, const CT *__restrict__ in,
                                                          elem_t<FT> *__restrict__ out)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.nsites) return;
  int xcb, y, z, t;
  site_coords(g, i, xcb, y, z, t);
  const long long base = spinor_block(g, xcb, y, z, t, S) * (ftraits<FT>::SPB * S) + xcb % S;
  double v[24];
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      // canonical (spin, colour, ri) -> tile component ((c*4 + s)*2 + ri)
      v[(c * 4 + s) * 2 + 0] = cd(in, (i * 12 + s * 3 + c) * 2 + 0);
      v[(c * 4 + s) * 2 + 1] = cd(in, (i * 12 + s * 3 + c) * 2 + 1);
    }
  double scale = 1.0;
  if (ftraits<FT>::SPB == 26) {
    double m = 0.0;
#pragma unroll
    for (int k = 0; k < 24; k++) m = fmax(m, fabs(v[k]));
    const float nrm = m > 0.0 ? (float)m : 1.0f;
    reinterpret_cast<float *>(out + base - xcb % S + 24 * S)[xcb % S] = nrm;
    scale = (double)nrm;
  }
#pragma unroll
  for (int k = 0; k < 24; k++) put<FT>(out, base + (long long)k * S, ftraits<FT>::SPB == 26 ? v[k] / scale : v[k]);
}

template <typename FT, typename CT>
__global__ void __launch_bounds__(kT) unpack_spinor_kernel(const GeoDev g, int S, const elem_t<FT> *__restrict__ in,
                                                            CT *__restrict__ out)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.nsites) return;
  int xcb, y, z, t;
  site_coords(g, i, xcb, y, z, t);
  const long long base = spinor_block(g, xcb, y, z, t, S) * (ftraits<FT>::SPB * S) + xcb % S;
  double nrm = 1.0;
  if (ftraits<FT>::SPB == 26) nrm = reinterpret_cast<const float *>(in + base - xcb % S + 24 * S)[xcb % S];
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int ri = 0; ri < 2; ri++)
        out[(i * 12 + s * 3 + c) * 2 + ri] =
            (CT)(nrm * (double)ftraits<FT>::cv(in[base + (long long)((c * 4 + s) * 2 + ri) * S]));
}

// one thread per (site of cb, direction)
template <typename FT, typename CT>
__global__ void __launch_bounds__(kT) pack_gauge_kernel(const GeoDev g, int S, int R, int cb, int ntg, int t0,
                                                         const CT *__restrict__ U, elem_t<FT> *__restrict__ out)
{
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= 8LL * g.nsites) return;
  const long long i = q >> 3;
  const int d = (int)(q & 7), mu = d >> 1;
  int xcb, y, z, t;
  site_coords(g, i, xcb, y, z, t);
  int c4[4] = {2 * xcb + ((y + z + t + cb) & 1), y, z, (t + t0) % ntg};
  const int L[4] = {g.nx, g.ny, g.nz, ntg};
  if (!(d & 1)) c4[mu] = (c4[mu] + L[mu] - 1) % L[mu]; // backward hop: U_mu(x - mu)
  const long long site = (((long long)c4[3] * g.nz + c4[2]) * g.ny + c4[1]) * g.nx + c4[0];
  const long long vol = (long long)ntg * g.nz * g.ny * g.nx;
  const CT *u = U + ((mu * vol + site) * 9) * 2;
  int lane;
  const long long tile = tile_index(g, xcb, y, z, t, S, &lane);
  elem_t<FT> *o = out + tile * (8LL * R * 6 * g.V) + lane;
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int ri = 0; ri < 2; ri++) // G[r][c] = U[c][r]
        put<FT>(o, (long long)(((d * R + r) * 3 + c) * 2 + ri) * g.V, cd(u, (c * 3 + r) * 2 + ri));
}

// one thread per site; FULL: dense FullCloverBlock, else Hermitian CloverBlock
template <typename FT, typename CT, bool FULL>
__global__ void __launch_bounds__(kT) pack_clover_kernel(const GeoDev g, int S, const CT *__restrict__ A,
                                                          elem_t<FT> *__restrict__ out)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.nsites) return;
  int xcb, y, z, t;
  site_coords(g, i, xcb, y, z, t);
  int lane;
  const long long tile = tile_index(g, xcb, y, z, t, S, &lane);
  const int K = FULL ? 144 : 72;
  elem_t<FT> *o = out + tile * ((long long)K * g.V) + lane;
  const CT *a = A + i * 144; // [2][6][6][2]
  if (FULL) {
    for (int k = 0; k < 144; k++) put<FT>(o, (long long)k * g.V, cd(a, k));
  } else {
    for (int b = 0; b < 2; b++) {
      for (int r = 0; r < 6; r++) put<FT>(o, (long long)(b * 36 + r) * g.V, cd(a, ((b * 6 + r) * 6 + r) * 2));
      for (int r = 1; r < 6; r++)
        for (int c = 0; c < r; c++) {
          const int j = r * (r - 1) / 2 + c;
          put<FT>(o, (long long)(b * 36 + 6 + 2 * j) * g.V, cd(a, ((b * 6 + r) * 6 + c) * 2 + 0));
          put<FT>(o, (long long)(b * 36 + 7 + 2 * j) * g.V, cd(a, ((b * 6 + r) * 6 + c) * 2 + 1));
        }
    }
  }
}

int blocks_for(long long n) { return (int)((n + kT - 1) / kT); }

template <typename CT>
cudaError_t spinor_dispatch(bool pack, const qb200_lattice *l, const GeoDev &g, const void *in, void *out,
                            cudaStream_t st)
{
  const int nb = blocks_for(g.nsites);
  const int S = l->soalen;
#define QB_SP(FT)                                                                                            \
  if (pack) pack_spinor_kernel<FT, CT><<<nb, kT, 0, st>>>(g, S, (const CT *)in, (elem_t<FT> *)out);          \
  else unpack_spinor_kernel<FT, CT><<<nb, kT, 0, st>>>(g, S, (const elem_t<FT> *)in, (CT *)out);
  switch (l->ftype) {
  case QB200_F32: QB_SP(float) break;
  case QB200_F64: QB_SP(double) break;
  case QB200_F16: QB_SP(__half) break;
  case QB200_F16N: QB_SP(half_norm) break;
  default: QB_SP(__nv_bfloat16) break;
  }
#undef QB_SP
  return cudaGetLastError();
}

template <typename CT>
cudaError_t gauge_dispatch(const qb200_lattice *l, const GeoDev &g, int cb, int ntg, int t0, const void *in,
                           void *out, cudaStream_t st)
{
  const int nb = blocks_for(8LL * g.nsites);
  const int S = l->soalen, R = l->compress12 ? 2 : 3;
#define QB_G(FT) pack_gauge_kernel<FT, CT><<<nb, kT, 0, st>>>(g, S, R, cb, ntg, t0, (const CT *)in, (elem_t<FT> *)out);
  switch (l->ftype) {
  case QB200_F32: QB_G(float) break;
  case QB200_F64: QB_G(double) break;
  case QB200_BF16: QB_G(__nv_bfloat16) break;
  default: QB_G(__half) break; // F16 and F16N store plain FP16 links
  }
#undef QB_G
  return cudaGetLastError();
}

template <typename CT>
cudaError_t clover_dispatch(bool full, const qb200_lattice *l, const GeoDev &g, const void *in, void *out,
                            cudaStream_t st)
{
  const int nb = blocks_for(g.nsites);
  const int S = l->soalen;
#define QB_C(FT)                                                                                              \
  if (full) pack_clover_kernel<FT, CT, true><<<nb, kT, 0, st>>>(g, S, (const CT *)in, (elem_t<FT> *)out);     \
  else pack_clover_kernel<FT, CT, false><<<nb, kT, 0, st>>>(g, S, (const CT *)in, (elem_t<FT> *)out);
  switch (l->ftype) {
  case QB200_F32: QB_C(float) break;
  case QB200_F64: QB_C(double) break;
  case QB200_BF16: QB_C(__nv_bfloat16) break;
  default: QB_C(__half) break;
  }
#undef QB_C
  return cudaGetLastError();
}

int check(const qb200_lattice *l, int ctype, const void *a, const void *b, GeoDev &g)
{
  int rc = api_geo(l, g);
  if (rc) return rc;
  if (ctype != QB200_F64 && ctype != QB200_F32) return api_fail(QB200_EINVAL, "ctype must be QB200_F64 or QB200_F32");
  if (!a || !b) return api_fail(QB200_ENULL, "field pointers must be non-NULL");
  if (l->ftype == QB200_F16N && ((uintptr_t)a % 4 || (uintptr_t)b % 4))
    return api_fail(QB200_EALIGN, "QB200_F16N spinor fields must be 4-byte aligned");
  return api_check_device();
}

int done(cudaError_t e)
{
  if (e != cudaSuccess) return api_fail(QB200_ECUDA, cudaGetErrorString(e));
  return QB200_OK;
}

} // namespace

extern "C" {

int qb200_pack_spinor(const qb200_lattice *lat, int ctype, const void *canon, void *spinor, void *stream)
{
  GeoDev g;
  int rc = check(lat, ctype, canon, spinor, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  return done(ctype == QB200_F64 ? spinor_dispatch<double>(true, lat, g, canon, spinor, st)
                                 : spinor_dispatch<float>(true, lat, g, canon, spinor, st));
}

int qb200_unpack_spinor(const qb200_lattice *lat, int ctype, const void *spinor, void *canon, void *stream)
{
  GeoDev g;
  int rc = check(lat, ctype, spinor, canon, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  return done(ctype == QB200_F64 ? spinor_dispatch<double>(false, lat, g, spinor, canon, st)
                                 : spinor_dispatch<float>(false, lat, g, spinor, canon, st));
}

int qb200_pack_gauge(const qb200_lattice *lat, int cb, int ctype, const void *links, int nt_global, int t0,
                     void *gauge, void *stream)
{
  GeoDev g;
  int rc = check(lat, ctype, links, gauge, g);
  if (rc) return rc;
  if (cb != 0 && cb != 1) return api_fail(QB200_EINVAL, "cb must be 0 or 1");
  if (nt_global < lat->nt || t0 < 0 || t0 + lat->nt > nt_global)
    return api_fail(QB200_EINVAL, "the local time slices [t0, t0 + nt) must lie in [0, nt_global)");
  cudaStream_t st = (cudaStream_t)stream;
  return done(ctype == QB200_F64 ? gauge_dispatch<double>(lat, g, cb, nt_global, t0, links, gauge, st)
                                 : gauge_dispatch<float>(lat, g, cb, nt_global, t0, links, gauge, st));
}

int qb200_pack_clover(const qb200_lattice *lat, int ctype, const void *blocks, void *clover, void *stream)
{
  GeoDev g;
  int rc = check(lat, ctype, blocks, clover, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  return done(ctype == QB200_F64 ? clover_dispatch<double>(false, lat, g, blocks, clover, st)
                                 : clover_dispatch<float>(false, lat, g, blocks, clover, st));
}

int qb200_pack_full_clover(const qb200_lattice *lat, int ctype, const void *blocks, void *clover, void *stream)
{
  GeoDev g;
  int rc = check(lat, ctype, blocks, clover, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  return done(ctype == QB200_F64 ? clover_dispatch<double>(true, lat, g, blocks, clover, st)
                                 : clover_dispatch<float>(true, lat, g, blocks, clover, st));
}

} // extern "C"
