// qb200_face_kernel.cuh -- halo (face) pack and unpack kernels.
//
// face_pack: pack_face_vec (codegen/dslash.cc:433-458): the sites of psi on
// the face towards `dir` are projected with the projector of the opposite
// direction, because the neighbour beyond that face applies its own hop in
// direction dir^1 to them.
// face_unpack: recons_add_face_vec (codegen/dslash.cc:463-553): multiply the
// received half spinors by the link of direction dir (adjoint for a back
// face), reconstruct with +beta for clover faces and -beta otherwise
// (codegen/dslash_common.cc:1975-1981), apply the clover / full clover /
// A^-1 term to that contribution and accumulate into out.
#pragma once

#include "qb200_site_kernel.cuh"

namespace qb200 {

struct FaceDev {
  int dir, mu, coord, par, nface;
  int cb;
};

// site of face entry i (sites enumerated in (t, z, y, xcb) order)
__device__ __forceinline__ Site face_site(const GeoDev &g, const FaceDev &f, int i)
{
  Site s;
  if (f.mu == 3) {
    s.t = f.coord;
    s.xcb = i % g.nxh;
    int r = i / g.nxh;
    s.y = r % g.ny;
    s.z = r / g.ny;
  } else if (f.mu == 2) {
    s.z = f.coord;
    s.xcb = i % g.nxh;
    int r = i / g.nxh;
    s.y = r % g.ny;
    s.t = r / g.ny;
  } else if (f.mu == 1) {
    s.y = f.coord;
    s.xcb = i % g.nxh;
    int r = i / g.nxh;
    s.z = r % g.nz;
    s.t = r / g.nz;
  } else {
    // x face: one site per (t,z,y) row of the right parity
    const int nyh = g.ny / 2;
    const int k = i % nyh;
    const int zt = i / nyh;
    s.z = zt % g.nz;
    s.t = zt / g.nz;
    s.y = 2 * k + ((f.par + s.z + s.t + f.cb) & 1);
    s.xcb = f.par ? g.nxh - 1 : 0;
  }
  s.par = (s.y + s.z + s.t + f.cb) & 1;
  return s;
}

// one face site: 12 values; with a per-site norm (FACE == 14) the values are
// stored divided by the norm and the FP32 norm follows in the last two halves
template <typename FT>
__device__ __forceinline__ void store_face(elem_t<FT> *o, const cx<comp_t<FT>> (&b)[2][3])
{
  typedef comp_t<FT> C;
  C scale = (C)1;
  if (ftraits<FT>::FACE == 14) {
    C m = 0;
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int c = 0; c < 3; c++) m = fmax(m, fmax(fabs(b[h][c].re), fabs(b[h][c].im)));
    const C nrm = m > (C)0 ? m : (C)1;
    *reinterpret_cast<float *>(o + 12) = (float)nrm;
    scale = (C)1 / nrm;
  }
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      ftraits<FT>::st(o + (h * 3 + c) * 2 + 0, b[h][c].re * scale);
      ftraits<FT>::st(o + (h * 3 + c) * 2 + 1, b[h][c].im * scale);
    }
}

template <typename FT>
__device__ __forceinline__ void load_face(const elem_t<FT> *in, cx<comp_t<FT>> (&b)[2][3])
{
  typedef comp_t<FT> C;
  C nrm = (C)1;
  if (ftraits<FT>::FACE == 14) nrm = __ldg(reinterpret_cast<const float *>(in + 12));
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      b[h][c].re = ftraits<FT>::ld(in + (h * 3 + c) * 2 + 0) * nrm;
      b[h][c].im = ftraits<FT>::ld(in + (h * 3 + c) * 2 + 1) * nrm;
    }
}

template <typename FT, int S, int D>
__device__ __forceinline__ void pack_one(const elem_t<FT> *__restrict__ psi, elem_t<FT> *__restrict__ buf,
                                         const GeoDev &g, const FaceDev &f, int isPlus, int i)
{
  typedef comp_t<FT> C;
  const Site s = face_site(g, f, i);
  cx<C> sp[4][3], b[2][3];
  load_spinor<FT, S>(psi, spinor_base<FT, S>(g, s), sp);
  // proj_ops_plus[D^1] for plus == proj_ops_plus[D] with sigma = -1
  project<C, D>(sp, isPlus ? (C)-1 : (C)1, b);
  store_face<FT>(buf + (long long)i * ftraits<FT>::FACE, b);
}

template <typename FT, int S>
__global__ void __launch_bounds__(128)
    face_pack_kernel(const elem_t<FT> *__restrict__ psi, elem_t<FT> *__restrict__ buf, const GeoDev g,
                     const FaceDev f, int isPlus)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.nface) return;
  switch (f.dir) {
  case 0: pack_one<FT, S, 0>(psi, buf, g, f, isPlus, i); break;
  case 1: pack_one<FT, S, 1>(psi, buf, g, f, isPlus, i); break;
  case 2: pack_one<FT, S, 2>(psi, buf, g, f, isPlus, i); break;
  case 3: pack_one<FT, S, 3>(psi, buf, g, f, isPlus, i); break;
  case 4: pack_one<FT, S, 4>(psi, buf, g, f, isPlus, i); break;
  case 5: pack_one<FT, S, 5>(psi, buf, g, f, isPlus, i); break;
  case 6: pack_one<FT, S, 6>(psi, buf, g, f, isPlus, i); break;
  default: pack_one<FT, S, 7>(psi, buf, g, f, isPlus, i); break;
  }
}

template <typename FT, int S, bool COMP12, int FAM, int D>
__device__ __forceinline__ void unpack_one(const elem_t<FT> *__restrict__ buf,
                                           const elem_t<FT> *__restrict__ gauge,
                                           const elem_t<FT> *__restrict__ clov, elem_t<FT> *__restrict__ out,
                                           const GeoDev &g, const FaceDev &f,
                                           const OpDev<typename ftraits<FT>::C> &p, int i)
{
  typedef typename ftraits<FT>::C C;
  constexpr int MU = D / 2;
  constexpr bool BACK = (D & 1) == 0;
  constexpr bool CLOV = (FAM == FAM_CLOVER || FAM == FAM_TMCLOV);
  constexpr bool TM = (FAM == FAM_TM || FAM == FAM_TMCLOV);
  const Site s = face_site(g, f, i);
  int lane;
  const long long tile = tile_of<S>(g, s, &lane);
  constexpr int R = COMP12 ? 2 : 3;
  const long long obase = spinor_base<FT, S>(g, s);

  cx<C> o[4][3], b[2][3], ub[2][3], G[3][3];
  load_spinor<FT, S>(out, obase, o);
  load_face<FT>(buf + (long long)i * ftraits<FT>::FACE, b);
  load_link<FT, COMP12, D>(gauge, tile * (8LL * R * 6 * g.V) + lane, g.V, G);
  mult_link<C, BACK>(G, b, ub);
  if ((p.tbc_mask >> MU) & 1u) {
    const C pr = p.tbc[MU][0];
    const C pi = BACK ? -p.tbc[MU][1] : p.tbc[MU][1];
    apply_phase<C>(ub, pr, pi);
  }
  const C tau = ((p.isPlus != 0) == BACK) ? (C)1 : (C)-1;
  const C beta = CLOV ? p.beta[0] : -p.beta[0];
  if (CLOV || TM) {
    cx<C> dout[4][3];
#pragma unroll
    for (int sp = 0; sp < 4; sp++)
#pragma unroll
      for (int c = 0; c < 3; c++) dout[sp][c] = mk<C>(0, 0);
    recons<C, MU>(ub, beta, tau, dout);
    if (FAM == FAM_CLOVER || FAM == FAM_TMCLOV) {
      const long long cbase = tile * ((FAM == FAM_CLOVER ? 72LL : 144LL) * g.V) + lane;
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        if (FAM == FAM_CLOVER) clover_block<FT, MODE_ADD, false>(clov, cbase, g.V, blk, (C)0, dout, o);
        else full_clover_block<FT, MODE_ADD, false>(clov, cbase, g.V, blk, (C)0, dout, o);
      }
    } else {
      inv_twisted<C, true>(dout, p.isPlus, p.mu, p.muinv, o);
    }
  } else {
    recons<C, MU>(ub, beta, tau, o);
  }
  store_spinor<FT, S>(out, obase, o);
}

template <typename FT, int S, bool COMP12, int FAM>
__global__ void __launch_bounds__(128)
    face_unpack_kernel(const elem_t<FT> *__restrict__ buf, const elem_t<FT> *__restrict__ gauge,
                       const elem_t<FT> *__restrict__ clov, elem_t<FT> *__restrict__ out, const GeoDev g,
                       const FaceDev f,
                       const OpDev<typename ftraits<FT>::C> p)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.nface) return;
  switch (f.dir) {
  case 0: unpack_one<FT, S, COMP12, FAM, 0>(buf, gauge, clov, out, g, f, p, i); break;
  case 1: unpack_one<FT, S, COMP12, FAM, 1>(buf, gauge, clov, out, g, f, p, i); break;
  case 2: unpack_one<FT, S, COMP12, FAM, 2>(buf, gauge, clov, out, g, f, p, i); break;
  case 3: unpack_one<FT, S, COMP12, FAM, 3>(buf, gauge, clov, out, g, f, p, i); break;
  case 4: unpack_one<FT, S, COMP12, FAM, 4>(buf, gauge, clov, out, g, f, p, i); break;
  case 5: unpack_one<FT, S, COMP12, FAM, 5>(buf, gauge, clov, out, g, f, p, i); break;
  case 6: unpack_one<FT, S, COMP12, FAM, 6>(buf, gauge, clov, out, g, f, p, i); break;
  default: unpack_one<FT, S, COMP12, FAM, 7>(buf, gauge, clov, out, g, f, p, i); break;
  }
}

} // namespace qb200
