// qphix_tile_driver.cpp -- a QPhiX-style caller of the per-tile kernels
// (TEST CODE, compiled by tests/test_qphix_tiles*.py).
//
// It includes the reference's own kernel declarations -- the
// codegen/jinja/*_decl.h.j2 templates rendered unchanged into
// oracle/_ref/include by oracle/ref_build.py -- and nothing of this
// library's headers, so the link against libqphix_b200.so resolves each call
// to the B200 specialisation by the reference's symbol names.  Like QPhiX
// it walks a checkerboard tile by tile (veclen = soalen sites per tile), fills
// the per-lane offset arrays in FT elements relative to the base pointers
// (split x loads included) and the accumulate lane masks, and calls the
// kernel of each tile.  Fields are device pointers in the QPhiX layouts.
#include <cstdint>
#include <cstring>
#include <vector>

#include "dslash_decl.h"
#include "clov_dslash_decl.h"
#include "tm_dslash_decl.h"
#include "tm_clov_dslash_decl.h"

extern "C" int qb200_qphix_status(void);

namespace {

using QPhiX::Types;

struct Lat {
  int nx, ny, nz, nt, S, pad_xy, pad_xyz;
  double t_boundary;
  int t_edge_lo, t_edge_hi;
};

template <typename FT> FT cvt(double v) { return (FT)v; }
template <> unsigned short cvt<unsigned short>(double v)
{
  _Float16 h = (_Float16)(float)v;
  unsigned short b;
  std::memcpy(&b, &h, 2);
  return b;
}

struct Scalars {
  double cs, ctf, ctb, alpha, mu, muinv, rho;
  const double *phases;
  const unsigned *acc;
};

// the tile's arguments, as QPhiX would compute them (cf. the reference's
// per-tile contract, codegen/data_types.cc:60-198)
struct Tile {
  long long base, zb, zf, tb, tf, gtile;
  int t;
  int xbO[16], xfO[16], ybO[16], yfO[16], offs[16], gO[16];
  unsigned acc[8];
};

void make_tile(const Lat &L, int cb, int xb, int y, int z, int t, const unsigned *acc_in, Tile &T)
{
  const int S = L.S, nxh = L.nx / 2, nvecs = nxh / S;
  const long long Pxy = (long long)L.ny * nvecs + L.pad_xy, Pxyz = (long long)L.nz * Pxy + L.pad_xyz;
  auto blk = [&](int xb_, int y_, int z_, int t_) { return t_ * Pxyz + z_ * Pxy + (long long)y_ * nvecs + xb_; };
  const long long be = 24LL * S;
  T.t = t;
  T.base = blk(xb, y, z, t);
  T.zb = blk(xb, y, (z + L.nz - 1) % L.nz, t);
  T.zf = blk(xb, y, (z + 1) % L.nz, t);
  T.tb = blk(xb, y, z, (t + L.nt - 1) % L.nt);
  T.tf = blk(xb, y, z, (t + 1) % L.nt);
  T.gtile = ((long long)(t * L.nz + z) * L.ny + y) * nvecs + xb;
  const int par = (y + z + t + cb) & 1;
  const int xbm = (xb + nvecs - 1) % nvecs, xbp = (xb + 1) % nvecs;
  const long long to_m = (xbm - xb) * be, to_p = (xbp - xb) * be;
  const long long ym = (blk(xb, (y + L.ny - 1) % L.ny, z, t) - T.base) * be;
  const long long yp = (blk(xb, (y + 1) % L.ny, z, t) - T.base) * be;
  unsigned xbm_mask = 0, xfm_mask = 0;
  for (int l = 0; l < S; l++) {
    T.offs[l] = 0;
    T.ybO[l] = (int)ym;
    T.yfO[l] = (int)yp;
    T.xbO[l] = 0;
    T.xfO[l] = 0;
    T.gO[l] = 0;
    const int x = 2 * (xb * S + l) + par;
    if (acc_in[0] || x != 0) xbm_mask |= 1u << l;
    if (acc_in[1] || x != L.nx - 1) xfm_mask |= 1u << l;
  }
  if (S == 1) {
    T.xbO[0] = (int)(par == 0 ? to_m : 0);
    T.xfO[0] = (int)(par == 1 ? to_p : 0);
  } else {
    T.xbO[0] = par == 1 ? 0 : (int)(to_m + S - 1);
    T.xbO[1] = par == 1 ? 1 : 0;
    T.xfO[0] = par == 0 ? 0 : 1;
    T.xfO[S - 1] = par == 0 ? S - 1 : (int)to_p;
  }
  const unsigned all = (S >= 32) ? 0xffffffffu : ((1u << S) - 1u);
  T.acc[0] = xbm_mask & all;
  T.acc[1] = xfm_mask & all;
  T.acc[2] = (acc_in[2] || y != 0) ? all : 0u;
  T.acc[3] = (acc_in[3] || y != L.ny - 1) ? all : 0u;
  T.acc[4] = (acc_in[4] || z != 0) ? all : 0u;
  T.acc[5] = (acc_in[5] || z != L.nz - 1) ? all : 0u;
  T.acc[6] = (acc_in[6] || t != 0) ? all : 0u;
  T.acc[7] = (acc_in[7] || t != L.nt - 1) ? all : 0u;
}

// one body call, template arguments fixed
template <typename FT, int V, bool C12, bool X, bool Y, bool Z, bool W>
void call_body(int fam, int ach, int plus, const Tile &T, const void *psi, const void *chi, void *out,
               const void *gauge, const void *clov, const FT ph[4][2], FT cs, FT ctf, FT ctb, FT alpha, FT mu,
               FT muinv, FT rho)
{
  typedef typename Types<FT, V, V, C12>::FourSpinorBlock B;
  typedef typename Types<FT, V, V, C12>::SU3MatrixBlock G;
  typedef typename Types<FT, V, V, C12>::CloverBlock CL;
  typedef typename Types<FT, V, V, C12>::FullCloverBlock FCL;
  const B *p = (const B *)psi, *c = (const B *)chi;
  B *o = (B *)out;
  const G *g = (const G *)gauge + T.gtile;
  const CL *cl = (const CL *)clov + T.gtile;
  const FCL *fcl = (const FCL *)clov + T.gtile;
  const B *xy = p + T.base, *zb = p + T.zb, *zf = p + T.zf, *tb = p + T.tb, *tf = p + T.tf;
  const B *ch = c ? c + T.base : nullptr;
  B *ob = o + T.base;
  const int *xbO = T.xbO, *xfO = T.xfO, *ybO = T.ybO, *yfO = T.yfO, *offs = T.offs, *gO = T.gO;
  const unsigned *acc = T.acc;
#define QTD_PF 0, 0, 0, 0
#define QTD_PFB offs, xy, xy, xy
  switch (fam * 4 + ach * 2 + (plus ? 1 : 0)) {
  case 0: QPhiX::dslash_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, QTD_PFB, acc, cs, ctf, ctb, ph); break;
  case 1: QPhiX::dslash_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, QTD_PFB, acc, cs, ctf, ctb, ph); break;
  case 2: QPhiX::dslash_achimbdpsi_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, xy, alpha, cs, ctf, ctb, ph, acc); break;
  case 3: QPhiX::dslash_achimbdpsi_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, xy, alpha, cs, ctf, ctb, ph, acc); break;
  case 4: QPhiX::clov_dslash_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, cl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, acc, cs, ctf, ctb, ph); break;
  case 5: QPhiX::clov_dslash_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, cl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, acc, cs, ctf, ctb, ph); break;
  case 6: QPhiX::clov_dslash_achimbdpsi_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, cl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, 0, QTD_PFB, xy, cs, ctf, ctb, ph, acc, rho); break;
  case 7: QPhiX::clov_dslash_achimbdpsi_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, cl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, 0, QTD_PFB, xy, cs, ctf, ctb, ph, acc, rho); break;
  case 8: QPhiX::tm_dslash_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, QTD_PFB, acc, cs, ctf, ctb, ph, mu, muinv); break;
  case 9: QPhiX::tm_dslash_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, QTD_PFB, acc, cs, ctf, ctb, ph, mu, muinv); break;
  case 10: QPhiX::tm_dslash_achimbdpsi_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, xy, alpha, cs, ctf, ctb, ph, mu, acc); break;
  case 11: QPhiX::tm_dslash_achimbdpsi_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, xy, alpha, cs, ctf, ctb, ph, mu, acc); break;
  case 12: QPhiX::tm_clov_dslash_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, fcl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, acc, cs, ctf, ctb, ph); break;
  case 13: QPhiX::tm_clov_dslash_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ob, g, fcl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, QTD_PFB, acc, cs, ctf, ctb, ph); break;
  case 14: QPhiX::tm_clov_dslash_achimbdpsi_minus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, fcl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, 0, QTD_PFB, xy, cs, ctf, ctb, ph, acc, rho); break;
  default: QPhiX::tm_clov_dslash_achimbdpsi_plus_vec<FT, V, V, C12, X, Y, Z, W>(xy, zb, zf, tb, tf, ch, ob, g, fcl, xbO, xfO, ybO, yfO, offs, gO, QTD_PF, 0, 0, 0, QTD_PFB, xy, cs, ctf, ctb, ph, acc, rho); break;
  }
#undef QTD_PF
#undef QTD_PFB
}

typedef void (*BodyFn)(int, int, int, const Tile &, const void *, const void *, void *, const void *,
                       const void *, const void *, const Scalars &, int);

template <typename FT, int V, bool C12, bool X, bool Y, bool Z, bool W>
void body_sweep_tile(int fam, int ach, int plus, const Tile &T, const void *psi, const void *chi, void *out,
                     const void *gauge, const void *clov, const void *, const Scalars &s, int edges)
{
  FT ph[4][2];
  for (int m = 0; m < 4; m++) {
    ph[m][0] = cvt<FT>(s.phases ? s.phases[2 * m] : 1.0);
    ph[m][1] = cvt<FT>(s.phases ? s.phases[2 * m + 1] : 0.0);
  }
  // the time-boundary factor goes into coeff_t on the edge tiles, as QPhiX does
  const double tf = (edges & 2) ? s.ctf * ((edges >> 8) ? -1.0 : 1.0) : s.ctf;
  const double tb = (edges & 1) ? s.ctb * ((edges >> 8) ? -1.0 : 1.0) : s.ctb;
  call_body<FT, V, C12, X, Y, Z, W>(fam, ach, plus, T, psi, chi, out, gauge, clov, ph, cvt<FT>(s.cs), cvt<FT>(tf),
                                    cvt<FT>(tb), cvt<FT>(s.alpha), cvt<FT>(s.mu), cvt<FT>(s.muinv),
                                    cvt<FT>(s.rho));
}

template <typename FT, int V, bool C12>
BodyFn body_fn(int tbc)
{
  switch (tbc & 15) {
  case 0: return body_sweep_tile<FT, V, C12, false, false, false, false>;
  case 1: return body_sweep_tile<FT, V, C12, true, false, false, false>;
  case 2: return body_sweep_tile<FT, V, C12, false, true, false, false>;
  case 3: return body_sweep_tile<FT, V, C12, true, true, false, false>;
  case 4: return body_sweep_tile<FT, V, C12, false, false, true, false>;
  case 5: return body_sweep_tile<FT, V, C12, true, false, true, false>;
  case 6: return body_sweep_tile<FT, V, C12, false, true, true, false>;
  case 7: return body_sweep_tile<FT, V, C12, true, true, true, false>;
  case 8: return body_sweep_tile<FT, V, C12, false, false, false, true>;
  case 9: return body_sweep_tile<FT, V, C12, true, false, false, true>;
  case 10: return body_sweep_tile<FT, V, C12, false, true, false, true>;
  case 11: return body_sweep_tile<FT, V, C12, true, true, false, true>;
  case 12: return body_sweep_tile<FT, V, C12, false, false, true, true>;
  case 13: return body_sweep_tile<FT, V, C12, true, false, true, true>;
  case 14: return body_sweep_tile<FT, V, C12, false, true, true, true>;
  default: return body_sweep_tile<FT, V, C12, true, true, true, true>;
  }
}

template <typename FT> BodyFn body_fn_v(int V, bool c12, int tbc)
{
  if (V == 4) return c12 ? body_fn<FT, 4, true>(tbc) : body_fn<FT, 4, false>(tbc);
  if (V == 8) return c12 ? body_fn<FT, 8, true>(tbc) : body_fn<FT, 8, false>(tbc);
  if (V == 16) return c12 ? body_fn<FT, 16, true>(tbc) : body_fn<FT, 16, false>(tbc);
  return nullptr;
}

BodyFn pick(int ftype, int V, bool c12, int tbc)
{
  if (ftype == 0) return body_fn_v<float>(V, c12, tbc);
  if (ftype == 1) return body_fn_v<double>(V, c12, tbc);
  if (ftype == 2) return body_fn_v<unsigned short>(V, c12, tbc);
  return nullptr;
}

// face tiles in (t, z, y, xb) order: is site lane l of the tile on the face
// of `dir` on checkerboard cb?
bool on_face(const Lat &L, int cb, int dir, int xb, int l, int y, int z, int t)
{
  const int x = 2 * (xb * L.S + l) + ((y + z + t + cb) & 1);
  const int c[4] = {x, y, z, t}, n[4] = {L.nx, L.ny, L.nz, L.nt};
  const int mu = dir / 2;
  return c[mu] == ((dir & 1) ? n[mu] - 1 : 0);
}

template <typename FT, int V, bool C12>
void face_tile(int fam, int plus, bool unpack, bool tbc, const Tile &T, unsigned mask, int dir, FT *buf,
               const void *psi_or_out, const void *gauge, const void *clov, FT beta, FT mu, FT muinv,
               const FT ph[4][2])
{
  typedef typename Types<FT, V, V, C12>::FourSpinorBlock B;
  typedef typename Types<FT, V, V, C12>::SU3MatrixBlock G;
  typedef typename Types<FT, V, V, C12>::CloverBlock CL;
  typedef typename Types<FT, V, V, C12>::FullCloverBlock FCL;
  if (!unpack) {
    const B *xy = (const B *)psi_or_out + T.base;
    if (plus) QPhiX::face_proj_dir_plus<FT, V, V, C12>(xy, T.offs, 0, buf, 0, mask, dir);
    else QPhiX::face_proj_dir_minus<FT, V, V, C12>(xy, T.offs, 0, buf, 0, mask, dir);
    return;
  }
  B *ob = (B *)psi_or_out + T.base;
  const G *g = (const G *)gauge + T.gtile;
  const CL *cl = (const CL *)clov + T.gtile;
  const FCL *fcl = (const FCL *)clov + T.gtile;
#define QTD_F(name) \
  (tbc ? name<FT, V, V, C12, true> : name<FT, V, V, C12, false>)
  switch (fam * 2 + (plus ? 1 : 0)) {
  case 0: QTD_F(QPhiX::face_finish_dir_minus)(buf, g, ob, T.gO, T.offs, 0, 0, 0, beta, mask, dir, ph); break;
  case 1: QTD_F(QPhiX::face_finish_dir_plus)(buf, g, ob, T.gO, T.offs, 0, 0, 0, beta, mask, dir, ph); break;
  case 2: QTD_F(QPhiX::face_clov_finish_dir_minus)(buf, g, ob, cl, T.gO, T.offs, 0, 0, 0, 0, beta, mask, dir, ph); break;
  case 3: QTD_F(QPhiX::face_clov_finish_dir_plus)(buf, g, ob, cl, T.gO, T.offs, 0, 0, 0, 0, beta, mask, dir, ph); break;
  case 4: QTD_F(QPhiX::tm_face_finish_dir_minus)(buf, g, ob, T.gO, T.offs, 0, 0, 0, beta, mu, muinv, mask, dir, ph); break;
  case 5: QTD_F(QPhiX::tm_face_finish_dir_plus)(buf, g, ob, T.gO, T.offs, 0, 0, 0, beta, mu, muinv, mask, dir, ph); break;
  case 6: QTD_F(QPhiX::tm_clov_face_finish_dir_minus)(buf, g, ob, fcl, T.gO, T.offs, 0, 0, 0, 0, beta, mask, dir, ph); break;
  default: QTD_F(QPhiX::tm_clov_face_finish_dir_plus)(buf, g, ob, fcl, T.gO, T.offs, 0, 0, 0, 0, beta, mask, dir, ph); break;
  }
#undef QTD_F
}

template <typename FT, int V, bool C12>
int face_sweep(const Lat &L, int fam, int plus, int cb, bool unpack, int tbc, int dir, void *buf,
               const void *field, const void *gauge, const void *clov, double beta, double mu, double muinv,
               const double *phases)
{
  FT ph[4][2];
  for (int m = 0; m < 4; m++) {
    ph[m][0] = cvt<FT>(phases ? phases[2 * m] : 1.0);
    ph[m][1] = cvt<FT>(phases ? phases[2 * m + 1] : 0.0);
  }
  const unsigned all_acc[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  const int nvecs = L.nx / 2 / L.S;
  FT *b = (FT *)buf;
  for (int t = 0; t < L.nt; t++)
    for (int z = 0; z < L.nz; z++)
      for (int y = 0; y < L.ny; y++)
        for (int xb = 0; xb < nvecs; xb++) {
          unsigned mask = 0;
          for (int l = 0; l < V; l++)
            if (on_face(L, cb, dir, xb, l, y, z, t)) mask |= 1u << l;
          if (!mask) continue;
          Tile T;
          make_tile(L, cb, xb, y, z, t, all_acc, T);
          face_tile<FT, V, C12>(fam, plus, unpack, tbc != 0, T, mask, dir, b, field, gauge, clov, cvt<FT>(beta),
                                cvt<FT>(mu), cvt<FT>(muinv), ph);
          // x faces hold the lanes of the mask, the other faces a whole tile
          b += 12 * (dir < 2 ? __builtin_popcount(mask) : V);
        }
  return qb200_qphix_status();
}

template <typename FT>
int face_sweep_v(const Lat &L, int V, bool c12, int fam, int plus, int cb, bool unpack, int tbc, int dir,
                 void *buf, const void *field, const void *gauge, const void *clov, double beta, double mu,
                 double muinv, const double *phases)
{
#define QTD_FS(VV, CC) face_sweep<FT, VV, CC>(L, fam, plus, cb, unpack, tbc, dir, buf, field, gauge, clov, beta, mu, muinv, phases)
  if (V == 4) return c12 ? QTD_FS(4, true) : QTD_FS(4, false);
  if (V == 8) return c12 ? QTD_FS(8, true) : QTD_FS(8, false);
  if (V == 16) return c12 ? QTD_FS(16, true) : QTD_FS(16, false);
#undef QTD_FS
  return -3;
}

} // namespace

extern "C" {

// body kernel over a whole checkerboard, one call per tile; returns the
// library's per-tile status
int qtd_body(int nx, int ny, int nz, int nt, int soalen, int pad_xy, int pad_xyz, double t_boundary,
             int t_edge_lo, int t_edge_hi, int ftype, int compress12, int family, int ach, int isign, int cb,
             int tbc, const void *psi, const void *chi, const void *gauge, const void *clov, void *out,
             double coeff_s, double coeff_t_f, double coeff_t_b, double alpha, double mu, double muinv,
             double rho, const double *tbc_phases, const unsigned *accumulate)
{
  const Lat L = {nx, ny, nz, nt, soalen, pad_xy, pad_xyz, t_boundary, t_edge_lo, t_edge_hi};
  BodyFn fn = pick(ftype, soalen, compress12 != 0, tbc);
  if (!fn) return -3;
  const unsigned all_acc[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  const unsigned *acc = accumulate ? accumulate : all_acc;
  const Scalars s = {coeff_s, coeff_t_f, coeff_t_b, alpha, mu, muinv, rho, tbc_phases, acc};
  const int nvecs = nx / 2 / soalen;
  const int neg = t_boundary < 0 ? 1 : 0;
  for (int t = 0; t < nt; t++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int xb = 0; xb < nvecs; xb++) {
          Tile T;
          make_tile(L, cb, xb, y, z, t, acc, T);
          const int edges = ((t == 0 && t_edge_lo) ? 1 : 0) | ((t == nt - 1 && t_edge_hi) ? 2 : 0) | (neg << 8);
          fn(family, ach, isign > 0, T, psi, chi, out, gauge, clov, nullptr, s, edges);
        }
  return qb200_qphix_status();
}

// face pack (unpack = 0) or finish (unpack = 1) over the face of `dir`; buf
// holds the faces tile by tile: [12][lanes] per tile, lanes = the mask's
// lanes for x, veclen otherwise
int qtd_face(int nx, int ny, int nz, int nt, int soalen, int pad_xy, int pad_xyz, int ftype, int compress12,
             int family, int isign, int cb, int unpack, int tbc, int dir, void *buf, const void *field,
             const void *gauge, const void *clov, double beta, double mu, double muinv, const double *tbc_phases)
{
  const Lat L = {nx, ny, nz, nt, soalen, pad_xy, pad_xyz, 1.0, 0, 0};
  const bool c = compress12 != 0, u = unpack != 0;
  const int p = isign > 0;
  if (ftype == 0)
    return face_sweep_v<float>(L, soalen, c, family, p, cb, u, tbc, dir, buf, field, gauge, clov, beta, mu, muinv, tbc_phases);
  if (ftype == 1)
    return face_sweep_v<double>(L, soalen, c, family, p, cb, u, tbc, dir, buf, field, gauge, clov, beta, mu, muinv, tbc_phases);
  if (ftype == 2)
    return face_sweep_v<unsigned short>(L, soalen, c, family, p, cb, u, tbc, dir, buf, field, gauge, clov, beta, mu, muinv, tbc_phases);
  return -3;
}

// number of distinct b200 specialisations referenced by this driver (each
// body template for every tbc combination, every face template), all of
// which the link resolved against the library
int qtd_symbols(void)
{
  int n = 0;
  for (int ft = 0; ft < 3; ft++)
    for (int V : {4, 8, 16})
      for (int c = 0; c < 2; c++)
        for (int tbc = 0; tbc < 16; tbc++)
          if (pick(ft, V, c != 0, tbc)) n++;
  return n;
}
}
