// ref_driver.cpp -- runs the reference's generated per-tile dslash kernels
// over a whole checkerboard (TEST INFRASTRUCTURE; built into oracle/_ref by
// oracle/ref_build.py; loaded only by tests/ and bench.py's reference arm).
//
// The reference kernels (codegen/jinja/*_decl.h.j2) compute one tile of
// VECLEN sites (VECLEN/SOALEN y rows of SOALEN x sites) per call and leave
// the lattice loop, per-lane neighbour offsets and per-tile boundary
// coefficients to the caller, QPhiX, which is not part of the reference.
// This driver plays that caller for the layout of include/qphix_b200.h:
//   - z/t neighbours: zbBase..tfBase point at the neighbour tile's first row,
//     `offs` holds the element offset of each row (only lanes i = j*SOALEN
//     are read, codegen/data_types.cc:75-85);
//   - y neighbours: ybOffs/yfOffs hold each row's neighbour row offset;
//   - x neighbours: split loads (codegen/data_types.cc:102-120,
//     inst_sp_vec16.cc:609-636): backward reads lane 0 from xbOffs[j*S] and
//     lanes 1..S-1 contiguously from xbOffs[j*S+1]; forward reads lanes
//     0..S-2 from xfOffs[j*S] and lane S-1 from xfOffs[j*S+S-1];
//   - accumulate[d] is a lane mask for x and y (codegen/dslash.cc:285-290)
//     and a flag for z and t;
//   - coeff_t_f / coeff_t_b carry the time-boundary factor on edge tiles.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"
#include "ref_driver.h"

TileFn rd_body[4][2][2][2][16];
TileFn rd_unpack[4][8][2][2][2];
TileFn rd_pack[8][2];

namespace {

struct Geo {
  int nx, ny, nz, nt, nxh, S, V, ngy, nvecs;
  long long Pxy, Pxyz;
};

bool make_geo(const qb200_lattice *l, Geo &g)
{
  if (!l || l->nx <= 0 || l->ny <= 0 || l->nz <= 0 || l->nt <= 0 || l->nx % 2)
    return false;
  if (l->soalen != RD_SOA || l->veclen != RD_VEC) return false;
  g.nx = l->nx; g.ny = l->ny; g.nz = l->nz; g.nt = l->nt;
  g.nxh = l->nx / 2; g.S = RD_SOA; g.V = RD_VEC; g.ngy = RD_VEC / RD_SOA;
  if (g.nxh % g.S || g.ny % g.ngy) return false;
  g.nvecs = g.nxh / g.S;
  g.Pxy = (long long)g.ny * g.nvecs + l->pad_xy;
  g.Pxyz = (long long)g.nz * g.Pxy + l->pad_xyz;
  return true;
}

FT to_ft(double v)
{
#if RD_HALF
  _Float16 h = (_Float16)(float)v;
  unsigned short b;
  std::memcpy(&b, &h, 2);
  return b;
#else
  return (FT)v;
#endif
}

bool tables_ready = false;
void init_tables()
{
  if (tables_ready) return;
  rd_fill_family0();
  rd_fill_family1();
  rd_fill_family2();
  rd_fill_family3();
  rd_fill_faces();
  tables_ready = true;
}

} // namespace

extern "C" {

int rd_info(int *vec, int *soa, int *ft_bytes, int *half)
{
  *vec = RD_VEC;
  *soa = RD_SOA;
  *ft_bytes = (int)sizeof(FT);
  *half = RD_HALF;
  return 0;
}

int rd_max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int rd_dslash(const qb200_lattice *lat, int family, int achimbdpsi, int isign,
              int cb, const void *psi, const void *chi, const void *gauge,
              const void *clov, void *out, const oracle_params *p,
              int nthreads)
{
  Geo g;
  if (!make_geo(lat, g) || family < 0 || family > 3) return QB200_EINVAL;
  if (!psi || !gauge || !out || (achimbdpsi && !chi)) return QB200_ENULL;
  if (family % 2 == 1 && !clov) return QB200_ENULL;
  init_tables();
  const int comp = lat->compress12 ? 1 : 0;
  const int isPlus = isign > 0 ? 1 : 0;
  const int tbc = (int)(p->tbc_mask & 15u);
  TileFn fn = rd_body[family][achimbdpsi ? 1 : 0][isPlus][comp][tbc];
  if (!fn) return QB200_ELAYOUT;

  const FSB *ps = (const FSB *)psi;
  const FSB *ch = (const FSB *)chi;
  FSB *o = (FSB *)out;
  const long long gtile = 8LL * (comp ? 2 : 3) * 6 * g.V * (long long)sizeof(FT);
  const long long ctile = (family == 1 ? 72LL : 144LL) * g.V * (long long)sizeof(FT);
  const int nyg = g.ny / g.ngy;
  const long long ntiles = (long long)g.nt * g.nz * nyg * g.nvecs;
  const long long blk_elems = 24LL * g.S;

  FT tbcph[4][2];
  for (int m = 0; m < 4; m++)
    for (int r = 0; r < 2; r++) tbcph[m][r] = to_ft(p->tbc_phases[m][r]);
  const FT c_s = to_ft(p->coeff_s);
  const FT c_tf = to_ft(p->coeff_t_f), c_tb = to_ft(p->coeff_t_b);
  const FT c_tf_edge = to_ft(p->coeff_t_f * lat->t_boundary);
  const FT c_tb_edge = to_ft(p->coeff_t_b * lat->t_boundary);
  const FT alpha = to_ft(p->alpha), mu = to_ft(p->mu), muinv = to_ft(p->muinv);
  const FT rho = to_ft(p->rho);
  const unsigned all_lanes = (g.V >= 32) ? 0xffffffffu : ((1u << g.V) - 1u);

#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (long long tile = 0; tile < ntiles; tile++) {
    int xb = (int)(tile % g.nvecs);
    long long r = tile / g.nvecs;
    int yg = (int)(r % nyg);
    r /= nyg;
    int z = (int)(r % g.nz);
    int t = (int)(r / g.nz);
    int y0 = yg * g.ngy;
    auto blk = [&](int xb_, int y_, int z_, int t_) -> long long {
      return t_ * g.Pxyz + z_ * g.Pxy + (long long)y_ * g.nvecs + xb_;
    };
    const long long base = blk(xb, y0, z, t);
    int offs[RD_VEC], xbO[RD_VEC], xfO[RD_VEC], ybO[RD_VEC], yfO[RD_VEC], gO[RD_VEC];
    unsigned acc[8];
    unsigned xb_mask = 0, xf_mask = 0;
    for (int j = 0; j < g.ngy; j++) {
      int y = y0 + j;
      long long row = (blk(xb, y, z, t) - base) * blk_elems;
      long long ym = (blk(xb, (y + g.ny - 1) % g.ny, z, t) - base) * blk_elems;
      long long yp = (blk(xb, (y + 1) % g.ny, z, t) - base) * blk_elems;
      int par = (y + z + t + cb) & 1; // x = 2*xcb + par
      int xbm = (xb + g.nvecs - 1) % g.nvecs, xbp = (xb + 1) % g.nvecs;
      long long to_m = (long long)(xbm - xb) * blk_elems;
      long long to_p = (long long)(xbp - xb) * blk_elems;
      for (int l = 0; l < g.S; l++) {
        int i = j * g.S + l;
        offs[i] = (int)row;
        ybO[i] = (int)ym;
        yfO[i] = (int)yp;
        xbO[i] = (int)row;
        xfO[i] = (int)row;
        gO[i] = 0;
        int x = 2 * (xb * g.S + l) + par;
        if (lat->nx > 0) {
          if (p->accumulate[0] || x != 0) xb_mask |= 1u << i;
          if (p->accumulate[1] || x != g.nx - 1) xf_mask |= 1u << i;
        }
      }
      int i0 = j * g.S;
      if (g.S == 1) {
        xbO[i0] = (int)(par == 0 ? row + to_m : row);
        xfO[i0] = (int)(par == 1 ? row + to_p : row);
      } else {
        if (par == 1) {
          xbO[i0] = (int)row;
          xbO[i0 + 1] = (int)(row + 1);
        } else {
          xbO[i0] = (int)(row + to_m + g.S - 1);
          xbO[i0 + 1] = (int)row;
        }
        if (par == 0) {
          xfO[i0] = (int)row;
          xfO[i0 + g.S - 1] = (int)(row + g.S - 1);
        } else {
          xfO[i0] = (int)(row + 1);
          xfO[i0 + g.S - 1] = (int)(row + to_p);
        }
      }
    }
    // y masks: rows at the local y edge drop the crossing hop
    unsigned yb_mask = 0, yf_mask = 0;
    for (int j = 0; j < g.ngy; j++) {
      int y = y0 + j;
      unsigned rowbits = ((g.S >= 32) ? 0xffffffffu : ((1u << g.S) - 1u)) << (j * g.S);
      if (p->accumulate[2] || y != 0) yb_mask |= rowbits;
      if (p->accumulate[3] || y != g.ny - 1) yf_mask |= rowbits;
    }
    acc[0] = xb_mask & all_lanes;
    acc[1] = xf_mask & all_lanes;
    acc[2] = yb_mask & all_lanes;
    acc[3] = yf_mask & all_lanes;
    acc[4] = (p->accumulate[4] || z != 0) ? all_lanes : 0u;
    acc[5] = (p->accumulate[5] || z != g.nz - 1) ? all_lanes : 0u;
    acc[6] = (p->accumulate[6] || t != 0) ? all_lanes : 0u;
    acc[7] = (p->accumulate[7] || t != g.nt - 1) ? all_lanes : 0u;

    TileArgs A;
    std::memset(&A, 0, sizeof(A));
    int zm = (z + g.nz - 1) % g.nz, zp = (z + 1) % g.nz;
    int tm = (t + g.nt - 1) % g.nt, tp = (t + 1) % g.nt;
    A.xyBase = ps + base;
    A.zbBase = ps + blk(xb, y0, zm, t);
    A.zfBase = ps + blk(xb, y0, zp, t);
    A.tbBase = ps + blk(xb, y0, z, tm);
    A.tfBase = ps + blk(xb, y0, z, tp);
    A.chiBase = ch ? ch + base : nullptr;
    A.oBase = o + base;
    A.gBase = (const char *)gauge + tile * gtile;
    A.clBase = clov ? (const void *)((const char *)clov + tile * ctile) : nullptr;
    A.xbOffs = xbO; A.xfOffs = xfO; A.ybOffs = ybO; A.yfOffs = yfO;
    A.offs = offs; A.gOffs = gO;
    A.accumulate = acc;
    A.coeff_s = c_s;
    A.coeff_t_f = (t == g.nt - 1 && lat->t_edge_hi) ? c_tf_edge : c_tf;
    A.coeff_t_b = (t == 0 && lat->t_edge_lo) ? c_tb_edge : c_tb;
    A.alpha = alpha; A.mu = mu; A.muinv = muinv; A.prec_mass_rho = rho;
    std::memcpy(A.tbc_phases, tbcph, sizeof(tbcph));
    fn(A);
  }
  return QB200_OK;
}

// Face kernels are driven one site per call, so only the VECLEN = 1
// (scalar ISA) build supports them.
static long long face_list(const Geo &g, int cb, int mu, int coord,
                           std::vector<int> &fs)
{
  fs.clear();
  for (int t = 0; t < g.nt; t++)
    for (int z = 0; z < g.nz; z++)
      for (int y = 0; y < g.ny; y++)
        for (int xcb = 0; xcb < g.nxh; xcb++) {
          int x = 2 * xcb + ((y + z + t + cb) & 1);
          int c[4] = {x, y, z, t};
          if (c[mu] != coord) continue;
          fs.push_back(xcb); fs.push_back(y); fs.push_back(z); fs.push_back(t);
        }
  return (long long)fs.size() / 4;
}

int rd_face_pack(const qb200_lattice *lat, int isign, int psi_cb,
                 const void *psi, void *outbuf, int dir)
{
  Geo g;
  if (!make_geo(lat, g) || g.V != 1) return QB200_EINVAL;
  if (dir < 0 || dir > 7) return QB200_EDIR;
  init_tables();
  TileFn fn = rd_pack[dir][isign > 0 ? 1 : 0];
  if (!fn) return QB200_ELAYOUT;
  int L[4] = {g.nx, g.ny, g.nz, g.nt};
  int mu = dir / 2;
  std::vector<int> fs;
  long long n = face_list(g, psi_cb, mu, (dir & 1) ? L[mu] - 1 : 0, fs);
  int offs[1] = {0};
  for (long long i = 0; i < n; i++) {
    int xcb = fs[4 * i], y = fs[4 * i + 1], z = fs[4 * i + 2], t = fs[4 * i + 3];
    TileArgs A;
    std::memset(&A, 0, sizeof(A));
    A.xyBase = (const FSB *)psi + (t * g.Pxyz + z * g.Pxy + (long long)y * g.nvecs + xcb);
    A.offs = offs;
    A.outbuf = (FT *)outbuf + 12 * i;
    A.mask = 1u;
    A.dir = dir;
    fn(A);
  }
  return QB200_OK;
}

int rd_face_unpack(const qb200_lattice *lat, int family, int isign, int cb,
                   const void *inbuf, const void *gauge, void *out,
                   const void *clov, double beta, double mu, double muinv,
                   int dir, int tbc, const double *tbc_phases)
{
  Geo g;
  if (!make_geo(lat, g) || g.V != 1 || family < 0 || family > 3) return QB200_EINVAL;
  if (dir < 0 || dir > 7) return QB200_EDIR;
  init_tables();
  const int comp = lat->compress12 ? 1 : 0;
  TileFn fn = rd_unpack[family][dir][isign > 0 ? 1 : 0][comp][tbc ? 1 : 0];
  if (!fn) return QB200_ELAYOUT;
  int L[4] = {g.nx, g.ny, g.nz, g.nt};
  int dim = dir / 2;
  std::vector<int> fs;
  long long n = face_list(g, cb, dim, (dir & 1) ? L[dim] - 1 : 0, fs);
  const long long gtile = 8LL * (comp ? 2 : 3) * 6 * (long long)sizeof(FT);
  const long long ctile = (family == 1 ? 72LL : 144LL) * (long long)sizeof(FT);
  int offs[1] = {0}, gO[1] = {0};
  for (long long i = 0; i < n; i++) {
    int xcb = fs[4 * i], y = fs[4 * i + 1], z = fs[4 * i + 2], t = fs[4 * i + 3];
    long long tile = ((long long)t * g.nz + z) * g.ny * g.nvecs + (long long)y * g.nvecs + xcb;
    TileArgs A;
    std::memset(&A, 0, sizeof(A));
    A.inbuf = (const FT *)inbuf + 12 * i;
    A.gBase = (const char *)gauge + tile * gtile;
    A.oBase = (FSB *)out + (t * g.Pxyz + z * g.Pxy + (long long)y * g.nvecs + xcb);
    A.clBase = clov ? (const void *)((const char *)clov + tile * ctile) : nullptr;
    A.offs = offs;
    A.gOffs = gO;
    A.beta = to_ft(beta);
    A.mu = to_ft(mu);
    A.muinv = to_ft(muinv);
    A.mask = 1u;
    A.dir = dir;
    if (tbc_phases)
      for (int m = 0; m < 4; m++)
        for (int r = 0; r < 2; r++) A.tbc_phases[m][r] = to_ft(tbc_phases[2 * m + r]);
    fn(A);
  }
  return QB200_OK;
}

} // extern "C"
