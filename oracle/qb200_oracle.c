/*
 * qb200_oracle.c -- CPU oracle for the dslash family (TEST INFRASTRUCTURE).
 *
 * This file is the checker, never the product: only tests/, the smoke check
 * in __graft_entry__.py and the cpu_baseline leg of bench.py load it.  It is
 * a plain-C restatement, in FP64 arithmetic, of the per-site operators that
 * JeffersonLab/qphix-codegen generates, applied to whole checkerboards in
 * the QPhiX tile layouts that include/qphix_b200.h describes.  It reads
 * and writes the storage type (float, double or IEEE binary16) of the field.
 *
 * Parity pin: tests/test_oracle_ref.py compares it with the reference's own
 * generated scalar (and AVX512) kernels, built from the reference sources by
 * oracle/ref_build.py, and tests/test_oracle_golden.py with the fixtures in
 * tests/golden/ that those kernels produced.
 *
 * Formulas followed (paths inside the reference project):
 *   projectors             codegen/dslash_common.cc:748-766 (proj_ops_plus/minus)
 *   reconstruction         codegen/dslash_common.cc:784-890 (rec_*_{p,m}beta_ops)
 *                          and :631-706 (add/sub/addi/subi _pbeta/_mbeta)
 *   project / recons_add   codegen/dslash_common.cc:958-1021, :1058-1089
 *   SU(3) x half spinor    codegen/dslash_common.cc:1678-1727 (matMultVec)
 *   12-real reconstruction codegen/dslash_common.cc:1657-1676, :701-718
 *   clover block           codegen/dslash_common.cc:1098-1186 (clover_term)
 *   full clover block      codegen/dslash_common.cc:1188-1232
 *   A^-1 twisted mass      codegen/dslash_common.cc:1234-1359
 *   A twisted mass         codegen/dslash_common.cc:1364-1489
 *   twisted BC phases      codegen/dslash_common.cc:1491-1524
 *   plain body             codegen/dslash_common.cc:1729-1826
 *   achimbdpsi body        codegen/dslash_common.cc:1830-1932 (rho term :1873-1906)
 *   face pack              codegen/dslash.cc:433-458
 *   face unpack            codegen/dslash.cc:463-553, dslash_common.cc:1934-1993
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

typedef double _Complex cplx;

enum {
  FAM_WILSON = ORACLE_WILSON,
  FAM_CLOVER = ORACLE_CLOVER,
  FAM_TM = ORACLE_TM,
  FAM_TMCLOV = ORACLE_TMCLOV
};

/* ------------------------------------------------------------------ */
/* geometry                                                            */

typedef struct geo {
  int nx, ny, nz, nt, nxh, S, V, ngy, nvecs;
  long long Pxy, Pxyz;
  int ft, comp12;
} geo;

static int make_geo(const qb200_lattice *l, geo *g)
{
  if (l->nx <= 0 || l->ny <= 0 || l->nz <= 0 || l->nt <= 0) return -1;
  if (l->nx % 2) return -1;
  if (l->soalen <= 0 || l->veclen <= 0 || l->veclen % l->soalen) return -1;
  g->nx = l->nx; g->ny = l->ny; g->nz = l->nz; g->nt = l->nt;
  g->nxh = l->nx / 2;
  g->S = l->soalen; g->V = l->veclen; g->ngy = l->veclen / l->soalen;
  if (g->nxh % g->S || g->ny % g->ngy) return -1;
  g->nvecs = g->nxh / g->S;
  g->Pxy = (long long)g->ny * g->nvecs + l->pad_xy;
  g->Pxyz = (long long)g->nz * g->Pxy + l->pad_xyz;
  g->ft = l->ftype; g->comp12 = l->compress12 ? 1 : 0;
  return 0;
}

/* elements per lane of a spinor block: 24, or 26 for F16N (24 halves plus
 * the FP32 norm in two halves) */
static int spb(const geo *g) { return g->ft == QB200_F16N ? 26 : 24; }

/* index of component (c, s, ri) of site (xcb,y,z,t) in a spinor field */
static long long sp_idx(const geo *g, int xcb, int y, int z, int t, int c,
                        int s, int ri)
{
  long long blk = t * g->Pxyz + z * g->Pxy + (long long)y * g->nvecs + xcb / g->S;
  return blk * spb(g) * g->S + ((c * 4 + s) * 2 + ri) * g->S + xcb % g->S;
}

/* the FP32 norm of an F16N site */
static float *sp_norm(const geo *g, const void *f, int xcb, int y, int z, int t)
{
  long long blk = t * g->Pxyz + z * g->Pxy + (long long)y * g->nvecs + xcb / g->S;
  return (float *)((const _Float16 *)f + blk * 26 * g->S + 24 * g->S) + xcb % g->S;
}

static long long tile_of(const geo *g, int xcb, int y, int z, int t)
{
  return (((long long)t * g->nz + z) * (g->ny / g->ngy) + y / g->ngy) * g->nvecs +
         xcb / g->S;
}

static int lane_of(const geo *g, int xcb, int y)
{
  return (y % g->ngy) * g->S + xcb % g->S;
}

/* ------------------------------------------------------------------ */
/* storage access                                                      */

/* bfloat16: the upper 16 bits of an IEEE binary32, rounded to nearest even */
static double bf16_to_d(uint16_t b)
{
  uint32_t u = (uint32_t)b << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

static uint16_t d_to_bf16(double v)
{
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

static double ld(const void *p, int ft, long long i)
{
  switch (ft) {
  case QB200_F32: return ((const float *)p)[i];
  case QB200_F64: return ((const double *)p)[i];
  case QB200_BF16: return bf16_to_d(((const uint16_t *)p)[i]);
  default: return (double)((const _Float16 *)p)[i]; /* F16 and the halves of F16N */
  }
}

static void st(void *p, int ft, long long i, double v)
{
  switch (ft) {
  case QB200_F32: ((float *)p)[i] = (float)v; break;
  case QB200_F64: ((double *)p)[i] = v; break;
  case QB200_BF16: ((uint16_t *)p)[i] = d_to_bf16(v); break;
  default: ((_Float16 *)p)[i] = (_Float16)(float)v; break;
  }
}

static void load_spinor(const geo *g, const void *f, int xcb, int y, int z,
                        int t, cplx sp[4][3])
{
  double nrm = g->ft == QB200_F16N ? *sp_norm(g, f, xcb, y, z, t) : 1.0;
  for (int c = 0; c < 3; c++)
    for (int s = 0; s < 4; s++)
      sp[s][c] = nrm * (ld(f, g->ft, sp_idx(g, xcb, y, z, t, c, s, 0)) +
                        I * ld(f, g->ft, sp_idx(g, xcb, y, z, t, c, s, 1)));
}

static void store_spinor(const geo *g, void *f, int xcb, int y, int z, int t,
                         cplx sp[4][3])
{
  double scale = 1.0;
  if (g->ft == QB200_F16N) {
    double m = 0.0;
    for (int c = 0; c < 3; c++)
      for (int s = 0; s < 4; s++) {
        m = fmax(m, fabs(creal(sp[s][c])));
        m = fmax(m, fabs(cimag(sp[s][c])));
      }
    float nrm = m > 0.0 ? (float)m : 1.0f;
    *sp_norm(g, f, xcb, y, z, t) = nrm;
    scale = 1.0 / nrm;
  }
  for (int c = 0; c < 3; c++)
    for (int s = 0; s < 4; s++) {
      st(f, g->ft, sp_idx(g, xcb, y, z, t, c, s, 0), scale * creal(sp[s][c]));
      st(f, g->ft, sp_idx(g, xcb, y, z, t, c, s, 1), scale * cimag(sp[s][c]));
    }
}

/* one face record: 12 values (F16N: scaled by a norm stored after them) */
static int face_elems(const geo *g) { return g->ft == QB200_F16N ? 14 : 12; }

static void store_face(const geo *g, void *buf, long long i, cplx b[2][3])
{
  long long o = i * face_elems(g);
  double scale = 1.0;
  if (g->ft == QB200_F16N) {
    double m = 0.0;
    for (int s = 0; s < 2; s++)
      for (int c = 0; c < 3; c++) m = fmax(m, fmax(fabs(creal(b[s][c])), fabs(cimag(b[s][c]))));
    float nrm = m > 0.0 ? (float)m : 1.0f;
    *(float *)((_Float16 *)buf + o + 12) = nrm;
    scale = 1.0 / nrm;
  }
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 3; c++) {
      st(buf, g->ft, o + (s * 3 + c) * 2 + 0, scale * creal(b[s][c]));
      st(buf, g->ft, o + (s * 3 + c) * 2 + 1, scale * cimag(b[s][c]));
    }
}

static void load_face(const geo *g, const void *buf, long long i, cplx b[2][3])
{
  long long o = i * face_elems(g);
  double nrm = g->ft == QB200_F16N ? *(const float *)((const _Float16 *)buf + o + 12) : 1.0;
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 3; c++)
      b[s][c] = nrm * (ld(buf, g->ft, o + (s * 3 + c) * 2) + I * ld(buf, g->ft, o + (s * 3 + c) * 2 + 1));
}

/* stored link G (= U^T) of direction d at an output site */
static void load_link(const geo *g, const void *u, int xcb, int y, int z,
                      int t, int d, cplx G[3][3])
{
  int rows = g->comp12 ? 2 : 3;
  long long base = tile_of(g, xcb, y, z, t) * (8LL * rows * 6 * g->V);
  int lane = lane_of(g, xcb, y);
  for (int r = 0; r < rows; r++)
    for (int c = 0; c < 3; c++) {
      long long e = base + ((((long long)d * rows + r) * 3 + c) * 2) * g->V + lane;
      G[r][c] = ld(u, g->ft, e) + I * ld(u, g->ft, e + g->V);
    }
  if (g->comp12)
    for (int c = 0; c < 3; c++) {
      int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      G[2][c] = conj(G[0][c1] * G[1][c2] - G[0][c2] * G[1][c1]);
    }
}

/* Hermitian clover block b (0: spins 0,1; 1: spins 2,3) as a dense 6x6 */
static void load_clover(const geo *g, const void *cl, int xcb, int y, int z,
                        int t, int b, cplx A[6][6])
{
  long long base = tile_of(g, xcb, y, z, t) * (72LL * g->V);
  int lane = lane_of(g, xcb, y);
  long long blk = base + (long long)b * 36 * g->V; /* diag(6) + off(30) */
  double dg[6];
  cplx od[15];
  for (int i = 0; i < 6; i++) dg[i] = ld(cl, g->ft, blk + (long long)i * g->V + lane);
  for (int i = 0; i < 15; i++)
    od[i] = ld(cl, g->ft, blk + (6LL + 2 * i) * g->V + lane) +
            I * ld(cl, g->ft, blk + (6LL + 2 * i + 1) * g->V + lane);
  for (int r = 0; r < 6; r++)
    for (int c = 0; c < 6; c++) {
      if (r == c) A[r][c] = dg[r];
      else if (r > c) A[r][c] = od[r * (r - 1) / 2 + c];
      else A[r][c] = conj(od[c * (c - 1) / 2 + r]);
    }
}

static void load_full_clover(const geo *g, const void *cl, int xcb, int y,
                             int z, int t, int b, cplx F[6][6])
{
  long long base = tile_of(g, xcb, y, z, t) * (144LL * g->V);
  int lane = lane_of(g, xcb, y);
  long long blk = base + (long long)b * 72 * g->V;
  for (int r = 0; r < 6; r++)
    for (int c = 0; c < 6; c++) {
      long long e = blk + ((long long)(r * 6 + c) * 2) * g->V + lane;
      F[r][c] = ld(cl, g->ft, e) + I * ld(cl, g->ft, e + g->V);
    }
}

/* ------------------------------------------------------------------ */
/* spin algebra tables                                                  */

/* one complex op: 0 add (a+b), 1 sub (a-b), 2 addi (a+ib), 3 subi (a-ib) */
static cplx op_apply(int op, cplx a, cplx b)
{
  switch (op) {
  case 0: return a + b;
  case 1: return a - b;
  case 2: return a + I * b;
  default: return a - I * b;
  }
}

/* proj_ops_plus (dslash_common.cc:748-756): spin pairs and ops per index */
static const int proj_spin[8][2][2] = {
    {{0, 3}, {1, 2}}, {{0, 3}, {1, 2}}, {{0, 3}, {1, 2}}, {{0, 3}, {1, 2}},
    {{0, 2}, {1, 3}}, {{0, 2}, {1, 3}}, {{0, 2}, {1, 3}}, {{0, 2}, {1, 3}}};
static const int proj_op[8][2] = {{2, 2}, {3, 3}, {1, 0}, {0, 1},
                                  {2, 3}, {3, 2}, {0, 0}, {1, 1}};

/* rec_plus_*beta / rec_minus_*beta (dslash_common.cc:784-890): per dim the
 * half-spinor row s2 that feeds spin 2 (the other row feeds spin 3) and the
 * ops F1 (spin 2) and F2 (spin 3); the top two spins always use "add". */
static const int rec_s2[4] = {1, 1, 0, 0};
static const int rec_plus_op[4][2] = {{3, 3}, {0, 1}, {3, 2}, {0, 0}};
static const int rec_minus_op[4][2] = {{2, 2}, {1, 0}, {2, 3}, {1, 1}};

/* b = projection of psi with proj_ops_plus[p] */
static void project(int p, cplx psi[4][3], cplx b[2][3])
{
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 3; c++)
      b[s][c] = op_apply(proj_op[p][s], psi[proj_spin[p][s][0]][c],
                         psi[proj_spin[p][s][1]][c]);
}

/* ub = G^T b (forward) or G^* b (backward, adj) */
static void mult_link(cplx G[3][3], int adj, cplx b[2][3], cplx ub[2][3])
{
  for (int s = 0; s < 2; s++)
    for (int c1 = 0; c1 < 3; c1++) {
      cplx acc = 0;
      for (int k = 0; k < 3; k++)
        acc += adj ? conj(G[c1][k]) * b[s][k] : G[k][c1] * b[s][k];
      ub[s][c1] = acc;
    }
}

/* out += beta-scaled reconstruction of ub (recons_add with *_pbeta ops;
 * *_mbeta is the same with beta -> -beta) */
static void recons(int dim, int plus_table, double beta, cplx ub[2][3],
                   cplx out[4][3])
{
  const int *ops = plus_table ? rec_plus_op[dim] : rec_minus_op[dim];
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 3; c++) {
      out[s][c] += beta * ub[s][c];
      if (rec_s2[dim] == s)
        out[2][c] = op_apply(ops[0], out[2][c], beta * ub[s][c]);
      else
        out[3][c] = op_apply(ops[1], out[3][c], beta * ub[s][c]);
    }
}

static void apply_tbc(int fwd, const double ph[2], cplx ub[2][3])
{
  cplx p = ph[0] + I * ph[1];
  if (!fwd) p = conj(p);
  for (int s = 0; s < 2; s++)
    for (int c = 0; c < 3; c++) ub[s][c] *= p;
}

static void clover_mult(cplx A[6][6], int b, cplx in[4][3], cplx res[4][3],
                        int accumulate)
{
  for (int r = 0; r < 6; r++) {
    cplx acc = 0;
    for (int c = 0; c < 6; c++) acc += A[r][c] * in[2 * b + c / 3][c % 3];
    if (accumulate) res[2 * b + r / 3][r % 3] += acc;
    else res[2 * b + r / 3][r % 3] = acc;
  }
}

/* out (+)= muinv (1 -/+ i mu g5) in : inverse_twisted_term */
static void inv_twisted(int isPlus, double mu, double muinv, cplx in[4][3],
                        cplx out[4][3], int accumulate)
{
  for (int s = 0; s < 4; s++) {
    int upper = s < 2;
    double sg = (upper == isPlus) ? -1.0 : 1.0; /* (1 + sg*i*mu) */
    for (int c = 0; c < 3; c++) {
      cplx v = muinv * (1.0 + sg * I * mu) * in[s][c];
      if (accumulate) out[s][c] += v;
      else out[s][c] = v;
    }
  }
}

/* ------------------------------------------------------------------ */
/* neighbour coordinates                                                */

/* neighbour of output site (xcb,y,z,t) on cb in direction d; returns 1 if
 * the hop leaves the local sub-lattice (crosses a local boundary) */
static int neighbour(const geo *g, int cb, int d, int xcb, int y, int z,
                     int t, int *nx_, int *ny_, int *nz_, int *nt_)
{
  int mu = d / 2, fwd = d & 1;
  int par = (y + z + t + cb) & 1; /* x = 2*xcb + par */
  int x = 2 * xcb + par;
  int n[4] = {x, y, z, t};
  int L[4] = {g->nx, g->ny, g->nz, g->nt};
  int cross = fwd ? (n[mu] == L[mu] - 1) : (n[mu] == 0);
  n[mu] = (n[mu] + (fwd ? 1 : L[mu] - 1)) % L[mu];
  *nx_ = n[0] / 2;
  *ny_ = n[1]; *nz_ = n[2]; *nt_ = n[3];
  return cross;
}

/* ------------------------------------------------------------------ */
/* body kernels                                                         */

/* The body kernels with the result stored in storage type out_ft (same
 * lattice and tile layout as the inputs): out_ft = QB200_F64 keeps the FP64
 * result unrounded, the reference against which 16-bit storage is judged. */
int oracle_dslash_out(const qb200_lattice *lat, int out_ft, int family,
                      int achimbdpsi, int isign, int cb, const void *psi,
                      const void *chi, const void *gauge, const void *clov,
                      void *out, const oracle_params *p)
{
  geo g, go;
  if (make_geo(lat, &g)) return QB200_EINVAL;
  if (out_ft < QB200_F32 || out_ft > QB200_BF16) return QB200_EINVAL;
  go = g;
  go.ft = out_ft;
  if (!psi || !gauge || !out) return QB200_ENULL;
  if (achimbdpsi && !chi) return QB200_ENULL;
  if ((family == FAM_CLOVER || family == FAM_TMCLOV) && !clov) return QB200_ENULL;
  int isPlus = isign > 0;
  int clover = family == FAM_CLOVER || family == FAM_TMCLOV;
  int tm = family == FAM_TM || family == FAM_TMCLOV;
  long long nsites = (long long)g.nxh * g.ny * g.nz * g.nt;

#pragma omp parallel for schedule(static)
  for (long long i = 0; i < nsites; i++) {
    int xcb = (int)(i % g.nxh);
    long long r = i / g.nxh;
    int y = (int)(r % g.ny); r /= g.ny;
    int z = (int)(r % g.nz);
    int t = (int)(r / g.nz);

    cplx res[4][3], hop[4][3], ch[4][3];
    memset(hop, 0, sizeof(hop));
    memset(res, 0, sizeof(res));

    /* hopping term with +beta (plain) or -beta (achimbdpsi) */
    for (int d = 0; d < 8; d++) {
      int mu = d / 2, fwd = d & 1;
      int ax, ay, az, at;
      int cross = neighbour(&g, cb, d, xcb, y, z, t, &ax, &ay, &az, &at);
      if (!p->accumulate[d] && cross) continue;
      double beta = mu < 3 ? p->coeff_s : (fwd ? p->coeff_t_f : p->coeff_t_b);
      if (mu == 3 && fwd && t == g.nt - 1 && lat->t_edge_hi) beta *= lat->t_boundary;
      if (mu == 3 && !fwd && t == 0 && lat->t_edge_lo) beta *= lat->t_boundary;
      if (achimbdpsi) beta = -beta;

      cplx nb[4][3], b[2][3], ub[2][3], G[3][3];
      load_spinor(&g, psi, ax, ay, az, at, nb);
      project(isPlus ? d : (d ^ 1), nb, b);
      load_link(&g, gauge, xcb, y, z, t, d, G);
      mult_link(G, !fwd, b, ub);
      if (p->tbc_mask & (1u << mu)) apply_tbc(fwd, p->tbc_phases[mu], ub);
      /* plus: backward hops use rec_plus, forward rec_minus; minus swaps */
      recons(mu, isPlus ? !fwd : fwd, beta, ub, hop);
    }

    if (achimbdpsi) {
      load_spinor(&g, chi, xcb, y, z, t, ch);
      if (family == FAM_WILSON) {
        for (int s = 0; s < 4; s++)
          for (int c = 0; c < 3; c++) res[s][c] = p->alpha * ch[s][c];
      } else if (family == FAM_TM) {
        /* twisted_term: alpha (1 +/- i mu g5) chi, upper sign + for plus */
        for (int s = 0; s < 4; s++) {
          double sg = ((s < 2) == isPlus) ? 1.0 : -1.0;
          for (int c = 0; c < 3; c++)
            res[s][c] = p->alpha * (1.0 + sg * I * p->mu) * ch[s][c];
        }
      } else {
        for (int b = 0; b < 2; b++) {
          cplx A[6][6];
          if (family == FAM_CLOVER) load_clover(&g, clov, xcb, y, z, t, b, A);
          else load_full_clover(&g, clov, xcb, y, z, t, b, A);
          clover_mult(A, b, ch, res, 0);
        }
        /* + i rho g5 chi for plus, - for minus */
        for (int s = 0; s < 4; s++) {
          double sg = (isPlus ^ (s >= 2)) ? 1.0 : -1.0;
          for (int c = 0; c < 3; c++) res[s][c] += sg * I * p->rho * ch[s][c];
        }
      }
      for (int s = 0; s < 4; s++)
        for (int c = 0; c < 3; c++) res[s][c] += hop[s][c];
    } else {
      if (clover) {
        for (int b = 0; b < 2; b++) {
          cplx A[6][6];
          if (family == FAM_CLOVER) load_clover(&g, clov, xcb, y, z, t, b, A);
          else load_full_clover(&g, clov, xcb, y, z, t, b, A);
          clover_mult(A, b, hop, res, 0);
        }
      } else if (tm) {
        inv_twisted(isPlus, p->mu, p->muinv, hop, res, 0);
      } else {
        memcpy(res, hop, sizeof(res));
      }
    }
    store_spinor(&go, out, xcb, y, z, t, res);
  }
  return QB200_OK;
}

int oracle_dslash(const qb200_lattice *lat, int family, int achimbdpsi,
                  int isign, int cb, const void *psi, const void *chi,
                  const void *gauge, const void *clov, void *out,
                  const oracle_params *p)
{
  return oracle_dslash_out(lat, lat->ftype, family, achimbdpsi, isign, cb, psi,
                           chi, gauge, clov, out, p);
}

/* ------------------------------------------------------------------ */
/* link derivative of the hopping term (no counterpart in the reference)  */

/* Re <chi, beta recons(tbc(mult_link(G, b)))> of one hop, for a given G:
 * the same steps as the hop loop of oracle_dslash (dslash_common.cc:
 * 1729-1826).  The derivative with respect to the link is taken below by
 * linearity: the hop is linear in G (forward) or in conj(G) (backward), so
 * evaluating it on the unit matrices gives dL/dRe G and dL/dIm G exactly. */
static double hop_value(int d, int isPlus, double beta, const oracle_params *p,
                        cplx G[3][3], cplx b[2][3], cplx ch[4][3])
{
  int mu = d / 2, fwd = d & 1;
  cplx ub[2][3], hop[4][3];
  memset(hop, 0, sizeof(hop));
  mult_link(G, !fwd, b, ub);
  if (p->tbc_mask & (1u << mu)) apply_tbc(fwd, p->tbc_phases[mu], ub);
  recons(mu, isPlus ? !fwd : fwd, beta, ub, hop);
  double v = 0;
  for (int s = 0; s < 4; s++)
    for (int c = 0; c < 3; c++) v += creal(conj(ch[s][c]) * hop[s][c]);
  return v;
}

/* force[((d*3+r)*3+c)*2+ri][i] = dL/dU (gauge == NULL) or TA(dL/dU U^dag)
 * for L = Re <chi, H psi>, H the plain Wilson hopping term on cb; see
 * qb200_hop_force in include/qphix_b200.h.  FP64 output. */
int oracle_hop_force(const qb200_lattice *lat, int isign, int cb, const void *chi,
                     const void *psi, const void *gauge, const oracle_params *p,
                     double *force)
{
  geo g;
  if (make_geo(lat, &g)) return QB200_EINVAL;
  if (!chi || !psi || !force) return QB200_ENULL;
  int isPlus = isign > 0;
  long long nsites = (long long)g.nxh * g.ny * g.nz * g.nt;

#pragma omp parallel for schedule(static)
  for (long long i = 0; i < nsites; i++) {
    int xcb = (int)(i % g.nxh);
    long long r = i / g.nxh;
    int y = (int)(r % g.ny); r /= g.ny;
    int z = (int)(r % g.nz);
    int t = (int)(r / g.nz);
    cplx ch[4][3];
    load_spinor(&g, chi, xcb, y, z, t, ch);
    for (int d = 0; d < 8; d++) {
      int mu = d / 2, fwd = d & 1;
      int ax, ay, az, at;
      neighbour(&g, cb, d, xcb, y, z, t, &ax, &ay, &az, &at);
      double beta = mu < 3 ? p->coeff_s : (fwd ? p->coeff_t_f : p->coeff_t_b);
      if (mu == 3 && fwd && t == g.nt - 1 && lat->t_edge_hi) beta *= lat->t_boundary;
      if (mu == 3 && !fwd && t == 0 && lat->t_edge_lo) beta *= lat->t_boundary;
      cplx nb[4][3], b[2][3];
      load_spinor(&g, psi, ax, ay, az, at, nb);
      project(isPlus ? d : (d ^ 1), nb, b);
      /* F_U[c][r] = dL/dRe G[r][c] + i dL/dIm G[r][c]  (U = G^T) */
      cplx F[3][3];
      for (int rr = 0; rr < 3; rr++)
        for (int cc = 0; cc < 3; cc++) {
          cplx E[3][3];
          memset(E, 0, sizeof(E));
          E[rr][cc] = 1.0;
          double dre = hop_value(d, isPlus, beta, p, E, b, ch);
          E[rr][cc] = I;
          double dim = hop_value(d, isPlus, beta, p, E, b, ch);
          F[cc][rr] = dre + I * dim;
        }
      if (gauge) {
        cplx G[3][3], M[3][3];
        load_link(&g, gauge, xcb, y, z, t, d, G);
        for (int a = 0; a < 3; a++)
          for (int c = 0; c < 3; c++) {
            cplx acc = 0;
            for (int k = 0; k < 3; k++) acc += F[a][k] * conj(G[k][c]); /* U^dag[k][c] = conj(G[k][c]) */
            M[a][c] = acc;
          }
        cplx tr = (M[0][0] - conj(M[0][0]) + M[1][1] - conj(M[1][1]) + M[2][2] - conj(M[2][2])) / 6.0;
        for (int a = 0; a < 3; a++)
          for (int c = 0; c < 3; c++) F[a][c] = 0.5 * (M[a][c] - conj(M[c][a])) - (a == c ? tr : 0.0);
      }
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++) {
          force[((long long)((d * 3 + a) * 3 + c) * 2 + 0) * nsites + i] = creal(F[a][c]);
          force[((long long)((d * 3 + a) * 3 + c) * 2 + 1) * nsites + i] = cimag(F[a][c]);
        }
    }
  }
  return QB200_OK;
}

/* ------------------------------------------------------------------ */
/* faces                                                                */

/* enumerate the sites of checkerboard cb whose coordinate in dim mu is
 * `coord`, in increasing (t, z, y, xcb) order; returns the count and fills
 * the coordinate arrays when they are non-NULL */
static long long face_sites(const geo *g, int cb, int mu, int coord, int *fx,
                            int *fy, int *fz, int *ft)
{
  long long n = 0;
  for (int t = 0; t < g->nt; t++)
    for (int z = 0; z < g->nz; z++)
      for (int y = 0; y < g->ny; y++)
        for (int xcb = 0; xcb < g->nxh; xcb++) {
          int x = 2 * xcb + ((y + z + t + cb) & 1);
          int c[4] = {x, y, z, t};
          if (c[mu] != coord) continue;
          if (fx) { fx[n] = xcb; fy[n] = y; fz[n] = z; ft[n] = t; }
          n++;
        }
  return n;
}

/* elements of one checkerboard spinor array of lat with FP64 storage */
long long oracle_spinor_elems_f64(const qb200_lattice *lat)
{
  geo g;
  if (make_geo(lat, &g)) return -1;
  return (long long)g.nt * g.Pxyz * 24 * g.S;
}

long long oracle_face_count(const qb200_lattice *lat, int cb, int dir)
{
  geo g;
  if (make_geo(lat, &g) || dir < 0 || dir > 7) return -1;
  int L[4] = {g.nx, g.ny, g.nz, g.nt};
  int mu = dir / 2;
  return face_sites(&g, cb, mu, (dir & 1) ? L[mu] - 1 : 0, 0, 0, 0, 0);
}

/* face_proj_dir: sites of psi (on psi_cb) on the face towards dir, projected
 * with the projector of the opposite direction (dslash.cc:451-454) */
int oracle_face_pack_out(const qb200_lattice *lat, int out_ft, int isign,
                         int psi_cb, const void *psi, void *outbuf, int dir,
                         int *scratch)
{
  geo g, go;
  if (make_geo(lat, &g)) return QB200_EINVAL;
  if (dir < 0 || dir > 7) return QB200_EDIR;
  if (out_ft < QB200_F32 || out_ft > QB200_BF16) return QB200_EINVAL;
  go = g;
  go.ft = out_ft;
  int L[4] = {g.nx, g.ny, g.nz, g.nt};
  int mu = dir / 2;
  int coord = (dir & 1) ? L[mu] - 1 : 0;
  long long n = face_sites(&g, psi_cb, mu, coord, 0, 0, 0, 0);
  int *fx = scratch, *fy = scratch + n, *fz = scratch + 2 * n, *ft = scratch + 3 * n;
  face_sites(&g, psi_cb, mu, coord, fx, fy, fz, ft);
  int pidx = isign > 0 ? (dir ^ 1) : dir; /* proj_ops_minus[k] == proj_ops_plus[k^1] */
  for (long long i = 0; i < n; i++) {
    cplx sp[4][3], b[2][3];
    load_spinor(&g, psi, fx[i], fy[i], fz[i], ft[i], sp);
    project(pidx, sp, b);
    store_face(&go, outbuf, i, b);
  }
  return QB200_OK;
}

int oracle_face_pack(const qb200_lattice *lat, int isign, int psi_cb,
                     const void *psi, void *outbuf, int dir, int *scratch)
{
  return oracle_face_pack_out(lat, lat->ftype, isign, psi_cb, psi, outbuf, dir,
                              scratch);
}

/* face_*finish_dir: accumulate the face contribution into out (on cb) */
/* out_ft: storage type of `out` (read and written), e.g. QB200_F64 for an
 * unrounded result; the other fields are in lat's storage type */
int oracle_face_unpack_out(const qb200_lattice *lat, int out_ft, int family,
                           int isign, int cb, const void *inbuf,
                           const void *gauge, void *out, const void *clov,
                           double beta, double mu, double muinv, int dir,
                           int tbc, const double *tbc_phases, int *scratch)
{
  geo g, go;
  if (make_geo(lat, &g)) return QB200_EINVAL;
  if (dir < 0 || dir > 7) return QB200_EDIR;
  if (out_ft < QB200_F32 || out_ft > QB200_BF16) return QB200_EINVAL;
  go = g;
  go.ft = out_ft;
  int L[4] = {g.nx, g.ny, g.nz, g.nt};
  int dim = dir / 2, isBack = !(dir & 1);
  int coord = isBack ? 0 : L[dim] - 1;
  int isPlus = isign > 0;
  int clover = family == FAM_CLOVER || family == FAM_TMCLOV;
  int tm = family == FAM_TM || family == FAM_TMCLOV;
  long long n = face_sites(&g, cb, dim, coord, 0, 0, 0, 0);
  int *fx = scratch, *fy = scratch + n, *fz = scratch + 2 * n, *ft = scratch + 3 * n;
  face_sites(&g, cb, dim, coord, fx, fy, fz, ft);
  /* pbeta for clover faces, mbeta otherwise (dslash_common.cc:1975-1981) */
  double b_eff = clover ? beta : -beta;
  for (long long i = 0; i < n; i++) {
    cplx o[4][3], dout[4][3], b[2][3], ub[2][3], G[3][3];
    load_spinor(&go, out, fx[i], fy[i], fz[i], ft[i], o);
    load_face(&g, inbuf, i, b);
    load_link(&g, gauge, fx[i], fy[i], fz[i], ft[i], dir, G);
    mult_link(G, isBack, b, ub);
    if (tbc) apply_tbc(!isBack, tbc_phases + 2 * dim, ub);
    memset(dout, 0, sizeof(dout));
    recons(dim, isPlus == isBack, b_eff, ub, (clover || tm) ? dout : o);
    if (clover) {
      for (int bl = 0; bl < 2; bl++) {
        cplx A[6][6];
        if (family == FAM_CLOVER) load_clover(&g, clov, fx[i], fy[i], fz[i], ft[i], bl, A);
        else load_full_clover(&g, clov, fx[i], fy[i], fz[i], ft[i], bl, A);
        clover_mult(A, bl, dout, o, 1);
      }
    } else if (tm) {
      inv_twisted(isPlus, mu, muinv, dout, o, 1);
    }
    store_spinor(&go, out, fx[i], fy[i], fz[i], ft[i], o);
  }
  return QB200_OK;
}

int oracle_face_unpack(const qb200_lattice *lat, int family, int isign,
                       int cb, const void *inbuf, const void *gauge,
                       void *out, const void *clov, double beta, double mu,
                       double muinv, int dir, int tbc,
                       const double *tbc_phases, int *scratch)
{
  return oracle_face_unpack_out(lat, lat->ftype, family, isign, cb, inbuf,
                                gauge, out, clov, beta, mu, muinv, dir, tbc,
                                tbc_phases, scratch);
}

int oracle_abi_version(void) { return QB200_ABI_VERSION; }
