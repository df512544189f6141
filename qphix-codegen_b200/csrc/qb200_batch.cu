// qb200_batch.cu -- several independent lattices in one persistent launch,
// and the launch-configuration autotuner.
//
// A batch holds up to QB200_MAX_BATCH problems of one operator (family,
// kernel, isign) whose fields share storage type, SOALEN, VECLEN and link
// compression but may differ in size (e.g. 3 x 16^3x32 + 2 x 24^3x48 +
// 1 x 32^3x64).  One launch of batch_dslash_kernel covers all their sites:
// the per-problem geometry, pointers and coefficients travel as one kernel
// parameter block, and the threads stride through the concatenated site
// ranges.  There is no counterpart in the reference, whose kernels work on
// one tile of one lattice per call (codegen/jinja/dslash_decl.h.j2:6-43); the
// per-site operator is the same as qb200_*dslash*_vec's.
//
// The tuner times candidate (grid, block) pairs on the caller's fields and
// remembers the fastest per (operator, layout, lattice sizes, device) in a
// process-wide table that can be saved to and loaded from a text file.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "qphix_b200.h"
#include "qb200_internal.h"

namespace qb200 {
int api_fail(int code, const char *msg);
int api_geo(const qb200_lattice *l, GeoDev &g);
int api_check_device();
void api_fill_op_f(OpDev<float> &p, const qb200_lattice *l, int isPlus, int cb, bool negate, double cs, double ctf,
                   double ctb, unsigned tbc_mask, const double *ph, const unsigned *acc);
void api_fill_op_d(OpDev<double> &p, const qb200_lattice *l, int isPlus, int cb, bool negate, double cs, double ctf,
                   double ctb, unsigned tbc_mask, const double *ph, const unsigned *acc);
} // namespace qb200

using namespace qb200;

static_assert(QB200_MAX_BATCH == kMaxBatch, "batch size limits differ");

namespace {

void fill(OpDev<float> &p, const qb200_lattice *l, int isPlus, int cb, bool neg, const qb200_coeffs &c)
{
  api_fill_op_f(p, l, isPlus, cb, neg, c.coeff_s, c.coeff_t_f, c.coeff_t_b, c.tbc_mask, &c.tbc_phases[0][0],
                nullptr);
  p.alpha = (float)c.alpha;
  p.mu = (float)c.mu;
  p.muinv = (float)c.muinv;
  p.rho = (float)c.rho;
}

void fill(OpDev<double> &p, const qb200_lattice *l, int isPlus, int cb, bool neg, const qb200_coeffs &c)
{
  api_fill_op_d(p, l, isPlus, cb, neg, c.coeff_s, c.coeff_t_f, c.coeff_t_b, c.tbc_mask, &c.tbc_phases[0][0],
                nullptr);
  p.alpha = c.alpha;
  p.mu = c.mu;
  p.muinv = c.muinv;
  p.rho = c.rho;
}

int check_batch(int family, int nitems, const qb200_batch_item *items)
{
  if (family < 0 || family > 3) return api_fail(QB200_EINVAL, "family must be 0..3");
  if (nitems < 1 || nitems > QB200_MAX_BATCH) return api_fail(QB200_EINVAL, "a batch holds 1..QB200_MAX_BATCH items");
  if (!items) return api_fail(QB200_ENULL, "items is NULL");
  const qb200_lattice &l0 = items[0].lat;
  for (int k = 0; k < nitems; k++) {
    const qb200_batch_item &it = items[k];
    const qb200_lattice &l = it.lat;
    if (l.ftype != l0.ftype || l.soalen != l0.soalen || l.veclen != l0.veclen || l.compress12 != l0.compress12)
      return api_fail(QB200_ELAYOUT, "batch items must share ftype, soalen, veclen and compress12");
    if (l.soalen >= 4 && l.veclen != l.soalen)
      return api_fail(QB200_ELAYOUT, "batched layouts with soalen >= 4 need veclen == soalen");
    GeoDev g;
    int rc = api_geo(&l, g);
    if (rc) return rc;
    if (it.cb != 0 && it.cb != 1) return api_fail(QB200_EINVAL, "cb must be 0 or 1");
    if (!it.psi || !it.gauge || !it.out) return api_fail(QB200_ENULL, "psi, gauge and out must be non-NULL");
    if ((family == 1 || family == 3) && !it.clov) return api_fail(QB200_ENULL, "clover field is NULL");
    if (it.out == it.psi) return api_fail(QB200_EINVAL, "out must not alias psi");
  }
  return QB200_OK;
}

template <typename FT>
cudaError_t launch_t(int family, int ach, int isign, int nitems, const qb200_batch_item *items, int grid, int block,
                     cudaStream_t st)
{
  typedef elem_t<FT> E;
  BatchDev<FT> b;
  std::memset(&b, 0, sizeof(b));
  long long first = 0;
  for (int k = 0; k < nitems; k++) {
    const qb200_batch_item &it = items[k];
    BatchItem<FT> &d = b.it[k];
    api_geo(&it.lat, d.g);
    d.a.psi = (const E *)it.psi;
    d.a.chi = (const E *)it.chi;
    d.a.gauge = (const E *)it.gauge;
    d.a.clov = (const E *)it.clov;
    d.a.out = (E *)it.out;
    fill(d.p, &it.lat, isign > 0, it.cb, ach != 0, it.coeffs);
    d.first = first;
    first += d.g.nsites;
  }
  b.n = nitems;
  b.total = first;
  LaunchSpec ls;
  ls.fam = family;
  ls.ach = ach != 0;
  ls.comp12 = items[0].lat.compress12 != 0;
  const bool vfixed = items[0].lat.veclen == items[0].lat.soalen;
  switch (items[0].lat.soalen) {
  case 1: return launch_dslash_batched<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 1)>(ls, b, vfixed, grid, block, st);
  case 2: return launch_dslash_batched<FT, (ftraits<FT>::WIDE_ONLY ? 4 : 2)>(ls, b, vfixed, grid, block, st);
  case 4: return launch_dslash_batched<FT, 4>(ls, b, vfixed, grid, block, st);
  case 8: return launch_dslash_batched<FT, 8>(ls, b, vfixed, grid, block, st);
  default: return launch_dslash_batched<FT, 16>(ls, b, vfixed, grid, block, st);
  }
}

long long total_sites(int nitems, const qb200_batch_item *items)
{
  long long n = 0;
  for (int k = 0; k < nitems; k++) {
    GeoDev g;
    api_geo(&items[k].lat, g);
    n += g.nsites;
  }
  return n;
}

int launch(int family, int ach, int isign, int nitems, const qb200_batch_item *items, int grid, int block,
           cudaStream_t st)
{
  cudaError_t e;
  switch (items[0].lat.ftype) {
  case QB200_F32: e = launch_t<float>(family, ach, isign, nitems, items, grid, block, st); break;
  case QB200_F64: e = launch_t<double>(family, ach, isign, nitems, items, grid, block, st); break;
  case QB200_F16: e = launch_t<__half>(family, ach, isign, nitems, items, grid, block, st); break;
  case QB200_F16N: e = launch_t<half_norm>(family, ach, isign, nitems, items, grid, block, st); break;
  default: e = launch_t<__nv_bfloat16>(family, ach, isign, nitems, items, grid, block, st); break;
  }
  if (e != cudaSuccess) return api_fail(QB200_ECUDA, cudaGetErrorString(e));
  return QB200_OK;
}

// ---- the tuning table ------------------------------------------------------

struct Tuned {
  int grid, block;
  double ms;
};

std::mutex g_tune_mu;
std::map<std::string, Tuned> g_tune;

// name of the current device (looked up once per device; the caller holds g_tune_mu)
std::string device_name()
{
  static std::map<int, std::string> names;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return "unknown";
  auto it = names.find(dev);
  if (it != names.end()) return it->second;
  cudaDeviceProp prop;
  std::string s = cudaGetDeviceProperties(&prop, dev) == cudaSuccess ? prop.name : "unknown";
  std::replace(s.begin(), s.end(), ' ', '_');
  names[dev] = s;
  return s;
}

// operator variant, layout, lattice sizes and device: the launch choice of
// one key does not depend on the field values
std::string tune_key(int family, int ach, int isign, int nitems, const qb200_batch_item *items)
{
  std::ostringstream o;
  const qb200_lattice &l = items[0].lat;
  o << "batch:f" << family << ":a" << ach << ":s" << (isign > 0 ? 1 : -1) << ":t" << l.ftype << ":S" << l.soalen
    << ":V" << l.veclen << ":c" << l.compress12 << ":" << device_name();
  for (int k = 0; k < nitems; k++) {
    const qb200_lattice &m = items[k].lat;
    o << ":" << m.nx << "x" << m.ny << "x" << m.nz << "x" << m.nt << "p" << m.pad_xy << "." << m.pad_xyz;
  }
  return o.str();
}

int sm_count()
{
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev))
    return 148;
  return n > 0 ? n : 148;
}

} // namespace

extern "C" {

int qb200_dslash_batched(int family, int achimbdpsi, int isign, int nitems, const qb200_batch_item *items,
                         const qb200_launch_cfg *cfg, void *stream)
{
  int rc = check_batch(family, nitems, items);
  if (rc) return rc;
  if ((rc = api_check_device())) return rc;
  for (int k = 0; k < nitems; k++)
    if (achimbdpsi && !items[k].chi) return api_fail(QB200_ENULL, "achimbdpsi needs chi");
  int grid = 0, block = 128;
  if (cfg) {
    grid = cfg->grid;
    block = cfg->block;
  } else {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(tune_key(family, achimbdpsi, isign, nitems, items));
    if (it != g_tune.end()) {
      grid = it->second.grid;
      block = it->second.block;
    }
  }
  if (block != 64 && block != 128) return api_fail(QB200_EINVAL, "block must be 64 or 128");
  if (grid < 0) return api_fail(QB200_EINVAL, "grid must be >= 0 (0: one thread per site)");
  const long long n = total_sites(nitems, items);
  if (grid == 0) grid = (int)std::min<long long>((n + block - 1) / block, 0x7fffffffLL);
  return launch(family, achimbdpsi, isign, nitems, items, grid, block, (cudaStream_t)stream);
}

int qb200_tune_batched(int family, int achimbdpsi, int isign, int nitems, const qb200_batch_item *items,
                       qb200_launch_cfg *best, double *best_ms, void *stream)
{
  int rc = check_batch(family, nitems, items);
  if (rc) return rc;
  if ((rc = api_check_device())) return rc;
  for (int k = 0; k < nitems; k++)
    if (achimbdpsi && !items[k].chi) return api_fail(QB200_ENULL, "achimbdpsi needs chi");
  cudaStream_t st = (cudaStream_t)stream;
  std::string key;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    key = tune_key(family, achimbdpsi, isign, nitems, items);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      if (best) {
        best->grid = it->second.grid;
        best->block = it->second.block;
      }
      if (best_ms) *best_ms = it->second.ms;
      return QB200_OK;
    }
  }
  // candidates: one thread per site, and persistent grids of m blocks per SM
  const long long n = total_sites(nitems, items);
  const int nsm = sm_count();
  std::vector<std::pair<int, int>> cand;
  for (int block : {128, 64}) {
    cand.push_back({(int)((n + block - 1) / block), block});
    for (int m : {1, 2, 4, 6, 8, 12, 16, 24, 32}) {
      const long long gr = (long long)m * nsm;
      if (gr * block < n) cand.push_back({(int)gr, block});
    }
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return api_fail(QB200_ECUDA, "cudaEventCreate failed");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return api_fail(QB200_ECUDA, "cudaEventCreate failed");
  }
  Tuned t{0, 128, 1e30};
  const int reps = 5;
  for (const auto &c : cand) {
    // one untimed launch, then reps timed ones
    if ((rc = launch(family, achimbdpsi, isign, nitems, items, c.first, c.second, st))) break;
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps && rc == QB200_OK; r++)
      rc = launch(family, achimbdpsi, isign, nitems, items, c.first, c.second, st);
    cudaEventRecord(e1, st);
    if (rc) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = api_fail(QB200_ECUDA, "tuning launch failed");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms / reps < t.ms) t = Tuned{c.first, c.second, ms / reps};
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = t;
  }
  if (best) {
    best->grid = t.grid;
    best->block = t.block;
  }
  if (best_ms) *best_ms = t.ms;
  return QB200_OK;
}

int qb200_tune_cache_save(const char *path)
{
  if (!path) return api_fail(QB200_ENULL, "path is NULL");
  FILE *f = std::fopen(path, "w");
  if (!f) return api_fail(QB200_EINVAL, "cannot open the tuning file for writing");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (const auto &kv : g_tune) std::fprintf(f, "%s %d %d %.6g\n", kv.first.c_str(), kv.second.grid, kv.second.block,
                                             kv.second.ms);
  std::fclose(f);
  return QB200_OK;
}

int qb200_tune_cache_load(const char *path)
{
  if (!path) return api_fail(QB200_ENULL, "path is NULL");
  FILE *f = std::fopen(path, "r");
  if (!f) return api_fail(QB200_EINVAL, "cannot open the tuning file");
  char key[1024];
  int grid, block;
  double ms;
  int loaded = 0;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  while (std::fscanf(f, "%1023s %d %d %lf", key, &grid, &block, &ms) == 4) {
    if ((block == 64 || block == 128) && grid >= 0) {
      g_tune[key] = Tuned{grid, block, ms};
      loaded++;
    }
  }
  std::fclose(f);
  return loaded;
}

void qb200_tune_cache_clear(void)
{
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
}

} // extern "C"
