// kk_engine.cu -- solve() orchestration on one device for one handle.
//
// Data flow of one solve (solve_base, kriging_base.F90:2064-2194):
//   prepare    host: variogram tables + search parameters; device: upload of
//              changed observations/targets, grid build per variable
//   search     k_search per variable (+ exact kd-tree replica for targets
//              whose selection boundary has equal distances)
//   bucket     size buckets of npp per target
//   solve      per bucket the planned kernel: warp per target (FP64, or
//              FP32 + FP64 refinement) up to 64 equations, CTA per target
//              up to 128, generic kernel beyond (and for Cholesky failures:
//              LDL^T + jitter); the plan can be tuned by timing candidates
//              on a sample of each bucket; FP64 re-solve of non-converged
//              FP32 targets
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "kk_host.h"
#include "kk_kernels.h"

namespace kk {

static_assert(KK_CNT_N_HOST == KK_CNT_N, "host copy of the device counters");

static alloc_fn g_alloc = nullptr;
static free_fn g_free = nullptr;
static void* g_actx = nullptr;

void set_allocator(alloc_fn a, free_fn f, void* ctx) {
  g_alloc = a;
  g_free = f;
  g_actx = ctx;
}

#define KK_CUDA(x)                                                                    \
  do {                                                                                \
    cudaError_t err__ = (x);                                                          \
    if (err__ != cudaSuccess) {                                                       \
      throw std::string("CUDA error ") + cudaGetErrorString(err__) + " at " #x;       \
    }                                                                                 \
  } while (0)

void DBuf::reserve(size_t b) {
  if (b <= bytes && p) return;
  release();
  size_t nb = b < 256 ? 256 : b;
  if (g_alloc) {
    p = g_alloc(nb, g_actx);
    if (!p) throw std::string("device allocation failed (registered allocator)");
  } else {
    KK_CUDA(cudaMalloc(&p, nb));
  }
  bytes = nb;
}

void DBuf::release() {
  if (!p) return;
  if (g_alloc) g_free(p, g_actx);
  else cudaFree(p);
  p = nullptr;
  bytes = 0;
}

static void upload(DBuf& d, const void* h, size_t bytes, cudaStream_t st) {
  d.reserve(bytes);
  if (bytes) KK_CUDA(cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, st));
}

// (D, nb) interleaved target coordinates -> one array per axis
__global__ void k_split_axes(const double* __restrict__ src, int nb, int D, double* __restrict__ x0,
                             double* __restrict__ x1, double* __restrict__ x2, double* __restrict__ x3) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    const double* p = src + (size_t)i * D;
    x0[i] = p[0];
    if (D > 1) x1[i] = p[1];
    if (D > 2) x2[i] = p[2];
    if (D > 3) x3[i] = p[3];
  }
}

static int sm_count(int dev) {
  static int cached[64] = {0};
  if (dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) cudaDeviceGetAttribute(&cached[dev], cudaDevAttrMultiProcessorCount, dev);
  return cached[dev];
}

// search parameters for variable v (set_search, kriging.F90:318-387;
// kriging_st.F90:322-403) and the matrix sizing (prepare_common,
// kriging_base.F90:3003-3012)
static void setup_search(Engine& e, int v, KkSearch& S) {
  const ObsVar& o = e.obs[v];
  std::memset(&S, 0, sizeof S);
  S.ndim = e.ndim;
  S.nlag = e.nlag;
  S.st = e.st;
  S.nobs = o.n;
  S.cv = (e.cross_validation != 0);
  int nmax = o.nmax;
  if (e.cross_validation && v == 0 && nmax > 0 && nmax < INT_MAX) nmax = nmax + 1;  // set_grid_cv_base
  if (nmax > o.n) nmax = o.n;
  if (nmax <= 0) nmax = o.n;
  const bool need = o.n > nmax;
  const double eps = 1.0e-10;
  S.aniso = ((std::fabs(o.anis1 - 1.0) > eps || std::fabs(o.anis2 - 1.0) > eps) && e.anisotropic_search) ? 1 : 0;
  double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(S.rotmat, eye, sizeof eye);
  if (e.st || (need && S.aniso)) calc_rotmat(o.az, o.dip, o.plunge, o.anis1, o.anis2, S.rotmat);
  S.maxd2 = o.maxdist * o.maxdist;
  S.ta = o.time_at;
  S.nmax = nmax;
  if (!need) {
    S.mode = 0;
    S.K = o.n;
    S.mmax = o.n;
  } else if (o.sector) {
    // the sector selection packs the sector id above bit 28 of the index
    if (o.n >= (1 << 28)) throw std::string("sector search supports fewer than 2^28 observations per variable");
    S.mode = 2;
    long long lim = (long long)(1 << e.ndim) * nmax * 4;
    S.K = (int)std::min<long long>(o.n, lim);
    S.mmax = (1 << e.ndim) * nmax;
  } else {
    S.mode = 1;
    S.K = nmax;
    S.mmax = nmax;
  }
}

// uniform grid over the search coordinates of variable v
static void build_grid(Engine& e, int v) {
  VarDevice& d = e.vd[v];
  KkSearch& S = d.search;
  const int n = S.nobs;
  const int D = e.nlag;
  cudaStream_t st = e.stream;
  DBuf scu;
  scu.reserve(sizeof(double) * (size_t)D * n);
  const double* xs[4] = {d.x[0].as<double>(), d.x[1].as<double>(), d.x[2].as<double>(), d.x[3].as<double>()};
  KkGrid& g = S.grid;
  g.D = D;
  launch_search_coords(S, xs, scu.as<double>(), n, st);
  std::vector<double> h((size_t)D * n);
  KK_CUDA(cudaMemcpyAsync(h.data(), scu.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
  KK_CUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < D; ++k) {
    double lo = h[(size_t)k * n], hi = lo;
    for (int i = 1; i < n; ++i) {
      double x = h[(size_t)k * n + i];
      lo = std::min(lo, x);
      hi = std::max(hi, x);
    }
    g.umin[k] = lo;
    g.umax[k] = hi;
  }
  g.G = std::min(D, 3);
  g.nobs = n;
  // grid axes: every search dimension, or with four (space-time in 3-D) the
  // three of widest extent -- a constant coordinate (z = 0 for 2-D data
  // given as 3-D) is then left out of the grid
  int gd[3] = {0, 1, 2};
  if (D > 3) {
    int order[4] = {0, 1, 2, 3};
    std::stable_sort(order, order + D, [&](int p, int q) {
      return (g.umax[p] - g.umin[p]) > (g.umax[q] - g.umin[q]);
    });
    std::sort(order, order + 3);
    for (int k = 0; k < 3; ++k) gd[k] = order[k];
  }
  g.gmask = 0;
  for (int k = 0; k < 3; ++k) {
    g.gd[k] = k < g.G ? gd[k] : 0;
    if (k < g.G) g.gmask |= 1 << gd[k];
    g.gumin[k] = k < g.G ? g.umin[gd[k]] : 0.0;
    g.gumax[k] = k < g.G ? g.umax[gd[k]] : 0.0;
  }
  // Cell size from the dense end of the point distribution: a coarse
  // histogram gives the density seen by the 99th-percentile point, and cells
  // are sized to hold about max(2, K/8) points there, so a K-nearest search
  // in the densest regions gathers a few K candidates while sparse regions
  // cost only extra (cheap, mostly empty) cell rows.
  double ext[3], vol = 1.0, emax = 0.0;
  for (int k = 0; k < g.G; ++k) emax = std::max(emax, g.gumax[k] - g.gumin[k]);
  if (emax <= 0.0) emax = 1.0;
  for (int k = 0; k < g.G; ++k) {
    ext[k] = std::max(g.gumax[k] - g.gumin[k], 1e-9 * emax);
    vol *= ext[k];
  }
  const int nc_axis = g.G == 1 ? 65536 : (g.G == 2 ? 256 : 48);
  long long ncoarse = 1;
  for (int k = 0; k < g.G; ++k) ncoarse *= nc_axis;
  std::vector<int> coarse(ncoarse, 0);
  for (int i = 0; i < n; ++i) {
    long long c = 0, stride = 1;
    for (int k = 0; k < g.G; ++k) {
      int ck = (int)((h[(size_t)gd[k] * n + i] - g.gumin[k]) / ext[k] * nc_axis);
      ck = ck < 0 ? 0 : (ck >= nc_axis ? nc_axis - 1 : ck);
      c += ck * stride;
      stride *= nc_axis;
    }
    coarse[c]++;
  }
  std::vector<int> cnt;
  cnt.reserve(4096);
  for (int v : coarse) if (v > 0) cnt.push_back(v);
  std::sort(cnt.begin(), cnt.end());
  long long acc = 0, p99 = 0;
  for (size_t q = 0; q < cnt.size(); ++q) {  // density of the cell holding the 99th-percentile point
    acc += cnt[q];
    if (acc >= (long long)(0.99 * n)) { p99 = cnt[q]; break; }
  }
  const double coarse_vol = vol / (double)ncoarse;
  const double rho = std::max((double)p99, 1.0) / coarse_vol;
  const double occ = std::max(2.0, S.K / 8.0);
  double hcell = std::pow(occ / rho, 1.0 / g.G);
  hcell = std::max(hcell, std::pow(vol * 2.0 / std::max(n, 1), 1.0 / g.G) * 0.05);
  long long ncell = 1;
  for (int k = 0; k < g.G; ++k) {
    long long c = (long long)std::ceil(ext[k] / hcell);
    c = std::max<long long>(1, std::min<long long>(c, g.G == 1 ? (1 << 24) : (1 << 14)));
    g.n[k] = (int)c;
    ncell *= c;
  }
  while (ncell > (1ll << 25)) {
    ncell = 1;
    for (int k = 0; k < g.G; ++k) { g.n[k] = std::max(1, g.n[k] / 2); ncell *= g.n[k]; }
  }
  for (int k = 0; k < 3; ++k) {
    if (k >= g.G) { g.n[k] = 1; g.lo[k] = 0; g.h[k] = 1; g.inv_h[k] = 1; continue; }
    g.lo[k] = g.gumin[k];
    g.h[k] = ext[k] / g.n[k] * (1.0 + 1e-12);
    g.inv_h[k] = 1.0 / g.h[k];
  }
  const long long nsat = (long long)(g.n[0] + 1) * (g.n[1] + 1) * (g.n[2] + 1);
  d.cell_of.reserve(sizeof(int) * n);
  DBuf count;
  count.reserve(sizeof(int) * ncell);
  d.cursor.reserve(sizeof(int) * ncell);
  d.cell_start.reserve(sizeof(int) * (ncell + 1));
  d.sc.reserve(sizeof(double) * (size_t)D * n);
  d.sidx.reserve(sizeof(int) * n);
  d.sat.reserve(sizeof(int) * nsat);
  launch_grid_build(g, scu.as<double>(), d.cell_of.as<int>(), count.as<int>(), d.cell_start.as<int>(),
                    d.cursor.as<int>(), d.sc.as<double>(), d.sidx.as<int>(), d.sat.as<int>(), n, st);
  g.cell_start = d.cell_start.as<int>();
  g.sat = d.sat.as<int>();
  g.sc = d.sc.as<double>();
  g.sidx = d.sidx.as<int>();
  KK_CUDA(cudaStreamSynchronize(st));
  // keep the search coordinates in original order for a kd-tree build on demand
  d.tree_rdata.reserve(sizeof(double) * h.size());
  KK_CUDA(cudaMemcpyAsync(d.tree_rdata.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, st));
  d.grid_ready = true;
  d.tree_ready = false;
}

// kd-tree for the exact tie fallback (kdtree2_create on the search coords)
static void build_tree(Engine& e, int v) {
  VarDevice& d = e.vd[v];
  KkSearch& S = d.search;
  const int n = S.nobs, D = e.nlag;
  std::vector<double> soa((size_t)D * n), pm((size_t)D * n);
  KK_CUDA(cudaMemcpyAsync(soa.data(), d.tree_rdata.p, sizeof(double) * soa.size(), cudaMemcpyDeviceToHost, e.stream));
  KK_CUDA(cudaStreamSynchronize(e.stream));
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < D; ++k) pm[(size_t)i * D + k] = soa[(size_t)k * n + i];
  std::vector<int> ni, ind;
  std::vector<double> nd, box, rdata;
  int root = 0;
  build_kdtree(pm.data(), D, n, ni, nd, box, ind, rdata, root);
  upload(d.tree_i, ni.data(), sizeof(int) * ni.size(), e.stream);
  upload(d.tree_d, nd.data(), sizeof(double) * nd.size(), e.stream);
  upload(d.tree_box, box.data(), sizeof(double) * box.size(), e.stream);
  upload(d.tree_ind, ind.data(), sizeof(int) * ind.size(), e.stream);
  DBuf tmp;
  upload(tmp, rdata.data(), sizeof(double) * rdata.size(), e.stream);
  KK_CUDA(cudaStreamSynchronize(e.stream));
  d.tree_rdata.release();
  std::swap(d.tree_rdata.p, tmp.p);
  std::swap(d.tree_rdata.bytes, tmp.bytes);
  KkTree& T = S.tree;
  T.D = D;
  T.n = n;
  T.nnodes = (int)(ni.size() / 5);
  T.root = root;
  T.node_i = d.tree_i.as<int>();
  T.node_d = d.tree_d.as<double>();
  T.box = d.tree_box.as<double>();
  T.ind = d.tree_ind.as<int>();
  T.rdata = d.tree_rdata.as<double>();
  d.tree_ready = true;
}

static void validate(const Engine& e) {
  if (e.nblock <= 0) throw std::string("Call set_grid() before solve().");
  for (int v = 0; v < e.nvar; ++v) {
    if (e.obs[v].n == 0) throw std::string("Call set_obs() for every variable before solve().");
    if (!e.obs[v].search_set) throw std::string("set_search() needs to be called before solve().");
    if (e.ndrift > 0 && e.obs[v].drift.empty())
      throw std::string("Observation drift is not set while ndrift > 0.");
  }
  if (e.ndrift > 0 && e.bdrift.empty()) throw std::string("Grid drift is not set while ndrift > 0.");
  for (int a = 0; a < e.nvar; ++a)
    for (int b = a; b < e.nvar; ++b)
      if (e.vgm[a][b].empty()) {
        char msg[160];
        snprintf(msg, sizeof msg, "variogram not set for ivar=%d, jvar=%d. Call set_vgm().", a + 1, b + 1);
        throw std::string(msg);
      }
}

// CUDA-event timer for the solve phases (enabled by krige_gpu_profile)
struct PhaseTimer {
  Engine& e;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  explicit PhaseTimer(Engine& en) : e(en) {
    if (e.profile) { cudaEventCreate(&ev[0]); cudaEventCreate(&ev[1]); }
  }
  ~PhaseTimer() {
    if (ev[0]) { cudaEventDestroy(ev[0]); cudaEventDestroy(ev[1]); }
  }
  void start() { if (ev[0]) cudaEventRecord(ev[0], e.stream); }
  void stop(int phase) {
    if (!ev[0]) return;
    cudaEventRecord(ev[1], e.stream);
    cudaEventSynchronize(ev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    e.phase_ms[phase] += ms;
  }
};

// Solve parameters from the engine's device buffers (after the search).
static void fill_params(Engine& e, SolveParams& P) {
  const int nv = e.nvar, nb = e.nblock;
  std::memset(&P, 0, sizeof P);
  P.nvar = nv;
  P.ndim = e.ndim;
  P.nlag = e.nlag;
  P.st = e.st;
  P.ndrift = e.ndrift;
  P.naug = e.naug();
  P.pa = e.pdrift();
  P.std_ck = e.std_ck;
  P.unbias = e.unbias;
  P.ck_isa = (!e.std_ck && e.unbias != 0 && nv > 1) ? 1 : 0;
  P.sk_any = 0;
  for (int v = 0; v < nv; ++v) {
    P.sk_mean[v] = e.obs[v].sk_mean;
    if (e.unbias == 0 && e.obs[v].sk_mean != 0.0) P.sk_any = 1;
  }
  P.nmin = e.nmin;
  P.neglect_error = e.neglect_error;
  P.bounds[0] = e.bounds[0];
  P.bounds[1] = e.bounds[1];
  P.models = e.st ? nullptr : e.models.as<KkModel>();
  P.smodels = e.st ? e.models.as<KkSTModel>() : nullptr;
  P.tables = e.tables.as<double2>();
  for (int v = 0; v < nv; ++v) {
    VarDevice& d = e.vd[v];
    for (int k = 0; k < 4; ++k) P.ox[v][k] = d.x[k].as<double>();
    P.oval[v] = d.value.as<double>();
    P.ovar[v] = d.variance.as<double>();
    P.odrift[v] = d.drift.as<double>();
    P.nobs[v] = e.obs[v].n;
    P.nbr[v] = d.nbr.as<int>();
    P.nnear[v] = d.nnear.as<int>();
    P.mmax[v] = std::max(d.search.mmax, 1);
  }
  P.nblock = nb;
  for (int k = 0; k < 4; ++k) P.tx[k] = e.tx[k].as<double>();
  P.rs = e.rangescale.empty() ? nullptr : e.trs.as<double>();
  P.ln = e.localnugget.empty() ? nullptr : e.tln.as<double>();
  P.tdrift = e.ndrift > 0 ? e.tdrift.as<double>() : nullptr;
  P.gstart = e.nblockpnt.empty() ? nullptr : e.gstart.as<int>();
  for (int k = 0; k < 4; ++k) P.gx[k] = e.nblockpnt.empty() ? nullptr : e.gx[k].as<double>();
  P.gw = e.nblockpnt.empty() ? nullptr : e.gw.as<double>();
  P.est = e.est.as<double>();
  P.var = e.var.as<double>();
  P.status = e.status.as<int>();
  P.counters = e.counters.as<int>();
  P.fb_list = e.npp.as<int>();
  P.fp64_list = e.npp.as<int>() + nb;
  P.refine_tol = 1.0e-10;
  // the refinement form's correction term c is about (cond * eps32)^2 of its
  // value and carries an error of about c^1.5: c <= tol^(2/3) keeps it <= tol
  P.refine_tol_corr = std::cbrt(P.refine_tol * P.refine_tol);
}

// Systems with more drift / variable columns than the register kernels hold
// (8: e.g. four-variable cokriging without standardisation) are solved by the
// general kernel.
static bool wide_columns(const SolveParams& P) {
  return P.pa + P.nvar + 1 + ((P.ck_isa || P.sk_any) ? P.nvar : 0) > 8;
}

// indicator kriging: the category probabilities after a solve or a re-estimate
static void indicator_post(Engine& e) {
  if (!e.indicator || e.nsim > 0) return;
  const int kcat = (e.ncat > 0 && e.ncat <= e.nvar) ? e.ncat : e.nvar;
  launch_indicator_post(e.est.as<double>(), e.nblock, e.nvar, kcat, sm_count(e.device), e.stream);
  KK_CUDA(cudaGetLastError());
  KK_CUDA(cudaStreamSynchronize(e.stream));
  e.launches += 1;
}

// ---------------------------------------------------------------------------
// solve plan: which kernel solves each neighbour-count list
// ---------------------------------------------------------------------------
// Equations a planned kernel holds (the assembly buffer's row count), and
// its form (1: FP32 factor + FP64 correction).
static int kernel_rows(int ker) {
  return (ker == KK_KER_W32 || ker == KK_KER_W32R) ? 32 : ((ker == KK_KER_W64 || ker == KK_KER_W64R) ? 64 : 128);
}
static int kernel_form(int ker) { return (ker == KK_KER_W32R || ker == KK_KER_W64R) ? 1 : 0; }
// Targets per assembly chunk: about 1.1 GB of packed FP64 K per chunk.
static int chunk_targets(int N) { return N == 128 ? (1 << 14) : (1 << 16); }
static size_t kbuf_bytes(int N, int n) { return sizeof(double) * (size_t)n * (N * (N + 1) / 2); }

// rform: the warp kernels' forms open to a solve: 0 FP64 only (precision
// fp64, the weight store, or more than six columns), 1 FP32 + correction,
// 2 either (precision auto: FP64 unless the tuner times the other faster).
//
// The plan without tuning: the smallest register kernel that holds the list,
// the general kernel for systems wider than eight columns, for more than 128
// equations, and for the weight store's 65..128 list (the CTA kernel keeps
// no weights).
static int default_kernel(int li, bool wide, bool wstore, int rform) {
  if (wide || li == KK_LIST_BIG) return KK_KER_GEN;
  if (li == KK_LIST_B32) return rform == 1 ? KK_KER_W32R : KK_KER_W32;
  if (li == KK_LIST_B64) return rform == 1 ? KK_KER_W64R : KK_KER_W64;
  return wstore ? KK_KER_GEN : KK_KER_BLOCK;
}

// Kernels that can solve list li: the default, the next larger one (a list
// of at most 32 equations on the 64-row warp kernel, 33..64 on the CTA
// kernel, 65..128 on the general kernel), so the tuner moves the bucket
// boundaries by one step where that is faster, and under rform 2 both forms
// of each warp kernel.
static int candidates(int li, bool wide, bool wstore, int rform, int* cand) {
  const int d = default_kernel(li, wide, wstore, rform);
  int n = 0;
  cand[n++] = d;
  if (d == KK_KER_GEN) return n;
  if (li == KK_LIST_B32) {
    if (rform == 2) {
      cand[n++] = KK_KER_W32R;
      cand[n++] = KK_KER_W64;
      cand[n++] = KK_KER_W64R;
    } else {
      cand[n++] = rform == 1 ? KK_KER_W64R : KK_KER_W64;
    }
    return n;
  }
  if (li == KK_LIST_B64) {
    if (rform == 2) cand[n++] = KK_KER_W64R;
    if (!wstore) cand[n++] = KK_KER_BLOCK;
    return n;
  }
  cand[n++] = KK_KER_GEN;
  return n;
}

constexpr int KK_TUNE_MIN = 2048;     // shorter lists keep the fixed plan (unless cached)
constexpr int KK_TUNE_SAMPLE = 8192;  // targets timed per candidate

// System signature the tuner's choice is cached under: what changes the
// work per target (form, columns, covariance path, dimensions, block
// targets) and the list's size class (a short list does not fill the GPU).
struct TuneKey {
  int v[9];
  bool operator<(const TuneKey& o) const { return std::lexicographical_compare(v, v + 9, o.v, o.v + 9); }
};
struct TuneEntry {
  int kernel = KK_KER_GEN;
  double us[KK_NKER];
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneEntry> g_tune;

static TuneKey tune_key(const SolveParams& P, int li, int rform, int st, int count) {
  const int C = P.pa + P.nvar + 1 + ((P.ck_isa || P.sk_any) ? P.nvar : 0);
  int dev = 0;
  cudaGetDevice(&dev);
  return TuneKey{{li, rform, C, P.nvar, P.fast_model, P.nlag + 8 * st, P.gstart ? 1 : 0,
                  count >= 65536 ? 2 : (count >= 8192 ? 1 : 0), dev}};
}
static bool tune_find(const TuneKey& k, TuneEntry& out) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tune.find(k);
  if (it == g_tune.end()) return false;
  out = it->second;
  return true;
}
static void tune_store(const TuneKey& k, const TuneEntry& e) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[k] = e;
}
void tune_clear() {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune.clear();
}

static void engine_replay(Engine& e);

static void engine_sgsim(Engine& e);

void engine_solve(Engine& e) {
  if (e.nsim > 0) {
    engine_sgsim(e);
    return;
  }
  auto t0 = std::chrono::steady_clock::now();
  for (double& x : e.phase_ms) x = 0.0;
  e.launches = 0;
  e.solved = false;
  std::memset(e.stats, 0, sizeof e.stats);
  if (e.use_old_weight) {
    // weight-store reuse: no search and no solve (load_block_weights)
    engine_replay(e);
    e.last_solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return;
  }
  validate(e);
  e.wstore_dev = false;  // this solve's neighbour lists replace the store's
  KK_CUDA(cudaSetDevice(e.device));
  PhaseTimer timer(e);
  cudaStream_t st = e.stream;
  const int nsm = sm_count(e.device);
  set_zones(st);
  const int nv = e.nvar, nb = e.nblock, D = e.nlag;

  // ---- variogram models and tables (prepare, kriging.F90:398-424)
  std::vector<KkModel> mdl;
  std::vector<KkSTModel> smdl;
  std::vector<double2> tabs;
  build_models(e, mdl, smdl, tabs);
  if (tabs.empty()) tabs.push_back(make_double2(0.0, 0.0));
  upload(e.tables, tabs.data(), sizeof(double2) * tabs.size(), st);
  if (e.st) upload(e.models, smdl.data(), sizeof(KkSTModel) * smdl.size(), st);
  else upload(e.models, mdl.data(), sizeof(KkModel) * mdl.size(), st);

  // ---- observations + search structures
  for (int v = 0; v < nv; ++v) {
    ObsVar& o = e.obs[v];
    VarDevice& d = e.vd[v];
    const int n = o.n;
    if (o.dirty) {
      std::vector<double> tmp(n);
      for (int k = 0; k < D; ++k) {
        for (int i = 0; i < n; ++i) tmp[i] = o.coord[(size_t)i * D + k];
        upload(d.x[k], tmp.data(), sizeof(double) * n, st);
      }
      for (int k = D; k < 4; ++k) d.x[k].reserve(8);
      upload(d.value, o.value.data(), sizeof(double) * n, st);
      upload(d.variance, o.variance.data(), sizeof(double) * n, st);
      if (e.ndrift > 0) {
        std::vector<double> dr((size_t)e.ndrift * n);
        for (int i = 0; i < n; ++i)
          for (int a = 0; a < e.ndrift; ++a) dr[(size_t)a * n + i] = o.drift[(size_t)i * e.ndrift + a];
        upload(d.drift, dr.data(), sizeof(double) * dr.size(), st);
      } else {
        d.drift.reserve(8);
      }
      KK_CUDA(cudaStreamSynchronize(st));
    }
    KkSearch S;
    setup_search(e, v, S);
    const bool rebuild = o.dirty || o.search_dirty || !d.grid_ready ||
                         std::memcmp(S.rotmat, d.search.rotmat, sizeof S.rotmat) != 0 ||
                         S.aniso != d.search.aniso || S.ta != d.search.ta;
    KkGrid keep_grid = d.search.grid;
    KkTree keep_tree = d.search.tree;
    d.search = S;
    if (S.mode != 0 && e.sim_nobs >= 0) {
      // the systems of a simulation search the kd-tree only: its search
      // coordinates, without the grid
      d.search.grid.D = D;  // k_search_coords writes D coordinates
      d.tree_rdata.reserve(sizeof(double) * (size_t)D * S.nobs);
      const double* xs[4] = {d.x[0].as<double>(), d.x[1].as<double>(), d.x[2].as<double>(), d.x[3].as<double>()};
      launch_search_coords(d.search, xs, d.tree_rdata.as<double>(), S.nobs, st);
      KK_CUDA(cudaGetLastError());
      d.grid_ready = false;
      d.tree_ready = false;
    } else if (S.mode != 0) {
      if (rebuild) build_grid(e, v);
      else { d.search.grid = keep_grid; d.search.tree = keep_tree; }
    } else {
      d.grid_ready = false;
    }
    o.dirty = false;
    o.search_dirty = false;
  }

  // ---- targets
  if (e.grid_dirty) {
    // target coordinates: through pinned staging, one array per axis on the
    // device; block targets add their nodes, weights and node offsets after
    // them in the same staging buffer (every region is in flight until the
    // synchronisation below)
    const bool blocks = !e.nblockpnt.empty();
    size_t ng = 0;
    if (blocks)
      for (int i = 0; i < nb; ++i) ng += (size_t)e.nblockpnt[i];
    const size_t need_t = sizeof(double) * (size_t)nb * D;
    const size_t need_n = blocks ? sizeof(double) * ng * (D + 1) : 0;
    const size_t need_g = blocks ? sizeof(int) * ((size_t)nb + 1) : 0;
    const size_t need = need_t + need_n + need_g;
    if (e.hstage_bytes < need) {
      // never reached with staged point targets: krige_set_grid sized the
      // buffer for them and they carry no nodes
      if (e.hstage) cudaFreeHost(e.hstage);
      e.hstage = nullptr;
      e.hstage_bytes = 0;
      KK_CUDA(cudaMallocHost(&e.hstage, need));
      e.hstage_bytes = need;
    }
    double* hs = static_cast<double*>(e.hstage);
    if (e.bcoord_staged) {
      // the caller's (D, nb) layout as staged by krige_set_grid: one copy,
      // then the per-axis split on the device
      upload(e.til, hs, need_t, st);
      for (int k = 0; k < D; ++k) e.tx[k].reserve(sizeof(double) * nb);
      if (nb > 0) {
        k_split_axes<<<std::min((nb + 255) / 256, 8 * nsm), 256, 0, st>>>(
            e.til.as<double>(), nb, D, e.tx[0].as<double>(), D > 1 ? e.tx[1].as<double>() : nullptr,
            D > 2 ? e.tx[2].as<double>() : nullptr, D > 3 ? e.tx[3].as<double>() : nullptr);
        KK_CUDA(cudaGetLastError());
        e.launches += 1;
      }
    } else {
      const double* bc = e.bcoord.data();
      par_for((size_t)nb, size_t(1) << 18, [=](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i)
          for (int k = 0; k < D; ++k) hs[(size_t)k * nb + i] = bc[i * D + k];
      });
      for (int k = 0; k < D; ++k) upload(e.tx[k], hs + (size_t)k * nb, sizeof(double) * nb, st);
    }
    for (int k = D; k < 4; ++k) e.tx[k].reserve(8);
    if (!e.rangescale.empty()) upload(e.trs, e.rangescale.data(), sizeof(double) * nb, st);
    if (!e.localnugget.empty()) upload(e.tln, e.localnugget.data(), sizeof(double) * nb, st);
    if (blocks) {
      double* hn = hs + (size_t)nb * D;  // nodes per axis, then the weights
      const double* gc = e.gcoord.data();
      par_for(ng, size_t(1) << 18, [=](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i)
          for (int k = 0; k < D; ++k) hn[(size_t)k * ng + i] = gc[i * D + k];
      });
      par_copy(hn + (size_t)D * ng, e.gweight.data(), sizeof(double) * ng);
      int* gs = reinterpret_cast<int*>(hn + (size_t)(D + 1) * ng);
      gs[0] = 0;
      for (int i = 0; i < nb; ++i) gs[i + 1] = gs[i] + e.nblockpnt[i];
      upload(e.gstart, gs, sizeof(int) * ((size_t)nb + 1), st);
      for (int k = 0; k < D; ++k) upload(e.gx[k], hn + (size_t)k * ng, sizeof(double) * ng, st);
      upload(e.gw, hn + (size_t)D * ng, sizeof(double) * ng, st);
    }
    KK_CUDA(cudaStreamSynchronize(st));
    e.grid_dirty = false;
  }
  if (e.ndrift > 0) upload(e.tdrift, e.bdrift.data(), sizeof(double) * e.bdrift.size(), st);

  // ---- outputs and work buffers
  e.est.reserve(sizeof(double) * (size_t)nb * nv);
  e.var.reserve(sizeof(double) * (size_t)nb * nv * nv);
  e.status.reserve(sizeof(int) * nb);
  e.counters.reserve(sizeof(int) * KK_CNT_N);
  e.bucket.reserve(sizeof(int) * (size_t)nb * KK_NLIST);
  e.npp.reserve(sizeof(int) * (size_t)nb * 2);  // fb + fp64 lists
  KK_CUDA(cudaMemsetAsync(e.counters.p, 0, sizeof(int) * KK_CNT_N, st));
  KK_CUDA(cudaMemsetAsync(e.status.p, 0, sizeof(int) * nb, st));
  int* redo = e.npp.as<int>();  // reuse the fallback list storage for search redo lists

  // ---- neighbour search per variable
  int mm_total = 0;
  for (int v = 0; v < nv; ++v) {
    VarDevice& d = e.vd[v];
    KkSearch& S = d.search;
    d.nbr.reserve(sizeof(int) * (size_t)nb * std::max(S.mmax, 1));
    d.nnear.reserve(sizeof(int) * nb);
    mm_total += S.mmax;
    const double* tx[4] = {e.tx[0].as<double>(), e.tx[1].as<double>(), e.tx[2].as<double>(), e.tx[3].as<double>()};
    const double* ox[4] = {d.x[0].as<double>(), d.x[1].as<double>(), d.x[2].as<double>(), d.x[3].as<double>()};
    if (e.sim_nobs >= 0) {
      // the systems of a sequential simulation: every target searches the
      // observations and the targets visited before it (exact kd-tree order)
      if (S.mode != 0 && !d.tree_ready) build_tree(e, v);
      // a thread per target up to the heap memory of 262 144 threads (one
      // round: a second round on part of the threads doubles the launch)
      const int stride = (S.mode == 2 ? S.K : S.nmax) + 2;
      const long long cap = std::max(32768LL, (long long)((size_t(1) << 30) / (kd_heap_entry_bytes() * stride)));
      const int nthreads = (int)std::max(1LL, std::min<long long>({(long long)nb, 262144LL, cap}));
      DBuf heaps;
      heaps.reserve(kd_heap_entry_bytes() * (size_t)stride * nthreads);
      timer.start();
      launch_search_sgsim(S, nb, e.sim_nobs, tx, ox, d.nbr.as<int>(), d.nnear.as<int>(), heaps.p, stride,
                          nthreads, st);
      KK_CUDA(cudaGetLastError());
      timer.stop(0);
      e.launches += 1;
      KK_CUDA(cudaStreamSynchronize(st));
      continue;
    }
    KK_CUDA(cudaMemsetAsync(e.counters.as<int>() + KK_CNT_REDO + v, 0, sizeof(int), st));
    timer.start();
    launch_search(S, nb, tx, ox, d.nbr.as<int>(), d.nnear.as<int>(), e.status.as<int>(), redo,
                  e.counters.as<int>() + KK_CNT_REDO + v, nsm, st);
    KK_CUDA(cudaGetLastError());
    timer.stop(0);
    e.launches += 1;
    int nredo = 0;
    KK_CUDA(cudaMemcpyAsync(&nredo, e.counters.as<int>() + KK_CNT_REDO + v, sizeof(int), cudaMemcpyDeviceToHost, st));
    KK_CUDA(cudaStreamSynchronize(st));
    e.stats[5] += nredo;
    if (nredo > 0) {
      if (!d.tree_ready) build_tree(e, v);
      const int nthreads = std::min(nredo, 32768);
      const int stride = S.K + 2;
      DBuf heaps;
      heaps.reserve(kd_heap_entry_bytes() * (size_t)stride * nthreads);
      timer.start();
      launch_search_kdtree(S, redo, e.counters.as<int>() + KK_CNT_REDO + v, tx, ox, d.nbr.as<int>(),
                           d.nnear.as<int>(), e.status.as<int>(), heaps.p, stride, nthreads, st);
      KK_CUDA(cudaGetLastError());
      timer.stop(3);
      e.launches += 1;
      KK_CUDA(cudaStreamSynchronize(st));
    }
  }
  e.mmax_total = mm_total;

  // ---- solve parameters
  SolveParams P;
  fill_params(e, P);
  // fast covariance paths of single-variable spatial kriging (with several
  // variables vgm(i, j), i > j, has no table and is evaluated analytically,
  // as in the reference: the general path)
  P.fast_model = 0;
  if (!e.st && nv == 1 && mdl[0].mode == KK_LEVEL_B) {
    P.fast_model = 1;
    for (int k = 0; k < 9; ++k) P.fm[k] = mdl[0].bmat[k];
    P.fm_ndim = mdl[0].ndim;
    P.fm_tail = mdl[0].btail;
    P.fm_tab_off = mdl[0].btab_off;
  } else if (!e.st && nv == 1 && mdl[0].mode == KK_LEVEL_A && mdl[0].nstruct >= 1 &&
             mdl[0].nstruct <= KK_FA_MAXS) {
    // Level A with every structure's transform a multiple k of one matrix
    // (structures that differ only in range): h_s = k_s * |B lag|
    const KkModel& m = mdl[0];
    const KkComp& c0 = m.comp[0];
    int big = 0;
    for (int q = 1; q < 9; ++q)
      if (std::fabs(c0.mat[q]) > std::fabs(c0.mat[big])) big = q;
    bool ok = c0.mat[big] != 0.0;
    P.fa_nst = m.nstruct;
    P.fa_tailmask = 0;
    for (int s = 0; s < m.nstruct && ok; ++s) {
      const KkComp& c = m.comp[s];
      const double k = c.mat[big] / c0.mat[big];
      ok = !c.is_product && c.tab_off >= 0 && k > 0.0;
      for (int r = 0; r < 9 && ok; ++r) ok = std::fabs(c.mat[r] - k * c0.mat[r]) <= 1e-12 * std::fabs(c.mat[big]);
      P.fa_off[s] = c.tab_off;
      P.fa_k[s] = k;
      if (c.tail) P.fa_tailmask |= 1 << s;
    }
    if (ok) {
      P.fast_model = 2;
      for (int k = 0; k < 9; ++k) P.fm[k] = c0.mat[k];
      P.fm_ndim = m.ndim;
    }
  } else if (e.st && nv == 1 && smdl[0].cs.mode == KK_LEVEL_B && smdl[0].ct.mode == KK_LEVEL_B &&
             (smdl[0].model == 1 || !smdl[0].has_joint)) {
    // space-time: spatial and temporal Level-B tables combined as product-sum
    // (or sum-metric without joint sills), like the general st_cov
    const KkSTModel& sm = smdl[0];
    P.fast_model = 4;
    for (int k = 0; k < 9; ++k) P.fm[k] = sm.cs.bmat[k];
    P.fm_ndim = sm.cs.ndim;
    P.fm_tail = sm.cs.btail;
    P.fm_tab_off = sm.cs.btab_off;
    P.ft_k = sm.ct.bmat[0];
    P.ft_off = sm.ct.btab_off;
    P.ft_tail = sm.ct.btail;
    P.st_kind = sm.model;
    P.st_kps = sm.k_ps;
  } else if (!e.st && nv == 2) {
    // two variables whose structures all have transforms k * B (structures
    // that differ only in range and sill, as in a linear model of
    // coregionalisation): per pair a Level-B table, Level-A tables, or (for
    // vgm(i, j), i > j) the analytic structures, each at h_s = k_s * |B lag|
    const KkComp& c0 = mdl[0].comp[0];
    int big = 0;
    for (int q = 1; q < 9; ++q)
      if (std::fabs(c0.mat[q]) > std::fabs(c0.mat[big])) big = q;
    bool ok = c0.mat[big] != 0.0;
    auto mult = [&](const double* mat, double& k) {
      k = mat[big] / c0.mat[big];
      bool good = k > 0.0;
      for (int r = 0; r < 9 && good; ++r) good = std::fabs(mat[r] - k * c0.mat[r]) <= 1e-12 * std::fabs(mat[big]);
      return good;
    };
    for (int q = 0; q < 4 && ok; ++q) {
      const KkModel& m = mdl[q];
      ok = m.ndim == mdl[0].ndim && m.nstruct >= 1 && m.nstruct <= KK_FA_MAXS;
      for (int s = 0; s < m.nstruct && ok; ++s) {
        double k;
        ok = !m.comp[s].is_product && mult(m.comp[s].mat, k);
      }
      if (!ok) break;
      P.fq_tail[q] = 0;
      if (m.mode == KK_LEVEL_B) {
        P.fq_kind[q] = 1;
        P.fq_nst[q] = 1;
        P.fq_off[q][0] = m.btab_off;
        ok = mult(m.bmat, P.fq_k[q][0]);
        if (m.btail) P.fq_tail[q] = 1;
      } else {
        P.fq_kind[q] = m.mode == KK_LEVEL_A ? 2 : 3;
        P.fq_nst[q] = m.nstruct;
        for (int s = 0; s < m.nstruct && ok; ++s) {
          const KkComp& c = m.comp[s];
          mult(c.mat, P.fq_k[q][s]);
          P.fq_off[q][s] = c.tab_off;
          if (P.fq_kind[q] == 2) ok = c.tab_off >= 0;
          if (c.tail) P.fq_tail[q] |= 1 << s;
        }
      }
    }
    if (ok) {
      P.fast_model = 3;
      for (int k = 0; k < 9; ++k) P.fm[k] = c0.mat[k];
      P.fm_ndim = mdl[0].ndim;
    }
  }

  // ---- bucket by neighbour count
  timer.start();
  launch_bucket(P, e.bucket.as<int>(), st);
  timer.stop(1);
  e.launches += 1;
  int cb[KK_CNT_N];
  KK_CUDA(cudaMemcpyAsync(cb, e.counters.p, sizeof cb, cudaMemcpyDeviceToHost, st));
  KK_CUDA(cudaStreamSynchronize(st));
  // ---- solve: per chunk of a bucket list, the assembly kernel writes packed
  // K64 to kbuf, then the factorisation kernel reads it
  if (e.store_weight) {
    // the weight store is filled by the FP64 form and the general kernel
    e.wstride = mm_total;
    for (int v = 0; v < nv; ++v) e.wmmax[v] = P.mmax[v];
    e.wbuf.reserve(sizeof(double) * (size_t)nb * nv * std::max(mm_total, 1));
    P.wout = e.wbuf.as<double>();
    P.wstride = mm_total;
  }
  const int rform = (e.store_weight || !solve_refine_form(P, e.precision)) ? 0 : e.precision;
  const int mtot = mm_total + P.pa;
  const size_t gstride = generic_stride(mtot, nv, P.pa);
  // threads of the general kernel for a list of count targets: one target
  // each at a time, as many as a 4 GiB workspace holds (at least 2 048, a
  // multiple of 64, at most 65 536)
  const int gen_cap = (int)std::max<size_t>(
      2048, std::min<size_t>(65536, ((size_t)4 << 30) / (sizeof(double) * gstride)) / 64 * 64);
  auto gen_threads = [&](int count) { return std::max(1, std::min(count, gen_cap)); };
  auto generic_scratch = [&](int nthreads) {
    e.scratch.reserve(sizeof(double) * gstride * gen_threads(nthreads));
    P.scratch = e.scratch.as<double>();
    P.scratch_stride = (int)gstride;
  };
  // one chunk of a list: assembly into kbuf, then the factorisation kernel
  // (each timed on its own when profiling)
  PhaseTimer ktimer(e);
  auto run_list = [&](const int* list, int count, int N, int form, int slot) {
    const int ch = chunk_targets(N);
    if (count > 0) e.kbuf.reserve(std::max(e.kbuf.bytes, kbuf_bytes(N, std::min(ch, count))));
    for (int c0 = 0; c0 < count; c0 += ch) {
      const int nit = std::min(ch, count - c0);
      KK_CUDA(cudaMemsetAsync(e.counters.as<int>() + slot, 0, sizeof(int), st));
      ktimer.start();
      launch_assemble(P, N, list, nullptr, c0, nit, e.kbuf.as<double>(), nsm, st);
      ktimer.stop(4);
      ktimer.start();
      launch_factor(P, form, N, list, nullptr, c0, nit, e.kbuf.as<double>(), slot, nsm, st);
      ktimer.stop(5);
      KK_CUDA(cudaGetLastError());
      e.launches += 2;
    }
  };
  // the first count entries of a list on one kernel (the tuner's runs)
  auto run_kernel = [&](int ker, const int* list, int count, int slot) {
    if (ker == KK_KER_GEN) {
      generic_scratch(count);
      KK_CUDA(cudaMemcpyAsync(e.counters.as<int>() + KK_CNT_TUNE, &count, sizeof(int), cudaMemcpyHostToDevice, st));
      launch_solve_generic(P, list, KK_CNT_TUNE, gen_threads(count), st);
      KK_CUDA(cudaGetLastError());
      e.launches += 1;
    } else {
      run_list(list, count, kernel_rows(ker), kernel_form(ker), slot);
    }
  };
  // ---- kernel per neighbour-count list: fixed, or chosen by timing the
  // candidates on a sample of the list (cached per system signature)
  const bool wide = wide_columns(P);
  int* lists = e.bucket.as<int>();
  for (int li = 0; li < KK_NLIST; ++li) {
    const int count = cb[list_slot(li)];
    e.plan[li] = count > 0 ? default_kernel(li, wide, e.store_weight != 0, rform) : -1;
    for (int k = 0; k < KK_NKER; ++k) e.plan_us[li][k] = NAN;
    int cand[KK_NKER];
    const int nc = candidates(li, wide, e.store_weight != 0, rform, cand);
    if (count <= 0 || nc < 2 || !e.autotune) continue;
    const TuneKey key = tune_key(P, li, rform, e.st, count);
    TuneEntry hit;
    if (e.autotune == 1 && tune_find(key, hit)) {
      e.plan[li] = hit.kernel;
      for (int k = 0; k < KK_NKER; ++k) e.plan_us[li][k] = hit.us[k];
      continue;
    }
    if (count < KK_TUNE_MIN) continue;
    // the candidates' side effects (status bits, fallback lists, counters)
    // are rolled back; the chosen kernel then solves the whole list
    const int ns = std::min(count, KK_TUNE_SAMPLE);
    int saved[KK_CNT_N];
    KK_CUDA(cudaMemcpyAsync(saved, e.counters.p, sizeof saved, cudaMemcpyDeviceToHost, st));
    KK_CUDA(cudaStreamSynchronize(st));
    // the fallback lists hold nb entries: each run below appends at most ns
    // to empty lists, and the counters are put back after every run
    if (saved[KK_CNT_FB] != 0 || saved[KK_CNT_FP64] != 0) continue;
    auto restore_counters = [&]() {
      KK_CUDA(cudaMemcpyAsync(e.counters.p, saved, sizeof saved, cudaMemcpyHostToDevice, st));
    };
    e.tunebuf.reserve(sizeof(int) * (size_t)nb);
    KK_CUDA(cudaMemcpyAsync(e.tunebuf.p, P.status, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToDevice, st));
    // buffers for the largest candidate first: no allocation inside a timing
    for (int c = 0; c < nc; ++c) {
      if (cand[c] == KK_KER_GEN) {
        generic_scratch(ns);
      } else {
        const int rows = kernel_rows(cand[c]);
        e.kbuf.reserve(std::max(e.kbuf.bytes, kbuf_bytes(rows, std::min(chunk_targets(rows), ns))));
      }
    }
    const int* l = lists + (size_t)li * nb;
    for (int c = 0; c < nc; ++c) {  // first launches (module loading) outside the timing
      run_kernel(cand[c], l, std::min(ns, 256), KK_CNT_WORK0 + 3);
      restore_counters();
    }
    cudaEvent_t ev[2];
    KK_CUDA(cudaEventCreate(&ev[0]));
    KK_CUDA(cudaEventCreate(&ev[1]));
    TuneEntry ent;
    ent.kernel = cand[0];
    for (int k = 0; k < KK_NKER; ++k) ent.us[k] = NAN;
    auto timed = [&](int ker, int count) {  // ms of one run on the first count targets
      KK_CUDA(cudaEventRecord(ev[0], st));
      run_kernel(ker, l, count, KK_CNT_WORK0 + 3);
      KK_CUDA(cudaEventRecord(ev[1], st));
      KK_CUDA(cudaEventSynchronize(ev[1]));
      float ms = 0.f;
      KK_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      restore_counters();
      return (double)ms;
    };
    // a candidate is timed on a quarter of the sample first and dropped there
    // when it is already more than eight times slower per target than the
    // best (the general kernel against a register kernel: 27-72x)
    const int nq = std::max(std::min(ns, 256), ns / 4);
    double best_us = 0.0;
    for (int c = 0; c < nc; ++c) {
      double us;
      if (c > 0 && nq < ns) {
        us = 1e3 * timed(cand[c], nq) / nq;
        if (us <= 8.0 * best_us) us = 1e3 * timed(cand[c], ns) / ns;
      } else {
        us = 1e3 * timed(cand[c], ns) / ns;
      }
      ent.us[cand[c]] = us;
      if (c == 0 || us < best_us) { best_us = us; ent.kernel = cand[c]; }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    KK_CUDA(cudaMemcpyAsync(P.status, e.tunebuf.p, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToDevice, st));
    KK_CUDA(cudaStreamSynchronize(st));
    e.tunebuf.release();
    tune_store(key, ent);
    e.plan[li] = ent.kernel;
    for (int k = 0; k < KK_NKER; ++k) e.plan_us[li][k] = ent.us[k];
  }
  if (e.autotune == 2) e.autotune = 1;
  timer.start();
  for (int li = 0; li < KK_NLIST; ++li) {
    if (e.plan[li] < 0 || e.plan[li] == KK_KER_GEN) continue;
    run_list(lists + (size_t)li * nb, cb[list_slot(li)], kernel_rows(e.plan[li]), kernel_form(e.plan[li]),
             KK_CNT_WORK0 + li);
  }
  timer.stop(2);
  bool any_r = false;
  for (int li = 0; li < KK_NLIST; ++li) any_r = any_r || (e.plan[li] >= 0 && kernel_form(e.plan[li]));
  if (any_r) {
    // targets whose FP32 factorisation failed or whose correction check did
    // not pass: FP64 form (they come from the lists of at most 64 equations)
    int nf = 0;
    KK_CUDA(cudaMemcpyAsync(&nf, e.counters.as<int>() + KK_CNT_FP64, sizeof(int), cudaMemcpyDeviceToHost, st));
    KK_CUDA(cudaStreamSynchronize(st));
    if (nf > 0) {
      timer.start();
      run_list(P.fp64_list, nf, 64, 0, KK_CNT_WORK0 + 4);
      timer.stop(3);
    }
  }
  int cnt[KK_CNT_N];
  KK_CUDA(cudaMemcpyAsync(cnt, e.counters.p, sizeof cnt, cudaMemcpyDeviceToHost, st));
  KK_CUDA(cudaStreamSynchronize(st));
  // general kernel: the lists planned on it (more than 128 equations, wide
  // systems, weight store) and Cholesky failures (LDL^T + jitter)
  int ngen = cnt[KK_CNT_FB];
  for (int li = 0; li < KK_NLIST; ++li)
    if (e.plan[li] == KK_KER_GEN) ngen = std::max(ngen, cnt[list_slot(li)]);
  if (ngen > 0) {
    generic_scratch(ngen);
    timer.start();
    for (int li = 0; li < KK_NLIST; ++li) {
      const int c = cnt[list_slot(li)];
      if (e.plan[li] != KK_KER_GEN || c <= 0) continue;
      launch_solve_generic(P, lists + (size_t)li * nb, list_slot(li), gen_threads(c), st);
      e.launches += 1;
    }
    if (cnt[KK_CNT_FB] > 0) {
      launch_solve_generic(P, P.fb_list, KK_CNT_FB, gen_threads(cnt[KK_CNT_FB]), st);
      e.launches += 1;
    }
    KK_CUDA(cudaGetLastError());
    timer.stop(3);
    KK_CUDA(cudaMemcpyAsync(cnt, e.counters.p, sizeof cnt, cudaMemcpyDeviceToHost, st));
    KK_CUDA(cudaStreamSynchronize(st));
  }
  // solver_stats: fail, chol_fact, chol_reuse, ssytrf_fact, ssytrf_reuse
  e.stats[0] = cnt[KK_CNT_FAIL];
  e.stats[1] = cnt[KK_CNT_CHOL];
  e.stats[2] = 0;
  e.stats[3] = cnt[KK_CNT_LDLT];
  e.stats[4] = 0;
  e.stats[6] = cnt[KK_CNT_FP64];
  e.stats[7] = cnt[KK_CNT_ITER];
  std::memcpy(e.counters_last, cnt, sizeof cnt);
  if (!e.neglect_error && cnt[KK_CNT_FAIL] > 0) throw std::string("Singular matrix or no neighbours at a block");
  if (e.store_weight) {
    e.wstore_dev = true;
    e.wstore_host = false;
  }
  indicator_post(e);
  e.solved = true;
  e.last_solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void engine_resolve_static(Engine& e, int ivar, int nobs, const double* value) {
  // Everything below works in buffers the last krige_solve left behind: no
  // DBuf::reserve, no allocator callback, no cudaMalloc.
  if (!e.solved) throw std::string("krige_resolve_static needs a completed krige_solve on this handle");
  if (e.grid_dirty) throw std::string("targets changed since the last krige_solve; call krige_solve");
  for (int v = 0; v < e.nvar; ++v)
    if (e.obs[v].dirty || e.obs[v].search_dirty)
      throw std::string("observations or search changed since the last krige_solve; call krige_solve");
  if (value) {
    if (ivar < 1 || ivar > e.nvar) throw std::string("ivar out of range");
    if (nobs != e.obs[ivar - 1].n) throw std::string("size(value) /= obs%n");
  }
  // Every check comes before the first change of state, so a rejected call
  // leaves the handle's values and results as they were.
  static_fit_check(e.mmax_total + e.pdrift(), e.nvar, e.pdrift());
  // the variogram may have been reset since the last solve: rebuild the
  // models on the host and copy them into the existing buffers when they fit
  std::vector<KkModel> mdl;
  std::vector<KkSTModel> smdl;
  std::vector<double2> tabs;
  build_models(e, mdl, smdl, tabs);
  if (tabs.empty()) tabs.push_back(make_double2(0.0, 0.0));
  const size_t tb = sizeof(double2) * tabs.size();
  const size_t mb = e.st ? sizeof(KkSTModel) * smdl.size() : sizeof(KkModel) * mdl.size();
  if (tb > e.tables.bytes || mb > e.models.bytes)
    throw std::string("the variogram tables outgrew the buffers of the last krige_solve; call krige_solve");
  // the grid drift may have been replaced by krige_set_grid_drift since the
  // last solve (same size: it is tied to the targets)
  const size_t db = sizeof(double) * e.bdrift.size();
  if (e.ndrift > 0 && db > e.tdrift.bytes)
    throw std::string("the grid drift outgrew the buffer of the last krige_solve; call krige_solve");
  KK_CUDA(cudaSetDevice(e.device));
  cudaStream_t st = e.stream;
  e.solved = false;
  set_zones(st);
  KK_CUDA(cudaMemcpyAsync(e.tables.p, tabs.data(), tb, cudaMemcpyHostToDevice, st));
  KK_CUDA(cudaMemcpyAsync(e.models.p, e.st ? (const void*)smdl.data() : (const void*)mdl.data(), mb,
                          cudaMemcpyHostToDevice, st));
  if (e.ndrift > 0 && db > 0) KK_CUDA(cudaMemcpyAsync(e.tdrift.p, e.bdrift.data(), db, cudaMemcpyHostToDevice, st));
  if (value) {
    ObsVar& o = e.obs[ivar - 1];
    std::copy(value, value + nobs, o.value.begin());
    KK_CUDA(cudaMemcpyAsync(e.vd[ivar - 1].value.p, o.value.data(), sizeof(double) * nobs,
                            cudaMemcpyHostToDevice, st));
  }
  SolveParams P;
  fill_params(e, P);
  int cnt[KK_CNT_N];
  solve_generic_static(P, e.device, st, e.mmax_total + P.pa, cnt);
  std::memset(e.stats, 0, sizeof e.stats);
  e.stats[0] = cnt[KK_CNT_FAIL];
  e.stats[1] = cnt[KK_CNT_CHOL];
  e.stats[3] = cnt[KK_CNT_LDLT];
  std::memcpy(e.counters_last, cnt, sizeof cnt);
  for (double& x : e.phase_ms) x = 0.0;
  e.launches = 2 * ((e.nblock + KK_STATIC_CHUNK - 1) / KK_STATIC_CHUNK);
  if (!e.neglect_error && cnt[KK_CNT_FAIL] > 0) throw std::string("Singular matrix or no neighbours at a block");
  e.solved = true;
}

// Neighbour-list length of every variable as the next solve would set it
// (set_search must have been called for the search mode; the default is the
// plain k-nearest search).
static void list_lengths(Engine& e, int* mm) {
  for (int v = 0; v < e.nvar; ++v) {
    KkSearch S;
    setup_search(e, v, S);
    mm[v] = std::max(S.mmax, 1);
  }
}

int engine_weight_nm(Engine& e) {
  int mm[KK_MAXVAR] = {0, 0, 0, 0};
  if (e.wstore_dev || e.wstore_host) std::memcpy(mm, e.wmmax, sizeof mm);
  else list_lengths(e, mm);
  int nm = 0;
  for (int v = 0; v < e.nvar; ++v) nm = std::max(nm, mm[v]);
  return nm;
}

// Estimates from the weight store (use_old_weight): the observation values
// of every variable are uploaded (update_obs_value may have replaced them),
// a store staged by set_weights is uploaded once, then one gather-dot kernel
// writes the estimates; the variances are the store's.
static void engine_replay(Engine& e) {
  if (!e.wstore_dev && !e.wstore_host)
    throw std::string("use_old_weight with no weight_file requires set_weights() to be called first.");
  if (e.nblock <= 0) throw std::string("Call set_grid() before solve().");
  for (int v = 0; v < e.nvar; ++v)
    if (e.obs[v].n == 0) throw std::string("Call set_obs() for every variable before solve().");
  KK_CUDA(cudaSetDevice(e.device));
  cudaStream_t st = e.stream;
  const int nb = e.nblock, nv = e.nvar;
  for (int v = 0; v < nv; ++v)
    upload(e.vd[v].value, e.obs[v].value.data(), sizeof(double) * e.obs[v].n, st);
  e.est.reserve(sizeof(double) * (size_t)nb * nv);
  e.var.reserve(sizeof(double) * (size_t)nb * nv * nv);
  e.status.reserve(sizeof(int) * nb);
  if (e.wstore_host) {
    const int ng = nv, nm = e.wh_nm;
    std::vector<int> nn((size_t)nb), nbr;
    std::vector<double> w((size_t)nb * nv * e.wstride, 0.0);
    std::vector<int> ist((size_t)nb * nv, 0);
    for (int ib = 0; ib < nb; ++ib)
      for (int v = 1; v < nv; ++v)
        ist[(size_t)ib * nv + v] = ist[(size_t)ib * nv + v - 1] + e.wh_nnear[(size_t)(v - 1) + (size_t)ng * ib];
    for (int v = 0; v < nv; ++v) {
      const int mm = e.wmmax[v];
      nbr.assign((size_t)nb * mm, 0);
      for (int ib = 0; ib < nb; ++ib) {
        const int k = e.wh_nnear[(size_t)v + (size_t)ng * ib];
        nn[ib] = k;
        for (int i = 0; i < k; ++i) {
          nbr[(size_t)ib * mm + i] = e.wh_inear[(size_t)i + (size_t)nm * (v + (size_t)ng * ib)] - 1;
          for (int jv = 0; jv < nv; ++jv)
            w[((size_t)ib * nv + jv) * e.wstride + ist[(size_t)ib * nv + v] + i] =
                e.wh_weight[(size_t)i + (size_t)nm * (v + (size_t)ng * (jv + (size_t)nv * ib))];
        }
      }
      upload(e.vd[v].nnear, nn.data(), sizeof(int) * nb, st);
      upload(e.vd[v].nbr, nbr.data(), sizeof(int) * nbr.size(), st);
      KK_CUDA(cudaStreamSynchronize(st));
    }
    upload(e.wbuf, w.data(), sizeof(double) * w.size(), st);
    // variance(nvar, nvar, nblock) -> per target [iv + jv nvar]
    std::vector<double> vv((size_t)nb * nv * nv);
    for (int ib = 0; ib < nb; ++ib)
      for (int jv = 0; jv < nv; ++jv)
        for (int iv = 0; iv < nv; ++iv)
          vv[((size_t)ib * nv + jv) * nv + iv] = e.wh_var[(size_t)iv + (size_t)nv * (jv + (size_t)nv * ib)];
    KK_CUDA(cudaMemcpyAsync(e.var.p, vv.data(), sizeof(double) * vv.size(), cudaMemcpyHostToDevice, st));
    KK_CUDA(cudaMemsetAsync(e.status.p, 0, sizeof(int) * nb, st));
    KK_CUDA(cudaStreamSynchronize(st));
    e.wstore_host = false;
    e.wstore_dev = true;
    e.wh_nnear.clear(); e.wh_inear.clear(); e.wh_weight.clear(); e.wh_var.clear();
  }
  SolveParams P;
  std::memset(&P, 0, sizeof P);
  P.nvar = nv;
  P.nblock = nb;
  P.unbias = e.unbias;
  P.ck_isa = (!e.std_ck && e.unbias != 0 && nv > 1) ? 1 : 0;
  P.bounds[0] = e.bounds[0];
  P.bounds[1] = e.bounds[1];
  for (int v = 0; v < nv; ++v) {
    P.sk_mean[v] = e.obs[v].sk_mean;
    P.oval[v] = e.vd[v].value.as<double>();
    P.nbr[v] = e.vd[v].nbr.as<int>();
    P.nnear[v] = e.vd[v].nnear.as<int>();
    P.mmax[v] = e.wmmax[v];
    P.nobs[v] = e.obs[v].n;
  }
  P.est = e.est.as<double>();
  P.var = e.var.as<double>();
  P.status = e.status.as<int>();
  P.wout = e.wbuf.as<double>();
  P.wstride = e.wstride;
  launch_replay(P, sm_count(e.device), st);
  KK_CUDA(cudaGetLastError());
  KK_CUDA(cudaStreamSynchronize(st));
  e.launches = 1;
  indicator_post(e);
  std::memset(e.counters_last, 0, sizeof e.counters_last);
  e.solved = true;
}

void engine_set_weights(Engine& e, int nm, int ng, int nv, int nb, const int* nnear, const int* inear,
                        const double* weight, const double* var) {
  if (e.obs.empty() || e.obs[0].n == 0) throw std::string("call set_obs() before set_weights() so nmax is set");
  if (nb != e.nblock || ng != e.nvar) throw std::string("nnear shape mismatch");
  int mm[KK_MAXVAR] = {0, 0, 0, 0};
  list_lengths(e, mm);
  int nmx = 0;
  for (int v = 0; v < e.nvar; ++v) nmx = std::max(nmx, mm[v]);
  if (nm != nmx) throw std::string("inear shape mismatch");
  if (nv != e.nvar) throw std::string("weight shape mismatch");
  for (int ib = 0; ib < nb; ++ib)
    for (int v = 0; v < ng; ++v) {
      const int k = nnear[(size_t)v + (size_t)ng * ib];
      if (k < 0 || k > mm[v]) throw std::string("nnear exceeds the neighbour-list length of its variable");
      for (int i = 0; i < k; ++i) {
        const int o = inear[(size_t)i + (size_t)nm * (v + (size_t)ng * ib)];
        if (o < 1 || o > e.obs[v].n) throw std::string("inear holds an index outside 1..nobs");
      }
    }
  e.wh_nm = nm;
  e.wh_nnear.assign(nnear, nnear + (size_t)ng * nb);
  e.wh_inear.assign(inear, inear + (size_t)nm * ng * nb);
  e.wh_weight.assign(weight, weight + (size_t)nm * ng * nv * nb);
  if (var) e.wh_var.assign(var, var + (size_t)nv * nv * nb);
  else e.wh_var.assign((size_t)nv * nv * nb, 0.0);
  std::memcpy(e.wmmax, mm, sizeof mm);
  e.wstride = 0;
  for (int v = 0; v < e.nvar; ++v) e.wstride += mm[v];
  e.wstore_host = true;
  e.wstore_dev = false;
  e.use_old_weight = 1;
  e.solved = false;
}

void engine_get_weights(Engine& e, int nm, int ng, int nv, int nb, int* nnear, int* inear, double* weight,
                        double* var) {
  if (!e.wstore_dev && !e.wstore_host) throw std::string("Weight store not allocated. Set store_weight=True.");
  if (nb != e.nblock || ng != e.nvar || nv != e.nvar || nm != engine_weight_nm(e))
    throw std::string("weight store dimensions do not match the buffers");
  if (e.wstore_host) {
    if (nnear) std::copy(e.wh_nnear.begin(), e.wh_nnear.end(), nnear);
    if (inear) std::copy(e.wh_inear.begin(), e.wh_inear.end(), inear);
    if (weight) std::copy(e.wh_weight.begin(), e.wh_weight.end(), weight);
    if (var) std::copy(e.wh_var.begin(), e.wh_var.end(), var);
    return;
  }
  KK_CUDA(cudaSetDevice(e.device));
  cudaStream_t st = e.stream;
  std::vector<std::vector<int>> nn(nv), nbr(nv);
  for (int v = 0; v < nv; ++v) {
    nn[v].resize(nb);
    KK_CUDA(cudaMemcpyAsync(nn[v].data(), e.vd[v].nnear.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
    if (inear || weight) {
      nbr[v].resize((size_t)nb * e.wmmax[v]);
      KK_CUDA(cudaMemcpyAsync(nbr[v].data(), e.vd[v].nbr.p, sizeof(int) * nbr[v].size(), cudaMemcpyDeviceToHost, st));
    }
  }
  std::vector<double> w;
  if (weight) {
    w.resize((size_t)nb * nv * e.wstride);
    KK_CUDA(cudaMemcpyAsync(w.data(), e.wbuf.p, sizeof(double) * w.size(), cudaMemcpyDeviceToHost, st));
  }
  std::vector<double> vv;
  if (var) {
    vv.resize((size_t)nb * nv * nv);
    KK_CUDA(cudaMemcpyAsync(vv.data(), e.var.p, sizeof(double) * vv.size(), cudaMemcpyDeviceToHost, st));
  }
  KK_CUDA(cudaStreamSynchronize(st));
  // unused slots are zero (test_weight_store.py: padding checks)
  if (inear) std::fill(inear, inear + (size_t)nm * ng * nb, 0);
  if (weight) std::fill(weight, weight + (size_t)nm * ng * nv * nb, 0.0);
  for (int ib = 0; ib < nb; ++ib) {
    int ist = 0;
    for (int v = 0; v < ng; ++v) {
      const int k = nn[v][ib];
      if (nnear) nnear[(size_t)v + (size_t)ng * ib] = k;
      for (int i = 0; i < k; ++i) {
        if (inear) inear[(size_t)i + (size_t)nm * (v + (size_t)ng * ib)] = nbr[v][(size_t)ib * e.wmmax[v] + i] + 1;
        if (weight)
          for (int jv = 0; jv < nv; ++jv)
            weight[(size_t)i + (size_t)nm * (v + (size_t)ng * (jv + (size_t)nv * ib))] =
                w[((size_t)ib * nv + jv) * e.wstride + ist + i];
      }
      ist += k;
    }
    if (var)
      for (int jv = 0; jv < nv; ++jv)
        for (int iv = 0; iv < nv; ++iv)
          var[(size_t)iv + (size_t)nv * (jv + (size_t)nv * ib)] = vv[((size_t)ib * nv + jv) * nv + iv];
  }
}

void engine_free_weight_store(Engine& e) {
  e.wbuf.release();
  e.wh_nnear.clear(); e.wh_inear.clear(); e.wh_weight.clear(); e.wh_var.clear();
  e.wstore_dev = false;
  e.wstore_host = false;
  e.use_old_weight = 0;
}

// ---------------------------------------------------------------------------
// sequential Gaussian simulation (nsim > 0)
// ---------------------------------------------------------------------------
// set_sim_base without a path or samples (kriging_base.F90:1255-1300): a
// random visiting order and N(0, 1) draws.  The reference draws them with its
// own generator and writes them to sgs_path.dat / sgs_sample.dat; here they
// come from a 64-bit Mersenne twister seeded by initialize's seed (a random
// seed when it is 0) and stay in memory, so a given seed repeats its
// realisations but does not repeat the reference's.
void engine_sim_defaults(Engine& e, bool path, bool sample) {
  const int nb = e.nblock;
  std::mt19937_64 rng(e.seed != 0 ? (uint64_t)(int64_t)e.seed : (uint64_t)std::random_device{}());
  if (path) {
    e.sim_path.resize(nb);
    for (int i = 0; i < nb; ++i) e.sim_path[i] = i + 1;
    std::shuffle(e.sim_path.begin(), e.sim_path.end(), rng);
  }
  if (sample) {
    std::normal_distribution<double> nd(0.0, 1.0);
    e.sim_sample.resize((size_t)nb * e.nsim * e.nvar);
    for (auto& x : e.sim_sample) x = nd(rng);
  }
}

// The simulation (solve_base with nsim > 0, kriging_base.F90:2055-2181): an
// internal engine holds the observations followed by the targets in visiting
// order and solves every target's system at once, with the search limited to
// the observations and the targets visited before it and the weights kept;
// then the values are drawn level by level (k_sgsim_level).
static void engine_sgsim(Engine& e) {
  auto t0 = std::chrono::steady_clock::now();
  for (double& x : e.phase_ms) x = 0.0;
  e.launches = 0;
  if (e.nvar != 1)
    throw std::string("sequential simulation of several variables (joint co-simulation) is not supported by the "
                      "GPU library; simulate one variable");
  if (e.st) throw std::string("space-time sequential simulation is not supported by the GPU library");
  if (!e.nblockpnt.empty()) throw std::string("sequential simulation needs point targets (set_grid)");
  if (e.store_weight || e.use_old_weight) throw std::string("the weight store is not used with sequential simulation");
  if (e.obs.empty() || e.obs[0].n == 0) throw std::string("Observations need to be set first.");
  if (e.nblock == 0) throw std::string("Grid needs to be set first.");
  ObsVar& o = e.obs[0];
  if (o.sector && !(o.nmax > 0 && o.nmax < o.n + e.nblock))
    throw std::string("sector search in sequential simulation needs nmax below the number of observations plus "
                      "targets (the search tree exists only then)");
  if (o.nmax > (int)(INT_MAX * 0.001)) throw std::string("`nmax` must be set for all observations for SGSIM.");
  validate(e);
  const int nb = e.nblock, D = e.nlag, nsim = e.nsim, nobs = o.n;
  if ((int)e.sim_path.size() != nb) engine_sim_defaults(e, true, false);
  if (e.sim_sample.size() != (size_t)nb * nsim) engine_sim_defaults(e, false, true);
  {
    std::vector<char> seen(nb, 0);
    for (int p = 0; p < nb; ++p) {
      const int t = e.sim_path[p];
      if (t < 1 || t > nb || seen[t - 1]) throw std::string("randpath must be a 1-based permutation of 1..nblocks");
      seen[t - 1] = 1;
    }
  }
  const double* bc = e.bcoord_staged ? static_cast<const double*>(e.hstage) : e.bcoord.data();
  cudaStream_t st = e.stream;
  KK_CUDA(cudaSetDevice(e.device));
  const int nsm = sm_count(e.device);

  // ---- the systems: observations + targets in visiting order, weights kept
  Engine s;
  struct Release {
    Engine& x;
    ~Release() { engine_release(x); }
  } release{s};
  s.ndim = e.ndim;
  s.nlag = e.nlag;
  s.nvar = 1;
  s.ndrift = e.ndrift;
  s.unbias = e.unbias;
  s.anisotropic_search = e.anisotropic_search;
  s.neglect_error = e.neglect_error;
  s.std_ck = e.std_ck;
  s.precision = 0;
  s.nmin = e.nmin;
  s.device = e.device;
  s.stream = e.stream;
  s.autotune = e.autotune;
  s.profile = e.profile;
  s.store_weight = 1;
  s.sim_nobs = nobs;
  s.obs.assign(1, o);
  ObsVar& so = s.obs[0];
  so.n = nobs + nb;
  so.coord.resize((size_t)D * so.n);
  for (int p = 0; p < nb; ++p)
    for (int k = 0; k < D; ++k) so.coord[(size_t)(nobs + p) * D + k] = bc[(size_t)(e.sim_path[p] - 1) * D + k];
  so.value.resize(so.n, 0.0);
  so.variance.resize(so.n, 0.0);  // simulated targets carry no measurement error
  const int nd = e.ndrift;
  if (nd > 0) {
    // a simulated member's drift row is the target drift at its node
    // (block%drift in visiting order, kriging.F90:789-794)
    if (e.bdrift.size() != (size_t)nd * nb) throw std::string("Grid drift is not set while ndrift > 0.");
    so.drift.resize((size_t)nd * so.n);
    s.bdrift.resize((size_t)nd * nb);
    for (int p = 0; p < nb; ++p)
      for (int a = 0; a < nd; ++a) {
        const double g = e.bdrift[(size_t)(e.sim_path[p] - 1) * nd + a];
        so.drift[(size_t)(nobs + p) * nd + a] = g;
        s.bdrift[(size_t)p * nd + a] = g;
      }
  }
  so.dirty = true;
  so.search_dirty = true;
  s.vgm[0][0] = e.vgm[0][0];
  s.nblock = nb;
  s.bcoord.resize((size_t)D * nb);
  for (int p = 0; p < nb; ++p)
    for (int k = 0; k < D; ++k) s.bcoord[(size_t)p * D + k] = bc[(size_t)(e.sim_path[p] - 1) * D + k];
  if (!e.rangescale.empty()) {
    s.rangescale.resize(nb);
    for (int p = 0; p < nb; ++p) s.rangescale[p] = e.rangescale[e.sim_path[p] - 1];
  }
  if (!e.localnugget.empty()) {
    s.localnugget.resize(nb);
    for (int p = 0; p < nb; ++p) s.localnugget[p] = e.localnugget[e.sim_path[p] - 1];
  }
  s.grid_dirty = true;
  engine_solve(s);

  // ---- dependency levels: one above the highest level among the target's
  // simulated neighbours (all visited before it, so one pass in visiting order)
  const int mm = std::max(s.vd[0].search.mmax, 1);
  std::vector<int> hn(nb), hl((size_t)nb * mm);
  KK_CUDA(cudaMemcpyAsync(hn.data(), s.vd[0].nnear.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
  KK_CUDA(cudaMemcpyAsync(hl.data(), s.vd[0].nbr.p, sizeof(int) * hl.size(), cudaMemcpyDeviceToHost, st));
  KK_CUDA(cudaStreamSynchronize(st));
  e.sim_mmax = mm;
  e.sim_nn.assign((size_t)nb * 2, 0);
  e.sim_nbr.assign((size_t)nb * mm, 0);
  for (int p = 0; p < nb; ++p) {
    const int t = e.sim_path[p] - 1;
    int no = 0;
    for (int i = 0; i < hn[p]; ++i) no += hl[(size_t)p * mm + i] < nobs;
    e.sim_nn[(size_t)t * 2] = no;
    e.sim_nn[(size_t)t * 2 + 1] = hn[p] - no;
    std::memcpy(&e.sim_nbr[(size_t)t * mm], &hl[(size_t)p * mm], sizeof(int) * hn[p]);
  }
  std::vector<int> lev(nb, 0);
  int nlev = 0;
  for (int p = 0; p < nb; ++p) {
    int L = 0;
    for (int i = 0; i < hn[p]; ++i) {
      const int idx = hl[(size_t)p * mm + i];
      if (idx >= nobs) L = std::max(L, lev[idx - nobs] + 1);
    }
    lev[p] = L;
    nlev = std::max(nlev, L + 1);
  }
  std::vector<int> off((size_t)nlev + 1, 0), order(nb);
  for (int p = 0; p < nb; ++p) off[lev[p] + 1]++;
  for (int L = 0; L < nlev; ++L) off[L + 1] += off[L];
  {
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int p = 0; p < nb; ++p) order[fill[lev[p]]++] = p;
  }

  // ---- the draws, level by level
  DBuf dorder, dpath, dsample, dsim;
  upload(dorder, order.data(), sizeof(int) * nb, st);
  upload(dpath, e.sim_path.data(), sizeof(int) * nb, st);
  upload(dsample, e.sim_sample.data(), sizeof(double) * e.sim_sample.size(), st);
  dsim.reserve(sizeof(double) * (size_t)nsim * nb);
  e.est.reserve(sizeof(double) * (size_t)nb * nsim);
  e.var.reserve(sizeof(double) * nb);
  e.status.reserve(sizeof(int) * nb);
  SimParams SP;
  SP.nbr = s.vd[0].nbr.as<int>();
  SP.nnear = s.vd[0].nnear.as<int>();
  SP.w = s.wbuf.as<double>();
  SP.var = s.var.as<double>();
  SP.z = s.vd[0].value.as<double>();
  SP.sample = dsample.as<double>();
  SP.path = dpath.as<int>();
  SP.sim = dsim.as<double>();
  SP.out = e.est.as<double>();
  SP.nb = nb;
  SP.nobs = nobs;
  SP.nsim = nsim;
  SP.mmax = mm;
  SP.wstride = s.wstride;
  SP.sk = e.unbias == 0 ? 1 : 0;
  SP.sk_mean = o.sk_mean;
  SP.lo = e.bounds[0];
  SP.hi = e.bounds[1];
  PhaseTimer timer(e);
  timer.start();
  // every level in one launch; level by level when the device cannot take a
  // cooperative launch or a wait ran past its limit
  DBuf dflags;
  dflags.reserve(sizeof(int) * ((size_t)nb + 2));
  KK_CUDA(cudaMemsetAsync(dflags.p, 0, sizeof(int) * ((size_t)nb + 2), st));
  int* flags = dflags.as<int>();
  bool flow = !e.sim_by_level && launch_sgsim_flow(SP, dorder.as<int>(), nb, flags, flags + nb, flags + nb + 1, nsm, st);
  int nlaunch = 1;
  if (flow) {
    KK_CUDA(cudaGetLastError());
    int ferr = 0;
    KK_CUDA(cudaMemcpyAsync(&ferr, flags + nb + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    KK_CUDA(cudaStreamSynchronize(st));
    flow = ferr == 0;
  } else {
    cudaGetLastError();
  }
  if (!flow) {
    for (int L = 0; L < nlev; ++L) {
      launch_sgsim_level(SP, dorder.as<int>() + off[L], off[L + 1] - off[L], nsm, st);
      KK_CUDA(cudaGetLastError());
    }
    nlaunch += nlev;
  }
  e.sim_flow = flow ? 1 : 0;
  timer.stop(2);

  // ---- variance and status in target order
  std::vector<double> hv(nb), tv(nb);
  std::vector<int> hs(nb), ts(nb);
  KK_CUDA(cudaMemcpyAsync(hv.data(), s.var.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
  KK_CUDA(cudaMemcpyAsync(hs.data(), s.status.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
  KK_CUDA(cudaStreamSynchronize(st));
  for (int p = 0; p < nb; ++p) {
    tv[e.sim_path[p] - 1] = hv[p];
    ts[e.sim_path[p] - 1] = hs[p];
  }
  upload(e.var, tv.data(), sizeof(double) * nb, st);
  upload(e.status, ts.data(), sizeof(int) * nb, st);
  KK_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < 4; ++i) e.phase_ms[i] += s.phase_ms[i];
  e.phase_ms[4] = s.phase_ms[4];
  e.phase_ms[5] = s.phase_ms[5];
  e.launches += s.launches + nlaunch;
  std::memcpy(e.stats, s.stats, sizeof e.stats);
  std::memcpy(e.counters_last, s.counters_last, sizeof e.counters_last);
  e.counters_last[24] = e.sim_flow;  // host-side slots of krige_gpu_counters
  e.counters_last[25] = nlev;
  for (int li = 0; li < KK_NLIST; ++li) {
    e.plan[li] = s.plan[li];
    for (int k = 0; k < KK_NKER; ++k) e.plan_us[li][k] = s.plan_us[li][k];
  }
  e.sim_levels = nlev;
  e.mmax_total = mm;
  e.solved = true;
  e.last_solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
void engine_release(Engine& e) {
  for (int v = 0; v < KK_MAXVAR; ++v) {
    VarDevice& d = e.vd[v];
    for (auto& b : d.x) b.release();
    d.value.release(); d.variance.release(); d.drift.release();
    d.sc.release(); d.sidx.release(); d.cell_start.release(); d.sat.release(); d.cell_of.release();
    d.cursor.release(); d.tree_i.release(); d.tree_d.release(); d.tree_box.release(); d.tree_ind.release();
    d.tree_rdata.release(); d.nbr.release(); d.nnear.release();
  }
  e.models.release(); e.tables.release();
  for (auto& b : e.tx) b.release();
  for (auto& b : e.gx) b.release();
  e.trs.release(); e.tln.release(); e.tdrift.release(); e.gstart.release(); e.gw.release();
  e.est.release(); e.var.release(); e.status.release(); e.npp.release(); e.bucket.release(); e.tunebuf.release();
  e.counters.release(); e.scratch.release(); e.kbuf.release(); e.til.release(); e.wbuf.release();
  if (e.hstage) cudaFreeHost(e.hstage);
  e.hstage = nullptr;
  e.hstage_bytes = 0;
  if (e.hres) cudaFreeHost(e.hres);
  e.hres = nullptr;
  e.hres_bytes = 0;
}

}  // namespace kk
