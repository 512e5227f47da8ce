// kk_host.h -- host-side engine state behind the krige_* C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cfloat>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "kk_common.h"

#define KK_CNT_N_HOST 32  // = KK_CNT_N (kk_kernels.h)

namespace kk {

// f(lo, hi) over [0, n) in up to eight host threads, pieces of at least
// `grain` items (inline below that): the host-side copies and transposes of
// millions of targets and nodes run at memory rather than single-core speed.
template <class F>
inline void par_for(size_t n, size_t grain, F f) {
  const size_t hc = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>({size_t(8), hc, grain ? n / grain : size_t(1)});
  if (nt <= 1) {
    if (n) f(size_t(0), n);
    return;
  }
  const size_t per = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  for (size_t i = 1; i < nt; ++i) {
    const size_t lo = i * per, hi = std::min(n, lo + per);
    if (lo < hi) th.emplace_back([=] { f(lo, hi); });
  }
  f(size_t(0), std::min(n, per));
  for (auto& t : th) t.join();
}

// memcpy of a large array over threads (a caller's freshly allocated pages
// are first touched here, which one core does at a few GB/s)
inline void par_copy(void* dst, const void* src, size_t bytes) {
  par_for(bytes, size_t(4) << 20, [=](size_t lo, size_t hi) {
    std::memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(src) + lo, hi - lo);
  });
}

struct StructSpec {
  int vtype = KK_SPH;
  double nugget = 0.0, sill = 1.0;
  double a_major = 1.0, a_minor1 = 1.0, a_minor2 = 1.0;
  double az = 0.0, dip = 0.0, plunge = 0.0;
  int is_product = 0;
};

struct ObsVar {
  int n = 0;
  std::vector<double> coord;     // (nlag, n) column-major, as passed to krige_set_obs
  std::vector<double> value, variance, drift;  // drift: (ndrift, n)
  int nmax = INT_MAX;
  double maxdist = DBL_MAX;
  double sk_mean = 0.0;
  bool search_set = false;
  double anis1 = 1.0, anis2 = 1.0, az = 0.0, dip = 0.0, plunge = 0.0, time_at = 1.0;
  int sector = 0;
  bool dirty = true;             // observation data changed since the last upload
  bool search_dirty = true;      // search parameters changed since the last grid build
};

// device buffer owned through the engine allocator
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void reserve(size_t b);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
  ~DBuf() { release(); }
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
};

struct VarDevice {
  DBuf x[4];          // observation coordinates SoA (nlag)
  DBuf value, variance, drift;  // drift SoA: (ndrift) x n
  DBuf sc, sidx, cell_start, sat, cell_of, cursor;
  DBuf tree_i, tree_d, tree_box, tree_ind, tree_rdata;
  DBuf nbr;           // (nblock, mmax) sorted neighbour indices
  DBuf nnear;         // (nblock)
  KkSearch search{};
  bool grid_ready = false;
  bool tree_ready = false;
  long long tree_n = 0;
};

struct Engine {
  // options (krige_initialize, kriging_base.F90:467-553)
  int ndim = 2, nlag = 2, nvar = 1, ndrift = 0, unbias = 1, nsim = 0;
  int anisotropic_search = 0, neglect_error = 1, std_ck = 0, cross_validation = 0;
  int verbose = 0;
  double bounds[2] = {-DBL_MAX, DBL_MAX};
  int st = 0;
  int precision = 2;   // 0 = FP64 plain, 1 = FP32 factor + FP64 refinement, 2 = the faster (tuned)
  int nmin = 0;
  int device = 0;
  cudaStream_t stream = nullptr;

  std::vector<ObsVar> obs;
  std::vector<StructSpec> vgm[KK_MAXVAR][KK_MAXVAR];
  // space-time model (kriging_st.F90)
  int st_model = 0, st_transform = KK_LIN;
  double st_at = 1.0, st_k_ps = 0.0, st_time_nugget = 0.0, st_time_sill = 1.0;
  std::vector<StructSpec> vgm_t[KK_MAXVAR][KK_MAXVAR];
  std::vector<double> joint[KK_MAXVAR][KK_MAXVAR];

  // targets
  int nblock = 0;
  std::vector<double> bcoord;       // (nlag, nblock); empty when bcoord_staged
  bool bcoord_staged = false;       // point targets held in hstage (nlag, nblock) instead
  std::vector<int> nblockpnt;       // empty -> point targets
  std::vector<double> gcoord, gweight;
  std::vector<double> rangescale, localnugget;
  std::vector<double> bdrift;       // (ndrift, nvar, nblock)
  bool grid_dirty = true;

  // device state
  VarDevice vd[KK_MAXVAR];
  DBuf models, tables, tx[4], trs, tln, tdrift, gstart, gx[4], gw;
  DBuf est, var, status, npp, bucket, counters, scratch;
  DBuf kbuf;  // packed K64 of one chunk of targets (assembly -> factorisation)
  DBuf til;  // point-target coordinates as given (nlag, nblock), before the per-axis split
  void* hstage = nullptr;  // pinned host staging for target uploads
  void* hres = nullptr;    // pinned host staging for multi-variable results
  size_t hres_bytes = 0;
  size_t hstage_bytes = 0;
  size_t scratch_bytes = 0;
  int mmax_total = 0;
  bool solved = false;
  int stats[8] = {0};
  int counters_last[KK_CNT_N_HOST] = {0};  // device counters of the last solve (KK_CNT_*)
  double last_solve_ms = 0.0;
  // per-phase device time of the last solve (CUDA events on the handle's
  // stream): search, bucket, solve kernels, fallbacks; and kernel launches
  int profile = 0;
  double phase_ms[6] = {0, 0, 0, 0, 0, 0};  // [4] assembly, [5] factorisation kernels (inside [2], [3])
  int launches = 0;
  // solve kernel per neighbour-count list (KK_KER_*, -1 for an empty list)
  // in the last solve, and the tuner's measured microseconds per target of
  // each candidate (NaN where not timed).  autotune: 0 fixed plan, 1 time
  // the candidates once per system signature (process-wide cache), 2 time
  // them again on the next solve
  int autotune = 1;
  int plan[KK_NLIST] = {-1, -1, -1, -1};
  double plan_us[KK_NLIST][KK_NKER] = {};
  DBuf tunebuf;  // status copy while the tuner runs

  // weight store (store_weight / use_old_weight, kriging_base.F90:2703-2990):
  // the weights of every target stay on the device after a store_weight
  // solve, wbuf[(t * nvar + jv) * wstride + row] with rows in matrix order,
  // together with the neighbour lists of that solve; set_weights stages a
  // caller's store on the host until the next solve uploads it
  int indicator = 0;  // krige_ind_create: probabilities normalised after each solve
  int ncat = 0;       // indicator categories (0: every variable)
  int store_weight = 0, use_old_weight = 0;
  bool wstore_dev = false;   // the device holds a complete store
  bool wstore_host = false;  // set_weights data waiting for upload
  int wstride = 0;           // weight rows per target variable (sum of mmax)
  int wmmax[KK_MAXVAR] = {0, 0, 0, 0};  // neighbour-list stride per variable of the store
  DBuf wbuf;
  std::vector<int> wh_nnear;      // (ngroups, nblock)
  std::vector<int> wh_inear;      // (nm, ngroups, nblock), 1-based
  std::vector<double> wh_weight;  // (nm, ngroups, nvar, nblock)
  std::vector<double> wh_var;     // (nvar, nvar, nblock)
  int wh_nm = 0;
  std::string info;               // krige_to_str text

  // sequential simulation (nsim > 0, krige_set_sim): visiting order (1-based
  // targets) and N(0, 1) draws sample[p * nsim + s] of the p-th visited
  // target; generated from seed when not given.  sim_nobs >= 0 marks the
  // internal engine that solves the simulation's systems: its observations
  // are the sim_nobs data followed by the targets in visiting order.
  int seed = 0;
  std::vector<int> sim_path;
  std::vector<double> sim_sample;
  int sim_nobs = -1;
  int sim_levels = 0;  // dependency levels of the last simulation
  int sim_flow = 0;    // 1 when its draws ran as one launch (k_sgsim_flow)
  int sim_by_level = 0;  // 1: draw level by level (k_sgsim_level) instead
  // neighbour sets of the last simulation by target: counts (observation,
  // simulated) and lists (sim_mmax per target; observations < nobs, then
  // nobs + visiting position), in the order of the target's system
  int sim_mmax = 0;
  std::vector<int> sim_nn, sim_nbr;

  int naug() const { return std_ck ? unbias * nvar : unbias; }
  int pdrift() const { return ndrift + naug(); }
};

// host-side model building (kk_host.cpp)
void calc_rotmat(double ang1, double ang2, double ang3, double anis1, double anis2, double* m);
void build_models(const Engine& e, std::vector<KkModel>& mdl, std::vector<KkSTModel>& smdl,
                  std::vector<double2>& tables);
void build_kdtree(const double* data, int D, int n, std::vector<int>& node_i,
                  std::vector<double>& node_d, std::vector<double>& box, std::vector<int>& ind,
                  std::vector<double>& rdata, int& root);

// engine entry points (kk_engine.cu)
void engine_solve(Engine& e);
// visiting order and draws of a sequential simulation when the caller gave
// none (krige_set_sim without them, or none before solve)
void engine_sim_defaults(Engine& e, bool path, bool sample);
// FP64 re-solve of the last solve's neighbour sets without any device
// allocation (workspace in a fixed static array); value (nobs) replaces the
// observation values of variable ivar first when it is not null.
void engine_resolve_static(Engine& e, int ivar, int nobs, const double* value);
void engine_release(Engine& e);
// forget every cached kernel plan (krige_autotune_clear)
void tune_clear();
// weight store (kk_engine.cu): nm = largest neighbour-list length over the
// variables; the getters copy the device store (or the staged one) into the
// reference's column-major layouts
int engine_weight_nm(Engine& e);
void engine_set_weights(Engine& e, int nm, int ng, int nv, int nb, const int* nnear, const int* inear,
                        const double* weight, const double* var);
void engine_get_weights(Engine& e, int nm, int ng, int nv, int nb, int* nnear, int* inear, double* weight,
                        double* var);
void engine_free_weight_store(Engine& e);

// allocator hook
typedef void* (*alloc_fn)(size_t bytes, void* ctx);
typedef void (*free_fn)(void* ptr, void* ctx);
void set_allocator(alloc_fn a, free_fn f, void* ctx);

// error slot (kriging_err.f90): first error since the last clear
void set_error(const std::string& msg);
void clear_error();
bool failed();

}  // namespace kk
