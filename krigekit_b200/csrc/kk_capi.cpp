// kk_capi.cpp -- the krige_* C-ABI of libkrigecuda.so.
//
// Entry points keep the names, argument order, array layouts (Fortran
// column-major) and error convention (int32 ierr, 0 = ok; message through
// krige_get_last_error) of the reference's ISO_C_BINDING layer
// (src/libkriging/kriging_capi.F90, kriging_capi_common.F90,
// kriging_st_capi.f90), so the reference's ctypes wrapper can bind this
// library unchanged for the kriging path.  Each function cites the
// reference routine it replaces; declarations live in include/krigekit_b200.h.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kk_host.h"

namespace kk {

static std::string g_err;
static std::mutex g_err_mu;

void set_error(const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  if (g_err.empty()) g_err = msg;
}
void clear_error() {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_err.clear();
}
bool failed() {
  std::lock_guard<std::mutex> lk(g_err_mu);
  return !g_err.empty();
}

// The registry is never destroyed: engines still alive at process exit keep
// their device buffers, because the allocator callbacks they would call (a
// Python allocator, for instance) may already be gone by then.
static std::vector<std::unique_ptr<Engine>>& g_reg = *new std::vector<std::unique_ptr<Engine>>();
static std::mutex g_reg_mu;

static Engine* get(int64_t h) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  if (h < 1 || h > (int64_t)g_reg.size() || !g_reg[h - 1]) {
    set_error("invalid kriging handle");
    return nullptr;
  }
  return g_reg[h - 1].get();
}

static int ierr() { return failed() ? 1 : 0; }

// device -> host copy of solve results, with the CUDA status checked
static void copy_d2h(void* dst, const void* src, size_t bytes) {
  const cudaError_t err = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
  if (err != cudaSuccess) throw std::string("CUDA error ") + cudaGetErrorString(err) + " reading results";
}

static const double* results_to_host(Engine* e, const void* src, size_t n, std::vector<double>& fallback);

// Device results straight into a caller's array: small ones by one copy,
// large ones through the handle's pinned buffer (full-rate DMA) and a
// threaded host copy instead of the driver's pageable staging.
static void results_to_caller(Engine* e, double* out, const void* src, size_t n) {
  if (sizeof(double) * n < (size_t(8) << 20)) {
    copy_d2h(out, src, sizeof(double) * n);
    return;
  }
  std::vector<double> fb;
  const double* tmp = results_to_host(e, src, n, fb);
  if (tmp == fb.data()) {
    std::memcpy(out, tmp, sizeof(double) * n);
    return;
  }
  par_copy(out, tmp, sizeof(double) * n);
}

// Device results of a multi-variable solve into host memory for reordering:
// the handle's pinned result buffer (kept across calls), or a caller-owned
// vector when pinned memory cannot be had.
static const double* results_to_host(Engine* e, const void* src, size_t n, std::vector<double>& fallback) {
  const size_t bytes = sizeof(double) * n;
  if (e->hres_bytes < bytes) {
    if (e->hres) cudaFreeHost(e->hres);
    e->hres = nullptr;
    e->hres_bytes = 0;
    if (cudaHostAlloc(&e->hres, bytes, cudaHostAllocPortable) == cudaSuccess) {
      e->hres_bytes = bytes;
    } else {
      cudaGetLastError();
      e->hres = nullptr;
    }
  }
  if (e->hres) {
    copy_d2h(e->hres, src, bytes);
    return static_cast<const double*>(e->hres);
  }
  fallback.resize(n);
  copy_d2h(fallback.data(), src, bytes);
  return fallback.data();
}

static int vtype_id(const char* s) {
  // vtype_from_str, vgmfunc.f90:83-99 (case-insensitive 3-character prefix)
  static const char* names[] = {"nug", "sph", "exp", "gau", "hol", "pow", "bsq", "cir", "lin", "cyc", "dco"};
  char b[4] = {0, 0, 0, 0};
  for (int i = 0; i < 3 && s && s[i]; ++i) b[i] = (char)std::tolower((unsigned char)s[i]);
  for (int k = 0; k < 11; ++k)
    if (std::strncmp(b, names[k], 3) == 0) return k;
  return -1;
}

}  // namespace kk

using namespace kk;

#define KK_GUARD_BEGIN \
  clear_error();       \
  try {
#define KK_GUARD_END_NORET                     \
  }                                            \
  catch (const std::string& m) { set_error(m); } \
  catch (const std::exception& x) { set_error(x.what()); }
#define KK_GUARD_END                           \
  }                                            \
  catch (const std::string& m) { set_error(m); } \
  catch (const std::exception& x) { set_error(x.what()); } \
  return ierr();

extern "C" {

// krige_create, kriging_capi.F90:43-57
int krige_create(int64_t* handle) {
  KK_GUARD_BEGIN
  std::lock_guard<std::mutex> lk(g_reg_mu);
  g_reg.emplace_back(new Engine());
  *handle = (int64_t)g_reg.size();
  KK_GUARD_END
}

// krige_ind_create, kriging_capi.F90:83-100: a handle whose solves end with
// the indicator post-processing (category probabilities clipped to [0, 1]
// and normalised, post_solve_indicator, kriging_indicator.F90:170-185)
int krige_ind_create(int64_t* handle) {
  if (krige_create(handle) != 0) return 1;
  Engine* e = get(*handle);
  if (!e) return 1;
  e->indicator = 1;
  return 0;
}

// krige_ind_set_ncat, kriging_capi.F90:113-: 1 <= ncat <= nvar; variables past
// ncat are secondary co-variates, left out of the normalisation
int krige_ind_set_ncat(int64_t h, int ncat) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (!e->indicator) throw std::string("handle was not created by krige_ind_create");
  if (ncat < 1 || ncat > e->nvar) throw std::string("ncat must satisfy 1 <= ncat <= nvar");
  e->ncat = ncat;
  KK_GUARD_END
}

// krige_destroy, kriging_capi_common.F90 (release_obj_base)
int krige_destroy(int64_t* handle) {
  KK_GUARD_BEGIN
  Engine* e = get(*handle);
  if (e) {
    engine_release(*e);
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_reg[*handle - 1].reset();
  }
  *handle = 0;
  KK_GUARD_END
}

// krige_initialize, kriging_capi.F90:143-192 -> initialize_base (kriging_base.F90:467-553)
int krige_initialize(int64_t h, int ndim, int nvar, int ndrift, int unbias, int nsim, int anisotropic_search,
                     int weight_correction, int use_old_weight, int store_weight, int cross_validation,
                     int write_mat, int neglect_error, int varying_vgm, int std_ck, int verbose, int pf_cache,
                     const char* weight_file, const double* bounds, int seed) {
  (void)pf_cache; (void)weight_file; (void)write_mat;
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (nsim < 0) throw std::string("nsim must be >= 0");
  if (nsim > 0 && cross_validation) throw std::string("cross_validation and nsim>0 are mutually exclusive");
  if (store_weight && use_old_weight) throw std::string("store_weight and use_old_weight are mutually exclusive");
  if ((store_weight || use_old_weight) && weight_file && weight_file[0])
    throw std::string("weight files are not written by the GPU library: keep the weight store in memory "
                      "(get_weights / set_weights)");
  if (weight_correction) throw std::string("weight_correction is not part of the GPU kriging path");
  if (varying_vgm) throw std::string("varying_vgm is not part of the GPU kriging path");
  if (ndim < 1 || ndim > 3) throw std::string("ndim must be 1, 2 or 3");
  if (nvar < 1 || nvar > KK_MAXVAR) throw std::string("nvar must be 1..4");
  engine_release(*e);
  for (int a = 0; a < KK_MAXVAR; ++a)
    for (int b = 0; b < KK_MAXVAR; ++b) {
      e->vgm[a][b].clear();
      e->vgm_t[a][b].clear();
      e->joint[a][b].clear();
      }
  for (int v = 0; v < KK_MAXVAR; ++v) {
    e->vd[v].grid_ready = false;
    e->vd[v].tree_ready = false;
  }
  e->st = 0;
  e->nblock = 0;
  e->bcoord.clear(); e->nblockpnt.clear(); e->gcoord.clear(); e->gweight.clear();
  e->bcoord_staged = false;
  e->rangescale.clear(); e->localnugget.clear(); e->bdrift.clear();
  e->grid_dirty = true;
  e->solved = false;
  e->ndim = ndim;
  e->nlag = ndim;
  e->nvar = nvar;
  e->ndrift = ndrift;
  e->unbias = unbias;
  e->nsim = nsim;
  e->seed = seed;
  e->sim_path.clear();
  e->sim_sample.clear();
  e->anisotropic_search = anisotropic_search;
  e->cross_validation = cross_validation;
  e->neglect_error = neglect_error;
  e->std_ck = std_ck;
  e->verbose = verbose;
  engine_free_weight_store(*e);
  e->ncat = 0;
  e->store_weight = store_weight ? 1 : 0;
  e->use_old_weight = use_old_weight ? 1 : 0;
  e->bounds[0] = bounds ? bounds[0] : -DBL_MAX;
  e->bounds[1] = bounds ? bounds[1] : DBL_MAX;
  e->obs.assign(nvar, ObsVar());
  KK_GUARD_END
}

// krige_set_obs, kriging_capi.F90:197-224 -> set_obs_base (kriging_base.F90:560-639)
int krige_set_obs(int64_t h, int ivar, int nobs, int ndim_c, const double* coord, const double* value,
                  const double* variance, int nmax, double maxdist, double sk_mean) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (ivar < 1 || ivar > e->nvar) throw std::string("ivar out of range");
  if (ndim_c != e->nlag) throw std::string("nlag /= size(coord, 1) for obs");
  ObsVar& o = e->obs[ivar - 1];
  o = ObsVar();
  o.n = nobs;
  o.coord.assign(coord, coord + (size_t)ndim_c * nobs);
  o.value.assign(value, value + nobs);
  if (variance) o.variance.assign(variance, variance + nobs);
  else o.variance.assign(nobs, 0.0);
  // duplicate coordinate check (check_duplicate_coordinates_base, utils.F90:43-133):
  // open-addressing hash tables over all coordinates, full comparison on a
  // matching slot (equal coordinates always hash alike).  The hash's top
  // bits split the points into partitions, one table and thread each; every
  // partition scans in index order, so the reported pair (the smallest index
  // that repeats an earlier point, and that point) is the sequential scan's.
  {
    const double* c = o.coord.data();
    auto hash_of = [=](int i) {
      uint64_t hsh = 0x9e3779b97f4a7c15ull;
      for (int k = 0; k < ndim_c; ++k) {
        double v = c[(size_t)i * ndim_c + k];
        if (v == 0.0) v = 0.0;  // -0.0 and 0.0 are the same coordinate
        uint64_t bits;
        std::memcpy(&bits, &v, sizeof bits);
        hsh ^= bits + 0x9e3779b97f4a7c15ull + (hsh << 6) + (hsh >> 2);
        hsh *= 0xff51afd7ed558ccdull;
        hsh ^= hsh >> 33;
      }
      return hsh;
    };
    const int nparts = nobs >= (1 << 16) ? 8 : 1;
    std::vector<int> dup_i(nparts, INT_MAX), dup_j(nparts, -1);
    par_for((size_t)nparts, 1, [&](size_t p0, size_t p1) {
      for (size_t part = p0; part < p1; ++part) {
        size_t cap = 1;
        while (cap < 2 * ((size_t)nobs / nparts + 1) + 2) cap <<= 1;
        std::vector<int> slot(cap, -1);
        size_t used = 0;
        for (int i = 0; i < nobs; ++i) {
          const uint64_t hsh = hash_of(i);
          if (nparts > 1 && (size_t)(hsh >> 61) != part) continue;
          if (2 * (used + 1) > cap) {  // a skewed partition: grow and reinsert
            std::vector<int> old;
            old.swap(slot);
            cap <<= 1;
            slot.assign(cap, -1);
            for (int j : old) {
              if (j < 0) continue;
              size_t q = hash_of(j) & (cap - 1);
              while (slot[q] >= 0) q = (q + 1) & (cap - 1);
              slot[q] = j;
            }
          }
          size_t q = hsh & (cap - 1);
          bool found = false;
          while (slot[q] >= 0) {
            const int j = slot[q];
            bool same = true;
            for (int k = 0; k < ndim_c; ++k)
              if (c[(size_t)i * ndim_c + k] != c[(size_t)j * ndim_c + k]) { same = false; break; }
            if (same) { dup_i[part] = i; dup_j[part] = j; found = true; break; }
            q = (q + 1) & (cap - 1);
          }
          if (found) break;
          slot[q] = i;
          ++used;
        }
      }
    });
    int bi = INT_MAX, bj = -1;
    for (int part = 0; part < nparts; ++part)
      if (dup_i[part] < bi) { bi = dup_i[part]; bj = dup_j[part]; }
    if (bj >= 0) {
      char msg[160];
      snprintf(msg, sizeof msg, "Duplicate observation coordinates at points %d and %d", bj + 1, bi + 1);
      o = ObsVar();
      throw std::string(msg);
    }
  }
  o.nmax = nmax;
  o.maxdist = maxdist;
  o.sk_mean = sk_mean;
  o.dirty = true;
  KK_GUARD_END
}

// krige_update_obs_value (kriging_base.F90:649-680): new values, same locations
int krige_update_obs_value(int64_t h, int ivar, int nobs, const double* value) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (ivar < 1 || ivar > e->nvar) throw std::string("ivar out of range");
  ObsVar& o = e->obs[ivar - 1];
  if (nobs != o.n) throw std::string("size(value) /= obs%n");
  o.value.assign(value, value + nobs);
  bool keep_search = o.search_set;
  o.dirty = true;
  o.search_set = keep_search;
  // with a complete weight store the next solve reuses the weights
  // (update_obs_value_base, kriging_base.F90:669-677)
  if (e->wstore_dev && e->solved) {
    e->use_old_weight = 1;
    e->store_weight = 0;
  }
  KK_GUARD_END
}

// krige_set_obs_drift, kriging_capi.F90 -> set_obs_drift_base (kriging_base.F90:718-752)
int krige_set_obs_drift(int64_t h, int ivar, int ndrift_c, int nobs, const double* drift) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (ivar < 1 || ivar > e->nvar) throw std::string("ivar out of range");
  ObsVar& o = e->obs[ivar - 1];
  if (o.n == 0) throw std::string("Observation needs to be set before adding drift.");
  if (e->ndrift == 0) throw std::string("Observation drift is specified but ndrift==0");
  if (ndrift_c != e->ndrift) throw std::string("size(drift, 1) /= ndrift");
  if (nobs != o.n) throw std::string("size(drift, 2) /= nobs");
  o.drift.assign(drift, drift + (size_t)ndrift_c * nobs);
  o.dirty = true;
  KK_GUARD_END
}

// krige_reset_vgm, kriging_capi.F90:230-243
int krige_reset_vgm(int64_t h, int ivar, int jvar) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  int a = std::min(ivar, jvar) - 1, b = std::max(ivar, jvar) - 1;
  if (a < 0 || b >= e->nvar) throw std::string("ivar/jvar out of range");
  e->vgm[a][b].clear();
  KK_GUARD_END
}

// krige_set_vgm, kriging_capi.F90:245-268 -> set_vgm (kriging.F90:211-276)
int krige_set_vgm(int64_t h, int ivar, int jvar, const char* vtype, double nugget, double sill, double a_major,
                  double a_minor1, double a_minor2, double azimuth, double dip, double plunge, int is_product) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (ivar < 1 || jvar < 1 || ivar > e->nvar || jvar > e->nvar) throw std::string("ivar/jvar out of range");
  if (jvar < ivar) throw std::string("jvar must be >= ivar to set the upper triangle of the variogram matrix");
  int id = vtype_id(vtype);
  if (id < 0) throw std::string("Unknown variogram type: ") + (vtype ? vtype : "");
  std::vector<StructSpec>& v = e->vgm[ivar - 1][jvar - 1];
  if (is_product && v.empty())
    throw std::string("first structure cannot be a product member (product=.true. requires a preceding structure)");
  if ((int)v.size() >= KK_MAXSTRUCT) throw std::string("exceeded the maximum number of nested structures");
  StructSpec s;
  s.vtype = id;
  s.nugget = nugget;
  s.sill = sill;
  s.a_major = a_major;
  s.a_minor1 = a_minor1;
  s.a_minor2 = a_minor2;
  s.az = azimuth;
  s.dip = dip;
  s.plunge = plunge;
  s.is_product = is_product ? 1 : 0;
  v.push_back(s);
  KK_GUARD_END
}

// Point-target coordinates straight into the handle's pinned staging buffer
// (one host copy; the solve uploads it as is and splits the axes on the
// device).  False when pinned memory cannot be had: the caller keeps the
// coordinates in bcoord instead.
static bool stage_targets(Engine* e, const double* coord, size_t nval) {
  const size_t need = sizeof(double) * nval;
  if (e->hstage_bytes < need) {
    if (e->hstage) cudaFreeHost(e->hstage);
    e->hstage = nullptr;
    e->hstage_bytes = 0;
    if (cudaHostAlloc(&e->hstage, need, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      e->hstage = nullptr;
      return false;
    }
    e->hstage_bytes = need;
  }
  par_copy(e->hstage, coord, need);
  return true;
}

static void grid_common(Engine* e, int nblock, const double* rangescale, const double* localnugget) {
  e->nblock = nblock;
  e->rangescale.clear();
  e->localnugget.clear();
  bool rs1 = true, ln0 = true;
  for (int i = 0; rangescale && i < nblock; ++i) rs1 = rs1 && rangescale[i] == 1.0;
  for (int i = 0; localnugget && i < nblock; ++i) ln0 = ln0 && localnugget[i] == 0.0;
  if (rangescale && !rs1) e->rangescale.assign(rangescale, rangescale + nblock);
  if (localnugget && !ln0) e->localnugget.assign(localnugget, localnugget + nblock);
  e->bdrift.clear();
  if (e->ndrift > 0) e->bdrift.assign((size_t)e->ndrift * e->nvar * nblock, 0.0);
  e->grid_dirty = true;
  e->solved = false;
}

// krige_set_grid, kriging_capi.F90:310-331 -> set_grid_point_base (kriging_base.F90:981-1004)
int krige_set_grid(int64_t h, int ngrid, int ndim_c, const double* coord, const double* rangescale,
                   const double* localnugget) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (e->obs.empty() || e->obs[0].n == 0) throw std::string("Observation needs to be set first.");
  if (ndim_c != e->nlag) throw std::string("nlag /= size(coord, 1) for self%grid");
  const size_t nval = (size_t)ndim_c * ngrid;
  e->bcoord_staged = stage_targets(e, coord, nval);
  if (e->bcoord_staged) e->bcoord.clear();
  else e->bcoord.assign(coord, coord + nval);
  e->nblockpnt.clear();
  e->gcoord.clear();
  e->gweight.clear();
  grid_common(e, ngrid, rangescale, localnugget);
  KK_GUARD_END
}

// krige_set_grid_block, kriging_capi.F90:334-378: GQ blocks (set_grid_gq_base,
// kriging_base.F90:1010-1068) or user blocks (set_grid_user_block_base)
int krige_set_grid_block(int64_t h, int block_type, int ngrid, int ndim_c, const double* coord, int nblock,
                         const int* nblockpnt, const double* pointweight, const double* blocksize,
                         const double* rangescale, const double* localnugget) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (e->obs.empty() || e->obs[0].n == 0) throw std::string("Observation needs to be set first.");
  if (ndim_c != e->nlag) throw std::string("nlag /= size(coord, 1) for self%grid");
  const int D = ndim_c;
  if (block_type == -4) {
    // Gauss-Legendre 4-point rule per axis (gaussian_quadrature.f90:1-41)
    const double frac[4] = {0.4305681558, 0.1699905218, -0.1699905218, -0.4305681558};
    const double wgq4[4] = {0.1739274226, 0.3260725774, 0.3260725774, 0.1739274226};
    const int nb = ngrid;
    int ngq = 1;
    for (int k = 0; k < D; ++k) ngq *= 4;
    e->bcoord.assign(coord, coord + (size_t)D * nb);
    e->bcoord_staged = false;
    e->nblockpnt.assign(nb, ngq);
    e->gcoord.assign((size_t)D * nb * ngq, 0.0);
    e->gweight.assign((size_t)nb * ngq, 0.0);
    for (int ib = 0; ib < nb; ++ib)
      for (int g = 0; g < ngq; ++g) {
        int ii[3] = {g % 4, (g / 4) % 4, g / 16};
        double w = 1.0;
        for (int k = 0; k < D; ++k) {
          e->gcoord[((size_t)ib * ngq + g) * D + k] = coord[(size_t)ib * D + k] + frac[ii[k]] * blocksize[(size_t)ib * D + k];
          w = w * wgq4[ii[k]];
        }
        e->gweight[(size_t)ib * ngq + g] = w;
      }
    grid_common(e, nb, rangescale, localnugget);
  } else {
    if (block_type <= 0) throw std::string("block_type must be >0 for user block grids.");
    long long tot = 0;
    for (int i = 0; i < nblock; ++i) {
      if (nblockpnt[i] <= 0) throw std::string("nblockpnt entries must be positive");
      tot += nblockpnt[i];
    }
    if (tot != ngrid) throw std::string("gridcoord columns != sum(nblockpnt)");
    e->nblockpnt.assign(nblockpnt, nblockpnt + nblock);
    e->gcoord.assign(coord, coord + (size_t)D * ngrid);
    if (pointweight) e->gweight.assign(pointweight, pointweight + ngrid);
    else {
      e->gweight.resize(ngrid);
      size_t g = 0;
      for (int i = 0; i < nblock; ++i)
        for (int k = 0; k < nblockpnt[i]; ++k) e->gweight[g++] = 1.0 / nblockpnt[i];
    }
    // weighted centroid (set_grid_centroid_common, kriging_base.F90:1546-1560)
    e->bcoord.assign((size_t)D * nblock, 0.0);
    e->bcoord_staged = false;
    size_t g0 = 0;
    for (int ib = 0; ib < nblock; ++ib) {
      const int nn = nblockpnt[ib];
      double denom = 0.0;
      for (int k = 0; k < nn; ++k) denom = denom + e->gweight[g0 + k];
      if (denom <= 0.0) throw std::string("sum(pointweight) must be positive for every block");
      for (int d = 0; d < D; ++d) {
        double s = 0.0;
        for (int k = 0; k < nn; ++k) s = s + e->gcoord[(g0 + k) * D + d] * e->gweight[g0 + k];
        e->bcoord[(size_t)ib * D + d] = s / denom;
      }
      g0 += nn;
    }
    grid_common(e, nblock, rangescale, localnugget);
  }
  KK_GUARD_END
}

// krige_set_grid_cv -> set_grid_cv_base (kriging_base.F90:1120-1135)
int krige_set_grid_cv(int64_t h) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (e->obs.empty() || e->obs[0].n == 0) throw std::string("Observation needs to be set first.");
  e->cross_validation = 1;
  e->bcoord = e->obs[0].coord;
  e->bcoord_staged = false;
  e->nblockpnt.clear();
  e->gcoord.clear();
  e->gweight.clear();
  grid_common(e, e->obs[0].n, nullptr, nullptr);
  if (e->ndrift > 0) {
    if (e->obs[0].drift.empty()) throw std::string("Observation drift is not set while ndrift > 0.");
    for (int ib = 0; ib < e->nblock; ++ib)
      for (int v = 0; v < e->nvar; ++v)
        for (int a = 0; a < e->ndrift; ++a)
          e->bdrift[((size_t)ib * e->nvar + v) * e->ndrift + a] = e->obs[0].drift[(size_t)ib * e->ndrift + a];
  }
  KK_GUARD_END
}

// krige_set_grid_drift, kriging_capi.F90:380-397 -> set_grid_drift_base (kriging_base.F90:1138-1186)
int krige_set_grid_drift(int64_t h, int ivar, int ndrift_c, int nblocks, const double* drift) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (e->nblock == 0) throw std::string("Grid needs to be set before adding drift.");
  if (e->ndrift == 0) throw std::string("grid/block drift is specified but ndrift==0");
  if (ndrift_c != e->ndrift) throw std::string("size(drift, 1) /= ndrift");
  if (nblocks != e->nblock) throw std::string("size(drift, 2) /= block%n; one drift value per block, not per grid node");
  if (ivar == 0 || ivar > e->nvar) throw std::string("ivar must be 1..nvar or < 0 (broadcast)");
  if (e->nvar == 1) {
    // (ndrift, nblock) is already the (ndrift, nvar, nblock) layout
    par_copy(e->bdrift.data(), drift, sizeof(double) * (size_t)nblocks * ndrift_c);
  } else {
    for (int ib = 0; ib < nblocks; ++ib)
      for (int v = 0; v < e->nvar; ++v) {
        if (ivar >= 1 && ivar != v + 1) continue;
        for (int a = 0; a < ndrift_c; ++a)
          e->bdrift[((size_t)ib * e->nvar + v) * e->ndrift + a] = drift[(size_t)ib * ndrift_c + a];
      }
  }
  KK_GUARD_END
}

// krige_set_search, kriging_capi.F90:448-467 -> set_search (kriging.F90:318-387)
int krige_set_search(int64_t h, int ivar, double anis1, double anis2, double azimuth, double dip, double plunge,
                     int sector_search) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (ivar < 1 || ivar > e->nvar) throw std::string("ivar out of range");
  ObsVar& o = e->obs[ivar - 1];
  if (o.n == 0) throw std::string("set_obs() needs to be called before set_search().");
  o.anis1 = anis1;
  o.anis2 = anis2;
  o.az = azimuth;
  o.dip = dip;
  o.plunge = plunge;
  o.sector = sector_search ? 1 : 0;
  o.search_set = true;
  o.search_dirty = true;
  KK_GUARD_END
}

// krige_solve, kriging_capi_common.F90:229-239 -> solve_base (kriging_base.F90:2064-2194)
int krige_solve(int64_t h, int nthread, int ncache) {
  (void)nthread; (void)ncache;  // CPU threading / factor-cache knobs: not used on the GPU
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_solve(*e);
  KK_GUARD_END
}

// krige_solver_stats, kriging_capi_common.F90:113-128
void krige_solver_stats(int64_t h, int* out) {
  Engine* e = get(h);
  for (int i = 0; i < 5; ++i) out[i] = e ? e->stats[i] : 0;
}

int krige_get_last_error(char* buffer, int nbuf) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  if (nbuf > 0) {
    size_t n = std::min<size_t>(g_err.size(), (size_t)nbuf - 1);
    std::memcpy(buffer, g_err.data(), n);
    buffer[n] = 0;
  }
  return g_err.empty() ? 0 : 1;
}

int krige_get_nblocks(int64_t h, int* nb) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  *nb = e->nblock;
  KK_GUARD_END
}

int krige_get_nsim(int64_t h, int* ns) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  *ns = e->nsim;
  KK_GUARD_END
}

// krige_get_block_coord, kriging_capi_common.F90:277-288
int krige_get_block_coord(int64_t h, int ndim_c, int nblocks, double* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  const double* bc = e->bcoord_staged ? static_cast<const double*>(e->hstage) : e->bcoord.data();
  if (nblocks > 0 && e->nblock > 0 &&
      (!bc || (!e->bcoord_staged && e->bcoord.size() < (size_t)e->nblock * e->nlag)))
    throw std::string("no target coordinates are set");
  if (ndim_c > e->nlag) throw std::string("ndim exceeds the coordinate dimension of the targets");
  for (int ib = 0; ib < nblocks && ib < e->nblock; ++ib)
    for (int k = 0; k < ndim_c; ++k) out[(size_t)ib * ndim_c + k] = bc[(size_t)ib * e->nlag + k];
  KK_GUARD_END
}

static void check_solved(Engine* e) {
  if (!e->solved) throw std::string("solve() has not been called; call solve() before retrieving results");
}

// krige_get_estimate_all, kriging_capi_common.F90:323-344: out(nblocks, nvar, nsim)
int krige_get_estimate_all(int64_t h, int nblocks, int nvar_c, int nsim_c, double* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  check_solved(e);
  const int nv = e->nvar;
  if (nblocks < 0 || nblocks > e->nblock || nvar_c < 0 || nvar_c > nv || nsim_c < 0)
    throw std::string("output dimensions exceed the solved blocks or variables");
  if (nblocks == 0 || nvar_c == 0 || nsim_c == 0) return 0;
  if (e->nsim > 0) {
    // sequential simulation: est is (nblock, nsim) on the device, one variable
    if (nsim_c > e->nsim) throw std::string("nsim exceeds the simulated realisations");
    std::vector<double> fb;
    const double* tmp = results_to_host(e, e->est.p, (size_t)e->nblock * e->nsim, fb);
    for (int is = 0; is < nsim_c; ++is)
      for (int ib = 0; ib < nblocks; ++ib) out[ib + (size_t)nblocks * nvar_c * is] = tmp[(size_t)ib * e->nsim + is];
    return 0;
  }
  if (nv == 1) {
    // est is (nblock) on the device: copy the first column straight into out
    results_to_caller(e, out, e->est.p, (size_t)nblocks);
  } else {
    std::vector<double> fb;
    const double* tmp = results_to_host(e, e->est.p, (size_t)e->nblock * nv, fb);
    par_for((size_t)nblocks, size_t(1) << 18, [=](size_t lo, size_t hi) {
      for (int iv = 0; iv < nvar_c; ++iv)
        for (size_t ib = lo; ib < hi; ++ib) out[ib + (size_t)nblocks * iv] = tmp[ib * nv + iv];
    });
  }
  // every realisation slot holds the kriging estimate (no simulation)
  for (int is = 1; is < nsim_c; ++is)
    std::memcpy(out + (size_t)nblocks * nvar_c * is, out, sizeof(double) * (size_t)nblocks * nvar_c);
  KK_GUARD_END
}

// krige_get_estimate, kriging_capi_common.F90:290-306: out(nblocks, nsim) of variable 1
int krige_get_estimate(int64_t h, int nsim_c, int nblocks, double* out) {
  return krige_get_estimate_all(h, nblocks, 1, nsim_c, out);
}

// Neighbour sets of the last sequential simulation (extension): nnear(2, nblocks) =
// observation and simulated members, inear(mmax, nblocks) 0-based in the order of each
// target's system: observations (< nobs), then nobs + visiting position.
int krige_get_sim_neighbours(int64_t h, int nblocks, int mmax, int* nnear, int* inear) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  check_solved(e);
  if (e->nsim <= 0 || e->sim_nn.empty()) throw std::string("no sequential simulation has been solved");
  if (nblocks != e->nblock) throw std::string("nblocks must match the solved blocks");
  if (mmax < e->sim_mmax) throw std::string("mmax is smaller than the simulation's neighbour capacity");
  std::memcpy(nnear, e->sim_nn.data(), sizeof(int) * e->sim_nn.size());
  for (int t = 0; t < nblocks; ++t) {
    const int n = e->sim_nn[(size_t)t * 2] + e->sim_nn[(size_t)t * 2 + 1];
    for (int i = 0; i < mmax; ++i) inear[(size_t)t * mmax + i] = i < n ? e->sim_nbr[(size_t)t * e->sim_mmax + i] : 0;
  }
  KK_GUARD_END
}

// How a simulation draws its values (no reference counterpart): 0 one
// cooperative launch for every level, 1 one launch per level.
int krige_set_sim_draw(int64_t h, int by_level) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (by_level != 0 && by_level != 1) throw std::string("by_level must be 0 or 1");
  e->sim_by_level = by_level;
  KK_GUARD_END
}

// krige_set_sim, kriging_capi.F90:410-443 -> set_sim_base (kriging_base.F90:1226-1320):
// randpath (nblocks, 1-based) and sample (nsim, nvar, nblocks), either may be NULL
int krige_set_sim(int64_t h, int nblocks, const int* randpath, int nsim_c, int nvar_c, const double* sample) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (e->nsim == 0) return 0;
  if (e->obs.empty()) throw std::string("call initialize() before set_sim().");
  if (e->nblock == 0) throw std::string("Grid needs to be set first.");
  for (const ObsVar& o : e->obs)
    if (o.n == 0) throw std::string("Observations need to be set first.");
  for (const ObsVar& o : e->obs)
    if (o.nmax > (int)(INT_MAX * 0.001)) throw std::string("`nmax` must be set for all observations for SGSIM.");
  const int nb = e->nblock;
  if (randpath) {
    if (nblocks != nb) throw std::string("size(randpath) /= nblock");
    std::vector<char> seen(nb, 0);
    for (int i = 0; i < nb; ++i) {
      if (randpath[i] < 1 || randpath[i] > nb || seen[randpath[i] - 1])
        throw std::string("randpath must be a 1-based permutation of 1..nblocks");
      seen[randpath[i] - 1] = 1;
    }
    e->sim_path.assign(randpath, randpath + nb);
  } else {
    engine_sim_defaults(*e, true, false);
  }
  if (sample) {
    if (nsim_c != e->nsim) throw std::string("size(sample, 1) /= nsim");
    if (nvar_c != e->nvar) throw std::string("size(sample, 2) /= nvar");
    if (nblocks != nb) throw std::string("size(sample, 3) /= nblock");
    e->sim_sample.assign(sample, sample + (size_t)nsim_c * nvar_c * nb);
  } else {
    engine_sim_defaults(*e, false, true);
  }
  e->solved = false;
  KK_GUARD_END
}

// krige_get_variance_all, kriging_capi_common.F90:372-392: out(nblocks, nvar, nvar)
int krige_get_variance_all(int64_t h, int nblocks, int nvar_c, double* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  check_solved(e);
  const int nv = e->nvar;
  if (nblocks < 0 || nblocks > e->nblock || nvar_c < 0 || nvar_c > nv)
    throw std::string("output dimensions exceed the solved blocks or variables");
  if (nblocks == 0 || nvar_c == 0) return 0;
  if (nv == 1) {
    results_to_caller(e, out, e->var.p, (size_t)nblocks);
  } else {
    std::vector<double> fb;
    const double* tmp = results_to_host(e, e->var.p, (size_t)e->nblock * nv * nv, fb);
    par_for((size_t)nblocks, size_t(1) << 18, [=](size_t lo, size_t hi) {
      for (int jv = 0; jv < nvar_c; ++jv)
        for (int iv = 0; iv < nvar_c; ++iv)
          for (size_t ib = lo; ib < hi; ++ib)
            out[ib + (size_t)nblocks * (iv + (size_t)nvar_c * jv)] = tmp[ib * nv * nv + iv + (size_t)jv * nv];
    });
  }
  KK_GUARD_END
}

// krige_get_variance, kriging_capi_common.F90:352-369: variance of variable 1
int krige_get_variance(int64_t h, int nblocks, double* out) {
  return krige_get_variance_all(h, nblocks, 1, out);
}

// ---------------------------------------------------------------------------
// extensions (no reference counterpart; see include/krigekit_b200.h)
// ---------------------------------------------------------------------------
int krige_set_precision(int64_t h, int mode) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (mode < 0 || mode > 2) throw std::string("precision mode must be 0 (fp64), 1 (fp32_refine) or 2 (auto)");
  e->precision = mode;
  KK_GUARD_END
}

int krige_set_nmin(int64_t h, int nmin) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  e->nmin = nmin;
  KK_GUARD_END
}

int krige_set_device(int64_t h, int device, void* stream) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  e->device = device;
  e->stream = (cudaStream_t)stream;
  KK_GUARD_END
}

void krige_set_allocator(void* (*alloc)(size_t, void*), void (*release)(void*, void*), void* ctx) {
  set_allocator(alloc, release, ctx);
}

// neighbour sets after solve(): nnear(nblocks), inear(mmax, nblocks) 1-based, ascending
int krige_get_neighbours(int64_t h, int ivar, int nblocks, int mmax, int* nnear, int* inear) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  check_solved(e);
  if (ivar < 1 || ivar > e->nvar) throw std::string("ivar out of range");
  VarDevice& d = e->vd[ivar - 1];
  const int mm = std::max(d.search.mmax, 1);
  std::vector<int> nn(e->nblock), nb((size_t)e->nblock * mm);
  copy_d2h(nn.data(), d.nnear.p, sizeof(int) * nn.size());
  copy_d2h(nb.data(), d.nbr.p, sizeof(int) * nb.size());
  for (int ib = 0; ib < nblocks && ib < e->nblock; ++ib) {
    nnear[ib] = nn[ib];
    for (int k = 0; k < mmax; ++k) inear[(size_t)ib * mmax + k] = (k < nn[ib] && k < mm) ? nb[(size_t)ib * mm + k] + 1 : 0;
  }
  KK_GUARD_END
}

int krige_get_mmax(int64_t h, int ivar, int* mmax) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (ivar < 1 || ivar > e->nvar) throw std::string("ivar out of range");
  *mmax = std::max(e->vd[ivar - 1].search.mmax, 1);
  KK_GUARD_END
}

// per-target status bits (KK_ST_* in kk_common.h)
int krige_get_status(int64_t h, int nblocks, int* status) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  check_solved(e);
  std::vector<int> s(e->nblock);
  copy_d2h(s.data(), e->status.p, sizeof(int) * s.size());
  for (int ib = 0; ib < nblocks && ib < e->nblock; ++ib) status[ib] = s[ib];
  KK_GUARD_END
}

// counters of the last solve: [fail, chol, 0, ldlt, 0, search redo, fp64 re-solve, refine iterations]
int krige_gpu_stats(int64_t h, int* out8, double* solve_ms) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  for (int i = 0; i < 8; ++i) out8[i] = e->stats[i];
  if (solve_ms) *solve_ms = e->last_solve_ms;
  KK_GUARD_END
}

// ---- weight store (kriging_capi_common.F90 weight-store entry points,
// kriging_base.F90:2703-2990); layouts as the reference's ctypes binding
// (kriging.py:259-274)
int krige_get_weight_dims(int64_t h, int* nm, int* ng, int* nb) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (!e->wstore_dev && !e->wstore_host) throw std::string("Weight store not allocated. Set store_weight=True.");
  *nm = engine_weight_nm(*e);
  *ng = e->nvar;
  *nb = e->nblock;
  KK_GUARD_END
}

int krige_get_weight_nnear(int64_t h, int ng, int nb, int* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_get_weights(*e, engine_weight_nm(*e), ng, e->nvar, nb, out, nullptr, nullptr, nullptr);
  KK_GUARD_END
}

int krige_get_weight_inear(int64_t h, int nm, int ng, int nb, int* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_get_weights(*e, nm, ng, e->nvar, nb, nullptr, out, nullptr, nullptr);
  KK_GUARD_END
}

int krige_get_weight_data(int64_t h, int nm, int ng, int nv, int nb, double* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_get_weights(*e, nm, ng, nv, nb, nullptr, nullptr, out, nullptr);
  KK_GUARD_END
}

int krige_get_weight_var(int64_t h, int nv, int nb, double* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_get_weights(*e, engine_weight_nm(*e), e->nvar, nv, nb, nullptr, nullptr, nullptr, out);
  KK_GUARD_END
}

int krige_set_weights(int64_t h, int nm, int ng, int nv, int nb, const int* nnear, const int* inear,
                      const double* weight, const int* order, const double* var) {
  (void)order;  // the visiting order only matters for sequential simulation
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_set_weights(*e, nm, ng, nv, nb, nnear, inear, weight, var);
  KK_GUARD_END
}

int krige_free_weight_store(int64_t h) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_free_weight_store(*e);
  KK_GUARD_END
}

// Configuration summary (to_str_base, kriging_base.F90:3601-3646); the text
// belongs to the handle and stays valid until the next call on it.
const char* krige_to_str(int64_t h) {
  Engine* e = get(h);
  if (!e) return nullptr;
  auto yn = [](int b) { return b ? "yes" : "no"; };
  char buf[256];
  std::string r = "\n==================== Configuration ====================\n";
  auto line = [&](const char* k, const std::string& v) { r += " "; r += k; r += " : " + v + "\n"; };
  line("Engine                ", "B200 (sm_100a) kriging solve path");
  line("Dimension             ", std::to_string(e->ndim));
  line("Number of Variables   ", std::to_string(e->nvar));
  line("Number of Simulations ", std::to_string(e->nsim));
  line("Number of Drifts      ", std::to_string(e->ndrift));
  line("Number of Blocks      ", std::to_string(e->nblock));
  line("Ordinary Kriging      ", yn(e->unbias == 1));
  line("Standard CoKriging    ", yn(e->std_ck));
  line("LOO-Cross Validation  ", yn(e->cross_validation));
  line("Use Old Weights       ", yn(e->use_old_weight));
  line("Store Weights         ", yn(e->store_weight));
  line("Precision             ", e->precision == 2 ? "auto (FP64 or FP32 factor + FP64 correction, tuned)"
                                : (e->precision ? "FP32 factor + FP64 correction" : "FP64"));
  snprintf(buf, sizeof buf, "%.17g", e->bounds[0]);
  line("Lower Bound           ", buf);
  snprintf(buf, sizeof buf, "%.17g", e->bounds[1]);
  line("Upper Bound           ", buf);
  for (int v = 0; v < (int)e->obs.size(); ++v) {
    const ObsVar& o = e->obs[v];
    r += "Variable " + std::to_string(v + 1) + ":\n";
    line("Number of data        ", std::to_string(o.n));
    line("Maximum neighbors     ", std::to_string(o.nmax));
    snprintf(buf, sizeof buf, "%.17g", o.maxdist);
    line("Maxdist               ", buf);
    snprintf(buf, sizeof buf, "%.17g", o.sk_mean);
    line("Simple Kriging Mean   ", buf);
    line("Sector Search         ", yn(o.sector));
  }
  r += "================== End Configuration ==================\n";
  e->info = r;
  return e->info.c_str();
}

// Device counters of the last solve (KK_CNT_* of kk_kernels.h), n <= 32.
int krige_gpu_counters(int64_t h, int n, int* out) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (n < 0 || n > KK_CNT_N_HOST) throw std::string("n must be 0..32");
  for (int i = 0; i < n; ++i) out[i] = e->counters_last[i];
  KK_GUARD_END
}

// Kernel plan of the solve: 0 fixed, 1 tuned once per system signature, 2
// tuned again on the next solve.
int krige_set_autotune(int64_t h, int mode) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  if (mode < 0 || mode > 2) throw std::string("autotune mode must be 0, 1 or 2");
  e->autotune = mode;
  KK_GUARD_END
}

// Kernel per neighbour-count list in the last solve and the tuner's
// microseconds per target of each candidate (NaN where not timed).
int krige_get_kernel_plan(int64_t h, int* kernel4, double* us24) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  for (int li = 0; li < KK_NLIST; ++li) {
    if (kernel4) kernel4[li] = e->plan[li];
    for (int k = 0; k < KK_NKER; ++k)
      if (us24) us24[li * KK_NKER + k] = e->plan_us[li][k];
  }
  KK_GUARD_END
}

int krige_autotune_clear(void) {
  KK_GUARD_BEGIN
  tune_clear();
  KK_GUARD_END
}

// Enable per-phase CUDA-event timing of solve() (adds one event sync per phase).
int krige_gpu_profile(int64_t h, int enable) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  e->profile = enable ? 1 : 0;
  KK_GUARD_END
}

// Device time per phase of the last solve (ms): search, bucket, solve kernels,
// fallbacks (kd-tree replica, FP64 re-solve, generic); kernel launches.
int krige_gpu_phases(int64_t h, double* out4, int* launches) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  for (int i = 0; i < 4; ++i) out4[i] = e->phase_ms[i];
  if (launches) *launches = e->launches;
  KK_GUARD_END
}

// Device ms of the assembly and the factorisation launches of the last
// profiled solve (both inside the solve and fallback phases).
int krige_gpu_kernel_ms(int64_t h, double* out2) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  out2[0] = e->phase_ms[4];
  out2[1] = e->phase_ms[5];
  KK_GUARD_END
}

// ---------------------------------------------------------------------------
// space-time kriging (kriging_st_capi.f90): coordinates are the spatial ones
// followed by time; the shared entry points (krige_solve, the getters,
// krige_set_grid_cv, krige_update_obs_value, krige_set_obs_drift) apply too
// ---------------------------------------------------------------------------

// krige_st_create / krige_st_destroy, kriging_st_capi.f90:43-75
int krige_st_create(int64_t* handle) { return krige_create(handle); }
int krige_st_destroy(int64_t* handle) { return krige_destroy(handle); }

// krige_st_initialize, kriging_st_capi.f90:80-123 -> t_kriging_st%initialize
// (the reference engine is 3-D spatial + time; here the spatial dimension is
// taken from the first krige_st_set_obs, 3 until then)
int krige_st_initialize(int64_t h, int nvar, int ndrift, int unbias, int nsim, int anisotropic_search,
                        int weight_correction, int use_old_weight, int store_weight, int cross_validation,
                        int write_mat, int neglect_error, int verbose, const char* weight_file,
                        const double* bounds, int seed) {
  if (krige_initialize(h, 3, nvar, ndrift, unbias, nsim, anisotropic_search, weight_correction, use_old_weight,
                       store_weight, cross_validation, write_mat, neglect_error, 0, 1, verbose, 0, weight_file,
                       bounds, seed) != 0)
    return 1;
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  e->st = 1;
  e->ndim = 3;
  e->nlag = 4;
  e->st_model = 0;
  e->st_transform = KK_LIN;
  e->st_at = 1.0;
  e->st_k_ps = 0.0;
  e->st_time_nugget = 0.0;
  e->st_time_sill = 1.0;
  KK_GUARD_END
}

static Engine* get_st(int64_t h) {
  Engine* e = get(h);
  if (e && !e->st) throw std::string("handle was not initialised by krige_st_initialize");
  return e;
}

// krige_st_set_st_model, kriging_st_capi.f90:128-162
int krige_st_set_st_model(int64_t h, const char* model, const char* transform, double at, double time_nugget,
                          double time_sill, double k_ps) {
  KK_GUARD_BEGIN
  const std::string m = model ? model : "";
  int imodel;
  if (m == "sum_metric") imodel = 0;
  else if (m == "product_sum") imodel = 1;
  else throw std::string("model must be \"sum_metric\" or \"product_sum\", got: ") + m;
  const int it = vtype_id(transform);
  if (it < 0) throw std::string("Unknown variogram type: ") + (transform ? transform : "");
  Engine* e = get_st(h);
  if (!e) return 1;
  e->st_model = imodel;
  e->st_transform = it;
  e->st_at = at;
  e->st_time_nugget = time_nugget;
  e->st_time_sill = time_sill;
  e->st_k_ps = k_ps;
  KK_GUARD_END
}

// krige_st_set_obs, kriging_st_capi.f90:167-189: coord(ndim+1, nobs)
int krige_st_set_obs(int64_t h, int ivar, int nobs, int ndim, const double* coord, const double* value,
                     const double* variance, int nmax, double maxdist, double sk_mean) {
  {
    KK_GUARD_BEGIN
    Engine* e = get_st(h);
    if (!e) return 1;
    if (ndim < 1 || ndim > 3) throw std::string("ndim must be 1, 2 or 3");
    bool any = false;
    for (const ObsVar& o : e->obs) any = any || o.n > 0;
    if (!any) {
      e->ndim = ndim;
      e->nlag = ndim + 1;
    } else if (ndim != e->ndim) {
      throw std::string("ndim differs from the observations already set");
    }
    KK_GUARD_END_NORET
  }
  if (failed()) return 1;
  return krige_set_obs(h, ivar, nobs, ndim + 1, coord, value, variance, nmax, maxdist, sk_mean);
}

// krige_st_reset_vgm, kriging_st_capi.f90:245-258
int krige_st_reset_vgm(int64_t h, int ivar, int jvar) {
  KK_GUARD_BEGIN
  Engine* e = get_st(h);
  if (!e) return 1;
  int a = std::min(ivar, jvar) - 1, b = std::max(ivar, jvar) - 1;
  if (a < 0 || b >= e->nvar) throw std::string("ivar/jvar out of range");
  e->vgm[a][b].clear();
  e->vgm_t[a][b].clear();
  e->joint[a][b].clear();
  KK_GUARD_END
}

// krige_st_set_vgm, kriging_st_capi.f90:260-287: one spatial structure
int krige_st_set_vgm(int64_t h, int ivar, int jvar, const char* vtype, double nugget, double sill, double a_major,
                     double a_minor1, double a_minor2, double azimuth, double dip, double plunge) {
  {
    KK_GUARD_BEGIN
    if (!get_st(h)) return 1;
    KK_GUARD_END_NORET
  }
  if (failed()) return 1;
  return krige_set_vgm(h, ivar, jvar, vtype, nugget, sill, a_major, a_minor1, a_minor2, azimuth, dip, plunge, 0);
}

// krige_st_set_vgm_temporal, kriging_st_capi.f90:289-309: one temporal structure
int krige_st_set_vgm_temporal(int64_t h, int ivar, int jvar, const char* vtype, double nugget, double sill,
                              double at_k) {
  KK_GUARD_BEGIN
  Engine* e = get_st(h);
  if (!e) return 1;
  if (ivar < 1 || jvar < 1 || ivar > e->nvar || jvar > e->nvar) throw std::string("ivar/jvar out of range");
  const int id = vtype_id(vtype);
  if (id < 0) throw std::string("Unknown variogram type: ") + (vtype ? vtype : "");
  std::vector<StructSpec>& v = e->vgm_t[std::min(ivar, jvar) - 1][std::max(ivar, jvar) - 1];
  if ((int)v.size() >= KK_MAXSTRUCT) throw std::string("exceeded the maximum number of nested structures");
  StructSpec sp;
  sp.vtype = id;
  sp.nugget = nugget;
  sp.sill = sill;
  sp.a_major = at_k;
  sp.a_minor1 = at_k;
  sp.a_minor2 = at_k;
  v.push_back(sp);
  KK_GUARD_END
}

// krige_st_set_vgm_joint_sills, kriging_st_capi.f90:311-325: one sill per spatial structure
int krige_st_set_vgm_joint_sills(int64_t h, int ivar, int jvar, int nsill, const double* sills) {
  KK_GUARD_BEGIN
  Engine* e = get_st(h);
  if (!e) return 1;
  if (ivar < 1 || jvar < 1 || ivar > e->nvar || jvar > e->nvar) throw std::string("ivar/jvar out of range");
  const int a = std::min(ivar, jvar) - 1, b = std::max(ivar, jvar) - 1;
  if (nsill != (int)e->vgm[a][b].size())
    throw std::string("the number of joint sills must equal the number of spatial structures");
  e->joint[a][b].assign(sills, sills + nsill);
  KK_GUARD_END
}

// spatial coordinates (ndim, n) and times (n) -> (ndim + 1, n)
// coord(nd, n) + time(n) -> c(nd + 1, n); c keeps its capacity across calls
static void st_coords(const Engine* e, int n, const double* coord, const double* time, std::vector<double>& c) {
  const int nd = e->ndim;
  c.resize((size_t)(nd + 1) * n);
  double* cp = c.data();
  par_for((size_t)n, size_t(1) << 18, [=](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) {
      for (int k = 0; k < nd; ++k) cp[i * (nd + 1) + k] = coord[i * nd + k];
      cp[i * (nd + 1) + nd] = time[i];
    }
  });
}

// krige_st_set_grid, kriging_st_capi.f90:331-353: coord(ndim, ngrid), time(ngrid)
int krige_st_set_grid(int64_t h, int ngrid, const double* coord, const double* time, const double* rangescale,
                      const double* localnugget) {
  std::vector<double> c;
  {
    KK_GUARD_BEGIN
    Engine* e = get_st(h);
    if (!e) return 1;
    st_coords(e, ngrid, coord, time, c);
    KK_GUARD_END_NORET
  }
  if (failed()) return 1;
  int ndim = 0;
  { Engine* e = get(h); ndim = e ? e->ndim : 0; }
  return krige_set_grid(h, ngrid, ndim + 1, c.data(), rangescale, localnugget);
}

// krige_st_set_grid_block, kriging_st_capi.f90:355-388: block centres
// coord(ndim, nblocks) + time, integration nodes blockcoord(ndim, npnts) +
// blocktime with pointweight; the given centres are the search centres
int krige_st_set_grid_block(int64_t h, int nblocks, const double* coord, const double* time, const int* nblockpnt,
                            int npnts_total, const double* blockcoord, const double* blocktime,
                            const double* pointweight, const double* rangescale, const double* localnugget) {
  KK_GUARD_BEGIN
  Engine* e = get_st(h);
  if (!e) return 1;
  if (e->obs.empty() || e->obs[0].n == 0) throw std::string("Observation needs to be set first.");
  long long tot = 0;
  for (int i = 0; i < nblocks; ++i) {
    if (nblockpnt[i] <= 0) throw std::string("nblockpnt entries must be positive");
    tot += nblockpnt[i];
  }
  if (tot != npnts_total) throw std::string("sum(nblockpnt) /= size(blockcoord, 2)");
  st_coords(e, nblocks, coord, time, e->bcoord);
  e->bcoord_staged = false;
  e->nblockpnt.resize(nblocks);
  par_copy(e->nblockpnt.data(), nblockpnt, sizeof(int) * (size_t)nblocks);
  st_coords(e, npnts_total, blockcoord, blocktime, e->gcoord);
  e->gweight.resize(npnts_total);
  par_copy(e->gweight.data(), pointweight, sizeof(double) * (size_t)npnts_total);
  grid_common(e, nblocks, rangescale, localnugget);
  KK_GUARD_END
}

// krige_st_set_grid_drift, kriging_st_capi.f90:392-406: drift(ndrift, nblocks), all variables
int krige_st_set_grid_drift(int64_t h, int ndrift_c, int nblocks, const double* drift) {
  return krige_set_grid_drift(h, -1, ndrift_c, nblocks, drift);
}

// krige_st_set_search, kriging_st_capi.f90:458-490 -> t_kriging_st%set_search
// (kriging_st.F90:322-403): time_at scales the time axis of the search space
int krige_st_set_search(int64_t h, int ivar, double time_at, double anis1, double anis2, double azimuth, double dip,
                        double plunge, int sector_search) {
  {
    KK_GUARD_BEGIN
    Engine* e = get_st(h);
    if (!e) return 1;
    if (!(time_at > 1.0e-10)) throw std::string("time_at must be positive.");
    KK_GUARD_END_NORET
  }
  if (failed()) return 1;
  if (krige_set_search(h, ivar, anis1, anis2, azimuth, dip, plunge, sector_search) != 0) return 1;
  Engine* e = get(h);
  e->obs[ivar - 1].time_at = time_at;
  return 0;
}

// Allocation-free FP64 re-solve of the last krige_solve's neighbour sets
// (no counterpart in the reference): for callers that must not have device
// memory allocated during the call.  value may be null.
int krige_resolve_static(int64_t h, int ivar, int nobs, const double* value) {
  KK_GUARD_BEGIN
  Engine* e = get(h);
  if (!e) return 1;
  engine_resolve_static(*e, ivar, nobs, value);
  KK_GUARD_END
}

}  // extern "C"
