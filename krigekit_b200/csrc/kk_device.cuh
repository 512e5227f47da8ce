// kk_device.cuh -- device helpers shared by the search and solve kernels.
//
// Arithmetic that must reproduce the reference bit for bit (search-space
// rotation, squared distances, covariance table lookups) uses explicit
// round-to-nearest intrinsics so that nvcc cannot contract a multiply and an
// add into one fused operation; the reference build (gfortran -O2 on x86-64)
// rounds every multiply and add separately.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kk_common.h"

namespace kk {

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// zone layout of every lookup table (variogram.f90:223-256)
struct KkZones {
  double zb[KK_TAB_NZ + 1];
  double inv_dh[KK_TAB_NZ];
  int off[KK_TAB_NZ];
  int zn[KK_TAB_NZ];
};
// one private copy per translation unit (set by set_zones in kk_solve.cu)
static __constant__ KkZones c_zones;

// corefunc_fn, vgmfunc.f90:28-67 (device math library for exp/cos/sin/pow)
__device__ __forceinline__ double corefunc(int vtype, double r) {
  const double pi = 3.141592653589793;
  switch (vtype) {
    case KK_NUG: return 0.0;
    case KK_SPH: return (r < 1.0) ? dadd(dsub(1.0, dmul(1.5, r)), dmul(0.5, dmul(dmul(r, r), r))) : 0.0;
    case KK_EXP: return exp(dmul(-3.0, r));
    case KK_GAU: return exp(dmul(-3.0625, dmul(r, r)));
    case KK_HOL: return cos(dmul(pi, r));
    case KK_POW: return (r < 1.0) ? 1.0 - pow(r, 1.5) : 0.0;
    case KK_BSQ: { double t = dsub(1.0, dmul(r, r)); return (r < 1.0) ? dmul(t, t) : 0.0; }
    case KK_CIR:
      return (r < 1.0) ? 1.0 - (2.0 * r * sqrt(1.0 - r * r) + 2.0 * asin(r)) / pi : 0.0;
    case KK_LIN: return (r < 1.0) ? dsub(1.0, r) : 0.0;
    case KK_CYC: { double s = sin(dmul(pi, r)); return exp(dmul(-2.0, dmul(s, s))); }
    case KK_DCO: return dmul(exp(dmul(-3.0, r)), cos(dmul(pi, r)));
    default: return 0.0;
  }
}

// aniso_h, variogram.f90:194-210
__device__ __forceinline__ double aniso_h(const double* m, int ndim, const double* lag) {
  if (ndim == 1) return fabs(dmul(lag[0], m[0]));
  if (ndim == 2) {
    double rx = dadd(dmul(m[0], lag[0]), dmul(m[3], lag[1]));
    double ry = dadd(dmul(m[1], lag[0]), dmul(m[4], lag[1]));
    return __dsqrt_rn(dadd(dmul(rx, rx), dmul(ry, ry)));
  }
  double rx = dadd(dadd(dmul(m[0], lag[0]), dmul(m[3], lag[1])), dmul(m[6], lag[2]));
  double ry = dadd(dadd(dmul(m[1], lag[0]), dmul(m[4], lag[1])), dmul(m[7], lag[2]));
  double rz = dadd(dadd(dmul(m[2], lag[0]), dmul(m[5], lag[1])), dmul(m[8], lag[2]));
  return __dsqrt_rn(dadd(dadd(dmul(rx, rx), dmul(ry, ry)), dmul(rz, rz)));
}

// comp_cov_h, variogram.f90:327-337
__device__ __forceinline__ double comp_cov_h(const KkComp& c, double h) {
  const double eps = 2.2250738585072014e-308 * 1.0e3;  // tiny(1.0) * 1e3
  if (h > eps) return dmul(c.sill, corefunc(c.vtype, h));
  return dadd(c.sill, c.nugget);
}

// Piecewise-linear table lookup shared by comp_cov_tab_h (variogram.f90:
// 353-382) and cov_struct_tab_h (variogram.f90:682-710).  Returns false when
// h lies past the last zone and the caller must use the analytic tail.
__device__ __forceinline__ bool tab_lookup(const double2* __restrict__ tab, double h, double* res) {
  if (h >= c_zones.zb[KK_TAB_NZ]) return false;
  if (h <= 0.0) { *res = __ldg(&tab[0].x); return true; }
  int k = (h < c_zones.zb[1]) ? 0 : ((h < c_zones.zb[2]) ? 1 : 2);
  double fi = dmul(dsub(h, c_zones.zb[k]), c_zones.inv_dh[k]);
  int ii = (int)fi;
  int i = c_zones.off[k] + min(ii, c_zones.zn[k] - 1);
  fi = dsub(fi, (double)ii);
  double2 t = __ldg(&tab[i]);
  *res = dadd(t.x, dmul(fi, t.y));
  return true;
}

// struct_cov_h, variogram.f90:713-729
__device__ __forceinline__ double model_cov_h(const KkModel& m, double h) {
  double res = 0.0;
  int iv = 0;
  while (iv < m.nstruct) {
    double g = comp_cov_h(m.comp[iv], h);
    while (iv < m.nstruct - 1 && m.comp[iv + 1].is_product) {
      ++iv;
      g = dmul(g, comp_cov_h(m.comp[iv], h));
    }
    res = dadd(res, g);
    ++iv;
  }
  return res;
}

__device__ __forceinline__ double comp_cov(const KkComp& c, int ndim, const double2* __restrict__ tabs,
                                           const double* lag, bool level_a) {
  double h = aniso_h(c.mat, ndim, lag);
  if (level_a && c.tab_off >= 0) {
    double r;
    if (tab_lookup(tabs + c.tab_off, h, &r)) return r;
    return c.tail ? comp_cov_h(c, h) : 0.0;
  }
  return comp_cov_h(c, h);
}

// COV(vgm, lag): struct_cov_tab (variogram.f90:750-771); KK_ANALYTIC is the
// path of a vgm(first, second) entry for which no table was built.
__device__ __forceinline__ double model_cov(const KkModel& m, const double2* __restrict__ tabs,
                                            const double* lag) {
  if (m.mode == KK_LEVEL_B) {
    double h = aniso_h(m.bmat, m.ndim, lag);
    double r;
    if (tab_lookup(tabs + m.btab_off, h, &r)) return r;
    return m.btail ? model_cov_h(m, h) : 0.0;
  }
  const bool la = (m.mode == KK_LEVEL_A);
  double res = 0.0;
  int iv = 0;
  while (iv < m.nstruct) {
    double g = comp_cov(m.comp[iv], m.ndim, tabs, lag, la);
    while (iv < m.nstruct - 1 && m.comp[iv + 1].is_product) {
      ++iv;
      g = dmul(g, comp_cov(m.comp[iv], m.ndim, tabs, lag, la));
    }
    res = dadd(res, g);
    ++iv;
  }
  return res;
}

// f_time_vgm_st, variogram_st.f90:127-143
__device__ __forceinline__ double st_ftime(const KkSTModel& s, double dt) {
  if (fabs(dt) <= 2.220446049250313e-16) return 0.0;
  double adt = fabs(dt) / s.at;
  double dw = dadd(s.t_nugget, dmul(s.t_sill, dsub(1.0, corefunc(s.tvtype, adt))));
  return dw > 0.0 ? dw : 0.0;
}

// cov_tab_vgm_st, variogram_st.f90:222-277
__device__ __forceinline__ double st_cov(const KkSTModel& s, int ndim, const double2* __restrict__ tabs,
                                         const double* lag) {
  double ls[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < ndim; ++d) ls[d] = lag[d];
  double dt = lag[ndim];
  double lt[3] = {fabs(dt), 0.0, 0.0};
  double cs = model_cov(s.cs, tabs, ls);
  double ct = model_cov(s.ct, tabs, lt);
  if (s.model == 1) return dadd(dadd(dmul(dmul(s.k_ps, cs), ct), cs), ct);
  double res = dadd(cs, ct);
  if (s.has_joint) {
    double dw = st_ftime(s, dt);
    for (int k = 0; k < s.cs.nstruct; ++k) {
      const KkComp& c = s.cs.comp[k];
      double hs = aniso_h(c.mat, ndim, ls);
      double hst = __dsqrt_rn(dadd(dmul(hs, hs), dmul(dw, dw)));
      if (s.cs.mode == KK_LEVEL_A && c.tab_off >= 0 && c.sill > 0.0) {
        double r;
        if (!tab_lookup(tabs + c.tab_off, hst, &r)) r = c.tail ? comp_cov_h(c, hst) : 0.0;
        res = dadd(res, dmul(s.joint[k], r) / c.sill);
      } else {
        res = dadd(res, dmul(s.joint[k], corefunc(c.vtype, hst)));
      }
    }
  }
  return res;
}

// search-space transform of one point: rotation.f90:224-246 (mat_mul)
__device__ __forceinline__ void rotate_pt(const double* m, int ndim, const double* x, double* r) {
  if (ndim == 1) {
    r[0] = dmul(m[0], x[0]);
  } else if (ndim == 2) {
    double r0 = dadd(dmul(m[0], x[0]), dmul(m[3], x[1]));
    double r1 = dadd(dmul(m[1], x[0]), dmul(m[4], x[1]));
    r[0] = r0;
    r[1] = r1;
  } else {
    double r0 = dadd(dadd(dmul(m[0], x[0]), dmul(m[3], x[1])), dmul(m[6], x[2]));
    double r1 = dadd(dadd(dmul(m[1], x[0]), dmul(m[4], x[1])), dmul(m[7], x[2]));
    double r2 = dadd(dadd(dmul(m[2], x[0]), dmul(m[5], x[1])), dmul(m[8], x[2]));
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
  }
}

}  // namespace kk
