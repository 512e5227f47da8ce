// kk_solve_common.cuh -- device helpers of the solve kernels (kk_solve.cu,
// kk_warp.cuh).
//
// Covariance lookups (fast paths and the general model), the right-hand-side
// and drift entries, the neighbour-row gather, the block prior covariance and
// the Schur-complement finish that turns the inner products of a target's
// solved columns into its estimate and variance.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "kk_device.cuh"
#include "kk_kernels.h"

// right-hand-side columns carried by the refinement form (F | k | u); systems
// with more columns are solved by the FP64 form
#define KK_REFINE_COLS 6

namespace kk {

__device__ __forceinline__ double cov_pair(const SolveParams& P, int first, int second, const double* lag) {
  if (P.st) return st_cov(P.smodels[first * P.nvar + second], P.ndim, P.tables, lag);
  return model_cov(P.models[first * P.nvar + second], P.tables, lag);
}
__device__ __forceinline__ double cov0_pair(const SolveParams& P, int first, int second) {
  if (P.st) return P.smodels[first * P.nvar + second].cov0;
  return P.models[first * P.nvar + second].cov0;
}

// lag = (a - b) / rangescale for spatial kriging (kriging.F90:783, 905);
// space-time lags are not scaled (kriging_st.F90:806)
__device__ __forceinline__ void make_lag(const SolveParams& P, const double* a, const double* b, double rs,
                                         double* lag) {
  for (int d = 0; d < P.nlag; ++d) {
    double t = dsub(a[d], b[d]);
    lag[d] = P.st ? t : t / rs;
  }
}

// F row entry a of a neighbour of variable v at observation o (obs%drift,
// kriging_base.F90:614-624)
__device__ __forceinline__ double f_entry(const SolveParams& P, int a, int v, int o) {
  if (a < P.ndrift) return __ldg(&P.odrift[v][(size_t)a * P.nobs[v] + o]);
  int ua = a - P.ndrift;
  return P.std_ck ? (ua == v ? 1.0 : 0.0) : (ua == 0 ? 1.0 : 0.0);
}
// g entry a for target variable iv (block%drift, kriging_base.F90:938-951)
__device__ __forceinline__ double g_entry(const SolveParams& P, int a, int iv, int t) {
  if (a < P.ndrift) return P.tdrift ? __ldg(&P.tdrift[((size_t)t * P.nvar + iv) * P.ndrift + a]) : 0.0;
  int ua = a - P.ndrift;
  return P.std_ck ? (ua == iv ? 1.0 : 0.0) : (ua == 0 ? 1.0 : 0.0);
}

__device__ __forceinline__ void write_nan(const SolveParams& P, int t) {
  for (int v = 0; v < P.nvar; ++v) P.est[(size_t)t * P.nvar + v] = __longlong_as_double(0x7ff8000000000000ll);
  for (int q = 0; q < P.nvar * P.nvar; ++q)
    P.var[(size_t)t * P.nvar * P.nvar + q] = __longlong_as_double(0x7ff8000000000000ll);
}

constexpr int MAXC = 8;  // forward-substituted columns: F + k + functionals (z, indicators)

// number of functional columns carried for the estimate
__device__ __forceinline__ int n_func(const SolveParams& P) {
  return 1 + ((P.ck_isa || P.sk_any) ? P.nvar : 0);
}

// prior covariance C_ij(x0, x0) for the variance (calc_variance,
// kriging.F90:989-1008): cov0 for points, node-pair sum for blocks.
static __device__ double base_cov(const SolveParams& P, int t, int iv, int jv) {
  if (!P.gstart) return cov0_pair(P, iv, jv);
  const int k0 = __ldg(&P.gstart[t]), k1 = __ldg(&P.gstart[t + 1]);
  if (k1 - k0 == 1) return cov0_pair(P, iv, jv);
  const double c0 = cov0_pair(P, iv, jv);
  double base = 0.0;
  for (int i = k0; i < k1; ++i) {
    double wi = __ldg(&P.gw[i]);
    base = dadd(base, dmul(dmul(c0, wi), wi));
    for (int j = i + 1; j < k1; ++j) {
      double lag[4];
      for (int d = 0; d < P.nlag; ++d) lag[d] = dsub(__ldg(&P.gx[d][i]), __ldg(&P.gx[d][j]));
      base = dadd(base, dmul(dmul(dmul(cov_pair(P, iv, jv, lag), wi), __ldg(&P.gw[j])), 2.0));
    }
  }
  return base;
}

// Solve the small p x p Schur system and produce est / var from the inner
// products G (FP64).  Column order: F (pa), k (nvar), u (nu).
// G is symmetric, stored full C x C.
static __device__ __noinline__ void finish_outputs(const SolveParams& P, int t, const double* G, int C, const double* zmean,
                               int* fail, double* lam_out = nullptr) {
  const int pa = P.pa, q = P.nvar, nu = n_func(P);
  const int kF = 0, kK = pa, kU = pa + q;
  double S[36], lam[KK_MAXVAR][6];
  // S = F^T K^-1 F, Cholesky (SPOTRF 'U' semantics on p x p)
  for (int a = 0; a < pa; ++a)
    for (int b = 0; b < pa; ++b) S[a * 6 + b] = G[(kF + a) * C + kF + b];
  for (int j = 0; j < pa; ++j) {
    double ajj = S[j * 6 + j];
    for (int k = 0; k < j; ++k) ajj -= S[k * 6 + j] * S[k * 6 + j];
    if (!(ajj > 0.0)) { *fail = 1; return; }
    ajj = sqrt(ajj);
    S[j * 6 + j] = ajj;
    for (int i = j + 1; i < pa; ++i) {
      double s = S[j * 6 + i];
      for (int k = 0; k < j; ++k) s -= S[k * 6 + j] * S[k * 6 + i];
      S[j * 6 + i] = s / ajj;
    }
  }
  for (int iv = 0; iv < q; ++iv) {
    // rhs_small = F^T K^-1 k - g  (solver.f90:282-286)
    double r[6];
    for (int a = 0; a < pa; ++a) r[a] = G[(kF + a) * C + kK + iv] - g_entry(P, a, iv, t);
    for (int i = 0; i < pa; ++i) {  // U^T y = r
      double s = r[i];
      for (int k = 0; k < i; ++k) s -= S[k * 6 + i] * r[k];
      r[i] = s / S[i * 6 + i];
    }
    for (int i = pa - 1; i >= 0; --i) {  // U x = y
      double s = r[i];
      for (int k = i + 1; k < pa; ++k) s -= S[i * 6 + k] * r[k];
      r[i] = s / S[i * 6 + i];
    }
    for (int a = 0; a < pa; ++a) lam[iv][a] = r[a];
  }
  // Lagrange multipliers of every target variable, lam_out[iv * 6 + a]
  if (lam_out)
    for (int iv = 0; iv < q; ++iv)
      for (int a = 0; a < pa; ++a) lam_out[iv * 6 + a] = lam[iv][a];
  // estimate (estimate_block_base, kriging_base.F90:3424-3468)
  for (int jv = 0; jv < q; ++jv) {
    // z^T w = z^T K^-1 k - (z^T K^-1 F) lambda
    double avg = G[kU * C + kK + jv];
    for (int a = 0; a < pa; ++a) avg -= G[kU * C + kF + a] * lam[jv][a];
    if (nu > 1) {
      double tw[KK_MAXVAR], tws = 0.0;
      for (int v = 0; v < q; ++v) {
        tw[v] = G[(kU + 1 + v) * C + kK + jv];
        for (int a = 0; a < pa; ++a) tw[v] -= G[(kU + 1 + v) * C + kF + a] * lam[jv][a];
        tws += tw[v];
      }
      if (P.ck_isa)
        for (int v = 0; v < q; ++v)
          if (v != jv && zmean[KK_MAXVAR + v] > 0.0) avg += (zmean[jv] - zmean[v]) * tw[v];
      if (P.unbias == 0 && P.sk_mean[jv] != 0.0) avg += (1.0 - tws) * P.sk_mean[jv];
    }
    if (avg < P.bounds[0]) avg = P.bounds[0];
    if (avg > P.bounds[1]) avg = P.bounds[1];
    P.est[(size_t)t * q + jv] = avg;
  }
  // variance: base - (w_iv^T k_jv + lambda_iv^T g_jv) (calc_variance)
  double* V = P.var + (size_t)t * q * q;
  for (int iv = 0; iv < q; ++iv)
    for (int jv = iv; jv < q; ++jv) {
      double d = G[(kK + iv) * C + kK + jv];
      for (int a = 0; a < pa; ++a) d -= lam[iv][a] * G[(kF + a) * C + kK + jv];
      for (int a = 0; a < pa; ++a) d += lam[iv][a] * g_entry(P, a, jv, t);
      double v = base_cov(P, t, iv, jv) - d;
      V[iv + jv * q] = v;
      V[jv + iv * q] = v;
    }
  for (int iv = 0; iv < q; ++iv) {
    double d = V[iv + iv * q];
    if (d < 0.0) V[iv + iv * q] = 0.0;
    for (int jv = iv + 1; jv < q; ++jv) {
      double o = V[jv + iv * q];
      if (o < 0.0) o = 0.0;
      V[jv + iv * q] = o;
      V[iv + jv * q] = o;
    }
  }
}

// finish_outputs for one variable with one unbiasedness row and z as the
// only functional column (ordinary kriging, columns F | k | z): the same
// arithmetic in the same order, in registers, with no call frame.
__device__ __forceinline__ void finish_ok(const SolveParams& P, int t, const double* G, int* fail) {
  const double s00 = G[0];
  if (!(s00 > 0.0)) {
    *fail = 1;
    return;
  }
  const double ajj = sqrt(s00);
  double lam = G[1] - g_entry(P, 0, 0, t);
  lam = lam / ajj;
  lam = lam / ajj;
  double avg = G[7];
  avg -= G[6] * lam;
  if (avg < P.bounds[0]) avg = P.bounds[0];
  if (avg > P.bounds[1]) avg = P.bounds[1];
  P.est[t] = avg;
  double d = G[4];
  d -= lam * G[1];
  d += lam * g_entry(P, 0, 0, t);
  const double v = base_cov(P, t, 0, 0) - d;
  P.var[t] = v < 0.0 ? 0.0 : v;
}

// Covariance of one neighbour row (coordinates xr, variable vr) with the
// target for target variable iv, averaged over block nodes (assemble_rhs,
// kriging.F90:889-910); defined after the fast covariance paths.
static __device__ __noinline__ double rhs_cov_row(const SolveParams& P, int t, const double* xr, int vr, int iv, double rs);

__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }

// zone constants of the lookup tables, held in registers
struct ZoneRegs {
  double zb1, zb2, zb3, zb3e, i0, i1, i2;
  int o1, o2, n0, n1, n2;
};

// The reference's lookup clamps the index to a zone's last cell but keeps
// the fraction of the unclamped index (variogram.f90:369-373), so a distance
// a few ulp below a zone's end whose index rounds up to the zone size reads
// one cell early.  The fast paths compute h to a few ulp of the reference's
// h: a table argument within 1e-6 of a cell index from a zone's ends could
// land on the other side, and the lookup returns NaN there so that the caller
// takes the exact path.  zb3e: arguments up to just past the table's end
// still go through the lookup (and its edge test).
constexpr double KK_ZONE_EDGE = 1e-6;

// The reference's zones are fixed (bounds 0, 0.1, 0.5, 3.5, steps 1e-5,
// 1e-4, 1e-3: kriging.F90:416-417, alloc_zones in variogram.f90:223-256), so
// the fast paths take them as compile-time constants, computed with the
// same operations as set_zones (which checks that they agree), and hold no
// registers for them.
constexpr double KK_ZB1 = 0.1, KK_ZB2 = 0.5, KK_ZB3 = 3.5;
constexpr int KK_ZN0 = 10000, KK_ZN1 = 4000, KK_ZN2 = 3000;
__host__ __device__ __forceinline__ ZoneRegs load_zones_host() {
  ZoneRegs z;
  z.zb1 = KK_ZB1;
  z.zb2 = KK_ZB2;
  z.zb3 = KK_ZB3;
  z.zb3e = KK_ZB3 * (1.0 + 1e-12);
  z.i0 = (double)KK_ZN0 / (KK_ZB1 - 0.0);
  z.i1 = (double)KK_ZN1 / (KK_ZB2 - KK_ZB1);
  z.i2 = (double)KK_ZN2 / (KK_ZB3 - KK_ZB2);
  z.o1 = KK_ZN0;
  z.o2 = KK_ZN0 + KK_ZN1;
  z.n0 = KK_ZN0;
  z.n1 = KK_ZN1;
  z.n2 = KK_ZN2;
  return z;
}
__device__ __forceinline__ ZoneRegs load_zones() { return load_zones_host(); }

// tab_lookup without divergent constant-memory indexing: the same zone
// choice, index and interpolation (variogram.f90:353-382, 682-710) from
// register selects.  Valid for 0 <= h < zb3.
// EDGE: the argument comes from a fast h (a few ulp from the reference's),
// so zone ends return NaN; arguments computed exactly as the reference does
// (the temporal |k_t dt|) read the table as it is.
template <bool EDGE = true>
__device__ __forceinline__ double tab_fast(const double2* __restrict__ tab, const ZoneRegs& z, double h) {
  const bool z0 = h < z.zb1, z1 = h < z.zb2;
  const double lo = z0 ? 0.0 : (z1 ? z.zb1 : z.zb2);
  const double inv = z0 ? z.i0 : (z1 ? z.i1 : z.i2);
  const int off = z0 ? 0 : (z1 ? z.o1 : z.o2);
  const int nm1 = (z0 ? z.n0 : (z1 ? z.n1 : z.n2)) - 1;
  double fi = dmul(dsub(h, lo), inv);
  if (EDGE && (fi > (double)(nm1 + 1) - KK_ZONE_EDGE || (!z0 && fi < KK_ZONE_EDGE)))
    return __longlong_as_double(0x7ff8000000000000ll);
  const int ii = (int)fi;
  const int i = off + min(ii, nm1);
  fi = dsub(fi, (double)ii);
  const double2 t = __ldg(&tab[i]);
  return dadd(t.x, dmul(fi, t.y));
}

// analytic tail past the last table zone (struct_cov_h), kept out of line so
// that the rarely taken shape code does not raise the kernels' register count
static __device__ __noinline__ double tail_cov(const KkModel* m, double h) { return model_cov_h(*m, h); }

// COV(vgm(first, second), lag) for models without the fast path; the lag
// travels by value so that callers keep it in registers
static __device__ __noinline__ double cov_pair_call(const SolveParams& P, int first, int second, double l0, double l1,
                                             double l2, double l3) {
  const double lag[4] = {l0, l1, l2, l3};
  return cov_pair(P, first, second, lag);
}

// h = |M lag| with fused multiply-adds and h = h2 * rsqrt(h2): within a few
// ulp of aniso_h, which moves the interpolated covariance by far less than
// the solve tolerance (the table is continuous in h)
__device__ __forceinline__ double aniso_h_fast(const double* m, int ndim, const double* lag) {
  double h2;
  if (ndim == 2) {
    const double rx = fma(m[0], lag[0], m[3] * lag[1]);
    const double ry = fma(m[1], lag[0], m[4] * lag[1]);
    h2 = fma(rx, rx, ry * ry);
  } else if (ndim == 3) {
    const double rx = fma(m[0], lag[0], fma(m[3], lag[1], m[6] * lag[2]));
    const double ry = fma(m[1], lag[0], fma(m[4], lag[1], m[7] * lag[2]));
    const double rz = fma(m[2], lag[0], fma(m[5], lag[1], m[8] * lag[2]));
    h2 = fma(rx, rx, fma(ry, ry, rz * rz));
  } else {
    return fabs(m[0] * lag[0]);
  }
  return h2 > 0.0 ? h2 * rsqrt(h2) : 0.0;
}

// The single model of single-variable spatial kriging (P.fast_model); its
// transform and table offsets travel in the kernel parameters, which the
// kernels read as constant operands instead of holding registers.
// Level B (1): COV(vgm, lag) = table(aniso_h(bmat, lag)), analytic tail past
// the table.
// Level A (2): COV(vgm, lag) = sum over the structures s of
// table_s(k_s * |fm lag|), in structure order like the general model_cov.
static __device__ __noinline__ double tail_comp(const KkComp* c, double h) { return comp_cov_h(*c, h); }
template <int FM>  // 1 or 2 when known at compile time, 0: read P.fast_model
__device__ __forceinline__ double fast_cov(const SolveParams& P, const ZoneRegs& z, const double* lag) {
  const double h = aniso_h_fast(P.fm, P.fm_ndim, lag);
  if (FM == 1 || (FM == 0 && P.fast_model == 1)) {
    if (h < z.zb3e) return tab_fast(P.tables + P.fm_tab_off, z, h);
    return P.fm_tail ? tail_cov(P.models, h) : 0.0;
  }
  double res = 0.0;
#pragma unroll
  for (int s = 0; s < KK_FA_MAXS; ++s) {
    if (s < P.fa_nst) {
      const double hs = P.fa_k[s] * h;
      double g;
      if (hs < z.zb3e) g = tab_fast(P.tables + P.fa_off[s], z, hs);
      else g = ((P.fa_tailmask >> s) & 1) ? tail_comp(&P.models[0].comp[s], hs) : 0.0;
      res = dadd(res, g);
    }
  }
  return res;
}

// Space-time (P.fast_model == 4): st_cov of one variable from the spatial
// table at |fm lag_s| and the temporal table at |ft_k dt| (dt = lag[P.ndim]),
// combined in st_cov's order.
__device__ __forceinline__ double fast_cov_st(const SolveParams& P, const ZoneRegs& z, const double* lag) {
  const double hs = aniso_h_fast(P.fm, P.fm_ndim, lag);
  const double dt = P.ndim == 1 ? lag[1] : (P.ndim == 2 ? lag[2] : lag[3]);
  const double ht = fabs(P.ft_k * fabs(dt));
  double cs, ct;
  if (hs < z.zb3e) cs = tab_fast(P.tables + P.fm_tab_off, z, hs);
  else cs = P.fm_tail ? tail_cov(&P.smodels[0].cs, hs) : 0.0;
  if (ht < z.zb3) ct = tab_fast<false>(P.tables + P.ft_off, z, ht);  // |k_t dt| as the reference forms it
  else ct = P.ft_tail ? tail_cov(&P.smodels[0].ct, ht) : 0.0;
  if (P.st_kind == 1) return dadd(dadd(dmul(dmul(P.st_kps, cs), ct), cs), ct);
  return dadd(cs, ct);
}

// Two variables (P.fast_model == 3): COV(vgm(i, j), lag) at pair = 2 i + j from
// that pair's Level-B table, its Level-A tables, or its analytic structures
// (vgm(i, j), i > j, as the general model_cov evaluates it), every structure
// at h_s = k_s * |fm lag|.
__device__ __forceinline__ double fast_cov_pair(const SolveParams& P, const ZoneRegs& z, const double* lag,
                                                int pair) {
  const double h = aniso_h_fast(P.fm, P.fm_ndim, lag);
  const int kind = P.fq_kind[pair];
  if (kind == 1) {
    const double hs = P.fq_k[pair][0] * h;
    if (hs < z.zb3e) return tab_fast(P.tables + P.fq_off[pair][0], z, hs);
    return (P.fq_tail[pair] & 1) ? tail_cov(P.models + pair, hs) : 0.0;
  }
  double res = 0.0;
  const int nst = P.fq_nst[pair];
#pragma unroll
  for (int s = 0; s < KK_FA_MAXS; ++s) {
    if (s < nst) {
      const double hs = P.fq_k[pair][s] * h;
      double g;
      if (kind == 3) g = comp_cov_h(P.models[pair].comp[s], hs);
      else if (hs < z.zb3e) g = tab_fast(P.tables + P.fq_off[pair][s], z, hs);
      else g = ((P.fq_tail[pair] >> s) & 1) ? tail_comp(&P.models[pair].comp[s], hs) : 0.0;
      res = dadd(res, g);
    }
  }
  return res;
}

// rhs_cov_row: the space-time fast path serves block nodes too
static __device__ __noinline__ double rhs_cov_row(const SolveParams& P, int t, const double* xr, int vr, int iv, double rs) {
  double tmp = 0.0;
  if (P.gstart) {
    const int k0 = __ldg(&P.gstart[t]), k1 = __ldg(&P.gstart[t + 1]);
    for (int k = k0; k < k1; ++k) {
      double node[4], lag[4];
      for (int d = 0; d < P.nlag; ++d) node[d] = __ldg(&P.gx[d][k]);
      make_lag(P, xr, node, rs, lag);
      double cv = P.fast_model == 4 ? fast_cov_st(P, load_zones(), lag) : cov_pair(P, vr, iv, lag);
      if (cv != cv) cv = cov_pair(P, vr, iv, lag);  // a table argument at a zone edge
      tmp = dadd(tmp, dmul(cv, __ldg(&P.gw[k])));
    }
  } else {
    double node[4], lag[4];
    for (int d = 0; d < P.nlag; ++d) node[d] = __ldg(&P.tx[d][t]);
    make_lag(P, xr, node, rs, lag);
    double cv = P.fast_model == 4 ? fast_cov_st(P, load_zones(), lag) : cov_pair(P, vr, iv, lag);
    if (cv != cv) cv = cov_pair(P, vr, iv, lag);  // a table argument at a zone edge
    tmp = dadd(tmp, dmul(cv, 1.0));
  }
  return tmp;
}

// sqrt(h2) from an FP32 reciprocal square root refined by one FP64 Newton
// step: h0 = h2 y, h = h0 + (h2 - h0^2) y / 2; relative error about 1.5 e^2
// for an FP32 error e of y.  Zero, extreme and non-finite inputs take the
// library square root.
__device__ __forceinline__ double sqrt_newton(double h2) {
  if (!(h2 > 1e-36 && h2 < 1e36)) return sqrt(h2);
  const double y = (double)rsqrtf((float)h2);
  const double h0 = h2 * y;
  return fma(fma(-h0, h0, h2), 0.5 * y, h0);
}

// table value at h, 0 <= h < zb3: the zone, index and linear interpolation
// of the reference's lookup (variogram.f90:353-382, 682-710)
template <bool EDGE = true>
__device__ __forceinline__ double tab_h(const double2* __restrict__ tab, const ZoneRegs& z, double h) {
  const bool z0 = h < z.zb1, z1 = h < z.zb2;
  const double lo = z0 ? 0.0 : (z1 ? z.zb1 : z.zb2);
  const double inv = z0 ? z.i0 : (z1 ? z.i1 : z.i2);
  const int off = z0 ? 0 : (z1 ? z.o1 : z.o2);
  const int nm1 = (z0 ? z.n0 : (z1 ? z.n1 : z.n2)) - 1;
  double fi = (h - lo) * inv;
  if (EDGE && (fi > (double)(nm1 + 1) - KK_ZONE_EDGE || (!z0 && fi < KK_ZONE_EDGE)))
    return __longlong_as_double(0x7ff8000000000000ll);
  const int ii = (int)fi;
  fi -= (double)ii;
  const double2 t = __ldg(&tab[off + min(ii, nm1)]);
  return fma(fi, t.y, t.x);
}

// per-pair description of the two-variable fast path, copied to shared
// memory so that the pair index can be dynamic
struct PairModel {
  int kind, nst, tail, pad_;
  int off[KK_FA_MAXS];
  double k[KK_FA_MAXS];
};

// COV at anisotropic distance h on the spatial fast paths: one Level-B table
// (FM 1), Level-A tables of structures at multiples of one transform (FM 2),
// two variables (FM 3, pair 2 i + j)
template <int FM>
__device__ __forceinline__ double cov_h(const SolveParams& P, const ZoneRegs& z, double h, const PairModel* pm,
                                        int pair) {
  if (FM == 1) {
    if (h < z.zb3e) return tab_h(P.tables + P.fm_tab_off, z, h);
    return P.fm_tail ? tail_cov(P.models, h) : 0.0;
  }
  if (FM == 2) {
    double res = 0.0;
#pragma unroll
    for (int s = 0; s < KK_FA_MAXS; ++s) {
      if (s < P.fa_nst) {
        const double hs = P.fa_k[s] * h;
        double g;
        if (hs < z.zb3e) g = tab_h(P.tables + P.fa_off[s], z, hs);
        else g = ((P.fa_tailmask >> s) & 1) ? tail_comp(&P.models[0].comp[s], hs) : 0.0;
        res += g;
      }
    }
    return res;
  }
  const PairModel& m = pm[pair];
  if (m.kind == 1) {
    const double hs = m.k[0] * h;
    if (hs < z.zb3e) return tab_h(P.tables + m.off[0], z, hs);
    return (m.tail & 1) ? tail_cov(P.models + pair, hs) : 0.0;
  }
  double res = 0.0;
#pragma unroll
  for (int s = 0; s < KK_FA_MAXS; ++s) {
    if (s < m.nst) {
      const double hs = m.k[s] * h;
      double g;
      if (m.kind == 3) g = comp_cov_h(P.models[pair].comp[s], hs);
      else if (hs < z.zb3e) g = tab_h(P.tables + m.off[s], z, hs);
      else g = ((m.tail >> s) & 1) ? tail_comp(&P.models[pair].comp[s], hs) : 0.0;
      res += g;
    }
  }
  return res;
}

// space-time fast path (FM 4): spatial table at hs, temporal table at
// |ft_k dt|, combined in st_cov's order
__device__ __forceinline__ double cov_st_h(const SolveParams& P, const ZoneRegs& z, double hs, double dt) {
  const double ht = fabs(P.ft_k * fabs(dt));
  double cs, ct;
  if (hs < z.zb3e) cs = tab_h(P.tables + P.fm_tab_off, z, hs);
  else cs = P.fm_tail ? tail_cov(&P.smodels[0].cs, hs) : 0.0;
  if (ht < z.zb3) ct = tab_h<false>(P.tables + P.ft_off, z, ht);  // |k_t dt| as the reference forms it
  else ct = P.ft_tail ? tail_cov(&P.smodels[0].ct, ht) : 0.0;
  if (P.st_kind == 1) return P.st_kps * cs * ct + cs + ct;
  return cs + ct;
}

// start of column c of the strictly-lower packed factor
template <int N>
__device__ __forceinline__ int lcol(int c) { return c * (N - 1) - (c * (c - 1)) / 2; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Neighbour rows of target t in matrix order (variable blocks in order,
// ascending index within a block: assemble_linear_system_base,
// kriging_base.F90:3159-3235) into per-warp shared arrays.  Returns the row
// count n and the block starts of variables 1..3.
template <int N>
__device__ __forceinline__ int gather_rows(const SolveParams& P, int t, int lane, double (*x)[N], double* z,
                                           int* obs, int* var, int& ist1, int& ist2, int& ist3) {
  const int q = P.nvar;
  int n = 0;
  ist1 = ist2 = ist3 = 0x7fffffff;
#pragma unroll
  for (int v = 0; v < KK_MAXVAR; ++v) {
    if (v < q) {
      if (v == 1) ist1 = n;
      if (v == 2) ist2 = n;
      if (v == 3) ist3 = n;
      n += __ldg(&P.nnear[v][t]);
    }
  }
  for (int r = lane; r < n; r += 32) {
    const int v = (r >= ist1) + (r >= ist2) + (r >= ist3);
    const int i0 = v == 0 ? 0 : (v == 1 ? ist1 : (v == 2 ? ist2 : ist3));
    const int o = __ldg(&P.nbr[v][(size_t)t * P.mmax[v] + (r - i0)]);
    obs[r] = o;
    var[r] = v;
    for (int d = 0; d < P.nlag; ++d) x[d][r] = __ldg(&P.ox[v][d][o]);
    if (z) z[r] = __ldg(&P.oval[v][o]);
  }
  __syncwarp();
  return n;
}

}  // namespace kk
