/*
 * krigekit_b200.h -- C-ABI of libkrigecuda.so, the B200 kriging solve path.
 *
 * The krige_* entry points keep the names, argument order, array layouts
 * (Fortran column-major, 1-based variable indices) and error convention of
 * the reference engine's ISO_C_BINDING layer (ougx/krigekit
 * src/libkriging/kriging_capi.F90, kriging_capi_common.F90): every function
 * returns 0 on success and 1 on error, with the message available through
 * krige_get_last_error().  A caller that binds the reference library with
 * ctypes (src/krigekit/kriging.py:142-286) can bind this library instead.
 * Inputs are copied at each set_* call; outputs go to caller buffers.
 * Device memory is allocated by the library (cudaMalloc, or the allocator
 * registered with krige_set_allocator).
 */
#ifndef KRIGEKIT_B200_H
#define KRIGEKIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kriging_capi.F90:43-57 krige_create: new handle (1-based registry slot). */
int krige_create(int64_t *handle);
/* kriging_capi.F90:83-100 krige_ind_create: handle for multiple indicator kriging; after
 * each solve the first ncat estimates per target (category probabilities) are clipped to
 * [0, 1] and normalised to sum to one (post_solve_indicator, kriging_indicator.F90:170-185). */
int krige_ind_create(int64_t *handle);
/* kriging_capi.F90:113- krige_ind_set_ncat: categories (1..nvar), after krige_initialize;
 * variables past ncat are secondary co-variates outside the normalisation. */
int krige_ind_set_ncat(int64_t handle, int ncat);
/* kriging_capi_common.F90 krige_destroy (release_obj_base): frees device and host state. */
int krige_destroy(int64_t *handle);

/* kriging_capi.F90:143-192 krige_initialize -> initialize_base (kriging_base.F90:467-553).
 * nsim > 0 selects sequential Gaussian simulation (krige_set_sim; one variable; seed seeds
 * the draws when the caller gives none); weight_correction, varying_vgm and a non-empty
 * weight_file are outside the GPU path and return an error; store_weight / use_old_weight
 * select the in-memory weight store (below). */
int krige_initialize(int64_t handle, int ndim, int nvar, int ndrift, int unbias, int nsim,
                     int anisotropic_search, int weight_correction, int use_old_weight,
                     int store_weight, int cross_validation, int write_mat, int neglect_error,
                     int varying_vgm, int std_ck, int verbose, int pf_cache,
                     const char *weight_file, const double *bounds /* [2] */, int seed);

/* kriging_capi.F90:197-224 krige_set_obs: coord(ndim_c, nobs), value(nobs), variance(nobs). */
int krige_set_obs(int64_t handle, int ivar, int nobs, int ndim_c, const double *coord,
                  const double *value, const double *variance, int nmax, double maxdist,
                  double sk_mean);
/* kriging_capi.F90 krige_update_obs_value -> update_obs_value_base (kriging_base.F90:649-680). */
int krige_update_obs_value(int64_t handle, int ivar, int nobs, const double *value);
/* kriging_capi.F90 krige_set_obs_drift: drift(ndrift_c, nobs). */
int krige_set_obs_drift(int64_t handle, int ivar, int ndrift_c, int nobs, const double *drift);

/* kriging_capi.F90:230-243 krige_reset_vgm. */
int krige_reset_vgm(int64_t handle, int ivar, int jvar);
/* kriging_capi.F90:245-268 krige_set_vgm -> set_vgm (kriging.F90:211-276); jvar >= ivar. */
int krige_set_vgm(int64_t handle, int ivar, int jvar, const char *vtype, double nugget,
                  double sill, double a_major, double a_minor1, double a_minor2,
                  double azimuth, double dip, double plunge, int is_product);

/* kriging_capi.F90:310-331 krige_set_grid: coord(ndim_c, ngrid), rangescale/localnugget(ngrid). */
int krige_set_grid(int64_t handle, int ngrid, int ndim_c, const double *coord,
                   const double *rangescale, const double *localnugget);
/* kriging_capi.F90:334-378 krige_set_grid_block: block_type -4 (Gauss quadrature,
 * coord = centres, blocksize(ndim_c, nblock)) or > 0 (coord = nodes, nblockpnt, pointweight). */
int krige_set_grid_block(int64_t handle, int block_type, int ngrid, int ndim_c,
                         const double *coord, int nblock, const int *nblockpnt,
                         const double *pointweight, const double *blocksize,
                         const double *rangescale, const double *localnugget);
/* kriging_capi.F90 krige_set_grid_cv -> set_grid_cv_base (kriging_base.F90:1120-1135). */
int krige_set_grid_cv(int64_t handle);
/* kriging_capi.F90:380-397 krige_set_grid_drift: drift(ndrift_c, nblocks); ivar < 0 = all. */
int krige_set_grid_drift(int64_t handle, int ivar, int ndrift_c, int nblocks, const double *drift);

/* kriging_capi.F90:448-467 krige_set_search -> set_search (kriging.F90:318-387). */
int krige_set_search(int64_t handle, int ivar, double anis1, double anis2, double azimuth,
                     double dip, double plunge, int sector_search);

/* kriging_capi_common.F90:229-239 krige_solve -> solve_base (kriging_base.F90:2064-2194).
 * nthread and ncache (CPU threads, factor-cache slots) are accepted and ignored. */
int krige_solve(int64_t handle, int nthread, int ncache);
/* kriging_capi_common.F90:113-128 krige_solver_stats: out[5] = fail, chol_fact,
 * chol_reuse, ssytrf_fact, ssytrf_reuse (the GPU solves every target: no reuse). */
void krige_solver_stats(int64_t handle, int *out);
/* kriging_capi_common.F90:90-96 krige_get_last_error. */
int krige_get_last_error(char *buffer, int nbuf);

/* ---- weight store (in memory; kriging_base.F90:2703-2990, bound in the reference by
 * src/krigekit/kriging.py:259-274).  krige_initialize with store_weight = 1 keeps the
 * kriging weights and neighbour lists of the next krige_solve on the device (that solve
 * runs the FP64 form); krige_update_obs_value then makes the next krige_solve a
 * re-estimate from the stored weights (no search, no solve).  use_old_weight = 1 with
 * krige_set_weights does the same with a caller's store.  Weight files are not written:
 * weight_file must be empty.  Layouts are Fortran column-major; nm = the largest
 * neighbour-list length (nmax, 2^ndim nmax with sectors, nobs when every observation
 * is a neighbour), ng = nvar groups.  "Weight store not allocated" without a store. */
/* krige_get_weight_dims: nm, ng = nvar, nb = nblocks. */
int krige_get_weight_dims(int64_t handle, int *nm, int *ng, int *nb);
/* nnear(ng, nb). */
int krige_get_weight_nnear(int64_t handle, int ng, int nb, int *out);
/* inear(nm, ng, nb), 1-based, zero past nnear. */
int krige_get_weight_inear(int64_t handle, int nm, int ng, int nb, int *out);
/* weight(nm, ng, nv, nb): weight of neighbour i of group g for target variable v. */
int krige_get_weight_data(int64_t handle, int nm, int ng, int nv, int nb, double *out);
/* var(nv, nv, nb): the conditional covariance stored with the weights. */
int krige_get_weight_var(int64_t handle, int nv, int nb, double *out);
/* Load a store (layouts as the getters; order(nb) is accepted and unused, var may be
 * NULL for zero variances); the next krige_solve re-estimates from it. */
int krige_set_weights(int64_t handle, int nm, int ng, int nv, int nb, const int *nnear, const int *inear,
                      const double *weight, const int *order, const double *var);
/* Release the store. */
int krige_free_weight_store(int64_t handle);
/* kriging_capi_common.F90 krige_to_str: configuration summary owned by the handle. */
const char *krige_to_str(int64_t handle);

/* kriging_capi_common.F90 krige_get_nblocks / krige_get_nsim. */
int krige_get_nblocks(int64_t handle, int *nblocks);
int krige_get_nsim(int64_t handle, int *nsim);
/* kriging_capi_common.F90:277-288 krige_get_block_coord: out(ndim_c, nblocks). */
int krige_get_block_coord(int64_t handle, int ndim_c, int nblocks, double *out);
/* kriging_capi_common.F90:290-306 krige_get_estimate: out(nblocks, nsim_c), variable 1
 * (the realisations of a sequential simulation when nsim > 0). */
int krige_get_estimate(int64_t handle, int nsim_c, int nblocks, double *out);
/* kriging_capi.F90:410-443 krige_set_sim: SGSIM visiting order randpath(nblocks), 1-based,
 * and N(0, 1) draws sample(nsim_c, nvar_c, nblocks) of the p-th visited target; either
 * pointer may be NULL (a seeded random order / draws, not the reference's generator).
 * One variable and point targets; sector search and external drift as in kriging. */
int krige_set_sim(int64_t handle, int nblocks, const int *randpath, int nsim_c, int nvar_c,
                  const double *sample);
/* No counterpart in the reference.  How a simulation draws its values: 0 (default) every
 * dependency level in one cooperative launch, 1 one launch per level.  Both give the same
 * values bit for bit. */
int krige_set_sim_draw(int64_t handle, int by_level);
/* No counterpart in the reference.  Neighbour sets of the last sequential simulation:
 * nnear(2, nblocks) = observation and simulated members; inear(mmax, nblocks), 0-based, in
 * each target's system order: observations (< nobs), then nobs + visiting position. */
int krige_get_sim_neighbours(int64_t handle, int nblocks, int mmax, int *nnear, int *inear);
/* kriging_capi_common.F90:323-344 krige_get_estimate_all: out(nblocks, nvar_c, nsim_c). */
int krige_get_estimate_all(int64_t handle, int nblocks, int nvar_c, int nsim_c, double *out);
/* kriging_capi_common.F90:352-369 krige_get_variance: out(nblocks), variable 1. */
int krige_get_variance(int64_t handle, int nblocks, double *out);
/* kriging_capi_common.F90:372-392 krige_get_variance_all: out(nblocks, nvar_c, nvar_c). */
int krige_get_variance_all(int64_t handle, int nblocks, int nvar_c, double *out);

/* ---- space-time kriging (kriging_st_capi.f90) ----
 * Coordinates are the spatial ones followed by time.  krige_solve, the
 * getters, krige_set_grid_cv, krige_update_obs_value and krige_set_obs_drift
 * are shared with spatial kriging.  The reference engine is 3-D spatial + time;
 * this library takes the spatial dimension (1..3) from the first
 * krige_st_set_obs and expects spatial coordinate arrays of that dimension. */
/* kriging_st_capi.f90:43-75 */
int krige_st_create(int64_t *handle);
int krige_st_destroy(int64_t *handle);
/* kriging_st_capi.f90:80-123 krige_st_initialize -> t_kriging_st%initialize (std_ck cokriging). */
int krige_st_initialize(int64_t handle, int nvar, int ndrift, int unbias, int nsim, int anisotropic_search,
                        int weight_correction, int use_old_weight, int store_weight, int cross_validation,
                        int write_mat, int neglect_error, int verbose, const char *weight_file,
                        const double *bounds /* [2] */, int seed);
/* kriging_st_capi.f90:128-162: model "sum_metric" | "product_sum", transform = variogram type of f(dt). */
int krige_st_set_st_model(int64_t handle, const char *model, const char *transform, double at,
                          double time_nugget, double time_sill, double k_ps);
/* kriging_st_capi.f90:167-189: coord(ndim+1, nobs), last row = time. */
int krige_st_set_obs(int64_t handle, int ivar, int nobs, int ndim, const double *coord, const double *value,
                     const double *variance, int nmax, double maxdist, double sk_mean);
/* kriging_st_capi.f90:245-258 */
int krige_st_reset_vgm(int64_t handle, int ivar, int jvar);
/* kriging_st_capi.f90:260-287: one spatial structure of vgm(ivar, jvar). */
int krige_st_set_vgm(int64_t handle, int ivar, int jvar, const char *vtype, double nugget, double sill,
                     double a_major, double a_minor1, double a_minor2, double azimuth, double dip,
                     double plunge);
/* kriging_st_capi.f90:289-309: one temporal structure (practical range at_k). */
int krige_st_set_vgm_temporal(int64_t handle, int ivar, int jvar, const char *vtype, double nugget,
                              double sill, double at_k);
/* kriging_st_capi.f90:311-325: joint sills of the sum-metric model, one per spatial structure. */
int krige_st_set_vgm_joint_sills(int64_t handle, int ivar, int jvar, int nsill, const double *sills);
/* kriging_st_capi.f90:331-353: coord(ndim, ngrid), time(ngrid). */
int krige_st_set_grid(int64_t handle, int ngrid, const double *coord, const double *time,
                      const double *rangescale, const double *localnugget);
/* kriging_st_capi.f90:355-388: block centres coord(ndim, nblocks) + time; integration nodes
 * blockcoord(ndim, npnts_total) + blocktime with pointweight. */
int krige_st_set_grid_block(int64_t handle, int nblocks, const double *coord, const double *time,
                            const int *nblockpnt, int npnts_total, const double *blockcoord,
                            const double *blocktime, const double *pointweight, const double *rangescale,
                            const double *localnugget);
/* kriging_st_capi.f90:392-406: drift(ndrift_c, nblocks), every variable. */
int krige_st_set_grid_drift(int64_t handle, int ndrift_c, int nblocks, const double *drift);
/* kriging_st_capi.f90:458-490 -> set_search (kriging_st.F90:322-403): search-space time = t * time_at. */
int krige_st_set_search(int64_t handle, int ivar, double time_at, double anis1, double anis2, double azimuth,
                        double dip, double plunge, int sector_search);

/* ---- extensions of the GPU library (no counterpart in the reference) ---- */
/* 0 = FP64 throughout, 1 = FP32 factorisation with an FP64 residual correction (systems of at
 * most six right-hand-side columns; wider ones stay FP64), 2 = auto (default): per neighbour-count
 * list the faster of the two as timed by the kernel tuner (FP64 when not tuned).  Every form
 * meets 1e-6 relative accuracy; 0 meets the FP64 one. */
int krige_set_precision(int64_t handle, int mode);
/* Targets with fewer than nmin neighbours return NaN (0 = reference behaviour). */
int krige_set_nmin(int64_t handle, int nmin);
/* CUDA device ordinal and cudaStream_t used by this handle. */
int krige_set_device(int64_t handle, int device, void *stream);
/* Route device allocations through caller callbacks (e.g. a framework allocator). */
void krige_set_allocator(void *(*alloc)(size_t bytes, void *ctx), void (*release)(void *ptr, void *ctx),
                         void *ctx);
/* Neighbour sets of the last solve: nnear(nblocks), inear(mmax, nblocks), 1-based ascending. */
int krige_get_neighbours(int64_t handle, int ivar, int nblocks, int mmax, int *nnear, int *inear);
/* Leading dimension of the neighbour list of variable ivar. */
int krige_get_mmax(int64_t handle, int ivar, int *mmax);
/* Per-target status bits of the last solve (tie/overflow search fallback, FP64
 * re-solve, LDL^T path, failure, no neighbours). */
int krige_get_status(int64_t handle, int nblocks, int *status);
/* Counters of the last solve: out8 = fail, cholesky, 0, ldlt, 0, search fallbacks,
 * FP64 re-solves, refinement iterations; solve_ms = wall time of krige_solve. */
int krige_gpu_stats(int64_t handle, int *out8, double *solve_ms);

/* No counterpart in the reference.  Raw device counters of the last solve, out[0..n), n <= 32:
 * [0..2] targets per size bucket (<= 32, 33..64, > 128 neighbours), [3] general-kernel
 * list, [4] FP32 systems re-solved in FP64, [5] failures (NaN), [6] Cholesky solves,
 * [7] LDL^T solves, [16..19] search fallbacks per variable, [20] refinement passes,
 * [21] LDL^T solves that needed the 1e-6 mean-diagonal jitter, [22] targets with
 * 65..128 neighbours; after a simulation (nsim > 0) [24] 1 when its draws ran as one
 * launch (0: level by level) and [25] its number of dependency levels. */
int krige_gpu_counters(int64_t handle, int n, int *out);
/* No counterpart in the reference (its solver has one CPU path).  How krige_solve picks
 * the kernel for each neighbour-count list (2..32, 33..64, > 128, 65..128 equations):
 * mode 0 = fixed plan (warp per target up to 64, CTA per target up to 128, general kernel
 * beyond), 1 = time the candidate kernels on a sample of each list once per system
 * signature and keep the fastest (process-wide cache; the default), 2 = time them again
 * on the next solve. */
int krige_set_autotune(int64_t handle, int mode);
/* Plan of the last solve: kernel4[list] = 0 warp/32, 1 warp/64, 2 CTA/128, 3 general,
 * 4 warp/32 FP32 + correction, 5 warp/64 FP32 + correction, -1 empty list;
 * us24[list * 6 + kernel] = tuner's microseconds per target (NaN where not timed).
 * Either pointer may be NULL. */
int krige_get_kernel_plan(int64_t handle, int *kernel4, double *us24);
/* Forget every cached plan (all handles). */
int krige_autotune_clear(void);
/* Enable per-phase CUDA-event timing of krige_solve (one event sync per phase). */
int krige_gpu_profile(int64_t handle, int enable);
/* Device ms per phase of the last solve: search, bucket, solve kernels, fallbacks;
 * launches = kernels launched by that solve. */
int krige_gpu_phases(int64_t handle, double *out4, int *launches);
/* Device ms of the last profiled solve's assembly launches (out2[0]) and factorisation
 * launches (out2[1]) of the register kernels, each timed on its own. */
int krige_gpu_kernel_ms(int64_t handle, double *out2);

/* No counterpart in the reference.  Allocation-free FP64 re-solve: repeats the
 * last krige_solve of this handle with the same neighbour sets, after replacing
 * the observation values of variable ivar with value[nobs] (value may be NULL
 * to keep them).  It allocates no device memory: the one-thread-per-target
 * kernel runs with its workspace, work list and counters in a fixed 32 MiB
 * static device array.  A system whose workspace exceeds that array (about
 * 1440 equations for one variable) is rejected with an error.  Needs a
 * completed krige_solve with no set_obs / set_grid / set_search since.  The
 * first call on a device looks up the array's address and belongs before any
 * stream capture on that device.  Calls on one device share the array and are
 * serialised inside the library; the call returns after its work has finished.
 * Results are read with the usual getters. */
int krige_resolve_static(int64_t handle, int ivar, int nobs, const double *value);

#ifdef __cplusplus
}
#endif
#endif
