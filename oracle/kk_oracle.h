/*
 * kk_oracle.h -- CPU oracle for the krigekit kriging solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * engine's per-target algorithm (ougx/krigekit, src/libkriging), used
 * by tests/ and by bench.py's cpu_baseline leg as the checker and the timed
 * CPU port.  The product (krigekit_b200/) never links, loads or calls it.
 *
 * One call, orc_solve(), runs a complete solve() for a fully specified
 * problem: neighbour search (kd-tree, sector filter, maxdist filter),
 * covariance assembly from the piecewise-linear lookup tables, the block
 * Cholesky / Schur-complement solver with its LDL^T + jitter fallback,
 * conditional variance, estimate and bound clipping.  Each function in
 * kk_oracle.c cites the reference file:line it follows.
 */
#ifndef KK_ORACLE_H
#define KK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXVAR 4
#define ORC_MAXSTRUCT 16

/* One nested variogram structure (kriging.F90:211-276 argument list). */
typedef struct {
  int vtype;            /* vgmfunc.f90:7-17 ids: 0 nug .. 10 dco        */
  double nugget, sill;
  double a_major, a_minor1, a_minor2;
  double azimuth, dip, plunge;
  int is_product;
} orc_struct_spec;

typedef struct {
  int ndim;             /* spatial dimension 1..3                       */
  int nlag;             /* ndim (spatial) or ndim + 1 (space-time)      */
  int nvar, ndrift, unbias, std_ck, neglect_error, anisotropic_search;
  int nmin;             /* extension: targets with fewer neighbours -> NaN (0 = off) */
  double bounds[2];

  /* observations, column-major (nlag, nobs) like the reference's obs%coord */
  int nobs[ORC_MAXVAR];
  const double *obs_coord[ORC_MAXVAR];
  const double *obs_value[ORC_MAXVAR];
  const double *obs_var[ORC_MAXVAR];     /* may be NULL -> zeros          */
  const double *obs_drift[ORC_MAXVAR];   /* (ndrift, nobs) or NULL        */
  int nmax[ORC_MAXVAR];                  /* as passed to set_obs          */
  double maxdist[ORC_MAXVAR];            /* as passed (not squared)       */
  double sk_mean[ORC_MAXVAR];

  /* search parameters (kriging.F90:318-387) */
  double s_anis1[ORC_MAXVAR], s_anis2[ORC_MAXVAR];
  double s_az[ORC_MAXVAR], s_dip[ORC_MAXVAR], s_plunge[ORC_MAXVAR];
  int sector[ORC_MAXVAR];
  double time_at[ORC_MAXVAR];            /* space-time search scale       */

  /* variogram structures per ordered pair (ivar, jvar) */
  int nstruct[ORC_MAXVAR][ORC_MAXVAR];
  orc_struct_spec vgm[ORC_MAXVAR][ORC_MAXVAR][ORC_MAXSTRUCT];

  /* space-time model (kriging_st.F90, variogram_st.f90); st = 0 -> spatial */
  int st;
  int st_model;                          /* 0 sum-metric, 1 product-sum   */
  int st_transform;
  double st_at, st_k_ps, st_time_nugget, st_time_sill;
  int nstruct_t[ORC_MAXVAR][ORC_MAXVAR];
  orc_struct_spec vgm_t[ORC_MAXVAR][ORC_MAXVAR][ORC_MAXSTRUCT];
  double st_joint[ORC_MAXVAR][ORC_MAXVAR][ORC_MAXSTRUCT];
  int st_has_joint[ORC_MAXVAR][ORC_MAXVAR];

  /* targets: block centres (nlag, nblock); integration nodes (nlag, ngrid) */
  int nblock;
  const double *block_coord;
  const int *nblockpnt;                  /* NULL -> point kriging          */
  const double *grid_coord;              /* NULL -> block_coord            */
  const double *grid_weight;             /* NULL -> 1                      */
  const double *rangescale;              /* NULL -> 1                      */
  const double *localnugget;             /* NULL -> 0                      */
  const double *block_drift;             /* (ndrift, nvar, nblock) or NULL */

  int nthread;                           /* 0 -> OpenMP default            */
  int ncache;                            /* factor-cache slots per thread  */
  int cross_validation;                  /* leave-one-out over obs(1)      */
  int analytic;                          /* 1 -> analytic covariance, the
                                            reference's USE_COV_TABLE=0 build */
} orc_problem;

typedef struct {
  double *value;        /* (nvar, nblock)            */
  double *variance;     /* (nvar, nvar, nblock)      */
  int *nnear;           /* (nvar, nblock) or NULL    */
  int *inear;           /* (mmax, nvar, nblock) or NULL, 1-based like the reference */
  int mmax;             /* leading dimension of inear */
  double *weight;       /* (mmax, nvar(groups), nvar(targets), nblock) or NULL */
  int stats[5];         /* fail, chol_fact, chol_reuse, ssytrf_fact, ssytrf_reuse */
  int err;
  char errmsg[256];
} orc_result;

int orc_solve(const orc_problem *prob, orc_result *res);

/* Sequential Gaussian simulation of one variable over the point targets of
 * prob (set_sim_base and the simulation branches of the reference engine):
 * path holds the 1-based visiting order, sample the N(0, 1) draws as
 * sample[p * nsim + isim] for the p-th visited target. */
typedef struct {
  double *value;        /* (nsim, nblock): value[ib * nsim + isim], target order */
  double *variance;     /* (nblock) conditional variance of each target          */
  int *nnear;           /* (2, nblock): observation and simulated neighbours, or NULL */
  int *inear;           /* (mmax, nblock): 0-based; observations < nobs, then nobs + visit position; or NULL */
  int mmax;
  int err;
  char errmsg[256];
} orc_sim_result;

int orc_sgsim(const orc_problem *prob, const int *path, const double *sample, int nsim, orc_sim_result *res);

/* Building blocks exported for unit tests. */
void orc_calc_rotmat(double ang1, double ang2, double ang3, double anis1,
                     double anis2, double *out /* column-major 3x3 */);
double orc_corefunc(int vtype, double rdist);
/* Evaluate the table covariance of one (ivar, jvar) model of a problem at lag. */
double orc_cov(const orc_problem *prob, int ivar, int jvar, const double *lag);
/* kd-tree nearest neighbours over (dim, n) data, results 1-based. */
int orc_kdtree_nn(const double *data, int dim, int n, const double *qv, int nn,
                  int sort, double *dis, int *idx);
/* Bunch-Kaufman LDL^T solve of a dense symmetric system (upper storage). */
int orc_sysv(int m, double *a, int nrhs, double *b);

#ifdef __cplusplus
}
#endif
#endif
