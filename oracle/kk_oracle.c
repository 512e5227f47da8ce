/*
 * kk_oracle.c -- CPU oracle for the krigekit kriging solve path.
 *
 * TEST INFRASTRUCTURE ONLY (see kk_oracle.h).  Plain C restatement of the
 * reference engine (ougx/krigekit, gfortran -O2 -fdefault-real-8, no FMA):
 * every routine below cites the Fortran it follows.  Compile with
 * -ffp-contract=off so that each multiply and add rounds separately, as in
 * the reference build.  The kd-tree section restates the published kdtree2
 * algorithm (M. Kennel 2004, AFL 1.1) bundled in the reference as
 * src/libkriging/kdtree2_maxidx.f90; the LDL^T section restates netlib
 * LAPACK dsytf2/dsytrs (BSD) bundled as src/libkriging/lapack.f.
 */
#include "kk_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* constants (common.f90:7-12)                                              */
/* ------------------------------------------------------------------------ */
static double orc_pi(void) { return 4.0 * atan(1.0); }
#define ORC_EPSLON 1.0e-10
#define ORC_MAT_TOL 1.0e-6  /* variogram.f90:54 */
#define ORC_ANG_TOL 1.0e-4  /* variogram.f90:56 */

enum { VGM_NUG = 0, VGM_SPH, VGM_EXP, VGM_GAU, VGM_HOL, VGM_POW, VGM_BSQ,
       VGM_CIR, VGM_LIN, VGM_CYC, VGM_DCO };

/* corefunc_fn, vgmfunc.f90:28-67 */
double orc_corefunc(int vtype, double r) {
  const double pi = orc_pi();
  switch (vtype) {
    case VGM_NUG: return 0.0;
    case VGM_SPH: return (r < 1.0) ? 1.0 - 1.5 * r + 0.5 * (r * r * r) : 0.0;
    case VGM_EXP: return exp(-3.0 * r);
    case VGM_GAU: return exp(-3.0625 * (r * r));
    case VGM_HOL: return cos(pi * r);
    case VGM_POW: return (r < 1.0) ? 1.0 - pow(r, 1.5) : 0.0;
    case VGM_BSQ: { double t = 1.0 - r * r; return (r < 1.0) ? t * t : 0.0; }
    case VGM_CIR:
      return (r < 1.0) ? 1.0 - (2.0 * r * sqrt(1.0 - r * r) + 2.0 * asin(r)) / pi : 0.0;
    case VGM_LIN: return (r < 1.0) ? 1.0 - r : 0.0;
    case VGM_CYC: { double s = sin(pi * r); return exp(-2.0 * (s * s)); }
    case VGM_DCO: return exp(-3.0 * r) * cos(pi * r);
    default: return 0.0;
  }
}

/* corefunc_has_analytic_tail, vgmfunc.f90:71-80 */
static int orc_has_tail(int vtype) {
  return vtype == VGM_EXP || vtype == VGM_GAU || vtype == VGM_HOL ||
         vtype == VGM_CYC || vtype == VGM_DCO;
}

/* ------------------------------------------------------------------------ */
/* rotation (rotation.f90)                                                  */
/* ------------------------------------------------------------------------ */
/* c = a*b for column-major 3x3, k summed in ascending order from zero. */
static void mat3_mul(const double *a, const double *b, double *c) {
  double t[9];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + a[i + 3 * k] * b[k + 3 * j];
      t[i + 3 * j] = s;
    }
  memcpy(c, t, sizeof t);
}

/* calc_rotmat, rotation.f90:51-95 (column-major out) */
void orc_calc_rotmat(double ang1, double ang2, double ang3, double anis1,
                     double anis2, double *m) {
  const double deg2rad = orc_pi() / 180.0;
  for (int i = 0; i < 9; ++i) m[i] = 0.0;
  m[0] = 1.0 / anis1;
  m[4] = 1.0;
  m[8] = 1.0 / anis2;
  double t[9];
  if (fabs(ang3) > ORC_EPSLON) {
    double alpha = -ang3 * deg2rad, sa = sin(alpha), ca = cos(alpha);
    double tt[9] = {ca, 0.0, sa, 0.0, 1.0, 0.0, -sa, 0.0, ca};
    memcpy(t, tt, sizeof t);
    mat3_mul(m, t, m);
  }
  if (fabs(ang2) > ORC_EPSLON) {
    double alpha = -ang2 * deg2rad, sa = sin(alpha), ca = cos(alpha);
    double tt[9] = {1.0, 0.0, 0.0, 0.0, ca, sa, 0.0, -sa, ca};
    memcpy(t, tt, sizeof t);
    mat3_mul(m, t, m);
  }
  if (fabs(ang1) > ORC_EPSLON) {
    double alpha = ang1 * deg2rad, sa = sin(alpha), ca = cos(alpha);
    double tt[9] = {ca, sa, 0.0, -sa, ca, 0.0, 0.0, 0.0, 1.0};
    memcpy(t, tt, sizeof t);
    mat3_mul(m, t, m);
  }
}

/* mat_mul for one point, rotation.f90:224-246 */
static void rotate_pt(const double *m, int ndim, const double *x, double *r) {
  if (ndim == 1) {
    r[0] = m[0] * x[0];
  } else if (ndim == 2) {
    double r0 = m[0] * x[0] + m[3] * x[1];
    double r1 = m[1] * x[0] + m[4] * x[1];
    r[0] = r0; r[1] = r1;
  } else {
    double r0 = m[0] * x[0] + m[3] * x[1] + m[6] * x[2];
    double r1 = m[1] * x[0] + m[4] * x[1] + m[7] * x[2];
    double r2 = m[2] * x[0] + m[5] * x[1] + m[8] * x[2];
    r[0] = r0; r[1] = r1; r[2] = r2;
  }
}

/* ------------------------------------------------------------------------ */
/* variogram model + lookup tables (variogram.f90)                          */
/* ------------------------------------------------------------------------ */
#define TAB_NZ 3
static const double TAB_HB[TAB_NZ + 1] = {0.0, 0.1, 0.5, 3.5}; /* kriging.F90:416-417 */
static const double TAB_DH[TAB_NZ] = {1e-5, 1e-4, 1e-3};

typedef struct {
  int nz, n;                 /* zones, total intervals                   */
  double bounds[TAB_NZ + 1];
  double inv_dh[TAB_NZ];
  int offset[TAB_NZ], zn[TAB_NZ];
  double hmax;
  double *tab;               /* tab[0..n]                                */
  int tail;
} orc_table;

typedef struct {
  int vtype;
  double sill, nugget;
  double a_major, a_minor1, a_minor2, az, dip, plunge;
  int is_product;
  int ndim;
  double mat[9];
  orc_table t;               /* Level-A per-component table              */
  int tab_ready;
} orc_comp;

typedef struct {
  int ndim, nstruct;
  double cov0;
  orc_comp c[ORC_MAXSTRUCT];
  int level_b;               /* struct_tab_ready                         */
  double bmat[9];            /* struct_aniso%mat                         */
  orc_table bt;
} orc_model;

/* build_aniso_mat, variogram.f90:185-192 */
static void comp_build_aniso(orc_comp *c) {
  orc_calc_rotmat(c->az, c->dip, c->plunge, c->a_minor1 / c->a_major,
                  c->a_minor2 / c->a_major, c->mat);
  for (int i = 0; i < 9; ++i) c->mat[i] = c->mat[i] / c->a_major;
}

/* aniso_h, variogram.f90:194-210 */
static double aniso_h(const double *m, int ndim, const double *lag) {
  if (ndim == 1) return fabs(lag[0] * m[0]);
  if (ndim == 2) {
    double rx = m[0] * lag[0] + m[3] * lag[1];
    double ry = m[1] * lag[0] + m[4] * lag[1];
    return sqrt(rx * rx + ry * ry);
  }
  double rx = m[0] * lag[0] + m[3] * lag[1] + m[6] * lag[2];
  double ry = m[1] * lag[0] + m[4] * lag[1] + m[7] * lag[2];
  double rz = m[2] * lag[0] + m[5] * lag[1] + m[8] * lag[2];
  return sqrt(rx * rx + ry * ry + rz * rz);
}

/* alloc_zones, variogram.f90:223-256 */
static void table_zones(orc_table *t) {
  t->nz = TAB_NZ;
  int off = 0;
  for (int k = 0; k < TAB_NZ; ++k) {
    int nk = (int)lround((TAB_HB[k + 1] - TAB_HB[k]) / TAB_DH[k]);
    if (nk < 1) nk = 1;
    t->zn[k] = nk;
    t->offset[k] = off;
    t->inv_dh[k] = (double)nk / (TAB_HB[k + 1] - TAB_HB[k]);
    off += nk;
  }
  for (int k = 0; k <= TAB_NZ; ++k) t->bounds[k] = TAB_HB[k];
  t->n = off;
  t->hmax = TAB_HB[TAB_NZ];
}

/* comp_cov_h, variogram.f90:327-337 */
static double comp_cov_h(const orc_comp *c, double h) {
  const double eps = DBL_MIN * 1.0e3;
  if (h > eps) return c->sill * orc_corefunc(c->vtype, h);
  return c->sill + c->nugget;
}

/* comp_build_table, variogram.f90:263-324 */
static void comp_build_table(orc_comp *c) {
  table_zones(&c->t);
  c->t.tab = (double *)malloc(sizeof(double) * (c->t.n + 1));
  c->t.tab[0] = c->sill + c->nugget;
  int off = 0;
  for (int k = 0; k < c->t.nz; ++k) {
    double hlo = c->t.bounds[k];
    double step = 1.0 / c->t.inv_dh[k];
    for (int i = 1; i <= c->t.zn[k]; ++i) {
      double r = hlo + (double)i * step;
      c->t.tab[off + i] = c->sill * orc_corefunc(c->vtype, r);
    }
    off += c->t.zn[k];
  }
  c->t.tail = orc_has_tail(c->vtype);
  c->tab_ready = 1;
}

/* table lookup shared by comp_cov_tab_h (variogram.f90:353-382) and
 * cov_struct_tab_h (variogram.f90:682-710); returns 1 when the caller must
 * fall back to the analytic tail. */
static int table_lookup(const orc_table *t, double h, double *res) {
  if (h >= t->hmax) return 1;
  if (h <= 0.0) { *res = t->tab[0]; return 0; }
  for (int k = 0; k < t->nz; ++k) {
    if (h < t->bounds[k + 1]) {
      double fi = (h - t->bounds[k]) * t->inv_dh[k];
      int ii = (int)fi;
      int i = t->offset[k] + (ii < t->zn[k] - 1 ? ii : t->zn[k] - 1);
      fi = fi - (double)ii;
      *res = t->tab[i] + fi * (t->tab[i + 1] - t->tab[i]);
      return 0;
    }
  }
  return 1;
}

static double comp_cov_tab_h(const orc_comp *c, double h) {
  if (!c->tab_ready) return comp_cov_h(c, h);
  double r;
  if (table_lookup(&c->t, h, &r)) return c->t.tail ? comp_cov_h(c, h) : 0.0;
  return r;
}

/* struct_cov_h, variogram.f90:713-729 */
static double model_cov_h(const orc_model *m, double h) {
  double res = 0.0;
  int iv = 0;
  while (iv < m->nstruct) {
    double g = comp_cov_h(&m->c[iv], h);
    while (iv < m->nstruct - 1 && m->c[iv + 1].is_product) {
      ++iv;
      g = g * comp_cov_h(&m->c[iv], h);
    }
    res = res + g;
    ++iv;
  }
  return res;
}

/* struct_recompute_cov0, variogram.f90:853-869 */
static void model_cov0(orc_model *m) {
  double total = 0.0;
  int iv = 0;
  while (iv < m->nstruct) {
    double g = m->c[iv].sill + m->c[iv].nugget;
    while (iv < m->nstruct - 1 && m->c[iv + 1].is_product) {
      ++iv;
      g = g * (m->c[iv].sill + m->c[iv].nugget);
    }
    total = total + g;
    ++iv;
  }
  m->cov0 = total;
}

/* build_composite_table, variogram.f90:572-679 */
static void model_build_composite(orc_model *m, int ref_idx) {
  orc_table *t = &m->bt;
  table_zones(t);
  double aref = m->c[ref_idx].a_major;
  t->tab = (double *)malloc(sizeof(double) * (t->n + 1));
  t->tab[0] = m->cov0;
  for (int k = 0; k < t->nz; ++k) {
    double hlo = t->bounds[k];
    double step = 1.0 / t->inv_dh[k];
    for (int i = 1; i <= t->zn[k]; ++i) {
      double r = hlo + (double)i * step;
      double val = 0.0;
      int iv = 0;
      while (iv < m->nstruct) {
        const orc_comp *c = &m->c[iv];
        if (c->vtype == VGM_NUG) { ++iv; continue; }
        double rk = r * aref / c->a_major;
        double g = c->sill * orc_corefunc(c->vtype, rk);
        while (iv < m->nstruct - 1) {
          if (!m->c[iv + 1].is_product) break;
          ++iv;
          const orc_comp *cc = &m->c[iv];
          rk = r * aref / cc->a_major;
          g = g * cc->sill * orc_corefunc(cc->vtype, rk);
        }
        val = val + g;
        ++iv;
      }
      t->tab[t->offset[k] + i] = val;
    }
  }
  /* analytic-tail flag (variogram.f90:655-673) */
  int tail = 0, iv = 0;
  while (iv < m->nstruct) {
    if (orc_has_tail(m->c[iv].vtype) && m->c[iv].vtype != VGM_NUG) {
      int gt = 1;
      while (iv < m->nstruct - 1 && m->c[iv + 1].is_product) {
        ++iv;
        gt = gt && orc_has_tail(m->c[iv].vtype);
      }
      tail = tail || gt;
    }
    ++iv;
  }
  t->tail = tail;
  memcpy(m->bmat, m->c[ref_idx].mat, sizeof m->bmat);
  m->level_b = 1;
}

/* struct_build_table, variogram.f90:497-537 */
static void model_build_table(orc_model *m) {
  int ref = -1;
  for (int iv = 0; iv < m->nstruct; ++iv) {
    const orc_comp *c = &m->c[iv];
    if (c->vtype == VGM_NUG) continue;
    if (ref < 0) { ref = iv; continue; }
    const orc_comp *r = &m->c[ref];
    int mismatch = 0;
    if (c->is_product) {
      mismatch = fabs(c->az - r->az) > ORC_ANG_TOL || fabs(c->dip - r->dip) > ORC_ANG_TOL ||
                 fabs(c->plunge - r->plunge) > ORC_ANG_TOL;
    } else {
      double mx = 0.0;
      for (int q = 0; q < 9; ++q) {
        double d = fabs(c->mat[q] - r->mat[q]);
        if (d > mx) mx = d;
      }
      mismatch = mx > ORC_MAT_TOL;
    }
    if (mismatch) { /* Level A: build_all_tables, variogram.f90:541-556 */
      for (int q = 0; q < m->nstruct; ++q) comp_build_table(&m->c[q]);
      return;
    }
  }
  if (ref >= 0) model_build_composite(m, ref);
}

/* struct_cov_tab, variogram.f90:750-771 (and the analytic struct_cov_lag
 * when no table has been built, variogram.f90:731-747) */
static double model_cov_tab(const orc_model *m, const double *lag) {
  if (m->level_b) {
    double h = aniso_h(m->bmat, m->ndim, lag);
    double r;
    if (table_lookup(&m->bt, h, &r)) return m->bt.tail ? model_cov_h(m, h) : 0.0;
    return r;
  }
  double res = 0.0;
  int iv = 0;
  while (iv < m->nstruct) {
    const orc_comp *c = &m->c[iv];
    double g = comp_cov_tab_h(c, aniso_h(c->mat, m->ndim, lag));
    while (iv < m->nstruct - 1 && m->c[iv + 1].is_product) {
      ++iv;
      c = &m->c[iv];
      g = g * comp_cov_tab_h(c, aniso_h(c->mat, m->ndim, lag));
    }
    res = res + g;
    ++iv;
  }
  return res;
}

static void model_free(orc_model *m) {
  for (int i = 0; i < m->nstruct; ++i)
    if (m->c[i].tab_ready) free(m->c[i].t.tab);
  if (m->level_b) free(m->bt.tab);
}

static void model_init(orc_model *m, int ndim, const orc_struct_spec *sp, int ns) {
  memset(m, 0, sizeof *m);
  m->ndim = ndim;
  m->nstruct = ns;
  for (int i = 0; i < ns; ++i) {
    orc_comp *c = &m->c[i];
    c->vtype = sp[i].vtype;
    c->sill = sp[i].sill;
    c->nugget = sp[i].nugget;
    c->a_major = sp[i].a_major;
    c->a_minor1 = sp[i].a_minor1;
    c->a_minor2 = sp[i].a_minor2;
    c->az = sp[i].azimuth;
    c->dip = sp[i].dip;
    c->plunge = sp[i].plunge;
    c->is_product = sp[i].is_product;
    c->ndim = ndim;
    comp_build_aniso(c);
  }
  model_cov0(m);
}

/* Space-time covariance, variogram_st.f90:222-277 (table form) */
typedef struct {
  orc_model cs, ct;
  int model;
  int tvtype;
  double t_nugget, t_sill, at, k_ps;
  double joint[ORC_MAXSTRUCT];
  int has_joint;
  double cov0;
} orc_stmodel;

/* f_time_vgm_st, variogram_st.f90:127-143 */
static double st_ftime(const orc_stmodel *s, double dt) {
  if (fabs(dt) <= DBL_EPSILON) return 0.0;
  double adt = fabs(dt) / s->at;
  double dw = s->t_nugget + s->t_sill * (1.0 - orc_corefunc(s->tvtype, adt));
  return dw > 0.0 ? dw : 0.0;
}

static double st_cov_tab(const orc_stmodel *s, int ndim, const double *lag) {
  double lag_s[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < ndim; ++d) lag_s[d] = lag[d];
  double dt = lag[ndim];
  double lag_t[3] = {fabs(dt), 0.0, 0.0};
  double cs = model_cov_tab(&s->cs, lag_s);
  double ct = model_cov_tab(&s->ct, lag_t);
  if (s->model == 1) return s->k_ps * cs * ct + cs + ct;
  double res = cs + ct;
  if (s->has_joint) {
    double dw = st_ftime(s, dt);
    for (int k = 0; k < s->cs.nstruct; ++k) {
      const orc_comp *c = &s->cs.c[k];
      double hs = aniso_h(c->mat, ndim, lag_s);
      double hst = sqrt(hs * hs + dw * dw);
      if (c->tab_ready && c->sill > 0.0)
        res = res + s->joint[k] * comp_cov_tab_h(c, hst) / c->sill;
      else
        res = res + s->joint[k] * orc_corefunc(c->vtype, hst);
    }
  }
  return res;
}

/* compute_cov0_vgm_st, variogram_st.f90:344-371 */
static void st_cov0(orc_stmodel *s) {
  if (s->model == 1) {
    s->cov0 = s->k_ps * s->cs.cov0 * s->ct.cov0 + s->cs.cov0 + s->ct.cov0;
  } else {
    s->cov0 = s->cs.cov0 + s->ct.cov0;
    if (s->has_joint)
      for (int k = 0; k < s->cs.nstruct; ++k)
        if (s->cs.c[k].vtype != VGM_NUG) s->cov0 = s->cov0 + s->joint[k];
  }
}

/* ------------------------------------------------------------------------ */
/* kd-tree (kdtree2_maxidx.f90; Kennel 2004, AFL 1.1)                       */
/* ------------------------------------------------------------------------ */
#define KD_BUCKET 12 /* kdtree2_maxidx.f90:534 */

typedef struct {
  int cut_dim;
  double cut_val, cut_val_left, cut_val_right;
  int l, u;          /* 0-based inclusive range into ind              */
  int left, right;   /* node indices, -1 = null                       */
} kd_node;

typedef struct {
  int dimen, n;
  const double *data;   /* (dimen, n) */
  int *ind;
  double *rdata;        /* rearranged (dimen, n) */
  kd_node *nodes;
  double *lo, *hi;      /* box per node: nodes x dimen */
  int nnodes, cap;
  int root;
} kd_tree;

static int kd_new_node(kd_tree *t) {
  if (t->nnodes == t->cap) {
    t->cap = t->cap ? 2 * t->cap : 64;
    t->nodes = (kd_node *)realloc(t->nodes, sizeof(kd_node) * t->cap);
    t->lo = (double *)realloc(t->lo, sizeof(double) * t->cap * t->dimen);
    t->hi = (double *)realloc(t->hi, sizeof(double) * t->cap * t->dimen);
  }
  return t->nnodes++;
}

#define KV(t, c, i) ((t)->data[(size_t)(i) * (t)->dimen + (c)])

/* spread_in_coordinate, kdtree2_maxidx.f90:951-999 */
static void kd_spread(const kd_tree *t, int c, int l, int u, double *smin_o, double *smax_o) {
  double smin = KV(t, c, t->ind[l]), smax = smin;
  int i;
  for (i = l + 2; i <= u; i += 2) {
    double lmin = KV(t, c, t->ind[i - 1]), lmax = KV(t, c, t->ind[i]);
    if (lmin > lmax) { double tt = lmin; lmin = lmax; lmax = tt; }
    if (smin > lmin) smin = lmin;
    if (smax < lmax) smax = lmax;
  }
  if (i == u + 1) {
    double last = KV(t, c, t->ind[u]);
    if (smin > last) smin = last;
    if (smax < last) smax = last;
  }
  *smin_o = smin;
  *smax_o = smax;
}

/* select_on_coordinate_value, kdtree2_maxidx.f90:857-916 (returns 0-based) */
static int kd_select_value(kd_tree *t, int c, double alpha, int li, int ui) {
  int lb = li, rb = ui;
  while (lb < rb) {
    if (KV(t, c, t->ind[lb]) <= alpha) {
      ++lb;
    } else {
      int tmp = t->ind[lb]; t->ind[lb] = t->ind[rb]; t->ind[rb] = tmp;
      --rb;
    }
  }
  return (KV(t, c, t->ind[lb]) <= alpha) ? lb : lb - 1;
}

/* build_tree_for_range, kdtree2_maxidx.f90:719-855 */
static int kd_build_range(kd_tree *t, int l, int u, int parent) {
  if (u < l) return -1;
  int me = kd_new_node(t);
  int D = t->dimen;
  kd_node *nd = &t->nodes[me];
  nd->left = nd->right = -1;
  nd->l = l; nd->u = u;
  if (u - l <= KD_BUCKET) {
    for (int i = 0; i < D; ++i) kd_spread(t, i, l, u, &t->lo[me * D + i], &t->hi[me * D + i]);
    nd->cut_dim = 0;
    nd->cut_val = 0.0;
    return me;
  }
  for (int i = 0; i < D; ++i) {
    int recompute = 1;
    if (parent >= 0 && i != t->nodes[parent].cut_dim) recompute = 0;
    if (recompute) kd_spread(t, i, l, u, &t->lo[me * D + i], &t->hi[me * D + i]);
    else { t->lo[me * D + i] = t->lo[parent * D + i]; t->hi[me * D + i] = t->hi[parent * D + i]; }
  }
  int c = 0;
  double best = t->hi[me * D] - t->lo[me * D];
  for (int i = 1; i < D; ++i) {
    double s = t->hi[me * D + i] - t->lo[me * D + i];
    if (s > best) { best = s; c = i; }
  }
  double sum = 0.0;
  for (int i = l; i <= u; ++i) sum = sum + KV(t, c, t->ind[i]);
  double average = sum / (double)(u - l + 1);
  t->nodes[me].cut_val = average;
  int m = kd_select_value(t, c, average, l, u);
  t->nodes[me].cut_dim = c;
  int left = kd_build_range(t, l, m, me);
  int right = kd_build_range(t, m + 1, u, me);
  nd = &t->nodes[me]; /* realloc may have moved */
  nd->left = left;
  nd->right = right;
  if (right < 0) {
    for (int i = 0; i < D; ++i) { t->lo[me * D + i] = t->lo[left * D + i]; t->hi[me * D + i] = t->hi[left * D + i]; }
    nd->cut_val_left = t->hi[left * D + c];
    nd->cut_val = nd->cut_val_left;
  } else if (left < 0) {
    for (int i = 0; i < D; ++i) { t->lo[me * D + i] = t->lo[right * D + i]; t->hi[me * D + i] = t->hi[right * D + i]; }
    nd->cut_val_right = t->lo[right * D + c];
    nd->cut_val = nd->cut_val_right;
  } else {
    nd->cut_val_right = t->lo[right * D + c];
    nd->cut_val_left = t->hi[left * D + c];
    nd->cut_val = (nd->cut_val_left + nd->cut_val_right) / 2.0;
    for (int i = 0; i < D; ++i) {
      double a = t->hi[left * D + i], b = t->hi[right * D + i];
      t->hi[me * D + i] = a > b ? a : b;
      a = t->lo[left * D + i]; b = t->lo[right * D + i];
      t->lo[me * D + i] = a < b ? a : b;
    }
  }
  return me;
}

/* kdtree2_create with rearrange=.true., kdtree2_maxidx.f90:629-700 */
static void kd_create(kd_tree *t, const double *data, int dimen, int n) {
  memset(t, 0, sizeof *t);
  t->dimen = dimen;
  t->n = n;
  t->data = data;
  t->ind = (int *)malloc(sizeof(int) * n);
  for (int j = 0; j < n; ++j) t->ind[j] = j;
  t->root = kd_build_range(t, 0, n - 1, -1);
  t->rdata = (double *)malloc(sizeof(double) * (size_t)dimen * n);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < dimen; ++d) t->rdata[(size_t)i * dimen + d] = KV(t, d, t->ind[i]);
}

static void kd_free(kd_tree *t) {
  free(t->ind); free(t->rdata); free(t->nodes); free(t->lo); free(t->hi);
  memset(t, 0, sizeof *t);
}

typedef struct { double dis; int idx; } kd_res;

typedef struct {
  const kd_tree *t;
  const double *qv;
  int nn, nfound;
  double ballsize;
  kd_res *heap;   /* 1-based, size nn+1 */
  int maxn;       /* only points with 0-based index < maxn (the _maxidx variants) */
} kd_search_rec;

/* pq_insert, kdtree2_maxidx.f90:307-349 */
static double pq_insert(kd_search_rec *sr, double dis, int idx) {
  kd_res *a = sr->heap;
  int i = sr->nfound; /* already incremented heap size */
  while (i > 1) {
    int ip = i / 2;
    double pd = a[ip].dis;
    if (dis > pd) { a[i] = a[ip]; i = ip; } else break;
  }
  a[i].dis = dis;
  a[i].idx = idx;
  return a[1].dis;
}

/* pq_replace_max, kdtree2_maxidx.f90:392-461 */
static double pq_replace_max(kd_search_rec *sr, double dis, int idx) {
  kd_res *a = sr->heap;
  int N = sr->nfound;
  if (N >= 1) {
    int parent = 1, child = 2;
    while (child <= N) {
      double pc = a[child].dis;
      if (child < N) {
        double pc1 = a[child + 1].dis;
        if (pc < pc1) { ++child; pc = pc1; }
      }
      if (dis >= pc) break;
      a[parent] = a[child];
      parent = child;
      child = 2 * parent;
    }
    a[parent].dis = dis;
    a[parent].idx = idx;
    return a[1].dis;
  }
  a[1].dis = dis;
  a[1].idx = idx;
  return dis;
}

/* process_terminal_node, kdtree2_maxidx.f90:1510-1612 (rearranged data) */
static void kd_terminal(kd_search_rec *sr, const kd_node *nd) {
  const kd_tree *t = sr->t;
  double ballsize = sr->ballsize;
  const int D = t->dimen;
  for (int i = nd->l; i <= nd->u; ++i) {
    if (t->ind[i] >= sr->maxn) continue; /* process_terminal_node_maxidx, kdtree2_maxidx.f90:2081 */
    double sd = 0.0;
    int skip = 0;
    for (int k = 0; k < D; ++k) {
      double d = t->rdata[(size_t)i * D + k] - sr->qv[k];
      sd = sd + d * d;
      if (sd > ballsize) { skip = 1; break; }
    }
    if (skip) continue;
    int indexofi = t->ind[i];
    if (sr->nfound < sr->nn) {
      sr->nfound++;
      double newpri = pq_insert(sr, sd, indexofi);
      if (sr->nfound == sr->nn) ballsize = newpri;
    } else {
      ballsize = pq_replace_max(sr, sd, indexofi);
    }
  }
  sr->ballsize = ballsize;
}

/* dis2_from_bnd, kdtree2_maxidx.f90:1479-1494 */
static double dis2_from_bnd(double x, double amin, double amax) {
  if (x > amax) return (x - amax) * (x - amax);
  if (x < amin) return (amin - x) * (amin - x);
  return 0.0;
}

/* search, kdtree2_maxidx.f90:1383-1476 */
static void kd_search(kd_search_rec *sr, int node) {
  const kd_tree *t = sr->t;
  const kd_node *nd = &t->nodes[node];
  if (!(nd->left >= 0 && nd->right >= 0)) { kd_terminal(sr, nd); return; }
  int cd = nd->cut_dim;
  double qval = sr->qv[cd];
  int closer, farther;
  double dis;
  if (qval < nd->cut_val) {
    closer = nd->left; farther = nd->right;
    dis = (nd->cut_val_right - qval) * (nd->cut_val_right - qval);
  } else {
    closer = nd->right; farther = nd->left;
    dis = (nd->cut_val_left - qval) * (nd->cut_val_left - qval);
  }
  if (closer >= 0) kd_search(sr, closer);
  if (farther >= 0) {
    double ballsize = sr->ballsize;
    if (dis <= ballsize) {
      for (int i = 0; i < t->dimen; ++i) {
        if (i == cd) continue;
        dis = dis + dis2_from_bnd(sr->qv[i], t->lo[node * t->dimen + i], t->hi[node * t->dimen + i]);
        if (dis > ballsize) return;
      }
      kd_search(sr, farther);
    }
  }
}

/* heapsort_struct, kdtree2_maxidx.f90:1860-1926 (a is 1-based, n entries) */
static void kd_heapsort(kd_res *a, int n) {
  if (n <= 1) return;
  int ileft = n / 2 + 1, iright = n;
  kd_res value;
  for (;;) {
    if (ileft > 1) {
      --ileft;
      value = a[ileft];
    } else {
      value = a[iright];
      a[iright] = a[1];
      --iright;
      if (iright == 1) { a[1] = value; return; }
    }
    int i = ileft, j = 2 * ileft;
    while (j <= iright) {
      if (j < iright && a[j].dis < a[j + 1].dis) ++j;
      if (value.dis < a[j].dis) { a[i] = a[j]; i = j; j = j + j; }
      else j = iright + 1;
    }
    a[i] = value;
  }
}

/* kdtree2_n_nearest, kdtree2_maxidx.f90:1043-1085, and
 * kdtree2_n_nearest_maxidx, :1928-1964 (maxn = max_idx as a 0-based bound);
 * heap is 1-based [nn+1] */
static void kd_n_nearest_max(const kd_tree *t, const double *qv, int nn, int sort, kd_res *heap, int maxn) {
  kd_search_rec sr;
  sr.t = t;
  sr.qv = qv;
  sr.nn = nn;
  sr.nfound = 0;
  sr.ballsize = DBL_MAX;
  sr.heap = heap;
  sr.maxn = maxn;
  kd_search(&sr, t->root);
  if (sort) kd_heapsort(heap, nn);
}

static void kd_n_nearest(const kd_tree *t, const double *qv, int nn, int sort, kd_res *heap) {
  kd_n_nearest_max(t, qv, nn, sort, heap, INT_MAX);
}

int orc_kdtree_nn(const double *data, int dim, int n, const double *qv, int nn,
                  int sort, double *dis, int *idx) {
  kd_tree t;
  kd_create(&t, data, dim, n);
  kd_res *h = (kd_res *)malloc(sizeof(kd_res) * (nn + 1));
  kd_n_nearest(&t, qv, nn, sort, h);
  for (int i = 0; i < nn; ++i) { dis[i] = h[i + 1].dis; idx[i] = h[i + 1].idx + 1; }
  free(h);
  kd_free(&t);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* dense solvers                                                            */
/* ------------------------------------------------------------------------ */
/* Upper Cholesky A = U^T U on the leading n x n of column-major a (lda);
 * SPOTRF('U') semantics: returns 0 or the 1-based order of the first
 * non-positive (or NaN) pivot (lapack.f:4422-4720). */
static int potrf_u(int n, double *a, int lda) {
  for (int j = 0; j < n; ++j) {
    double ajj = a[j + j * lda];
    for (int k = 0; k < j; ++k) ajj = ajj - a[k + j * lda] * a[k + j * lda];
    if (ajj <= 0.0 || isnan(ajj)) { a[j + j * lda] = ajj; return j + 1; }
    ajj = sqrt(ajj);
    a[j + j * lda] = ajj;
    for (int i = j + 1; i < n; ++i) {
      double s = a[j + i * lda];
      for (int k = 0; k < j; ++k) s = s - a[k + j * lda] * a[k + i * lda];
      a[j + i * lda] = s / ajj;
    }
  }
  return 0;
}

/* SPOTRS('U'): solve U^T U X = B, B column-major (ldb) with nrhs columns */
static void potrs_u(int n, int nrhs, const double *a, int lda, double *b, int ldb) {
  for (int c = 0; c < nrhs; ++c) {
    double *x = b + (size_t)c * ldb;
    for (int i = 0; i < n; ++i) {
      double s = x[i];
      for (int k = 0; k < i; ++k) s = s - a[k + i * lda] * x[k];
      x[i] = s / a[i + i * lda];
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = x[i];
      for (int k = i + 1; k < n; ++k) s = s - a[i + k * lda] * x[k];
      x[i] = s / a[i + i * lda];
    }
  }
}

/* DSYTF2('U') Bunch-Kaufman factorisation, restated from netlib LAPACK
 * (lapack.f SSYTF2/SSYTRF); a is column-major m x m, ipiv 1-based. */
static int sytf2_u(int n, double *a, int lda, int *ipiv) {
#define A_(i, j) a[((i) - 1) + ((j) - 1) * (size_t)lda]
  const double alpha = (1.0 + sqrt(17.0)) / 8.0;
  int info = 0;
  int k = n;
  while (k >= 1) {
    int kstep = 1, kp;
    double absakk = fabs(A_(k, k));
    int imax = 0;
    double colmax = 0.0;
    if (k > 1) {
      imax = 1;
      colmax = fabs(A_(1, k));
      for (int i = 2; i <= k - 1; ++i)
        if (fabs(A_(i, k)) > colmax) { colmax = fabs(A_(i, k)); imax = i; }
    }
    if ((absakk > colmax ? absakk : colmax) == 0.0 || isnan(absakk)) {
      if (info == 0) info = k;
      kp = k;
    } else {
      if (absakk >= alpha * colmax) {
        kp = k;
      } else {
        double rowmax = 0.0;
        for (int j = imax + 1; j <= k; ++j)
          if (fabs(A_(imax, j)) > rowmax) rowmax = fabs(A_(imax, j));
        for (int j = 1; j <= imax - 1; ++j)
          if (fabs(A_(j, imax)) > rowmax) rowmax = fabs(A_(j, imax));
        if (absakk >= alpha * colmax * (colmax / rowmax)) {
          kp = k;
        } else if (fabs(A_(imax, imax)) >= alpha * rowmax) {
          kp = imax;
        } else {
          kp = imax;
          kstep = 2;
        }
      }
      int kk = k - kstep + 1;
      if (kp != kk) {
        for (int i = 1; i <= kp - 1; ++i) { double t = A_(i, kk); A_(i, kk) = A_(i, kp); A_(i, kp) = t; }
        for (int j = kp + 1; j <= kk - 1; ++j) { double t = A_(j, kk); A_(j, kk) = A_(kp, j); A_(kp, j) = t; }
        double t = A_(kk, kk); A_(kk, kk) = A_(kp, kp); A_(kp, kp) = t;
        if (kstep == 2) { t = A_(k - 1, k); A_(k - 1, k) = A_(kp, k); A_(kp, k) = t; }
      }
      if (kstep == 1) {
        double r1 = 1.0 / A_(k, k);
        for (int j = 1; j <= k - 1; ++j) {
          double xj = A_(j, k);
          if (xj != 0.0) {
            double tmp = -r1 * xj;
            for (int i = 1; i <= j; ++i) A_(i, j) = A_(i, j) + A_(i, k) * tmp;
          }
        }
        for (int i = 1; i <= k - 1; ++i) A_(i, k) = r1 * A_(i, k);
      } else if (k > 2) {
        double d12 = A_(k - 1, k);
        double d22 = A_(k - 1, k - 1) / d12;
        double d11 = A_(k, k) / d12;
        double t = 1.0 / (d11 * d22 - 1.0);
        d12 = t / d12;
        for (int j = k - 2; j >= 1; --j) {
          double wkm1 = d12 * (d11 * A_(j, k - 1) - A_(j, k));
          double wk = d12 * (d22 * A_(j, k) - A_(j, k - 1));
          for (int i = j; i >= 1; --i) A_(i, j) = A_(i, j) - A_(i, k) * wk - A_(i, k - 1) * wkm1;
          A_(j, k) = wk;
          A_(j, k - 1) = wkm1;
        }
      }
    }
    if (kstep == 1) ipiv[k - 1] = kp;
    else { ipiv[k - 1] = -kp; ipiv[k - 2] = -kp; }
    k -= kstep;
  }
  return info;
#undef A_
}

/* DSYTRS('U') for nrhs columns, restated from netlib LAPACK (lapack.f SSYTRS) */
static void sytrs_u(int n, int nrhs, const double *a, int lda, const int *ipiv,
                    double *b, int ldb) {
#define A_(i, j) a[((i) - 1) + ((j) - 1) * (size_t)lda]
#define B_(i, j) b[((i) - 1) + ((j) - 1) * (size_t)ldb]
  int k = n;
  while (k >= 1) {
    if (ipiv[k - 1] > 0) {
      int kp = ipiv[k - 1];
      if (kp != k)
        for (int j = 1; j <= nrhs; ++j) { double t = B_(k, j); B_(k, j) = B_(kp, j); B_(kp, j) = t; }
      for (int j = 1; j <= nrhs; ++j) {
        double bk = B_(k, j);
        for (int i = 1; i <= k - 1; ++i) B_(i, j) = B_(i, j) - A_(i, k) * bk;
      }
      double r = 1.0 / A_(k, k);
      for (int j = 1; j <= nrhs; ++j) B_(k, j) = r * B_(k, j);
      k -= 1;
    } else {
      int kp = -ipiv[k - 1];
      if (kp != k - 1)
        for (int j = 1; j <= nrhs; ++j) { double t = B_(k - 1, j); B_(k - 1, j) = B_(kp, j); B_(kp, j) = t; }
      for (int j = 1; j <= nrhs; ++j) {
        double bk = B_(k, j), bkm1 = B_(k - 1, j);
        for (int i = 1; i <= k - 2; ++i) B_(i, j) = B_(i, j) - A_(i, k) * bk;
        for (int i = 1; i <= k - 2; ++i) B_(i, j) = B_(i, j) - A_(i, k - 1) * bkm1;
      }
      double akm1k = A_(k - 1, k);
      double akm1 = A_(k - 1, k - 1) / akm1k;
      double ak = A_(k, k) / akm1k;
      double denom = akm1 * ak - 1.0;
      for (int j = 1; j <= nrhs; ++j) {
        double bkm1 = B_(k - 1, j) / akm1k;
        double bk = B_(k, j) / akm1k;
        B_(k - 1, j) = (ak * bkm1 - bk) / denom;
        B_(k, j) = (akm1 * bk - bkm1) / denom;
      }
      k -= 2;
    }
  }
  k = 1;
  while (k <= n) {
    if (ipiv[k - 1] > 0) {
      for (int j = 1; j <= nrhs; ++j) {
        double s = 0.0;
        for (int i = 1; i <= k - 1; ++i) s = s + A_(i, k) * B_(i, j);
        B_(k, j) = B_(k, j) - s;
      }
      int kp = ipiv[k - 1];
      if (kp != k)
        for (int j = 1; j <= nrhs; ++j) { double t = B_(k, j); B_(k, j) = B_(kp, j); B_(kp, j) = t; }
      k += 1;
    } else {
      for (int j = 1; j <= nrhs; ++j) {
        double s = 0.0, s1 = 0.0;
        for (int i = 1; i <= k - 1; ++i) s = s + A_(i, k) * B_(i, j);
        for (int i = 1; i <= k - 1; ++i) s1 = s1 + A_(i, k + 1) * B_(i, j);
        B_(k, j) = B_(k, j) - s;
        B_(k + 1, j) = B_(k + 1, j) - s1;
      }
      int kp = -ipiv[k - 1];
      if (kp != k)
        for (int j = 1; j <= nrhs; ++j) { double t = B_(k, j); B_(k, j) = B_(kp, j); B_(kp, j) = t; }
      k += 2;
    }
  }
#undef A_
#undef B_
}

int orc_sysv(int m, double *a, int nrhs, double *b) {
  int *ipiv = (int *)malloc(sizeof(int) * m);
  int info = sytf2_u(m, a, m, ipiv);
  if (info == 0) sytrs_u(m, nrhs, a, m, ipiv, b, m);
  free(ipiv);
  return info;
}


/* ------------------------------------------------------------------------ */
/* solve driver (kriging_base.F90:2064-2194, 3159-3503; kriging.F90)        */
/* ------------------------------------------------------------------------ */
typedef struct {
  const orc_problem *p;
  int nvar, ndim, nlag, pa, naug, st;
  int nobs[ORC_MAXVAR], nmax[ORC_MAXVAR], need_search[ORC_MAXVAR], aniso[ORC_MAXVAR];
  int sector[ORC_MAXVAR];
  double maxd2[ORC_MAXVAR];
  double rotmat[ORC_MAXVAR][9];
  double ta[ORC_MAXVAR];
  double *scoord[ORC_MAXVAR];
  kd_tree tree[ORC_MAXVAR];
  int has_tree[ORC_MAXVAR];
  orc_model mdl[ORC_MAXVAR][ORC_MAXVAR];     /* built for a <= b          */
  orc_stmodel smdl[ORC_MAXVAR][ORC_MAXVAR];  /* space-time: every pair    */
  int mmax, nppmax, mmat, heapn;
  int *gstart;                                /* first node of each block  */
} orc_ctx;

/* One prepared factorisation (t_factor_cache, kriging_base.F90:114-140). */
typedef struct {
  int valid, used_sysv, npp, p;
  unsigned hash;
  long last;
  double rs, ln;
  int nnear[ORC_MAXVAR];
  int *inear;
  double *L, *Y, *S, *Afac;
  int *ipiv;
} orc_fac;

typedef struct {
  double *matA, *rhsB, *x, *sqd;
  int *inear;
  int nnear[ORC_MAXVAR];
  kd_res *heap;
  orc_fac scratch;
  orc_fac *slot;
  int nslot;
  long clock;
  int stats[5];
} orc_ws;

static void fac_alloc(orc_fac *f, const orc_ctx *c) {
  memset(f, 0, sizeof *f);
  int pp = c->pa > 0 ? c->pa : 1;
  f->inear = (int *)malloc(sizeof(int) * c->mmax * c->nvar);
  f->L = (double *)malloc(sizeof(double) * (size_t)c->nppmax * c->nppmax);
  f->Y = (double *)malloc(sizeof(double) * (size_t)c->nppmax * pp);
  f->S = (double *)malloc(sizeof(double) * pp * pp);
  f->Afac = (double *)malloc(sizeof(double) * (size_t)c->mmat * c->mmat);
  f->ipiv = (int *)malloc(sizeof(int) * c->mmat);
}
static void fac_free(orc_fac *f) {
  free(f->inear); free(f->L); free(f->Y); free(f->S); free(f->Afac); free(f->ipiv);
}

/* fhcache_hash_key-style FNV mix (kriging_base.F90:1746-1773); any hash works
 * because matches are always verified element by element. */
static unsigned key_hash(const orc_ws *w, const orc_ctx *c, int npp, double rs, double ln) {
  unsigned h = 2166136261u;
#define MIX(x) do { h ^= (unsigned)(x); h *= 16777619u; } while (0)
  MIX(npp); MIX(c->pa); MIX((int)lround(rs * 1e6)); MIX((int)lround(ln * 1e6));
  for (int v = 0; v < c->nvar; ++v) {
    MIX(w->nnear[v]);
    for (int i = 0; i < w->nnear[v]; ++i) MIX(w->inear[v * c->mmax + i]);
  }
#undef MIX
  return h;
}

/* fcache_matches, kriging_base.F90:2445-2464 */
static int fac_matches(const orc_fac *f, const orc_ws *w, const orc_ctx *c, unsigned h, int npp,
                       double rs, double ln) {
  if (!f->valid || f->hash != h || f->npp != npp || f->rs != rs || f->ln != ln) return 0;
  for (int v = 0; v < c->nvar; ++v) {
    if (f->nnear[v] != w->nnear[v]) return 0;
    for (int i = 0; i < w->nnear[v]; ++i)
      if (f->inear[v * c->mmax + i] != w->inear[v * c->mmax + i]) return 0;
  }
  return 1;
}

/* search_neighbors, kriging.F90:490-666 (spatial) and kriging_st.F90:467-686
 * (space-time); returns nnear after the maxdist filter. */
static int search_one(const orc_ctx *c, orc_ws *w, int v, const double *xloc, int ib, int *inear,
                      double *dist) {
  const int ndim = c->ndim, nlag = c->nlag, nobs = c->nobs[v], nmax = c->nmax[v];
  const double *obs = c->p->obs_coord[v];
  double newloc[4];
  if (c->aniso[v]) rotate_pt(c->rotmat[v], ndim, xloc, newloc);
  else for (int d = 0; d < ndim; ++d) newloc[d] = xloc[d];
  if (c->st) newloc[nlag - 1] = xloc[nlag - 1] * c->ta[v];
  int nnear = 0;
  kd_res *h = w->heap;
  if (c->sector[v] && (c->need_search[v] || c->st)) {
    int ncand;
    if (c->need_search[v]) {
      int lim = (1 << ndim) * nmax * 4;
      ncand = nobs < lim ? nobs : lim;
      kd_n_nearest(&c->tree[v], newloc, ncand, 1, h);
    } else { /* space-time sector search over all observations, kriging_st.F90:590-597 */
      ncand = nobs;
      for (int i = 0; i < nobs; ++i) {
        double diff[3], r[3];
        for (int d = 0; d < ndim; ++d) diff[d] = obs[(size_t)i * nlag + d] - xloc[d];
        rotate_pt(c->rotmat[v], ndim, diff, r);
        double s = 0.0;
        for (int d = 0; d < ndim; ++d) s = s + r[d] * r[d];
        double tt = obs[(size_t)i * nlag + nlag - 1] * c->ta[v] - newloc[nlag - 1];
        h[i + 1].dis = s + tt * tt;
        h[i + 1].idx = i;
      }
      kd_heapsort(h, ncand);
    }
    /* apply_sector_filter, kriging.F90:1093-1154 */
    int count[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 1; i <= ncand; ++i) {
      int idx = h[i].idx;
      if (c->p->cross_validation && idx == ib) continue;
      if (h[i].dis > c->maxd2[v]) continue;
      double pr[3];
      if (c->aniso[v]) rotate_pt(c->rotmat[v], ndim, obs + (size_t)idx * nlag, pr);
      else for (int d = 0; d < ndim; ++d) pr[d] = obs[(size_t)idx * nlag + d];
      double dx = pr[0] - newloc[0];
      double dy = ndim > 1 ? pr[1] - newloc[1] : 0.0;
      double dz = ndim == 3 ? pr[2] - newloc[2] : 0.0;
      int ix = dx < 0.0 ? 1 : 0, iy = dy < 0.0 ? 1 : 0, iz = dz < 0.0 ? 1 : 0;
      int sector = ndim == 3 ? ix + 2 * iy + 4 * iz : ix + 2 * iy;
      if (count[sector] < nmax) {
        count[sector]++;
        inear[nnear] = idx;
        dist[nnear] = h[i].dis;
        ++nnear;
      }
    }
  } else if (c->need_search[v]) {
    kd_n_nearest(&c->tree[v], newloc, nmax, 0, h);
    nnear = nmax;
    for (int i = 0; i < nmax; ++i) { inear[i] = h[i + 1].idx; dist[i] = h[i + 1].dis; }
  } else {
    /* all observations: rotated_dists (rotation.f90:193-218) */
    nnear = nobs;
    for (int i = 0; i < nobs; ++i) {
      double diff[3], r[3];
      for (int d = 0; d < ndim; ++d)
        diff[d] = obs[(size_t)i * nlag + d] - (c->st ? xloc[d] : newloc[d]);
      rotate_pt(c->rotmat[v], ndim, diff, r);
      double s = 0.0;
      for (int d = 0; d < ndim; ++d) s = s + r[d] * r[d];
      if (c->st) {
        double tt = obs[(size_t)i * nlag + nlag - 1] * c->ta[v] - newloc[nlag - 1];
        s = s + tt * tt;
      }
      inear[i] = i;
      dist[i] = s;
    }
  }
  /* cross-validation: drop the target observation, kriging.F90:647-657 */
  if (c->p->cross_validation && !(c->sector[v] && (c->need_search[v] || c->st))) {
    for (int i = 0; i < nnear; ++i)
      if (inear[i] == ib) {
        for (int j = i; j < nnear - 1; ++j) { inear[j] = inear[j + 1]; dist[j] = dist[j + 1]; }
        --nnear;
        break;
      }
  }
  /* filter_by_maxlag, kriging_base.F90:2491-2505 */
  int kk = 0;
  for (int i = 0; i < nnear; ++i)
    if (dist[i] <= c->maxd2[v]) { inear[kk] = inear[i]; dist[kk] = dist[i]; ++kk; }
  return kk;
}

/* isort, kriging_base.F90:3510-3524 */
static void isort(int *a, int n) {
  for (int i = 1; i < n; ++i) {
    int tmp = a[i], j = i - 1;
    while (j >= 0 && a[j] > tmp) { a[j + 1] = a[j]; --j; }
    a[j + 1] = tmp;
  }
}

/* lag = (a - b) / rangescale (kriging.F90:783, 905); space-time lags are not
 * scaled (kriging_st.F90:806). */
static void lag_of(const orc_ctx *c, const double *a, const double *b, double rs, double *lag) {
  for (int d = 0; d < c->nlag; ++d) lag[d] = c->st ? (a[d] - b[d]) : (a[d] - b[d]) / rs;
}

/* struct_cov_lag, variogram.f90:731-747: per-component analytic covariance */
static double model_cov_lag(const orc_model *m, const double *lag) {
  double res = 0.0;
  int iv = 0;
  while (iv < m->nstruct) {
    const orc_comp *cp = &m->c[iv];
    double g = comp_cov_h(cp, aniso_h(cp->mat, m->ndim, lag));
    while (iv < m->nstruct - 1 && m->c[iv + 1].is_product) {
      ++iv;
      cp = &m->c[iv];
      g = g * comp_cov_h(cp, aniso_h(cp->mat, m->ndim, lag));
    }
    res = res + g;
    ++iv;
  }
  return res;
}

/* COV(vgm(first, second), lag).  The spatial engine builds lookup tables
 * only for vgm(iv, jv) with jv >= iv (kriging.F90:412-421); vgm(first,
 * second) with first > second therefore evaluates analytically through
 * comp_cov_h (variogram.f90:358).  Space-time builds every pair
 * (kriging_st.F90:438-449). */
static double pair_cov(const orc_ctx *c, int first, int second, const double *lag) {
  if (c->st) return st_cov_tab(&c->smdl[first][second], c->ndim, lag);
  if (first > second || c->p->analytic) {
    const orc_model *m = first <= second ? &c->mdl[first][second] : &c->mdl[second][first];
    return model_cov_lag(m, lag);
  }
  return model_cov_tab(&c->mdl[first][second], lag);
}

static double pair_cov0(const orc_ctx *c, int first, int second) {
  if (c->st) return c->smdl[first][second].cov0;
  return first <= second ? c->mdl[first][second].cov0 : c->mdl[second][first].cov0;
}

double orc_cov(const orc_problem *prob, int ivar, int jvar, const double *lag) {
  orc_model m;
  model_init(&m, prob->ndim, prob->vgm[ivar][jvar], prob->nstruct[ivar][jvar]);
  model_build_table(&m);
  double r = model_cov_tab(&m, lag);
  model_free(&m);
  return r;
}

/* kriging_setup + kriging_solve_prepared, solver.f90:224-300; returns info */
static int chol_setup(int npp, int pa, const double *A, int m, orc_fac *f) {
  for (int j = 0; j < npp; ++j)
    for (int i = 0; i < npp; ++i) f->L[i + (size_t)j * npp] = A[i + (size_t)j * m];
  int info = potrf_u(npp, f->L, npp);
  if (info != 0 || pa == 0) return info;
  for (int j = 0; j < pa; ++j)
    for (int i = 0; i < npp; ++i) f->Y[i + (size_t)j * npp] = A[i + (size_t)(npp + j) * m];
  potrs_u(npp, pa, f->L, npp, f->Y, npp);
  for (int j = 0; j < pa; ++j)
    for (int i = 0; i < pa; ++i) {
      double s = 0.0;
      for (int k = 0; k < npp; ++k) s = s + A[k + (size_t)(npp + i) * m] * f->Y[k + (size_t)j * npp];
      f->S[i + (size_t)j * pa] = s;
    }
  return potrf_u(pa, f->S, pa);
}

static void chol_solve(int npp, int pa, int q, const orc_fac *f, const double *B, double *X,
                       double *work) {
  double *Z = work;                       /* (npp, q) */
  double *rs = work + (size_t)npp * q;    /* (pa, q)  */
  for (int i = 0; i < q; ++i)
    for (int k = 0; k < npp; ++k) Z[k + (size_t)i * npp] = B[i + (size_t)k * q];
  potrs_u(npp, q, f->L, npp, Z, npp);
  if (pa == 0) {
    for (int i = 0; i < q; ++i)
      for (int k = 0; k < npp; ++k) X[i + (size_t)k * q] = Z[k + (size_t)i * npp];
    return;
  }
  for (int i = 0; i < q; ++i)
    for (int a = 0; a < pa; ++a) {
      double s = 0.0;
      for (int k = 0; k < npp; ++k) s = s + f->Y[k + (size_t)a * npp] * B[i + (size_t)k * q];
      rs[a + (size_t)i * pa] = s;
    }
  for (int i = 0; i < q; ++i)
    for (int a = 0; a < pa; ++a) rs[a + (size_t)i * pa] = rs[a + (size_t)i * pa] - B[i + (size_t)(npp + a) * q];
  potrs_u(pa, q, f->S, pa, rs, pa);
  for (int i = 0; i < q; ++i) {
    for (int k = 0; k < npp; ++k) {
      double s = 0.0;
      for (int a = 0; a < pa; ++a) s = s + f->Y[k + (size_t)a * npp] * rs[a + (size_t)i * pa];
      X[i + (size_t)k * q] = Z[k + (size_t)i * npp] - s;
    }
    for (int a = 0; a < pa; ++a) X[i + (size_t)(npp + a) * q] = rs[a + (size_t)i * pa];
  }
}

/* ssytrs_solve, solver.f90:376-406 */
static void ldl_solve(int m, int q, const orc_fac *f, const double *B, double *X, double *work) {
  for (int i = 0; i < q; ++i)
    for (int k = 0; k < m; ++k) work[k + (size_t)i * m] = B[i + (size_t)k * q];
  sytrs_u(m, q, f->Afac, m, f->ipiv, work, m);
  for (int i = 0; i < q; ++i)
    for (int k = 0; k < m; ++k) X[i + (size_t)k * q] = work[k + (size_t)i * m];
}

static void fac_save_key(orc_fac *f, const orc_ws *w, const orc_ctx *c, unsigned h, int npp,
                         double rs, double ln) {
  f->valid = 1;
  f->hash = h;
  f->npp = npp;
  f->p = c->pa;
  f->rs = rs;
  f->ln = ln;
  for (int v = 0; v < c->nvar; ++v) {
    f->nnear[v] = w->nnear[v];
    memcpy(f->inear + v * c->mmax, w->inear + v * c->mmax, sizeof(int) * w->nnear[v]);
  }
}

/* One target: assemble_linear_system_base + solve_linear_system_base +
 * calc_variance + estimate_block_base (kriging_base.F90:3159-3503). */
static void solve_target(const orc_ctx *c, orc_ws *w, int ib, orc_result *res, int *err_flag,
                         char *errmsg) {
  const orc_problem *P = c->p;
  const int nvar = c->nvar, nlag = c->nlag, mmax = c->mmax, pa = c->pa;
  const double *xloc = P->block_coord + (size_t)ib * nlag;
  const double rs = P->rangescale ? P->rangescale[ib] : 1.0;
  const double ln = P->localnugget ? P->localnugget[ib] : 0.0;
  double *val = res->value + (size_t)ib * nvar;
  double *var = res->variance + (size_t)ib * nvar * nvar;
  const int nbp = P->nblockpnt ? P->nblockpnt[ib] : 1;
  const int k0 = P->nblockpnt ? c->gstart[ib] : ib;
  const double *gc = P->grid_coord ? P->grid_coord : P->block_coord;

  int istart[ORC_MAXVAR];
  int npp = 0;
  for (int v = 0; v < nvar; ++v) {
    w->nnear[v] = search_one(c, w, v, xloc, ib, w->inear + v * mmax, w->sqd);
    istart[v] = npp;
    npp += w->nnear[v];
  }
  for (int v = 0; v < nvar; ++v) isort(w->inear + v * mmax, w->nnear[v]);
  if (res->nnear)
    for (int v = 0; v < nvar; ++v) res->nnear[(size_t)ib * nvar + v] = w->nnear[v];
  if (res->inear)
    for (int v = 0; v < nvar; ++v)
      for (int i = 0; i < w->nnear[v]; ++i)
        res->inear[((size_t)ib * nvar + v) * res->mmax + i] = w->inear[v * mmax + i] + 1;
  if (npp == 0 || (P->nmin > 0 && npp < P->nmin) || npp == 1) {
    /* zero neighbours: kriging_base.F90:3198-3207; npp == 1 reuses a stale
     * solution in the reference (kriging_base.F90:2130) and is reported as NaN */
    if (npp == 0 && !P->neglect_error) {
      *err_flag = 1;
      snprintf(errmsg, 256, "not enough neighbors for kriging at block %d", ib + 1);
    }
    for (int v = 0; v < nvar; ++v) val[v] = NAN;
    for (int q = 0; q < nvar * nvar; ++q) var[q] = NAN;
    return;
  }
  const int m = npp + pa;
  double *A = w->matA, *B = w->rhsB, *X = w->x;

  /* assemble_rhs, kriging.F90:864-939 / kriging_st.F90:887-958 */
  for (int iv = 0; iv < nvar; ++iv) {
    for (int kv = 0; kv < nvar; ++kv)
      for (int i = 0; i < w->nnear[kv]; ++i) {
        const double *xo = P->obs_coord[kv] + (size_t)w->inear[kv * mmax + i] * nlag;
        double tmp = 0.0;
        for (int k = k0; k < k0 + nbp; ++k) {
          double lag[4];
          lag_of(c, xo, gc + (size_t)k * nlag, rs, lag);
          double wk = P->grid_weight ? P->grid_weight[k] : 1.0;
          tmp = tmp + pair_cov(c, kv, iv, lag) * wk;
        }
        B[iv + (size_t)(istart[kv] + i) * nvar] = tmp;
      }
    for (int r = 0; r < pa; ++r) {
      double g;
      if (r < P->ndrift) {
        g = P->block_drift ? P->block_drift[((size_t)ib * nvar + iv) * P->ndrift + r] : 0.0;
      } else {
        int ua = r - P->ndrift;
        g = P->std_ck ? (ua == iv ? 1.0 : 0.0) : (ua == 0 ? 1.0 : 0.0);
      }
      B[iv + (size_t)(npp + r) * nvar] = g;
    }
  }

  /* cache lookup (kriging_base.F90:3213-3225) */
  unsigned h = key_hash(w, c, npp, rs, ln);
  orc_fac *f = NULL;
  for (int s = 0; s < w->nslot; ++s)
    if (fac_matches(&w->slot[s], w, c, h, npp, rs, ln)) { f = &w->slot[s]; break; }
  int info = 0;
  double *work = w->sqd + mmax;
  if (f) {
    f->last = ++w->clock;
    if (f->used_sysv) { ldl_solve(m, nvar, f, B, X, work); w->stats[4]++; }
    else { chol_solve(npp, pa, nvar, f, B, X, work); w->stats[2]++; }
  } else {
    /* assemble_lhs, kriging.F90:714-849 / kriging_st.F90:739-872 */
    for (size_t q = 0; q < (size_t)m * m; ++q) A[q] = 0.0;
    for (int kv = 0; kv < nvar; ++kv) {
      if (w->nnear[kv] == 0) continue;
      for (int lv = kv; lv < nvar; ++lv) {
        if (w->nnear[lv] == 0) continue;
        for (int i = 0; i < w->nnear[kv]; ++i) {
          int oi = w->inear[kv * mmax + i];
          const double *xi = P->obs_coord[kv] + (size_t)oi * nlag;
          int jstart = 0;
          if (lv == kv) {
            double ov = P->obs_var[kv] ? P->obs_var[kv][oi] : 0.0;
            A[(istart[lv] + i) + (size_t)(istart[kv] + i) * m] = pair_cov0(c, lv, kv) + ov + ln;
            jstart = i + 1;
          }
          for (int j = jstart; j < w->nnear[lv]; ++j) {
            const double *xj = P->obs_coord[lv] + (size_t)w->inear[lv * mmax + j] * nlag;
            double lag[4];
            lag_of(c, xi, xj, rs, lag);
            A[(istart[lv] + j) + (size_t)(istart[kv] + i) * m] = pair_cov(c, lv, kv, lag);
          }
        }
      }
      for (int i = 0; i < w->nnear[kv]; ++i) {
        int oi = w->inear[kv * mmax + i];
        for (int r = 0; r < pa; ++r) {
          double fv;
          if (r < P->ndrift) fv = P->obs_drift[kv] ? P->obs_drift[kv][(size_t)oi * P->ndrift + r] : 0.0;
          else {
            int ua = r - P->ndrift;
            fv = P->std_ck ? (ua == kv ? 1.0 : 0.0) : (ua == 0 ? 1.0 : 0.0);
          }
          A[(npp + r) + (size_t)(istart[kv] + i) * m] = fv;
        }
      }
    }
    for (int ir = 0; ir < npp; ++ir)
      for (int ic = ir + 1; ic < m; ++ic) A[ir + (size_t)ic * m] = A[ic + (size_t)ir * m];

    /* pick the LRU victim slot (fhcache_insert, kriging_base.F90:1862-1917) */
    if (w->nslot > 0) {
      f = &w->slot[0];
      for (int s = 0; s < w->nslot; ++s) {
        if (!w->slot[s].valid) { f = &w->slot[s]; break; }
        if (w->slot[s].last < f->last) f = &w->slot[s];
      }
    } else {
      f = &w->scratch;
    }
    f->valid = 0;
    /* solve_linear_system_base, kriging_base.F90:3244-3398 */
    info = chol_setup(npp, pa, A, m, f);
    if (info == 0) {
      f->used_sysv = 0;
      chol_solve(npp, pa, nvar, f, B, X, work);
      w->stats[1]++;
    } else {
      for (size_t q = 0; q < (size_t)m * m; ++q) f->Afac[q] = A[q];
      info = sytf2_u(m, f->Afac, m, f->ipiv);
      if (info != 0 && npp > 0) {
        double dscale = 0.0;
        for (int ii = 0; ii < npp; ++ii) dscale = dscale + A[ii + (size_t)ii * m];
        if (dscale > 0.0) {
          dscale = 1.0e-6 * (dscale / (double)npp);
          for (int ii = 0; ii < npp; ++ii) A[ii + (size_t)ii * m] = A[ii + (size_t)ii * m] + dscale;
          for (size_t q = 0; q < (size_t)m * m; ++q) f->Afac[q] = A[q];
          info = sytf2_u(m, f->Afac, m, f->ipiv);
        }
      }
      if (info == 0) {
        f->used_sysv = 1;
        ldl_solve(m, nvar, f, B, X, work);
        w->stats[3]++;
      }
    }
    if (info == 0) {
      fac_save_key(f, w, c, h, npp, rs, ln);
      f->last = ++w->clock;
      if (f == &w->scratch) f->valid = 0;
    }
  }
  int nn_est[ORC_MAXVAR];
  for (int v = 0; v < nvar; ++v) nn_est[v] = w->nnear[v];
  if (info != 0) {
    if (P->neglect_error) {
      for (int q = 0; q < nvar * m; ++q) X[q] = NAN;
      for (int v = 0; v < nvar; ++v) nn_est[v] = 1;
      w->stats[0]++;
    } else {
      *err_flag = 1;
      snprintf(errmsg, 256, "Singular matrix at block %d", ib + 1);
      return;
    }
  }

  /* calc_variance, kriging.F90:968-1028 / kriging_st.F90:986-1044 */
  for (int iv = 0; iv < nvar; ++iv)
    for (int jv = iv; jv < nvar; ++jv) {
      double base;
      if (nbp == 1) {
        base = pair_cov0(c, iv, jv);
      } else {
        base = 0.0;
        double c0 = pair_cov0(c, iv, jv);
        for (int i = 0; i < nbp; ++i) {
          double wi = P->grid_weight[k0 + i];
          base = base + c0 * wi * wi;
          for (int j = i + 1; j < nbp; ++j) {
            double lag[4];
            for (int d = 0; d < nlag; ++d)
              lag[d] = gc[(size_t)(k0 + i) * nlag + d] - gc[(size_t)(k0 + j) * nlag + d];
            base = base + pair_cov(c, iv, jv, lag) * wi * P->grid_weight[k0 + j] * 2.0;
          }
        }
      }
      double s = 0.0;
      for (int k = 0; k < m; ++k) s = s + X[iv + (size_t)k * nvar] * B[jv + (size_t)k * nvar];
      var[iv + jv * nvar] = base - s;
      if (iv != jv) var[jv + iv * nvar] = var[iv + jv * nvar];
    }
  for (int iv = 0; iv < nvar; ++iv) {
    if (!(var[iv + iv * nvar] >= 0.0) && !isnan(var[iv + iv * nvar])) var[iv + iv * nvar] = 0.0;
    for (int jv = iv + 1; jv < nvar; ++jv) {
      double t = var[jv + iv * nvar];
      if (t < 0.0) t = 0.0;
      var[jv + iv * nvar] = t;
      var[iv + jv * nvar] = t;
    }
  }

  /* assign_weight_ctx + estimate_block_base, kriging_base.F90:2428-2439, 3407-3503 */
  const int ck_isa = !P->std_ck && P->unbias != 0 && nvar > 1;
  double tmean[ORC_MAXVAR];
  if (ck_isa)
    for (int v = 0; v < nvar; ++v) {
      double s = 0.0;
      for (int k = 0; k < nn_est[v]; ++k) s = s + P->obs_value[v][w->inear[v * mmax + k]];
      tmean[v] = nn_est[v] > 0 ? s / nn_est[v] : 0.0;
    }
  for (int jv = 0; jv < nvar; ++jv) {
    double tw[ORC_MAXVAR];
    double avg = 0.0;
    for (int v = 0; v < nvar; ++v) {
      tw[v] = 0.0;
      double sw = 0.0, dp = 0.0;
      for (int k = 0; k < nn_est[v]; ++k) {
        double wt = X[jv + (size_t)(istart[v] + k) * nvar];
        sw = sw + wt;
        dp = dp + P->obs_value[v][w->inear[v * mmax + k]] * wt;
      }
      tw[v] = tw[v] + sw;
      avg = avg + dp;
      if (ck_isa && v != jv && nn_est[v] > 0) avg = avg + (tmean[jv] - tmean[v]) * tw[v];
    }
    if (P->unbias == 0 && P->sk_mean[jv] != 0.0) {
      double st = 0.0;
      for (int v = 0; v < nvar; ++v) st = st + tw[v];
      avg = avg + (1.0 - st) * P->sk_mean[jv];
    }
    if (avg < P->bounds[0]) avg = P->bounds[0];
    if (avg > P->bounds[1]) avg = P->bounds[1];
    val[jv] = avg;
  }
  if (res->weight) {
    for (int jv = 0; jv < nvar; ++jv)
      for (int v = 0; v < nvar; ++v)
        for (int k = 0; k < res->mmax; ++k) {
          double wt = k < nn_est[v] ? X[jv + (size_t)(istart[v] + k) * nvar] : 0.0;
          res->weight[(((size_t)ib * nvar + jv) * nvar + v) * res->mmax + k] = wt;
        }
  }
}

int orc_solve(const orc_problem *P, orc_result *R) {
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->p = P;
  c->nvar = P->nvar;
  c->ndim = P->ndim;
  c->nlag = P->nlag > 0 ? P->nlag : P->ndim;
  c->st = P->st;
  c->naug = P->std_ck ? P->unbias * P->nvar : P->unbias;
  c->pa = P->ndrift + c->naug;
  R->err = 0;
  R->errmsg[0] = 0;
  for (int i = 0; i < 5; ++i) R->stats[i] = 0;
  if (P->nvar < 1 || P->nvar > ORC_MAXVAR) { R->err = 1; snprintf(R->errmsg, 256, "bad nvar"); free(c); return 1; }

  /* set_search per variable: kriging.F90:318-387, kriging_st.F90:322-403 */
  int mmax = 0, heapn = 1;
  for (int v = 0; v < P->nvar; ++v) {
    int nobs = P->nobs[v];
    c->nobs[v] = nobs;
    int nmax = P->nmax[v];
    if (P->cross_validation && v == 0 && nmax > 0 && nmax < 2147483647) nmax = nmax + 1;
    if (nmax > nobs) nmax = nobs;
    if (nmax <= 0) nmax = nobs;
    c->nmax[v] = nmax;
    c->need_search[v] = nobs > nmax;
    c->sector[v] = P->sector[v];
    c->maxd2[v] = P->maxdist[v] * P->maxdist[v];
    c->ta[v] = P->time_at[v] > 0.0 ? P->time_at[v] : 1.0;
    double a1 = P->s_anis1[v] != 0.0 ? P->s_anis1[v] : 1.0;
    double a2 = P->s_anis2[v] != 0.0 ? P->s_anis2[v] : 1.0;
    c->aniso[v] = (fabs(a1 - 1.0) > ORC_EPSLON || fabs(a2 - 1.0) > ORC_EPSLON) && P->anisotropic_search;
    double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    memcpy(c->rotmat[v], eye, sizeof eye);
    if (c->st || (c->need_search[v] && c->aniso[v]))
      orc_calc_rotmat(P->s_az[v], P->s_dip[v], P->s_plunge[v], a1, a2, c->rotmat[v]);
    if (c->need_search[v]) {
      const int nlag = c->nlag, ndim = c->ndim;
      double *sc = (double *)malloc(sizeof(double) * (size_t)nlag * nobs);
      for (int i = 0; i < nobs; ++i) {
        const double *x = P->obs_coord[v] + (size_t)i * nlag;
        if (c->aniso[v]) rotate_pt(c->rotmat[v], ndim, x, sc + (size_t)i * nlag);
        else for (int d = 0; d < ndim; ++d) sc[(size_t)i * nlag + d] = x[d];
        if (c->st) sc[(size_t)i * nlag + nlag - 1] = x[nlag - 1] * c->ta[v];
      }
      c->scoord[v] = sc;
      kd_create(&c->tree[v], sc, nlag, nobs);
      c->has_tree[v] = 1;
    }
    int on = c->sector[v] ? (1 << c->ndim) * nmax : nmax;
    if (on > mmax) mmax = on;
    int hn = c->sector[v] ? ((1 << c->ndim) * nmax * 4 > nobs ? (1 << c->ndim) * nmax * 4 : nobs) : nobs;
    if (hn > heapn) heapn = hn;
  }
  /* the all-observation branch can return every observation */
  for (int v = 0; v < P->nvar; ++v) if (!c->need_search[v] && c->nobs[v] > mmax) mmax = c->nobs[v];
  c->mmax = mmax;
  c->nppmax = mmax * P->nvar;
  c->mmat = c->nppmax + c->pa;
  c->heapn = heapn;

  /* prepare: tables, kriging.F90:398-424 / kriging_st.F90:414-447 */
  for (int a = 0; a < P->nvar; ++a)
    for (int b = 0; b < P->nvar; ++b) {
      if (!c->st) {
        if (b < a) continue;
        if (P->nstruct[a][b] == 0) {
          R->err = 1;
          snprintf(R->errmsg, 256, "variogram not set for ivar=%d, jvar=%d", a + 1, b + 1);
        }
        model_init(&c->mdl[a][b], c->ndim, P->vgm[a][b], P->nstruct[a][b]);
        model_build_table(&c->mdl[a][b]);
      } else {
        orc_stmodel *s = &c->smdl[a][b];
        model_init(&s->cs, c->ndim, P->vgm[a][b], P->nstruct[a][b]);
        model_init(&s->ct, 1, P->vgm_t[a][b], P->nstruct_t[a][b]);
        s->model = P->st_model;
        s->tvtype = P->st_transform;
        s->t_nugget = P->st_time_nugget;
        s->t_sill = P->st_time_sill;
        s->at = P->st_at;
        s->k_ps = P->st_k_ps;
        s->has_joint = P->st_has_joint[a][b];
        for (int k = 0; k < ORC_MAXSTRUCT; ++k) s->joint[k] = P->st_joint[a][b][k];
        st_cov0(s);
        model_build_table(&s->cs);
        model_build_table(&s->ct);
      }
    }
  if (R->err) goto done;
  if (P->nblockpnt) {
    c->gstart = (int *)malloc(sizeof(int) * (P->nblock + 1));
    int acc = 0;
    for (int ib = 0; ib < P->nblock; ++ib) { c->gstart[ib] = acc; acc += P->nblockpnt[ib]; }
  }

  int nthread = 1;
#ifdef _OPENMP
  nthread = P->nthread > 0 ? P->nthread : omp_get_max_threads();
#endif
  int err_flag = 0;
  char errmsg[256] = {0};
  int stats[5] = {0, 0, 0, 0, 0};
#pragma omp parallel num_threads(nthread)
  {
    orc_ws w;
    memset(&w, 0, sizeof w);
    size_t mm = (size_t)c->mmat;
    w.matA = (double *)malloc(sizeof(double) * mm * mm);
    w.rhsB = (double *)malloc(sizeof(double) * mm * P->nvar);
    w.x = (double *)malloc(sizeof(double) * mm * P->nvar);
    w.sqd = (double *)malloc(sizeof(double) * ((size_t)c->mmax + mm * (P->nvar + 1) + mm * mm));
    w.inear = (int *)malloc(sizeof(int) * (size_t)c->mmax * P->nvar);
    w.heap = (kd_res *)malloc(sizeof(kd_res) * ((size_t)c->heapn + 1));
    fac_alloc(&w.scratch, c);
    w.nslot = P->ncache > 0 ? P->ncache : 0;
    /* slot memory is bounded like MAX_HCACHE_BYTES (kriging_base.F90:2350) */
    double slot_bytes = 8.0 * ((double)c->nppmax * c->nppmax + (double)mm * mm);
    while (w.nslot > 0 && w.nslot * slot_bytes > 64.0 * 1024 * 1024) --w.nslot;
    w.slot = w.nslot ? (orc_fac *)malloc(sizeof(orc_fac) * w.nslot) : NULL;
    for (int s = 0; s < w.nslot; ++s) fac_alloc(&w.slot[s], c);
    int my_err = 0;
    char my_msg[256];
#pragma omp for schedule(dynamic, 1)
    for (int ib = 0; ib < P->nblock; ++ib) {
      if (err_flag) continue;
      solve_target(c, &w, ib, R, &my_err, my_msg);
      if (my_err) {
#pragma omp critical(orc_err)
        {
          if (!err_flag) { err_flag = 1; memcpy(errmsg, my_msg, 256); }
        }
        my_err = 0;
      }
    }
#pragma omp critical(orc_stats)
    for (int i = 0; i < 5; ++i) stats[i] += w.stats[i];
    free(w.matA); free(w.rhsB); free(w.x); free(w.sqd); free(w.inear); free(w.heap);
    fac_free(&w.scratch);
    for (int s = 0; s < w.nslot; ++s) fac_free(&w.slot[s]);
    free(w.slot);
  }
  for (int i = 0; i < 5; ++i) R->stats[i] = stats[i];
  if (err_flag) { R->err = 1; memcpy(R->errmsg, errmsg, 256); }
done:
  for (int v = 0; v < P->nvar; ++v) {
    if (c->has_tree[v]) kd_free(&c->tree[v]);
    free(c->scoord[v]);
  }
  for (int a = 0; a < P->nvar; ++a)
    for (int b = 0; b < P->nvar; ++b) {
      if (!c->st) { if (b >= a) model_free(&c->mdl[a][b]); }
      else { model_free(&c->smdl[a][b].cs); model_free(&c->smdl[a][b].ct); }
    }
  free(c->gstart);
  free(c);
  return R->err;
}

/* ------------------------------------------------------------------------ */
/* sequential Gaussian simulation of one variable                           */
/* ------------------------------------------------------------------------ */
/* set_sim_base (kriging_base.F90:1226-1320): the targets are visited in the
 * order of path (1-based), the simulated targets join the observations as a
 * second neighbour group (obs%coord extended by the block centres in path
 * order).  Per visited target (search_neighbors, kriging.F90:524-612):
 * the nmax nearest among the observations and the targets visited before it
 * (kdtree2_n_nearest_maxidx), or all of them when nmax does not cut; the
 * simulated group keeps the heap order, is cut by maxdist, and loses members
 * co-located with an observation neighbour.  The system carries the
 * observation group (sorted, with its measurement variance) and the
 * simulated group (no measurement variance) (assemble_lhs / assemble_rhs,
 * kriging.F90:740-939); the draw adds the simulated group's values and the
 * square root of the conditional variance times the sample
 * (estimate_block_base + sim_draw_base, kriging_base.F90:3473-3495, 2320-2327);
 * results return to target order (reorder_sgsim_base, :2268-2282). */
int orc_sgsim(const orc_problem *P, const int *path, const double *sample, int nsim, orc_sim_result *R) {
  R->err = 0;
  R->errmsg[0] = 0;
  if (P->nvar != 1 || P->st || P->nblockpnt || P->cross_validation) {
    R->err = 1;
    snprintf(R->errmsg, 256, "sgsim: one variable, point targets, no cross-validation");
    return 1;
  }
  const int nb = P->nblock, nobs = P->nobs[0], ndim = P->ndim, nlag = ndim;
  const int ntot = nobs + nb;
  int nmax = P->nmax[0];
  if (nmax <= 0 || nmax > ntot) nmax = ntot;
  /* sector search: the sorted candidates of kdtree2_n_nearest_maxidx (the
   * tree is built with sort = sector_search, kriging.F90:378-381) through
   * apply_sector_filter; the tree exists only when nmax cuts (need_search,
   * kriging.F90:362-363) */
  const int sector = P->sector[0];
  if (sector && ntot <= nmax) {
    R->err = 1;
    snprintf(R->errmsg, 256, "sgsim: sector search needs nmax below the observations plus targets");
    return 1;
  }
  const int lim4 = (1 << ndim) * nmax * 4;
  const int ncmax = sector ? (ntot < lim4 ? ntot : lim4) : nmax;
  const int mcap = sector ? (1 << ndim) * nmax : nmax;
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->p = P;
  c->nvar = 1;
  c->ndim = ndim;
  c->nlag = nlag;
  c->naug = P->unbias;
  c->pa = P->ndrift + c->naug;
  const int pa = c->pa, ndr = P->ndrift;
  if (P->nstruct[0][0] == 0) {
    R->err = 1;
    snprintf(R->errmsg, 256, "variogram not set for ivar=1, jvar=1");
    free(c);
    return 1;
  }
  model_init(&c->mdl[0][0], ndim, P->vgm[0][0], P->nstruct[0][0]);
  model_build_table(&c->mdl[0][0]);
  double a1 = P->s_anis1[0] != 0.0 ? P->s_anis1[0] : 1.0;
  double a2 = P->s_anis2[0] != 0.0 ? P->s_anis2[0] : 1.0;
  const int aniso = (fabs(a1 - 1.0) > ORC_EPSLON || fabs(a2 - 1.0) > ORC_EPSLON) && P->anisotropic_search;
  double rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  /* the rotation exists only with the tree (need_search, kriging.F90:371-376) */
  if (aniso && ntot > nmax) orc_calc_rotmat(P->s_az[0], P->s_dip[0], P->s_plunge[0], a1, a2, rot);
  const double maxd2 = P->maxdist[0] * P->maxdist[0];

  /* observations, then the targets in visiting order */
  double *xc = (double *)malloc(sizeof(double) * (size_t)ntot * nlag);
  double *sc = (double *)malloc(sizeof(double) * (size_t)ntot * nlag);
  for (int i = 0; i < nobs; ++i)
    for (int d = 0; d < nlag; ++d) xc[(size_t)i * nlag + d] = P->obs_coord[0][(size_t)i * nlag + d];
  for (int p = 0; p < nb; ++p)
    for (int d = 0; d < nlag; ++d)
      xc[(size_t)(nobs + p) * nlag + d] = P->block_coord[(size_t)(path[p] - 1) * nlag + d];
  for (int i = 0; i < ntot; ++i) {
    if (aniso) rotate_pt(rot, ndim, xc + (size_t)i * nlag, sc + (size_t)i * nlag);
    else for (int d = 0; d < ndim; ++d) sc[(size_t)i * nlag + d] = xc[(size_t)i * nlag + d];
  }
  kd_tree tree;
  kd_create(&tree, sc, nlag, ntot);
  double *vals = (double *)malloc(sizeof(double) * (size_t)nsim * nb);  /* [isim][path position] */
  kd_res *h = (kd_res *)malloc(sizeof(kd_res) * ((size_t)ncmax + 1));
  double *dob = (double *)malloc(sizeof(double) * ((size_t)ntot + 1));
  int *io = (int *)malloc(sizeof(int) * ((size_t)ntot + 1));
  int *ib_ = (int *)malloc(sizeof(int) * ((size_t)ntot + 1));
  double *db = (double *)malloc(sizeof(double) * ((size_t)ntot + 1));
  const int mm = mcap + pa;
  double *A = (double *)malloc(sizeof(double) * (size_t)mm * mm);
  double *B = (double *)malloc(sizeof(double) * mm);
  double *X = (double *)malloc(sizeof(double) * mm);
  double *work = (double *)malloc(sizeof(double) * ((size_t)mm * 2 + (size_t)mm * mm));
  orc_fac f;
  memset(&f, 0, sizeof f);
  f.L = (double *)malloc(sizeof(double) * (size_t)mm * mm);
  f.Y = (double *)malloc(sizeof(double) * (size_t)mm * (pa > 0 ? pa : 1));
  f.S = (double *)malloc(sizeof(double) * (pa > 0 ? pa * pa : 1));
  f.Afac = (double *)malloc(sizeof(double) * (size_t)mm * mm);
  f.ipiv = (int *)malloc(sizeof(int) * mm);
  const double cov0 = c->mdl[0][0].cov0;

  for (int p = 0; p < nb && !R->err; ++p) {
    const int node = path[p] - 1;
    const double *xloc = P->block_coord + (size_t)node * nlag;
    const double rs = P->rangescale ? P->rangescale[node] : 1.0;
    const double ln = P->localnugget ? P->localnugget[node] : 0.0;
    double newloc[3];
    if (aniso) rotate_pt(rot, ndim, xloc, newloc);
    else for (int d = 0; d < ndim; ++d) newloc[d] = xloc[d];
    int no = 0, nbk = 0;
    const int lim = nobs + p;
    if (sector) {
      const int ncand = lim < ncmax ? lim : ncmax;
      kd_n_nearest_max(&tree, newloc, ncand, 1, h, lim);
      /* apply_sector_filter, kriging.F90:1093-1154, over observations and
       * earlier targets alike (obsloc holds both) */
      int count[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = 1; i <= ncand; ++i) {
        const int idx = h[i].idx;
        if (h[i].dis > maxd2) continue;
        double pr[3];
        if (aniso) rotate_pt(rot, ndim, xc + (size_t)idx * nlag, pr);
        else for (int d = 0; d < ndim; ++d) pr[d] = xc[(size_t)idx * nlag + d];
        const double dx = pr[0] - newloc[0];
        const double dy = ndim > 1 ? pr[1] - newloc[1] : 0.0;
        const double dz = ndim == 3 ? pr[2] - newloc[2] : 0.0;
        const int sec = (dx < 0.0 ? 1 : 0) + (dy < 0.0 ? 2 : 0) + (ndim == 3 && dz < 0.0 ? 4 : 0);
        if (count[sec] < nmax) {
          count[sec]++;
          if (idx < nobs) { dob[no] = h[i].dis; io[no++] = idx; }
          else { ib_[nbk] = idx - nobs; db[nbk] = h[i].dis; ++nbk; }
        }
      }
    } else if (nmax < lim) {
      kd_n_nearest_max(&tree, newloc, nmax, 0, h, lim);
      for (int i = 1; i <= nmax; ++i) {
        if (h[i].idx < nobs) { dob[no] = h[i].dis; io[no++] = h[i].idx; }
        else { ib_[nbk] = h[i].idx - nobs; db[nbk] = h[i].dis; ++nbk; }
      }
    } else {
      for (int i = 0; i < nobs; ++i) {  /* rotated_dists of the raw observations */
        double diff[3], r[3];
        for (int d = 0; d < ndim; ++d) diff[d] = xc[(size_t)i * nlag + d] - newloc[d];
        rotate_pt(rot, ndim, diff, r);
        double s2 = 0.0;
        for (int d = 0; d < ndim; ++d) s2 = s2 + r[d] * r[d];
        dob[no] = s2;
        io[no++] = i;
      }
      for (int q = 0; q < p; ++q) {  /* rotated_dists of the raw block centres (rotation.f90:193-218) */
        double diff[3], r[3];
        for (int d = 0; d < ndim; ++d) diff[d] = xc[(size_t)(nobs + q) * nlag + d] - newloc[d];
        rotate_pt(rot, ndim, diff, r);
        double s2 = 0.0;
        for (int d = 0; d < ndim; ++d) s2 = s2 + r[d] * r[d];
        ib_[nbk] = q;
        db[nbk] = s2;
        ++nbk;
      }
    }
    /* filter_by_maxlag on the simulated group (kriging_base.F90:2491-2505) */
    int k2 = 0;
    for (int i = 0; i < nbk; ++i)
      if (db[i] <= maxd2) { ib_[k2] = ib_[i]; db[k2] = db[i]; ++k2; }
    nbk = k2;
    /* simulated targets co-located with an observation neighbour, kriging.F90:584-609 */
    if (no > 0 && nbk > 0) {
      k2 = 0;
      for (int jb = 0; jb < nbk; ++jb) {
        int dup = 0;
        for (int oo = 0; oo < no; ++oo) {
          dup = 1;
          for (int d = 0; d < ndim; ++d) {
            const double xo = xc[(size_t)io[oo] * nlag + d];
            if (fabs(xc[(size_t)(nobs + ib_[jb]) * nlag + d] - xo) > 1.0e-6 * (1.0 + fabs(xo))) { dup = 0; break; }
          }
          if (dup) break;
        }
        if (!dup) { ib_[k2] = ib_[jb]; db[k2] = db[jb]; ++k2; }
      }
      nbk = k2;
    }
    /* filter_by_maxlag on the observation group (kriging.F90:660-661, after
     * the simulation branch) */
    k2 = 0;
    for (int i = 0; i < no; ++i)
      if (dob[i] <= maxd2) io[k2++] = io[i];
    no = k2;
    isort(io, no);
    if (R->nnear) { R->nnear[(size_t)node * 2] = no; R->nnear[(size_t)node * 2 + 1] = nbk; }
    if (R->inear) {
      for (int i = 0; i < no; ++i) R->inear[(size_t)node * R->mmax + i] = io[i];
      for (int i = 0; i < nbk; ++i) R->inear[(size_t)node * R->mmax + no + i] = nobs + ib_[i];
    }
    const int npp = no + nbk, m = npp + pa;
    double var = NAN;
    double *vrow = R->value + (size_t)node * nsim;
    if (npp == 0) {
      for (int is = 0; is < nsim; ++is) { vrow[is] = NAN; vals[(size_t)is * nb + p] = NAN; }
      R->variance[node] = NAN;
      continue;
    }
    /* row coordinates: observation group, then the simulated group */
#define SG_X(k) ((k) < no ? xc + (size_t)io[(k)] * nlag : xc + (size_t)(nobs + ib_[(k) - no]) * nlag)
    for (size_t q = 0; q < (size_t)m * m; ++q) A[q] = 0.0;
    for (int i = 0; i < npp; ++i) {
      const double ov = (i < no && P->obs_var[0]) ? P->obs_var[0][io[i]] : 0.0;
      A[i + (size_t)i * m] = cov0 + ov + ln;
      for (int j = i + 1; j < npp; ++j) {
        double lag[4];
        lag_of(c, SG_X(i), SG_X(j), rs, lag);
        A[j + (size_t)i * m] = pair_cov(c, 0, 0, lag);
      }
      /* drift rows, then unbiasedness (kriging.F90:789-794): the observation
       * drift for observation members, the target drift at the simulated
       * target's node for simulated members (block%drift in visiting order) */
      for (int r = 0; r < pa; ++r) {
        double fv = 1.0;
        if (r < ndr)
          fv = i < no ? P->obs_drift[0][(size_t)io[i] * ndr + r]
                      : P->block_drift[(size_t)(path[ib_[i - no]] - 1) * ndr + r];
        A[(npp + r) + (size_t)i * m] = fv;
      }
    }
    for (int ir = 0; ir < npp; ++ir)
      for (int ic = ir + 1; ic < m; ++ic) A[ir + (size_t)ic * m] = A[ic + (size_t)ir * m];
    for (int k = 0; k < npp; ++k) {
      double lag[4];
      lag_of(c, SG_X(k), xloc, rs, lag);
      B[k] = pair_cov(c, 0, 0, lag);
    }
    for (int r = 0; r < pa; ++r) B[npp + r] = r < ndr ? P->block_drift[(size_t)node * ndr + r] : 1.0;
#undef SG_X
    int info = chol_setup(npp, pa, A, m, &f);
    if (info == 0) {
      chol_solve(npp, pa, 1, &f, B, X, work);
    } else {
      for (size_t q = 0; q < (size_t)m * m; ++q) f.Afac[q] = A[q];
      info = sytf2_u(m, f.Afac, m, f.ipiv);
      if (info != 0) {
        double dscale = 0.0;
        for (int ii = 0; ii < npp; ++ii) dscale = dscale + A[ii + (size_t)ii * m];
        if (dscale > 0.0) {
          dscale = 1.0e-6 * (dscale / (double)npp);
          for (int ii = 0; ii < npp; ++ii) A[ii + (size_t)ii * m] = A[ii + (size_t)ii * m] + dscale;
          for (size_t q = 0; q < (size_t)m * m; ++q) f.Afac[q] = A[q];
          info = sytf2_u(m, f.Afac, m, f.ipiv);
        }
      }
      if (info == 0) ldl_solve(m, 1, &f, B, X, work);
    }
    if (info != 0) {
      if (!P->neglect_error) {
        R->err = 1;
        snprintf(R->errmsg, 256, "Singular matrix at block %d", node + 1);
        break;
      }
      for (int is = 0; is < nsim; ++is) { vrow[is] = NAN; vals[(size_t)is * nb + p] = NAN; }
      R->variance[node] = NAN;
      continue;
    }
    double s = 0.0;
    for (int k = 0; k < m; ++k) s = s + X[k] * B[k];
    var = cov0 - s;
    if (!(var >= 0.0) && !isnan(var)) var = 0.0;
    R->variance[node] = var;
    double avg = 0.0, tw = 0.0;
    for (int k = 0; k < no; ++k) {
      tw = tw + X[k];
      avg = avg + P->obs_value[0][io[k]] * X[k];
    }
    if (P->unbias == 0 && P->sk_mean[0] != 0.0) avg = avg + (1.0 - tw) * P->sk_mean[0];
    const double L = sqrt(var > 0.0 ? var : 0.0);
    for (int is = 0; is < nsim; ++is) {
      double v = avg, dp = 0.0;
      for (int k = 0; k < nbk; ++k) dp = dp + vals[(size_t)is * nb + ib_[k]] * X[no + k];
      v = v + dp;
      v = v + L * sample[(size_t)p * nsim + is];
      if (v < P->bounds[0]) v = P->bounds[0];
      if (v > P->bounds[1]) v = P->bounds[1];
      vals[(size_t)is * nb + p] = v;
      vrow[is] = v;
    }
  }
  free(f.L); free(f.Y); free(f.S); free(f.Afac); free(f.ipiv);
  free(A); free(B); free(X); free(work); free(h); free(dob); free(io); free(ib_); free(db); free(vals);
  kd_free(&tree);
  free(xc); free(sc);
  model_free(&c->mdl[0][0]);
  free(c);
  return R->err;
}
