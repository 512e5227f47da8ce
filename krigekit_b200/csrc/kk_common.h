// kk_common.h -- types shared by the host engine and the sm_100a kernels.
//
// Layout of every device-resident object of the kriging solve path:
//   * variogram models, one descriptor per ORDERED variable pair (first,
//     second) = the reference's vgm(first, second); lookup tables in one
//     global double2 array {tab[i], tab[i+1]-tab[i]} (variogram.f90:263-324,
//     572-679), zones fixed at h = [0, 0.1, 0.5, 3.5] (kriging.F90:416-417);
//   * observations per variable, structure-of-arrays FP64;
//   * a uniform grid over the search-space coordinates of each variable
//     (CSR cell_start over cells, x fastest, plus a summed-area table);
//   * targets as structure-of-arrays FP64 with optional block nodes (CSR).
#pragma once
#include <stdint.h>

#define KK_MAXVAR 4
#define KK_MAXSTRUCT 16
#define KK_TAB_NZ 3
#define KK_TAB_N 17000  // intervals: 10000 + 4000 + 3000

// variogram shape ids, vgmfunc.f90:7-17
enum { KK_NUG = 0, KK_SPH, KK_EXP, KK_GAU, KK_HOL, KK_POW, KK_BSQ, KK_CIR, KK_LIN, KK_CYC, KK_DCO };

// model evaluation modes
enum { KK_LEVEL_B = 0, KK_LEVEL_A = 1, KK_ANALYTIC = 2 };

struct KkComp {
  int vtype;
  int is_product;
  int tab_off;   // Level A: offset (in double2 entries) of this component's table, -1 if none
  int tail;      // corefunc_has_analytic_tail
  double sill, nugget, a_major;
  double mat[9];  // column-major aniso transform (variogram.f90:185-192)
};

struct KkModel {
  int mode;      // KK_LEVEL_B / KK_LEVEL_A / KK_ANALYTIC
  int nstruct;
  int ndim;
  int btab_off;  // Level B table offset
  int btail;
  int pad_;
  double cov0;
  double bmat[9];
  KkComp comp[KK_MAXSTRUCT];
};

// space-time model, variogram_st.f90:66-98
struct KkSTModel {
  KkModel cs, ct;
  int model;     // 0 sum-metric, 1 product-sum
  int tvtype;
  int has_joint;
  int pad_;
  double t_nugget, t_sill, at, k_ps, cov0;
  double joint[KK_MAXSTRUCT];
};

// uniform grid over the search-space coordinates of one variable
struct KkGrid {
  int G;          // gridded dimensions (1..3)
  int D;          // search dimensions (nlag)
  int gd[3];      // search dimension of each grid axis (the widest three when D = 4)
  int gmask;      // bit d set when search dimension d is a grid axis
  double gumin[3], gumax[3];  // bounding box of the grid axes
  int nobs;
  int n[3];       // cells per gridded dimension
  double lo[3], h[3], inv_h[3];
  double umin[4], umax[4];  // bounding box of every search dimension
  const int* cell_start;    // ncells + 1
  const int* sat;           // (n0+1)(n1+1)(n2+1) summed-area table of cell counts
  const double* sc;         // sorted search coords, SoA: sc[d * nobs + j]
  const int* sidx;          // original index of sorted point j
};

// kd-tree flattened for the device tie fallback (kdtree2_maxidx.f90)
struct KkTree {
  int D, n, nnodes, root;
  const int* node_i;        // per node: cut_dim, l, u, left, right (5 ints)
  const double* node_d;     // per node: cut_val, cut_val_left, cut_val_right
  const double* box;        // per node: D x {lo, hi}
  const int* ind;           // permuted indices
  const double* rdata;      // rearranged data (D, n) point-major
};

struct KkSearch {
  int mode;       // 0 all observations, 1 k nearest, 2 sector
  int K;          // candidates to select (nmax, or 2^ndim * nmax * 4 for sectors)
  int nmax;       // per-sector cap for sectors
  int ndim;       // spatial dimension
  int nlag;
  int aniso;
  int st;
  int nobs;
  int mmax;       // leading dimension of this variable's neighbour list
  int cv;         // cross-validation (skip the target's own index)
  double maxd2;
  double ta;
  double rotmat[9];
  KkGrid grid;
  KkTree tree;
};

// per-target status bits written by the search and solve kernels
enum {
  KK_ST_TIE = 1,         // equal distances at a selection boundary -> kd-tree path
  KK_ST_OVERFLOW = 2,    // candidate buffer overflow -> kd-tree path
  KK_ST_FP64 = 4,        // FP32 refinement did not converge -> FP64 solve
  KK_ST_LDLT = 8,        // Cholesky failed -> LDL^T path
  KK_ST_FAIL = 16,       // singular after jitter -> NaN
  KK_ST_EMPTY = 32,      // no neighbours
  KK_ST_BIG = 64,        // more neighbours than the register kernels hold (> 128)
};

// Neighbour-count lists written by the bucketing kernel, list li at
// lists + li * nblock: 2..32, 33..64, > 128 and 65..128 equations
enum { KK_LIST_B32 = 0, KK_LIST_B64 = 1, KK_LIST_BIG = 2, KK_LIST_B128 = 3, KK_NLIST = 4 };

// Solve kernels a list can be planned on: warp per target holding 32 or 64
// equations (FP64, or FP32 factor + FP64 correction: the R forms), CTA per
// target holding 128 (FP64), and the general thread-per-target kernel (FP64,
// any size)
enum {
  KK_KER_W32 = 0,
  KK_KER_W64 = 1,
  KK_KER_BLOCK = 2,
  KK_KER_GEN = 3,
  KK_KER_W32R = 4,
  KK_KER_W64R = 5,
  KK_NKER = 6
};
