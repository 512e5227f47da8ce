// kk_kernels.h -- launchers of the sm_100a kernels (kk_search.cu, kk_solve.cu).
#pragma once
#include <cuda_runtime.h>

#include "kk_common.h"

namespace kk {

// Everything the solve kernels read for one solve() call.
#define KK_FA_MAXS 4  // structures per vgm(i, j) on the Level-A fast path

struct SolveParams {
  int nvar, ndim, nlag, st;
  int ndrift, pa, naug, std_ck, unbias;
  int ck_isa;        // Isaaks & Srivastava mean correction (estimate_block_base)
  int sk_any;        // simple kriging with a non-zero mean
  int nmin;
  int neglect_error;
  double bounds[2];
  double sk_mean[KK_MAXVAR];
  const KkModel* models;     // nvar * nvar, [first * nvar + second]
  const KkSTModel* smodels;  // space-time models or null
  const double2* tables;
  // observations per variable (SoA)
  const double* ox[KK_MAXVAR][4];
  const double* oval[KK_MAXVAR];
  const double* ovar[KK_MAXVAR];
  const double* odrift[KK_MAXVAR];  // (ndrift) x nobs SoA
  int nobs[KK_MAXVAR];
  // neighbour lists
  const int* nbr[KK_MAXVAR];
  const int* nnear[KK_MAXVAR];
  int mmax[KK_MAXVAR];
  // targets
  int nblock;
  const double* tx[4];
  const double* rs;          // rangescale or null
  const double* ln;          // localnugget or null
  const double* tdrift;      // (ndrift, nvar, nblock) or null
  const int* gstart;         // block node CSR (nblock + 1) or null
  const double* gx[4];
  const double* gw;
  // outputs
  double* est;               // (nblock, nvar)
  double* var;               // (nblock, nvar, nvar)
  int* status;
  int* counters;             // see KK_CNT_*
  int* fb_list;              // targets needing the generic FP64 / LDL^T path
  int* fp64_list;            // FP32 targets that need the FP64 register kernel
  double* wout;              // kriging weights (weight store) or null: row r of target
                             // variable jv of target t at wout[(t * nvar + jv) * wstride + r],
                             // rows in matrix order (variable blocks, ascending index)
  int wstride;
  double* scratch;           // generic-path workspace
  int scratch_stride;        // doubles per generic-path thread
  double refine_tol;
  double refine_tol_corr;    // bound on the FP32 correction term relative to its value
  int fast_model;            // fast covariance path of single-variable spatial kriging:
                             // 1 = one Level-B table; 2 = Level-A tables of structures
                             // whose transforms are multiples k * fm of one matrix
  int fm_ndim, fm_tail, fm_tab_off;  // transform dimension; Level B: analytic tail, table offset
  double fm[9];              // the anisotropy transform (bmat, or the Level-A common matrix)
  int fa_nst, fa_tailmask;   // Level A: structures, bit s = structure s has an analytic tail
  int fa_off[KK_FA_MAXS];    // their table offsets
  double fa_k[KK_FA_MAXS];   // and transform multiples
  // fast_model 3 (2 variables, every structure's transform a multiple of fm):
  // per pair i * 2 + j its kind (1 Level-B table, 2 Level-A tables, 3
  // analytic), structures, table offsets, multiples and tail bits
  int fq_kind[4], fq_nst[4], fq_tail[4];
  // fast_model 4 (space-time, one variable, Level-B spatial and temporal
  // tables, product-sum or sum-metric without joint sills): the spatial
  // table is fm / fm_tab_off / fm_tail, the temporal one ft_*
  int ft_off, ft_tail, st_kind;
  double ft_k, st_kps;
  int fq_off[4][KK_FA_MAXS];
  double fq_k[4][KK_FA_MAXS];
};

enum {
  KK_CNT_B16 = 0,   // bucket sizes (targets with npp in 2..32)
  KK_CNT_B64 = 1,   // npp in 33..64
  KK_CNT_BIG = 2,   // npp > 128
  KK_CNT_FB = 3,    // generic fallback list length
  KK_CNT_FP64 = 4,  // FP32 targets re-solved in FP64
  KK_CNT_FAIL = 5,
  KK_CNT_CHOL = 6,
  KK_CNT_LDLT = 7,
  KK_CNT_WORK0 = 8,  // persistent-kernel work counters (8..15)
  KK_CNT_REDO = 16,  // search tie/overflow count per variable (16..19)
  KK_CNT_ITER = 20,  // total refinement iterations
  KK_CNT_JITTER = 21,  // LDL^T systems solved after the 1e-6 mean-diagonal jitter
  KK_CNT_B128 = 22,    // npp in 65..128
  KK_CNT_TUNE = 23,    // list length of a kernel-tuning sample
  KK_CNT_N = 32
};

// the counter that holds the length of neighbour-count list li (KK_LIST_*)
__host__ __device__ inline int list_slot(int li) { return li == KK_LIST_B128 ? (int)KK_CNT_B128 : li; }

void launch_search_coords(const KkSearch& S, const double* const* x, double* scu, int n, cudaStream_t st);
void launch_grid_build(const KkGrid& g, const double* scu, int* cell_of, int* count, int* start, int* cursor,
                       double* sc, int* sidx, int* sat, int n, cudaStream_t st);
void launch_search(const KkSearch& S, int ntarget, const double* const* tx, const double* const* ox, int* nbr,
                   int* nnear, int* status, int* redo_list, int* redo_count, int nsm, cudaStream_t st);
void launch_search_kdtree(const KkSearch& S, const int* list, const int* count, const double* const* tx,
                          const double* const* ox, int* nbr, int* nnear, int* status, void* heaps,
                          int heap_stride, int nthreads, cudaStream_t st);
size_t kd_heap_entry_bytes();
// Neighbour lists of a sequential simulation's targets (in visiting order)
// over the nobs observations followed by the targets; heaps: nthreads x
// heap_stride (>= nmax + 2) entries of kd_heap_entry_bytes().
void launch_search_sgsim(const KkSearch& S, int ntarget, int nobs, const double* const* tx, const double* const* ox,
                         int* nbr, int* nnear, void* heaps, int heap_stride, int nthreads, cudaStream_t st);
// One dependency level of a sequential simulation: for every target p of
// list[0, count) (visiting positions) and realisation s, the kriged value
// from the stored weights over the observations and the simulated targets,
// plus sqrt(max(var, 0)) * sample[p * nsim + s]; written to sim[s * nb + p]
// and to out[(path[p] - 1) * nsim + s].
struct SimParams {
  const int* nbr;       // (nb, mmax) neighbour lists, row order of the weights
  const int* nnear;     // (nb)
  const double* w;      // (nb, wstride) kriging weights
  const double* var;    // (nb) conditional variance
  const double* z;      // (nobs) observation values
  const double* sample; // (nb, nsim)
  const int* path;      // (nb) 1-based target of each visiting position
  double* sim;          // (nsim, nb) simulated values by visiting position
  double* out;          // (nb targets, nsim)
  int nb, nobs, nsim, mmax, wstride;
  int sk;               // simple kriging: the mean term on the observation weights
  double sk_mean, lo, hi;
};
void launch_sgsim_level(const SimParams& S, const int* list, int count, int nsm, cudaStream_t st);
// All levels in one cooperative launch (positions in level order; done, work
// and err zeroed); false when the device cannot take it.  *err turns 1 when a
// wait for a neighbour ran past its limit (the values are then NaN).
bool launch_sgsim_flow(const SimParams& S, const int* order, int count, int* done, int* work, int* err, int nsm,
                       cudaStream_t st);

void launch_bucket(const SolveParams& P, int* lists, cudaStream_t st);
// Estimates of every target from the weight store (P.wout, P.nbr, P.nnear)
// and the current observation values (weight-store reuse).
void launch_replay(const SolveParams& P, int nsm, cudaStream_t st);
// Indicator kriging: clip the first kcat estimates per target to [0, 1] and
// normalise them to sum to one.
void launch_indicator_post(double* est, int nb, int nvar, int kcat, int nsm, cudaStream_t st);
// Register-kernel solve of the targets list[item0 + i], i < nitems (or
// < *cnt - item0 when cnt is given): k_assemble writes each target's packed
// K64 to Kg + i * N (N + 1) / 2, then the factorisation kernel factors and
// solves; N is 32 or 64 (k_solve_warp, a warp per target) or 128
// (k_solve_block, a CTA per target, FP64 only); slot is the work counter,
// which must start at zero.
void launch_assemble(const SolveParams& P, int N, const int* list, const int* cnt, int item0, int nitems,
                     double* Kg, int nsm, cudaStream_t st);
void launch_factor(const SolveParams& P, int refine, int N, const int* list, const int* cnt, int item0, int nitems,
                   const double* Kg, int slot, int nsm, cudaStream_t st);
// 1 when the FP32 + refinement form applies (precision 1 and few enough columns)
int solve_refine_form(const SolveParams& P, int precision);
void launch_solve_generic(const SolveParams& P, const int* list, int list_cnt_slot, int nthreads, cudaStream_t st);
void set_zones(cudaStream_t st);


// Doubles of generic-kernel workspace per thread for systems of at most mtot
// equations (neighbours + drift/unbiasedness rows) with nv right-hand sides
// and pa drift/unbiasedness rows.
inline size_t generic_stride(int mtot, int nv, int pa) {
  return (size_t)mtot * mtot * 2 + (size_t)nv * mtot * 3 + (size_t)mtot * (pa + 2) + (size_t)(pa + 1) * (pa + 1) +
         (size_t)(pa + 1) * nv + (size_t)mtot + 64;
}

// Size of the fixed device array behind solve_generic_static (per device).
constexpr size_t KK_STATIC_SCRATCH_BYTES = (size_t)32 << 20;
constexpr int KK_STATIC_CHUNK = 1 << 16;  // targets per work-list chunk (two launches each)

// FP64 re-solve of every target through the generic kernel with workspace,
// work list and counters in the fixed static array instead of engine
// buffers; copies the counters of the run into cnt[KK_CNT_N] and
// synchronises st.  The caller has made `device` current.
void solve_generic_static(SolveParams P, int device, cudaStream_t st, int mtot, int* cnt);
// Throws the same error as solve_generic_static when one system of mtot
// equations does not fit in the static array (no device work).
void static_fit_check(int mtot, int nv, int pa);

}  // namespace kk
