// kk_solve.cu -- fused covariance assembly + factorisation + solve kernels.
//
// Per target the reference (kriging_base.F90:3159-3503, kriging.F90:714-1028,
// solver.f90:224-300) assembles K (covariances between neighbours, table
// lookup per pair), F (drift / unbiasedness rows) and the right-hand sides
// k (covariance to the target, averaged over block nodes) and g, factors K
// by Cholesky, forms the Schur complement S = F^T K^-1 F, and returns the
// estimate sum z_i w_i and the conditional variance.
//
// Kernels here:
//   k_bucket          npp per target -> size-bucket work lists
//   k_assemble, k_solve_warp (kk_warp.cuh)
//                     warp per target: covariance matrix, register Cholesky,
//                     right-hand sides forward-substituted in the same sweep;
//                     FP64, or FP32 factor with an FP64 residual correction
//   k_solve_block (kk_block.cuh)
//                     CTA per target for 65..128 equations: the same register
//                     layout over four warps, FP64
//   k_solve_generic   one thread per target in global workspace: Cholesky
//                     failures (Bunch-Kaufman LDL^T + jitter retry) and the
//                     allocation-free re-solve
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

#include "kk_solve_common.cuh"

namespace kk {

void set_zones(cudaStream_t st) {
  KkZones z;
  const double hb[4] = {0.0, 0.1, 0.5, 3.5};
  const double dh[3] = {1e-5, 1e-4, 1e-3};
  int o = 0;
  for (int k = 0; k < 3; ++k) {
    int n = (int)llround((hb[k + 1] - hb[k]) / dh[k]);
    if (n < 1) n = 1;
    z.zn[k] = n;
    z.off[k] = o;
    z.inv_dh[k] = (double)n / (hb[k + 1] - hb[k]);
    o += n;
  }
  for (int k = 0; k < 4; ++k) z.zb[k] = hb[k];
  // the fast paths' compile-time copy of these zones (load_zones)
  const ZoneRegs c = load_zones_host();
  if (z.zn[0] != c.n0 || z.zn[1] != c.n1 || z.zn[2] != c.n2 || z.off[1] != c.o1 || z.off[2] != c.o2 ||
      z.inv_dh[0] != c.i0 || z.inv_dh[1] != c.i1 || z.inv_dh[2] != c.i2 || z.zb[1] != c.zb1 || z.zb[2] != c.zb2 ||
      z.zb[3] != c.zb3)
    throw std::string("covariance table zones differ from the fast paths' constants");
  cudaMemcpyToSymbolAsync(c_zones, &z, sizeof z, 0, cudaMemcpyHostToDevice, st);
}

// ---------------------------------------------------------------------------
// bucketing
// ---------------------------------------------------------------------------
__global__ void k_bucket(SolveParams P, int* __restrict__ lists) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int slot = -1;  // no list: past the targets, or no system to solve
  if (t < P.nblock) {
    int npp = 0;
    for (int v = 0; v < P.nvar; ++v) npp += P.nnear[v][t];
    if (npp == 0 || npp == 1 || (P.nmin > 0 && npp < P.nmin)) {
      // zero neighbours (kriging_base.F90:3198-3207); npp == 1 reuses a stale
      // solution in the reference and is reported as NaN here
      write_nan(P, t);
      P.status[t] |= KK_ST_EMPTY;
      if (npp == 0 && !P.neglect_error) atomicAdd(&P.counters[KK_CNT_FAIL], 1);
    } else {
      slot = npp <= 32 ? KK_LIST_B32 : (npp <= 64 ? KK_LIST_B64 : (npp <= 128 ? KK_LIST_B128 : KK_LIST_BIG));
      if (slot == KK_LIST_BIG) P.status[t] |= KK_ST_BIG;
    }
  }
  // one atomic per warp and list (the order within a list is free: every
  // target is solved on its own)
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int li = 0; li < KK_NLIST; ++li) {
    const unsigned m = __ballot_sync(0xffffffffu, slot == li);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&P.counters[list_slot(li)], __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (slot == li) lists[(size_t)li * P.nblock + base + __popc(m & lt)] = t;
  }
}

void launch_bucket(const SolveParams& P, int* lists, cudaStream_t st) {
  k_bucket<<<(P.nblock + 255) / 256, 256, 0, st>>>(P, lists);
}

// ---------------------------------------------------------------------------
// weight-store reuse: estimates from stored weights and neighbours
// ---------------------------------------------------------------------------
// load_block_weights + estimate_block_base (kriging_base.F90:2780-2797,
// 3407-3503): est_j = sum_v sum_i z_v[inear_v(i)] w_ij, plus the Isaaks &
// Srivastava shift (std_ck off, several variables), the simple-kriging mean
// and the bounds.  HBM-bound gather-dot: a group of eight lanes per target,
// four targets per warp, each lane four neighbour rows per step with every
// load of the step issued before the first use (weights read contiguously,
// neighbour indices, then the values gathered from L2); group sums by three
// shuffles.  Targets without neighbours, or marked empty or failed by the
// solve that filled the store, give NaN.
__device__ __forceinline__ double group8_sum(double v) {
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  return v;
}

__global__ void __launch_bounds__(256) k_replay(const __grid_constant__ SolveParams P) {
  constexpr int G = 8, U = 4;  // lanes per target, rows per lane and step
  const int lane = threadIdx.x & 31, gl = lane & (G - 1);
  const int q = P.nvar;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  // warp-uniform loop over groups of four targets: every lane reaches every shuffle
  for (int tb = w0 * 4; tb < P.nblock; tb += nwarp * 4) {
    const int t = tb + (lane >> 3);
    const bool valid = t < P.nblock;
    int nn[KK_MAXVAR], ist[KK_MAXVAR], npp = 0;
#pragma unroll
    for (int v = 0; v < KK_MAXVAR; ++v) {
      nn[v] = (valid && v < q) ? __ldg(&P.nnear[v][t]) : 0;
      ist[v] = npp;
      npp += nn[v];
    }
    const bool nan_out = valid && (npp == 0 || (__ldg(&P.status[t]) & (KK_ST_EMPTY | KK_ST_FAIL)));
    if (nan_out) npp = 0;
    // variable loops unrolled to the maximum so nn / ist / tmean stay in registers
    double tmean[KK_MAXVAR] = {0.0, 0.0, 0.0, 0.0};
    if (P.ck_isa) {
#pragma unroll
      for (int v = 0; v < KK_MAXVAR; ++v) {
        if (v >= q) break;
        const int nv = nan_out ? 0 : nn[v];
        const int* nb = P.nbr[v] + (size_t)(valid ? t : 0) * P.mmax[v];
        double sz = 0.0;
        for (int i = gl; i < nv; i += G) sz += __ldg(&P.oval[v][__ldg(&nb[i])]);
        sz = group8_sum(sz);
        tmean[v] = nv > 0 ? sz / nv : 0.0;
      }
    }
#pragma unroll
    for (int jv = 0; jv < KK_MAXVAR; ++jv) {
      if (jv >= q) break;
      const double* w = P.wout + ((size_t)(valid ? t : 0) * q + jv) * P.wstride;
      double avg = 0.0, tws = 0.0;
#pragma unroll
      for (int v = 0; v < KK_MAXVAR; ++v) {
        if (v >= q) break;
        const int nv = nan_out ? 0 : nn[v];
        const int* nb = P.nbr[v] + (size_t)(valid ? t : 0) * P.mmax[v];
        const double* z = P.oval[v];
        double dot = 0.0, sw = 0.0;
        for (int i0 = 0; i0 < nv; i0 += G * U) {
          double wt[U];
          int o[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int i = i0 + u * G + gl;
            wt[u] = i < nv ? __ldg(&w[ist[v] + i]) : 0.0;
            o[u] = i < nv ? __ldg(&nb[i]) : -1;
          }
          double zv[U];
#pragma unroll
          for (int u = 0; u < U; ++u) zv[u] = o[u] >= 0 ? __ldg(&z[o[u]]) : 0.0;
#pragma unroll
          for (int u = 0; u < U; ++u) {
            dot = fma(zv[u], wt[u], dot);
            sw += wt[u];
          }
        }
        dot = group8_sum(dot);
        sw = group8_sum(sw);
        avg += dot;
        tws += sw;
        if (P.ck_isa && v != jv && nv > 0) avg += (tmean[jv] - tmean[v]) * sw;
      }
      if (P.unbias == 0 && P.sk_mean[jv] != 0.0) avg += (1.0 - tws) * P.sk_mean[jv];
      if (avg < P.bounds[0]) avg = P.bounds[0];
      if (avg > P.bounds[1]) avg = P.bounds[1];
      if (valid && gl == 0) P.est[(size_t)t * q + jv] = nan_out ? __longlong_as_double(0x7ff8000000000000ll) : avg;
    }
  }
}

// post_solve_indicator (kriging_indicator.F90:170-185): the first kcat
// estimates of every target (the category probabilities of indicator
// kriging) clipped to [0, 1] and scaled to sum to one when the sum is
// positive; NaN targets stay NaN.
__global__ void k_indicator_post(double* __restrict__ est, int nb, int nvar, int kcat) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += gridDim.x * blockDim.x) {
    double* v = est + (size_t)t * nvar;
    double sum = 0.0;
    for (int k = 0; k < kcat; ++k) {
      const double c = fmax(0.0, fmin(1.0, v[k]));
      v[k] = c;
      sum += c;
    }
    if (sum > 0.0)
      for (int k = 0; k < kcat; ++k) v[k] = v[k] / sum;
  }
}

void launch_indicator_post(double* est, int nb, int nvar, int kcat, int nsm, cudaStream_t st) {
  const int blocks = std::max(1, std::min((nb + 255) / 256, nsm * 8));
  k_indicator_post<<<blocks, 256, 0, st>>>(est, nb, nvar, kcat);
}

void launch_replay(const SolveParams& P, int nsm, cudaStream_t st) {
  const int need = (P.nblock + 31) / 32;  // eight warps of four targets per block
  const int blocks = std::max(1, std::min(need, nsm * 8));
  k_replay<<<blocks, 256, 0, st>>>(P);
}

}  // namespace kk

#include "kk_warp.cuh"
#include "kk_block.cuh"

namespace kk {

// ---------------------------------------------------------------------------
// generic path: one thread per target, reference algorithm in global memory
// ---------------------------------------------------------------------------
__device__ int potrf_u(int n, double* a, int lda) {
  for (int j = 0; j < n; ++j) {
    double ajj = a[j + j * lda];
    for (int k = 0; k < j; ++k) ajj = ajj - a[k + j * lda] * a[k + j * lda];
    if (!(ajj > 0.0)) { a[j + j * lda] = ajj; return j + 1; }
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

__device__ void potrs_u(int n, int nrhs, const double* a, int lda, double* b, int ldb) {
  for (int c = 0; c < nrhs; ++c) {
    double* x = b + (size_t)c * ldb;
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

// Bunch-Kaufman LDL^T ('U'), netlib LAPACK xSYTF2 algorithm (bundled in the
// reference as lapack.f SSYTRF/SSYTF2), column-major m x m.
__device__ int sytf2_u(int n, double* a, int lda, int* ipiv) {
#define A_(i, j) a[((i) - 1) + ((j) - 1) * (size_t)lda]
  const double alpha = (1.0 + sqrt(17.0)) / 8.0;
  int info = 0, k = n;
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
    if (fmax(absakk, colmax) == 0.0 || isnan(absakk)) {
      if (info == 0) info = k;
      kp = k;
    } else {
      if (absakk >= alpha * colmax) {
        kp = k;
      } else {
        double rowmax = 0.0;
        for (int j = imax + 1; j <= k; ++j) rowmax = fmax(rowmax, fabs(A_(imax, j)));
        for (int j = 1; j <= imax - 1; ++j) rowmax = fmax(rowmax, fabs(A_(j, imax)));
        if (absakk >= alpha * colmax * (colmax / rowmax)) kp = k;
        else if (fabs(A_(imax, imax)) >= alpha * rowmax) kp = imax;
        else { kp = imax; kstep = 2; }
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

__device__ void sytrs_u(int n, int nrhs, const double* a, int lda, const int* ipiv, double* b, int ldb) {
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

// one target, reference algorithm (solve_linear_system_base,
// kriging_base.F90:3244-3398) including the SSYTRF + jitter ladder
__global__ void k_solve_generic(SolveParams P, const int* __restrict__ list, const int* __restrict__ list_count) {
  const int n_items = *list_count;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  double* ws = P.scratch + (size_t)gt * P.scratch_stride;
  for (int item = gt; item < n_items; item += gridDim.x * blockDim.x) {
    const int t = list[item];
    const int q = P.nvar, pa = P.pa;
    int nn[KK_MAXVAR], ist[KK_MAXVAR], npp = 0;
    for (int v = 0; v < q; ++v) { nn[v] = P.nnear[v][t]; ist[v] = npp; npp += nn[v]; }
    const int m = npp + pa;
    const double rs = P.rs ? P.rs[t] : 1.0, ln = P.ln ? P.ln[t] : 0.0;
    double* A = ws;
    double* Bm = A + (size_t)m * m;          // (q, m)
    double* X = Bm + (size_t)q * m;          // (q, m)
    double* L = X + (size_t)q * m;           // (npp, npp)
    double* Y = L + (size_t)m * m;           // (npp, pa); L doubles as the m x m LDL^T factor
    double* S = Y + (size_t)npp * (pa > 0 ? pa : 1);
    double* Z = S + (size_t)(pa > 0 ? pa * pa : 1);  // (m, q)
    double* rsm = Z + (size_t)m * q;         // (pa, q)
    int* ipiv = (int*)(rsm + (size_t)(pa > 0 ? pa : 1) * q + 1);
    auto row_vo = [&](int r, int& v, int& o) {
      v = 0;
      while (v + 1 < q && r >= ist[v + 1]) ++v;
      o = P.nbr[v][(size_t)t * P.mmax[v] + (r - ist[v])];
    };
    auto xcoord = [&](int v, int o, double* x) { for (int d = 0; d < P.nlag; ++d) x[d] = P.ox[v][d][o]; };
    // RHS
    for (int iv = 0; iv < q; ++iv) {
      for (int r = 0; r < npp; ++r) {
        int v, o;
        row_vo(r, v, o);
        double xr[4];
        xcoord(v, o, xr);
        double tmp = 0.0;
        int k0 = P.gstart ? P.gstart[t] : 0, k1 = P.gstart ? P.gstart[t + 1] : 1;
        for (int k = k0; k < k1; ++k) {
          double node[4], lag[4];
          for (int d = 0; d < P.nlag; ++d) node[d] = P.gstart ? P.gx[d][k] : P.tx[d][t];
          make_lag(P, xr, node, rs, lag);
          tmp = dadd(tmp, dmul(cov_pair(P, v, iv, lag), P.gstart ? P.gw[k] : 1.0));
        }
        Bm[iv + (size_t)r * q] = tmp;
      }
      for (int a = 0; a < pa; ++a) Bm[iv + (size_t)(npp + a) * q] = g_entry(P, a, iv, t);
    }
    // LHS lower + mirror
    for (size_t e = 0; e < (size_t)m * m; ++e) A[e] = 0.0;
    for (int c = 0; c < npp; ++c) {
      int vc, oc;
      row_vo(c, vc, oc);
      double xc[4];
      xcoord(vc, oc, xc);
      A[c + (size_t)c * m] = dadd(dadd(cov0_pair(P, vc, vc), P.ovar[vc][oc]), ln);
      for (int r = c + 1; r < npp; ++r) {
        int vr, orr;
        row_vo(r, vr, orr);
        double xr[4], lag[4];
        xcoord(vr, orr, xr);
        make_lag(P, xc, xr, rs, lag);
        A[r + (size_t)c * m] = cov_pair(P, vr, vc, lag);
      }
      for (int a = 0; a < pa; ++a) A[(npp + a) + (size_t)c * m] = f_entry(P, a, vc, oc);
    }
    for (int ir = 0; ir < npp; ++ir)
      for (int ic = ir + 1; ic < m; ++ic) A[ir + (size_t)ic * m] = A[ic + (size_t)ir * m];
    // kriging_setup + kriging_solve_prepared (solver.f90:224-300)
    for (int j = 0; j < npp; ++j)
      for (int r = 0; r < npp; ++r) L[r + (size_t)j * npp] = A[r + (size_t)j * m];
    int info = potrf_u(npp, L, npp);
    if (info == 0 && pa > 0) {
      for (int j = 0; j < pa; ++j)
        for (int r = 0; r < npp; ++r) Y[r + (size_t)j * npp] = A[r + (size_t)(npp + j) * m];
      potrs_u(npp, pa, L, npp, Y, npp);
      for (int j = 0; j < pa; ++j)
        for (int r = 0; r < pa; ++r) {
          double s = 0.0;
          for (int k = 0; k < npp; ++k) s = s + A[k + (size_t)(npp + r) * m] * Y[k + (size_t)j * npp];
          S[r + (size_t)j * pa] = s;
        }
      info = potrf_u(pa, S, pa);
    }
    if (info == 0) {
      for (int c = 0; c < q; ++c)
        for (int k = 0; k < npp; ++k) Z[k + (size_t)c * npp] = Bm[c + (size_t)k * q];
      potrs_u(npp, q, L, npp, Z, npp);
      if (pa == 0) {
        for (int c = 0; c < q; ++c)
          for (int k = 0; k < npp; ++k) X[c + (size_t)k * q] = Z[k + (size_t)c * npp];
      } else {
        for (int c = 0; c < q; ++c)
          for (int a = 0; a < pa; ++a) {
            double s = 0.0;
            for (int k = 0; k < npp; ++k) s = s + Y[k + (size_t)a * npp] * Bm[c + (size_t)k * q];
            rsm[a + (size_t)c * pa] = s - Bm[c + (size_t)(npp + a) * q];
          }
        potrs_u(pa, q, S, pa, rsm, pa);
        for (int c = 0; c < q; ++c) {
          for (int k = 0; k < npp; ++k) {
            double s = 0.0;
            for (int a = 0; a < pa; ++a) s = s + Y[k + (size_t)a * npp] * rsm[a + (size_t)c * pa];
            X[c + (size_t)k * q] = Z[k + (size_t)c * npp] - s;
          }
          for (int a = 0; a < pa; ++a) X[c + (size_t)(npp + a) * q] = rsm[a + (size_t)c * pa];
        }
      }
      atomicAdd(&P.counters[KK_CNT_CHOL], 1);
    } else {
      // SSYTRF on the augmented system, jitter retry (kriging_base.F90:3289-3342)
      double* Af = L;  // reuse (needs m*m: workspace sized for it)
      for (size_t e = 0; e < (size_t)m * m; ++e) Af[e] = A[e];
      info = sytf2_u(m, Af, m, ipiv);
      if (info != 0 && npp > 0) {
        double dscale = 0.0;
        for (int ii = 0; ii < npp; ++ii) dscale = dscale + A[ii + (size_t)ii * m];
        if (dscale > 0.0) {
          dscale = 1.0e-6 * (dscale / (double)npp);
          for (int ii = 0; ii < npp; ++ii) A[ii + (size_t)ii * m] = A[ii + (size_t)ii * m] + dscale;
          for (size_t e = 0; e < (size_t)m * m; ++e) Af[e] = A[e];
          info = sytf2_u(m, Af, m, ipiv);
          if (info == 0) atomicAdd(&P.counters[KK_CNT_JITTER], 1);
        }
      }
      if (info == 0) {
        for (int c = 0; c < q; ++c)
          for (int k = 0; k < m; ++k) Z[k + (size_t)c * m] = Bm[c + (size_t)k * q];
        sytrs_u(m, q, Af, m, ipiv, Z, m);
        for (int c = 0; c < q; ++c)
          for (int k = 0; k < m; ++k) X[c + (size_t)k * q] = Z[k + (size_t)c * m];
        atomicAdd(&P.counters[KK_CNT_LDLT], 1);
      }
    }
    if (info != 0) {
      atomicAdd(&P.counters[KK_CNT_FAIL], 1);
      P.status[t] |= KK_ST_FAIL;
      write_nan(P, t);
      if (P.wout)  // the reference's failed system keeps NaN weights
        for (int c = 0; c < q; ++c)
          for (int k = 0; k < npp; ++k)
            P.wout[((size_t)t * q + c) * P.wstride + k] = __longlong_as_double(0x7ff8000000000000ll);
      continue;
    }
    if (P.wout)  // kriging weights of the neighbour rows (assign_weight_ctx)
      for (int c = 0; c < q; ++c)
        for (int k = 0; k < npp; ++k) P.wout[((size_t)t * q + c) * P.wstride + k] = X[c + (size_t)k * q];
    // calc_variance + estimate_block_base
    double* Vt = P.var + (size_t)t * q * q;
    for (int iv = 0; iv < q; ++iv)
      for (int jv = iv; jv < q; ++jv) {
        double s = 0.0;
        for (int k = 0; k < m; ++k) s = s + X[iv + (size_t)k * q] * Bm[jv + (size_t)k * q];
        double v = base_cov(P, t, iv, jv) - s;
        Vt[iv + jv * q] = v;
        Vt[jv + iv * q] = v;
      }
    for (int iv = 0; iv < q; ++iv) {
      if (Vt[iv + iv * q] < 0.0) Vt[iv + iv * q] = 0.0;
      for (int jv = iv + 1; jv < q; ++jv) {
        double o = Vt[jv + iv * q];
        if (o < 0.0) o = 0.0;
        Vt[jv + iv * q] = o;
        Vt[iv + jv * q] = o;
      }
    }
    double tmean[KK_MAXVAR];
    for (int v = 0; v < q; ++v) {
      double s = 0.0;
      for (int k = 0; k < nn[v]; ++k) s = s + P.oval[v][P.nbr[v][(size_t)t * P.mmax[v] + k]];
      tmean[v] = nn[v] > 0 ? s / nn[v] : 0.0;
    }
    for (int jv = 0; jv < q; ++jv) {
      double tw[KK_MAXVAR], avg = 0.0, tws = 0.0;
      for (int v = 0; v < q; ++v) {
        double sw = 0.0, dp = 0.0;
        for (int k = 0; k < nn[v]; ++k) {
          double wt = X[jv + (size_t)(ist[v] + k) * q];
          sw = sw + wt;
          dp = dp + P.oval[v][P.nbr[v][(size_t)t * P.mmax[v] + k]] * wt;
        }
        tw[v] = sw;
        tws += sw;
        avg = avg + dp;
        if (P.ck_isa && v != jv && nn[v] > 0) avg = avg + (tmean[jv] - tmean[v]) * tw[v];
      }
      if (P.unbias == 0 && P.sk_mean[jv] != 0.0) avg = avg + (1.0 - tws) * P.sk_mean[jv];
      if (avg < P.bounds[0]) avg = P.bounds[0];
      if (avg > P.bounds[1]) avg = P.bounds[1];
      P.est[(size_t)t * q + jv] = avg;
    }
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename T, int N, bool REFINE, int CB, bool WT = false>
static void launch_warp(const SolveParams& P, const int* list, const int* cnt, int item0, int nitems,
                        const double* Kg, int slot, int nsm, cudaStream_t st) {
  constexpr int WPC = warp_cta<T, N, REFINE>();
  const size_t smem = sizeof(WarpSmem<T, N, REFINE, CB, WT>) * WPC;
  // per instantiation and device: function attributes belong to a context
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr_set[dev]) {
    cudaFuncSetAttribute(k_solve_warp<T, N, REFINE, CB, WT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_solve_warp<T, N, REFINE, CB, WT>, 32 * WPC, smem);
  if (occ < 1) occ = 1;
  int blocks = nsm * occ;
  const int need = (nitems + WPC - 1) / WPC;
  if (need < blocks) blocks = need > 0 ? need : 1;
  k_solve_warp<T, N, REFINE, CB, WT><<<blocks, 32 * WPC, smem, st>>>(P, list, cnt, item0, nitems, Kg, slot);
}

template <int CB>
static void launch_block(const SolveParams& P, const int* list, const int* cnt, int item0, int nitems,
                         const double* Kg, int slot, int nsm, cudaStream_t st) {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_solve_block<CB>, 128, 0);
  if (occ < 1) occ = 1;
  int blocks = nsm * occ;
  if (nitems < blocks) blocks = nitems > 0 ? nitems : 1;
  k_solve_block<CB><<<blocks, 128, 0, st>>>(P, list, cnt, item0, nitems, Kg, slot);
}

int solve_refine_form(const SolveParams& P, int precision) {
  const int C = P.pa + P.nvar + 1 + ((P.ck_isa || P.sk_any) ? P.nvar : 0);
  return precision != 0 && C <= KK_REFINE_COLS;
}

void launch_assemble(const SolveParams& P, int N, const int* list, const int* cnt, int item0, int nitems,
                     double* Kg, int nsm, cudaStream_t st) {
  // the launch bound's residency: three CTAs of eight warps (six of four
  // for N = 128)
  const int wpc = N == 128 ? 4 : 8;
  int blocks = nsm * (N == 128 ? 6 : 3);
  const int need = (nitems + wpc - 1) / wpc;
  if (need < blocks) blocks = need > 0 ? need : 1;
  // the fast covariance variant is a template parameter (the general path
  // runs in the first instantiation with P.fast_model == 0)
  if (N == 128) {
    if (P.fast_model == 2) k_assemble<128, 2><<<blocks, 128, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else if (P.fast_model == 3) k_assemble<128, 3><<<blocks, 128, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else if (P.fast_model == 4) k_assemble<128, 4><<<blocks, 128, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else k_assemble<128, 1><<<blocks, 128, 0, st>>>(P, list, cnt, item0, nitems, Kg);
  } else if (N == 32) {
    if (P.fast_model == 2) k_assemble<32, 2><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else if (P.fast_model == 3) k_assemble<32, 3><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else if (P.fast_model == 4) k_assemble<32, 4><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else k_assemble<32, 1><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
  } else {
    if (P.fast_model == 2) k_assemble<64, 2><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else if (P.fast_model == 3) k_assemble<64, 3><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else if (P.fast_model == 4) k_assemble<64, 4><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
    else k_assemble<64, 1><<<blocks, 256, 0, st>>>(P, list, cnt, item0, nitems, Kg);
  }
}

void launch_factor(const SolveParams& P, int refine, int N, const int* list, const int* cnt, int item0, int nitems,
                   const double* Kg, int slot, int nsm, cudaStream_t st) {
  const int C = P.pa + P.nvar + 1 + ((P.ck_isa || P.sk_any) ? P.nvar : 0);
  const bool narrow = C <= 3;
  if (N == 128) {
    // CTA per target, FP64 (no weight-store form: those targets take the
    // general kernel)
    if (narrow) launch_block<3>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
    else launch_block<MAXC>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
  } else if (refine) {
    // the refinement's sweeps and residual cost in proportion to the columns
    // carried: 3 (one variable, ordinary or simple), 5 (drift or two-variable
    // cokriging), 6
    if (N == 32) {
      if (narrow) launch_warp<float, 32, true, 3>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else if (C <= 5) launch_warp<float, 32, true, 5>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else launch_warp<float, 32, true, KK_REFINE_COLS>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
    } else {
      if (narrow) launch_warp<float, 64, true, 3>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else if (C <= 5) launch_warp<float, 64, true, 5>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else launch_warp<float, 64, true, KK_REFINE_COLS>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
    }
  } else if (P.wout) {
    // FP64 form with the kriging weights of every target (weight store)
    if (N == 32) {
      if (narrow) launch_warp<double, 32, false, 3, true>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else launch_warp<double, 32, false, MAXC, true>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
    } else {
      if (narrow) launch_warp<double, 64, false, 3, true>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else launch_warp<double, 64, false, MAXC, true>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
    }
  } else {
    if (N == 32) {
      if (narrow) launch_warp<double, 32, false, 3>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else launch_warp<double, 32, false, MAXC>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
    } else {
      if (narrow) launch_warp<double, 64, false, 3>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
      else launch_warp<double, 64, false, MAXC>(P, list, cnt, item0, nitems, Kg, slot, nsm, st);
    }
  }
}

void launch_solve_generic(const SolveParams& P, const int* list, int list_cnt_slot, int nthreads, cudaStream_t st) {
  int blocks = (nthreads + 63) / 64;
  k_solve_generic<<<blocks, 64, 0, st>>>(P, list, P.counters + list_cnt_slot);
}

// ---------------------------------------------------------------------------
// allocation-free re-solve: the generic kernel on a fixed static array
// ---------------------------------------------------------------------------
// Some callers cannot let the library allocate device memory in the middle of
// a call.  A serving loop that keeps other streams busy would be stalled,
// because cudaMalloc and cudaFree may synchronise the whole device; a process
// whose HBM is already reserved by another allocator's pool would see the
// allocation fail, or force that pool to give back its cached blocks.  For
// those callers krige_resolve_static runs k_solve_generic with its workspace,
// its work list and its counters in this one array, sized once when the
// module is loaded.  The array exists once per device and per process, so
// calls on one device must not overlap in time: solve_generic_static holds a
// process-wide lock until the call's work on the device has finished.
constexpr size_t KK_STATIC_HEADER = 256;      // counters (KK_CNT_N ints), then the list count
constexpr size_t KK_STATIC_LIST_BYTES = sizeof(int) * KK_STATIC_CHUNK;
static __device__ __align__(256) unsigned char g_static_scratch[KK_STATIC_SCRATCH_BYTES];

static std::mutex g_static_mu;
static void* g_static_addr[64];

// Work list of the targets t0 <= t < t1 that have a solvable neighbour set;
// the others get NaN exactly as in k_bucket.  Status bits of the previous
// solve are cleared except those the search set.
__global__ void k_static_list(SolveParams P, int t0, int t1, int* __restrict__ list, int* __restrict__ count) {
  const int t = t0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= t1) return;
  int npp = 0;
  for (int v = 0; v < P.nvar; ++v) npp += P.nnear[v][t];
  P.status[t] &= (KK_ST_TIE | KK_ST_OVERFLOW);
  if (npp == 0 || npp == 1 || (P.nmin > 0 && npp < P.nmin)) {
    write_nan(P, t);
    P.status[t] |= KK_ST_EMPTY;
    if (npp == 0 && !P.neglect_error) atomicAdd(&P.counters[KK_CNT_FAIL], 1);
    return;
  }
  list[atomicAdd(count, 1)] = t;
}

static void static_check(cudaError_t err, const char* what) {
  if (err != cudaSuccess) throw std::string("CUDA error ") + cudaGetErrorString(err) + " at " + what;
}

// Workspace slots of the static array for systems of at most mtot equations;
// throws when not even one target fits.
static size_t static_slots(int mtot, int nv, int pa) {
  const size_t ws_bytes = KK_STATIC_SCRATCH_BYTES - KK_STATIC_HEADER - KK_STATIC_LIST_BYTES;
  const size_t stride = generic_stride(mtot, nv, pa);
  const size_t slots = ws_bytes / (stride * sizeof(double));
  if (slots < 1) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "krige_resolve_static: one target needs %zu bytes of workspace (%d equations), more than the %zu "
             "bytes of static scratch; use krige_solve",
             stride * sizeof(double), mtot, ws_bytes);
    throw std::string(msg);
  }
  return slots;
}

void static_fit_check(int mtot, int nv, int pa) { static_slots(mtot, nv, pa); }

void solve_generic_static(SolveParams P, int device, cudaStream_t st, int mtot, int* cnt) {
  const size_t slots = static_slots(mtot, P.nvar, P.pa);
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (device < 0 || device >= 64) throw std::string("device ordinal out of range for the static scratch");
  if (!g_static_addr[device]) {
    // Set-up, once per device with that device current: the address of this
    // device's copy of the array.  It may load the module, so the first call
    // on a device belongs before any stream capture on it.
    void* addr = nullptr;
    static_check(cudaGetSymbolAddress(&addr, g_static_scratch), "cudaGetSymbolAddress(g_static_scratch)");
    g_static_addr[device] = addr;
  }
  unsigned char* base = static_cast<unsigned char*>(g_static_addr[device]);
  const size_t stride = generic_stride(mtot, P.nvar, P.pa);
  int* counters = reinterpret_cast<int*>(base);
  int* list_count = counters + KK_CNT_N;
  int* list = reinterpret_cast<int*>(base + KK_STATIC_HEADER);
  P.counters = counters;
  P.fb_list = nullptr;
  P.fp64_list = nullptr;
  P.scratch = reinterpret_cast<double*>(base + KK_STATIC_HEADER + KK_STATIC_LIST_BYTES);
  P.scratch_stride = (int)stride;
  // thread g of the generic kernel owns workspace slot g: never more threads than slots
  const int threads = (int)std::min<size_t>(slots, (size_t)KK_STATIC_CHUNK);
  const int bs = std::min(64, threads);
  const int blocks = threads / bs;
  // the counters and the list count start at zero
  static_check(cudaMemsetAsync(base, 0, KK_STATIC_HEADER, st), "cudaMemsetAsync(static header)");
  for (int t0 = 0; t0 < P.nblock; t0 += KK_STATIC_CHUNK) {
    const int t1 = std::min(P.nblock, t0 + KK_STATIC_CHUNK);
    static_check(cudaMemsetAsync(list_count, 0, sizeof(int), st), "cudaMemsetAsync(static list count)");
    k_static_list<<<(t1 - t0 + 255) / 256, 256, 0, st>>>(P, t0, t1, list, list_count);
    k_solve_generic<<<blocks, bs, 0, st>>>(P, list, list_count);
    static_check(cudaGetLastError(), "k_solve_generic (static scratch)");
  }
  static_check(cudaMemcpyAsync(cnt, counters, sizeof(int) * KK_CNT_N, cudaMemcpyDeviceToHost, st),
               "cudaMemcpyAsync(static counters)");
  static_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

}  // namespace kk
