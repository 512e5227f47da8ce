// kk_warp.cuh -- warp-per-target kriging solve (included by kk_solve.cu).
//
// One warp owns one target system at a time and pulls the next target from
// a device work counter, so the solve needs no block-wide barrier at all.
//
// Register layout of the N x N covariance matrix K (N = 32 or 64): the warp
// is a 4 x 8 grid of lanes, pr = lane & 3 (row class), pc = lane >> 2
// (column class).  Lane (pr, pc) owns entry (r, c) = (4 ri + pr, 8 ci + pc)
// in register slot a[ri][ci]; only slots with ri >= 2 ci can hold lower-
// triangle entries, so a lane keeps 72 slots for N = 64 (20 for N = 32) and
// the trailing update of every Cholesky column is spread evenly over the
// 32 lanes.  Right-hand-side rows are owned one per (lane, m):
// r = 32 m + 4 pc + pr.
//
// Per target:
//   1. gather the neighbour rows (ascending index per variable block, as
//      assemble_linear_system_base, kriging_base.F90:3159-3235);
//   2. every lane evaluates its own K entries (assemble_lhs, kriging.F90:
//      714-849) and its right-hand-side rows F | k | u (assemble_rhs,
//      kriging.F90:864-939) -- no shared-memory round trip;
//   3. right-looking Cholesky, one __syncwarp per column: the lanes of
//      column class j % 8 publish column j of L to shared memory, every lane
//      applies the rank-1 update to its slots and forward-substitutes its
//      right-hand-side rows in the same sweep;
//   4. FP64: the outputs are inner products of forward-substituted columns
//      (S = F^T K^-1 F, lambda, variance, estimate); FP32 + refinement: the
//      FP32 factor is kept packed in shared memory, the solution of
//      K [W] = [F k] is refined with FP64 residuals against K64 (also kept in
//      shared memory) until the estimated error is below refine_tol; then
//      the same inner products are taken against the refined W.
#pragma once

namespace kk {

template <typename T, int N, bool REFINE, int CB, bool WT = false>
struct __align__(16) WarpSmem {
  double x[4][N];          // neighbour coordinates (nlag)
  double z[N];             // neighbour values
  int obs[N];
  int var[N];
  T col[2][4 * (N / 4 + (sizeof(T) == 8 ? 2 : 4))];  // column j of L, layout [pr][ri], padded rows
  double ybc[2][CB];       // forward-substituted right-hand sides of row j
  double G[CB * CB];
  double zmean[2 * KK_MAXVAR];
  float L[REFINE ? N * (N - 1) / 2 : 1];   // FP32 factor, strictly lower, packed by column
  float invd[REFINE ? N : 1];              // 1 / L[j][j]
  double W[REFINE ? CB * N : 1];           // current solution, broadcast for the residual
  // weight store (WT): strictly lower L packed by column after one leading
  // zero entry (L[r][j] at lcol(j) - j + r), 1 / L[j][j], Lagrange multipliers
  double Lw[WT ? N * (N - 1) / 2 + 2 : 1];
  double invw[WT ? N : 1];
  double lam[WT ? KK_MAXVAR * 6 : 1];
};

// Triangular sweeps of the refinement form over a lane's right-hand-side
// rows r = 32 m + 4 pc + pr, with L (strictly lower, packed by column) and
// 1 / L[j][j] in shared memory; the pivot row's values are broadcast by
// shuffle from the lane that owns that row.
template <typename T, int N, int RM, int CB>
__device__ __forceinline__ void sweep_back(T (&v)[RM][CB], const float* __restrict__ L, const float* __restrict__ invd,
                                           int n, int C, int lane) {  // v <- L^-T v
  const int pr = lane & 3, pc = lane >> 2;
  for (int j = n - 1; j >= 0; --j) {
    const int owner = ((j >> 2) & 7) * 4 + (j & 3);
    const T ij = (T)invd[j];
    T xj[CB];
#pragma unroll
    for (int k = 0; k < CB; ++k) {
      T mine = v[0][k];
      if (RM > 1 && (j >> 5) == 1) mine = v[RM - 1][k];
      xj[k] = __shfl_sync(0xffffffffu, mine, owner) * ij;
    }
#pragma unroll
    for (int m = 0; m < RM; ++m) {
      const int r = 32 * m + 4 * pc + pr;
      const T l = r < j ? (T)L[lcol<N>(r) + (j - r - 1)] : T(0);
#pragma unroll
      for (int k = 0; k < CB; ++k) {
        if (k < C) v[m][k] = (r == j) ? xj[k] : v[m][k] - l * xj[k];
      }
    }
  }
}

template <typename T, int N, int RM, int CB>
__device__ __forceinline__ void sweep_fwd(T (&v)[RM][CB], const float* __restrict__ L, const float* __restrict__ invd,
                                          int n, int C, int lane) {  // v <- L^-1 v
  const int pr = lane & 3, pc = lane >> 2;
  for (int j = 0; j < n; ++j) {
    const int owner = ((j >> 2) & 7) * 4 + (j & 3);
    const T ij = (T)invd[j];
    T yj[CB];
#pragma unroll
    for (int k = 0; k < CB; ++k) {
      T mine = v[0][k];
      if (RM > 1 && (j >> 5) == 1) mine = v[RM - 1][k];
      yj[k] = __shfl_sync(0xffffffffu, mine, owner) * ij;
    }
#pragma unroll
    for (int m = 0; m < RM; ++m) {
      const int r = 32 * m + 4 * pc + pr;
      const T l = (r > j && r < n) ? (T)L[lcol<N>(j) + (r - j - 1)] : T(0);
#pragma unroll
      for (int k = 0; k < CB; ++k) {
        if (k < C) v[m][k] = (r == j) ? yj[k] : v[m][k] - l * yj[k];
      }
    }
  }
}

// Covariance matrix K (assemble_lhs, kriging.F90:714-849; lag = x_c - x_r,
// diagonal cov0 + observation variance + local nugget) of the targets
// list[item0 + i], i < count, written packed row-major lower to
// Kg + i * N (N + 1) / 2.  One warp per target; the packed entries are
// spread evenly over the lanes (stores are contiguous across the warp).
// Eight warps per CTA (four for N = 128, to stay within 48 KB of static
// shared memory).
// This is the part of the solve that is bound by covariance-table latency,
// so it runs as its own kernel with many resident warps; the factorisation
// kernel then reads K from this buffer.  On the fast covariance paths an
// entry follows the reference's table lookup (zones, index, linear
// interpolation) at the distance |u_c - u_r| of target-centred transformed
// coordinates, with its square root from an FP32 seed and one FP64 Newton
// step: a few ulp from the reference's arithmetic, which moves the solution
// by about the condition number times 1e-15.
template <int N, int FM>
__global__ void __launch_bounds__(256, 3) k_assemble(const __grid_constant__ SolveParams P,
                                                     const int* __restrict__ list,
                                                     const int* __restrict__ list_count, int item0, int nitems,
                                                     double* __restrict__ Kg) {
  constexpr int NK = N * (N + 1) / 2;
  struct Rows {
    double x[4][N];
    double u[3][N];  // target-centred transformed coordinates (fast paths)
    int obs[N];
    int var[N];
  };
  __shared__ Rows rows[N == 128 ? 4 : 8];
  __shared__ PairModel s_pm[4];  // two-variable fast path (FM 3), dynamic pair index
  if (FM == 3 && threadIdx.x < 4) {
    PairModel& m = s_pm[threadIdx.x];
    m.kind = P.fq_kind[threadIdx.x];
    m.nst = P.fq_nst[threadIdx.x];
    m.tail = P.fq_tail[threadIdx.x];
    for (int q2 = 0; q2 < KK_FA_MAXS; ++q2) {
      m.off[q2] = P.fq_off[threadIdx.x][q2];
      m.k[q2] = P.fq_k[threadIdx.x][q2];
    }
  }
  __syncthreads();
  Rows& s = rows[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  int count = nitems;
  if (list_count) count = min(nitems, *list_count - item0);
  const bool fast = P.fast_model != 0;
  const int fd = P.fm_ndim;                       // transformed dimensions
  const int nsp = FM == 4 ? P.nlag - 1 : P.nlag;  // spatial coordinates
  const ZoneRegs zr = load_zones();
  const int nwarp = gridDim.x * (blockDim.x >> 5);
  for (int it = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < count; it += nwarp) {
    const int t = __ldg(&list[item0 + it]);
    int ist1, ist2, ist3;
    const int n = gather_rows<N>(P, t, lane, s.x, nullptr, s.obs, s.var, ist1, ist2, ist3);
    const double rs = P.rs ? __ldg(&P.rs[t]) : 1.0;
    const double ln = P.ln ? __ldg(&P.ln[t]) : 0.0;
    const bool scale_lag = !P.st && rs != 1.0;  // warp-uniform
    if (fast) {
      // u = M (x - x_t) / rangescale: the anisotropic distance of a pair is
      // |u_c - u_r|, one transform per neighbour instead of one per pair
      double xt[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < nsp) xt[d] = __ldg(&P.tx[d][t]);
      for (int r = lane; r < n; r += 32) {
        double l[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          if (d < nsp) {
            l[d] = s.x[d][r] - xt[d];
            if (scale_lag) l[d] = l[d] / rs;
          }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (d < fd) s.u[d][r] = fma(P.fm[d], l[0], fma(P.fm[3 + d], l[1], P.fm[6 + d] * l[2]));
      }
      __syncwarp();
    }
    double* K = Kg + (size_t)it * NK;
    const int E = n * (n + 1) / 2;
    int r = 0, c = lane;
    while (c > r) { c -= r + 1; ++r; }
    for (int e = lane; e < E; e += 32) {
      const int vr = s.var[r];
      double kv;
      if (c == r) {
        kv = dadd(dadd(cov0_pair(P, vr, vr), __ldg(&P.ovar[vr][s.obs[r]])), ln);
      } else if (fast) {
        const double d0 = s.u[0][c] - s.u[0][r];
        double h2 = d0 * d0;
        if (fd > 1) {
          const double d1 = s.u[1][c] - s.u[1][r];
          h2 = fma(d1, d1, h2);
        }
        if (fd > 2) {
          const double d2 = s.u[2][c] - s.u[2][r];
          h2 = fma(d2, d2, h2);
        }
        const double hh = fd == 1 ? fabs(d0) : sqrt_newton(h2);
        kv = FM == 4 ? cov_st_h(P, zr, hh, s.x[nsp][c] - s.x[nsp][r])
                     : cov_h<FM == 4 ? 1 : FM>(P, zr, hh, s_pm, FM == 3 ? vr * 2 + s.var[c] : 0);
        if (kv != kv) {  // a table argument at a zone edge: the reference's arithmetic
          double lag[4];
#pragma unroll
          for (int d = 0; d < 4; ++d) lag[d] = d < P.nlag ? dsub(s.x[d][c], s.x[d][r]) : 0.0;
          if (scale_lag) {
#pragma unroll
            for (int d = 0; d < 4; ++d) lag[d] = lag[d] / rs;
          }
          kv = cov_pair_call(P, vr, s.var[c], lag[0], lag[1], lag[2], lag[3]);
        }
      } else {
        double lag[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) lag[d] = d < P.nlag ? dsub(s.x[d][c], s.x[d][r]) : 0.0;
        if (scale_lag) {  // lag / rangescale (kriging.F90:783), only when a target sets it
#pragma unroll
          for (int d = 0; d < 4; ++d) lag[d] = lag[d] / rs;
        }
        kv = cov_pair_call(P, vr, s.var[c], lag[0], lag[1], lag[2], lag[3]);
      }
      K[e] = kv;
      c += 32;
      while (c > r) { c -= r + 1; ++r; }
    }
    __syncwarp();
  }
}

// warps per CTA of the factorisation kernel
template <typename T, int N, bool REFINE>
constexpr int warp_cta() { return 4; }

// CTAs per SM the register budget is sized for (the launch bound caps the
// registers at 64 K / (threads * this)): the FP64 N = 64 form needs the whole
// register file of a lane for the matrix; the FP32 one with three
// right-hand-side columns fits in 128 registers and 55 KB of shared memory
// per CTA (four CTAs per SM), the wider ones in 168 (three); the N = 32 forms
// in 128
template <typename T, int N, bool REFINE, int CB>
constexpr int warp_min_ctas() { return N == 64 ? (REFINE ? (CB == 3 ? 4 : 3) : 1) : 4; }

// CB: right-hand-side columns held per row at compile time (F | k | u);
// 3 covers ordinary and simple kriging of one variable, the wider forms
// cover drift and cokriging.
// WT (FP64 form only): also the kriging weights of every target, for the
// weight store (P.wout)
template <typename T, int N, bool REFINE, int CB, bool WT = false>
__global__ void __launch_bounds__(32 * warp_cta<T, N, REFINE>(), warp_min_ctas<T, N, REFINE, CB>())
    k_solve_warp(const __grid_constant__ SolveParams P, const int* __restrict__ list,
                 const int* __restrict__ list_count, int item0, int nitems, const double* __restrict__ Kg,
                 int work_slot) {
  static_assert(!(WT && REFINE), "the weight store is filled by the FP64 form");
  using WS = WarpSmem<T, N, REFINE, CB, WT>;
  constexpr int RI = N / 4, CI = N / 8, RM = N / 32;
  // column-buffer row stride: padded so the four row classes fall in
  // different banks and stay 16-byte aligned
  constexpr int RIP = RI + (sizeof(T) == 8 ? 2 : 4);
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WS& s = reinterpret_cast<WS*>(smem_raw)[threadIdx.x >> 5];
  constexpr int NK = N * (N + 1) / 2;  // packed K64 of one target in Kg (from k_assemble)
  const bool fast = P.fast_model == 1 || P.fast_model == 2;  // right-hand side: one variable only
  const int lane = threadIdx.x & 31;
  const int pr = lane & 3, pc = lane >> 2;
  int n_items = nitems;
  if (list_count) n_items = min(nitems, *list_count - item0);
  const int q = P.nvar, pa = P.pa;
  const int nu = n_func(P);
  const int C = pa + q + nu;  // forward-substituted columns (FP64 form)
  const ZoneRegs zr = load_zones();


  int n_chol = 0, n_iter = 0;
  if constexpr (WT) {
    if (lane == 0) s.Lw[0] = 0.0;
  }
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(&P.counters[work_slot], 1);
    item = __shfl_sync(FULL, item, 0);
    if (item >= n_items) break;
    const int t = __ldg(&list[item0 + item]);
    const double* Ks = Kg + (size_t)item * NK;

    // ---- neighbour rows: variable blocks in order, ascending index
    int ist1, ist2, ist3;
    const int n = gather_rows<N>(P, t, lane, s.x, s.z, s.obs, s.var, ist1, ist2, ist3);
    const double rs = P.rs ? __ldg(&P.rs[t]) : 1.0;
    const bool scale_lag = !P.st && rs != 1.0;  // warp-uniform
    const int nri = (n + 3) >> 2, nci = (n + 7) >> 3;

    // ---- right-hand-side rows r = 32 m + 4 pc + pr: F (pa), k (q), u (nu)
    T b[RM][CB];
    double b64[REFINE ? RM : 1][REFINE ? CB : 1];
#pragma unroll
    for (int m = 0; m < RM; ++m) {
      const int r = 32 * m + 4 * pc + pr;
#pragma unroll
      for (int k = 0; k < CB; ++k) b[m][k] = T(0);
      if constexpr (REFINE) {
#pragma unroll
        for (int k = 0; k < CB; ++k) b64[m][k] = 0.0;
      }
      if (r < n) {
        const int vr = s.var[r], orr = s.obs[r];
        double xr[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < 4; ++d)
          if (d < P.nlag) xr[d] = s.x[d][r];
#pragma unroll
        for (int k = 0; k < CB; ++k) {
          if (k >= C) break;
          double v;
          if (k < pa) {
            v = f_entry(P, k, vr, orr);
          } else if (k < pa + q) {
            const int iv = k - pa;
            if (fast && !P.gstart) {
              double lag[4];
#pragma unroll
              for (int d = 0; d < 4; ++d) lag[d] = dsub(xr[d], d < P.nlag ? __ldg(&P.tx[d][t]) : 0.0);
              if (scale_lag) {
#pragma unroll
                for (int d = 0; d < 4; ++d) lag[d] = lag[d] / rs;
              }
              v = dadd(0.0, dmul(fast_cov<0>(P, zr, lag), 1.0));
              if (v != v) v = rhs_cov_row(P, t, xr, vr, iv, rs);  // a table argument at a zone edge
            } else {
              v = rhs_cov_row(P, t, xr, vr, iv, rs);
            }
          } else {
            const int u = k - pa - q;
            v = u == 0 ? s.z[r] : (vr == u - 1 ? 1.0 : 0.0);
          }
          b[m][k] = (T)v;
          if constexpr (REFINE) b64[m][k] = v;
        }
      }
    }
    // ---- K from the assembly kernel (packed row-major lower, FP64)
    T a[RI][CI];
#pragma unroll
    for (int ri = 0; ri < RI; ++ri) {
      const int r = 4 * ri + pr;
#pragma unroll
      for (int ci = 0; ci < CI; ++ci) {
        if (ri >= 2 * ci) {
          const int c = 8 * ci + pc;
          a[ri][ci] = (ri < nri && r < n && c <= r) ? (T)__ldg(&Ks[r * (r + 1) / 2 + c]) : T(0);
        }
      }
    }
    if (P.ck_isa && lane == 0) {
      for (int v = 0; v < q; ++v) {
        const int i0 = v == 0 ? 0 : (v == 1 ? ist1 : (v == 2 ? ist2 : ist3));
        const int i1 = v + 1 >= q ? n : (v == 0 ? ist1 : (v == 1 ? ist2 : ist3));
        double sz = 0.0;
        for (int k = i0; k < i1; ++k) sz = dadd(sz, s.z[k]);
        s.zmean[v] = i1 > i0 ? sz / (i1 - i0) : 0.0;
        s.zmean[KK_MAXVAR + v] = (double)(i1 - i0);
      }
    }

    // ---- right-looking Cholesky + forward substitution of b
    bool fail = false;
#pragma unroll
    for (int jb = 0; jb < CI; ++jb) {
      if (jb >= nci) break;
      const int jm = (8 * jb) >> 5;  // right-hand-side slot of rows 8 jb .. 8 jb + 7
#pragma unroll 1
      for (int jj = 0; jj < 8; ++jj) {
        const int j = 8 * jb + jj;
        if (j >= n) break;
        T* cw = s.col[j & 1];
        const T dsel = (jj < 4) ? a[2 * jb][jb] : a[2 * jb + 1][jb];
        const T d = __shfl_sync(FULL, dsel, jj * 4 + (jj & 3));
        if (!(d > T(0))) { fail = true; break; }
        const T inv = rsqrt_t(d);
        if constexpr (REFINE) {
          if (lane == 0) s.invd[j] = (float)inv;
        }
        if constexpr (WT) {
          if (lane == 0) s.invw[j] = (double)inv;
        }
        if (pc == jj) {
#pragma unroll
          for (int ri = 2 * jb; ri < RI; ++ri) {
            const int r = 4 * ri + pr;
            const T l = (r > j) ? a[ri][jb] * inv : T(0);
            if (REFINE) a[ri][jb] = l;
            cw[pr * RIP + ri] = l;
            if constexpr (WT) {
              if (r > j) s.Lw[lcol<N>(j) - j + r] = (double)l;
            }
          }
        }
        const int owner = ((j >> 2) & 7) * 4 + (j & 3);
        if (lane == owner) {
#pragma unroll
          for (int k = 0; k < CB; ++k) {
            if (k < C) {
              const T yv = b[jm][k] * inv;
              b[jm][k] = yv;
              s.ybc[j & 1][k] = (double)yv;
            }
          }
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < RM; ++m) {
          if (m < jm) continue;  // rows below 32 jm are finished
          // L[r][j] for this lane's row r; the buffer holds column j only
          // from row 8 jb on, and finished rows take no update
          const T lb = (32 * m + 4 * pc + pr > j) ? cw[pr * RIP + 8 * m + pc] : T(0);
#pragma unroll
          for (int k = 0; k < CB; ++k)
            if (k < C) b[m][k] -= lb * (T)s.ybc[j & 1][k];
        }
        T lc[CI], lr[RI];
#pragma unroll
        for (int ci = jb; ci < CI; ++ci) lc[ci] = cw[(pc & 3) * RIP + 2 * ci + (pc >> 2)];
#pragma unroll
        for (int ri = 2 * jb; ri < RI; ++ri) lr[ri] = cw[pr * RIP + ri];
        // rows past n are zero: skip whole groups of four row slots
#pragma unroll
        for (int ci = jb; ci < CI; ++ci) {
          if (ci >= nci) break;
#pragma unroll
          for (int ri = 2 * ci; ri < RI; ++ri) {
            if ((ri & 3) == 0 && ri >= nri) break;
            a[ri][ci] -= lr[ri] * lc[ci];
          }
        }
      }
      if (fail) break;
    }
    if (fail) {
      // Cholesky failed: FP32 -> FP64 register kernel; FP64 -> generic LDL^T path
      if (lane == 0) {
        if (REFINE) {
          P.status[t] |= KK_ST_FP64;
          const int p = atomicAdd(&P.counters[KK_CNT_FP64], 1);
          P.fp64_list[p] = t;
        } else {
          P.status[t] |= KK_ST_LDLT;
          const int p = atomicAdd(&P.counters[KK_CNT_FB], 1);
          P.fb_list[p] = t;
        }
      }
      __syncwarp();
      continue;
    }

    if constexpr (!REFINE) {
      // ---- G = Y^T Y over the forward-substituted columns
#pragma unroll
      for (int ka = 0; ka < CB; ++ka) {
        if (ka >= C) break;
#pragma unroll
        for (int kb = ka; kb < CB; ++kb) {
          if (kb >= C) break;
          double g = 0.0;
#pragma unroll
          for (int m = 0; m < RM; ++m) g = fma((double)b[m][ka], (double)b[m][kb], g);
          g = warp_sum(g);
          if (lane == 0) {
            s.G[ka * C + kb] = g;
            s.G[kb * C + ka] = g;
          }
        }
      }
    } else {
      // ---- keep L (FP32, strictly lower, packed by column) for the sweeps
#pragma unroll
      for (int ri = 0; ri < RI; ++ri) {
        if (ri >= nri) break;
        const int r = 4 * ri + pr;
#pragma unroll
        for (int ci = 0; ci < CI; ++ci) {
          if (ri >= 2 * ci) {
            const int c = 8 * ci + pc;
            if (r > c && r < n) s.L[lcol<N>(c) + (r - c - 1)] = (float)a[ri][ci];
          }
        }
      }
      __syncwarp();
      const float* Lp = s.L;
      const float* id = s.invd;
      // x = (L L^T)^-1 [F k u]: b holds L^-1 [F k u] from the factor sweep
      sweep_back<T, N, RM, CB>(b, Lp, id, n, C, lane);
#pragma unroll
      for (int m = 0; m < RM; ++m) {
        const int r = 32 * m + 4 * pc + pr;
        if (r < n) {
#pragma unroll
          for (int k = 0; k < CB; ++k)
            if (k < C) s.W[k * N + r] = (double)b[m][k];
        }
      }
      __syncwarp();
      // K64 x (FP64) for this lane's rows, and the residuals r = col - K64 x
      double kx[RM][CB];
      T res[RM][CB];
#pragma unroll
      for (int m = 0; m < RM; ++m) {
        const int r = 32 * m + 4 * pc + pr;
#pragma unroll
        for (int k = 0; k < CB; ++k) kx[m][k] = 0.0;
        if (r < n) {
          const int rowoff = r * (r + 1) / 2;
          for (int c = 0; c < n; ++c) {
            const double kv = c <= r ? __ldg(&Ks[rowoff + c]) : __ldg(&Ks[c * (c + 1) / 2 + r]);
#pragma unroll
            for (int k = 0; k < CB; ++k)
              if (k < C) kx[m][k] = fma(kv, s.W[k * N + c], kx[m][k]);
          }
        }
#pragma unroll
        for (int k = 0; k < CB; ++k) res[m][k] = (r < n && k < C) ? (T)(b64[m][k] - kx[m][k]) : T(0);
      }
      sweep_fwd<T, N, RM, CB>(res, Lp, id, n, C, lane);
      // a^T K^-1 b = x_a^T b + x_b^T a - x_a^T K x_b + r_a^T K^-1 r_b exactly;
      // the last term, taken with the FP32 factor, leaves an error of third
      // order in the FP32 solution error
      bool ok = true;
#pragma unroll
      for (int ka = 0; ka < CB; ++ka) {
        if (ka >= C) break;
#pragma unroll
        for (int kb = ka; kb < CB; ++kb) {
          if (kb >= C) break;
          double g = 0.0, cr = 0.0;
#pragma unroll
          for (int m = 0; m < RM; ++m) {
            const double xa = (double)b[m][ka], xb = (double)b[m][kb];
            g = fma(xa, b64[m][kb], g);
            g = fma(xb, b64[m][ka], g);
            g = fma(-xa, kx[m][kb], g);
            cr = fma((double)res[m][ka], (double)res[m][kb], cr);
          }
          g = warp_sum(g);
          cr = warp_sum(cr);
          g += cr;
          // the correction is about (cond * eps32)^2 of the value and its own
          // error one order higher: refine_tol_corr keeps that below refine_tol
          if (ka == kb && !(cr <= P.refine_tol_corr * fabs(g))) ok = false;
          if (lane == 0) {
            s.G[ka * C + kb] = g;
            s.G[kb * C + ka] = g;
          }
        }
      }
      ++n_iter;
      if (!ok) {
        if (lane == 0) {
          P.status[t] |= KK_ST_FP64;
          const int p = atomicAdd(&P.counters[KK_CNT_FP64], 1);
          P.fp64_list[p] = t;
        }
        __syncwarp();
        continue;
      }
    }
    __syncwarp();
    int f = 0;
    if (lane == 0) {
      // the FP64 forms finish ordinary kriging in registers; the refinement
      // form keeps the out-of-line routine (its 128-register budget is full)
      if (!REFINE && !WT && C == 3 && P.pa == 1 && q == 1) finish_ok(P, t, s.G, &f);
      else finish_outputs(P, t, s.G, C, s.zmean, &f, WT ? s.lam : nullptr);
      if (f) {
        P.status[t] |= KK_ST_LDLT;
        const int p = atomicAdd(&P.counters[KK_CNT_FB], 1);
        P.fb_list[p] = t;
      } else {
        ++n_chol;
      }
    }
    __syncwarp();
    if constexpr (WT) {
      // kriging weights w = K^-1 (k - F lambda) = L^-T (y_k - Y_F lambda)
      // (assign_weight_ctx, kriging_base.F90:2428-2439): back sweep on the
      // unit-diagonal factor, rows scaled by 1 / L[r][r] at the end; a target
      // sent to the general kernel gets its weights there
      f = __shfl_sync(FULL, f, 0);
      if (!f) {
        int lrow[RM];
#pragma unroll
        for (int m = 0; m < RM; ++m) lrow[m] = lcol<N>(32 * m + lane) - (32 * m + lane);
        for (int jv = 0; jv < q; ++jv) {
          double v[RM];
#pragma unroll
          for (int m = 0; m < RM; ++m) {
            double vm = 0.0;
#pragma unroll
            for (int k = 0; k < CB; ++k)
              if (k == pa + jv) vm = (double)b[m][k];
#pragma unroll
            for (int k = 0; k < CB; ++k)
              if (k < pa) vm = fma(-(double)b[m][k], s.lam[jv * 6 + k], vm);
            v[m] = vm;
          }
          for (int j = n - 1; j >= 0; --j) {
            const double mine = (RM > 1 && (j >> 5) == 1) ? v[RM - 1] : v[0];
            const double nx = -__shfl_sync(FULL, mine, j & 31) * s.invw[j];
#pragma unroll
            for (int m = 0; m < RM; ++m) {
              const int r = 32 * m + lane;
              v[m] = fma(s.Lw[r < j ? lrow[m] + j : 0], nx, v[m]);
            }
          }
#pragma unroll
          for (int m = 0; m < RM; ++m) {
            const int r = 32 * m + lane;
            if (r < n) P.wout[((size_t)t * q + jv) * P.wstride + r] = v[m] * s.invw[r];
          }
        }
      }
      __syncwarp();
    }
  }
  if (lane == 0) {
    if (n_chol) atomicAdd(&P.counters[KK_CNT_CHOL], n_chol);
    if (REFINE && n_iter) atomicAdd(&P.counters[KK_CNT_ITER], n_iter);
  }
}

}  // namespace kk
