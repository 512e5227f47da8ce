// kk_block.cuh -- block-per-target FP64 solve of systems of 65..128
// equations (included by kk_solve.cu).
//
// The warp kernel's register layout scaled to one CTA of four warps: thread
// tid = pr + 8 pc (pr < 8 row classes, pc < 16 column classes) owns entry
// (8 ri + pr, 16 ci + pc) of the 128 x 128 covariance matrix in register slot
// a[ri][ci]; only slots with ri >= 2 ci can hold lower-triangle entries, so a
// thread keeps 72 FP64 slots -- the warp kernel's footprint at N = 64 -- and
// every trailing update is spread evenly over the 128 threads.  Thread tid
// also owns right-hand-side row tid.
//
// Per target (the reference's solve, solver.f90:224-300 and
// kriging_base.F90:3244-3503):
//   1. gather the neighbour rows; K comes packed from the assembly kernel;
//   2. right-looking Cholesky, one __syncthreads per column: the eight owner
//      threads of column j (one warp) take the pivot by shuffle and publish
//      the scaled column to a double-buffered shared column; the owner of
//      right-hand-side row j published that row just before;
//   3. the outputs are inner products of the forward-substituted columns
//      (block reduction), finished by thread 0 (Schur complement, estimate,
//      variance); a Cholesky failure goes to the general kernel's LDL^T path.
#pragma once

namespace kk {

template <int CB>
struct __align__(16) BlockSmem {
  double x[4][128];
  double z[128];
  int obs[128];
  int var[128];
  double col[2][8 * 18];   // column j of L, layout [pr][ri] with padded rows
  double yb[2][CB];        // right-hand-side row j before scaling
  double inv[2];           // 1 / L[j][j]
  double G[CB * CB];
  double red[4][CB * (CB + 1) / 2];
  double zmean[2 * KK_MAXVAR];
  int item, fail;
};

template <int CB>
__global__ void __launch_bounds__(128, 2)
    k_solve_block(const __grid_constant__ SolveParams P, const int* __restrict__ list,
                  const int* __restrict__ list_count, int item0, int nitems, const double* __restrict__ Kg,
                  int work_slot) {
  constexpr int N = 128, RI = 16, CI = 8, RIP = 18;
  constexpr int NK = N * (N + 1) / 2;
  constexpr int NG = CB * (CB + 1) / 2;
  __shared__ BlockSmem<CB> s;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int pr = tid & 7, pc = tid >> 3;
  int n_items = nitems;
  if (list_count) n_items = min(nitems, *list_count - item0);
  const int q = P.nvar, pa = P.pa;
  const int nu = n_func(P);
  const int C = pa + q + nu;
  const bool fast = P.fast_model == 1 || P.fast_model == 2;
  const ZoneRegs zr = load_zones();
  int n_chol = 0;
  for (;;) {
    if (tid == 0) s.item = atomicAdd(&P.counters[work_slot], 1);
    __syncthreads();
    const int item = s.item;
    if (item >= n_items) break;
    const int t = __ldg(&list[item0 + item]);
    const double* Ks = Kg + (size_t)item * NK;

    // ---- neighbour rows (variable blocks in order, ascending index)
    int nn[KK_MAXVAR], ist[KK_MAXVAR], n = 0;
#pragma unroll
    for (int v = 0; v < KK_MAXVAR; ++v) {
      nn[v] = v < q ? __ldg(&P.nnear[v][t]) : 0;
      ist[v] = n;
      n += nn[v];
    }
    if (tid < n) {
      const int r = tid;
      const int v = (q > 1 && r >= ist[1]) + (q > 2 && r >= ist[2]) + (q > 3 && r >= ist[3]);
      const int o = __ldg(&P.nbr[v][(size_t)t * P.mmax[v] + (r - ist[v])]);
      s.obs[r] = o;
      s.var[r] = v;
      for (int d = 0; d < P.nlag; ++d) s.x[d][r] = __ldg(&P.ox[v][d][o]);
      s.z[r] = __ldg(&P.oval[v][o]);
    }
    if (tid == 0) s.fail = 0;
    __syncthreads();
    const double rs = P.rs ? __ldg(&P.rs[t]) : 1.0;

    // ---- right-hand-side row tid: F (pa), k (q), u (nu)
    double b[CB];
#pragma unroll
    for (int k = 0; k < CB; ++k) b[k] = 0.0;
    if (tid < n) {
      const int r = tid, vr = s.var[r], orr = s.obs[r];
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
          if (fast && !P.gstart) {
            double lag[4];
#pragma unroll
            for (int d = 0; d < 4; ++d) lag[d] = dsub(xr[d], d < P.nlag ? __ldg(&P.tx[d][t]) : 0.0);
            if (!P.st && rs != 1.0) {
#pragma unroll
              for (int d = 0; d < 4; ++d) lag[d] = lag[d] / rs;
            }
            v = dadd(0.0, dmul(fast_cov<0>(P, zr, lag), 1.0));
            if (v != v) v = rhs_cov_row(P, t, xr, vr, k - pa, rs);  // a table argument at a zone edge
          } else {
            v = rhs_cov_row(P, t, xr, vr, k - pa, rs);
          }
        } else {
          const int u = k - pa - q;
          v = u == 0 ? s.z[r] : (vr == u - 1 ? 1.0 : 0.0);
        }
        b[k] = v;
      }
    }
    // ---- K (packed row-major lower, from the assembly kernel)
    double a[RI][CI];
#pragma unroll
    for (int ri = 0; ri < RI; ++ri) {
      const int r = 8 * ri + pr;
#pragma unroll
      for (int ci = 0; ci < CI; ++ci) {
        if (ri >= 2 * ci) {
          const int c = 16 * ci + pc;
          a[ri][ci] = (r < n && c <= r) ? __ldg(&Ks[r * (r + 1) / 2 + c]) : 0.0;
        }
      }
    }
    if (P.ck_isa && tid == 0) {
      for (int v = 0; v < q; ++v) {
        double sz = 0.0;
        for (int k = ist[v]; k < ist[v] + nn[v]; ++k) sz = dadd(sz, s.z[k]);
        s.zmean[v] = nn[v] > 0 ? sz / nn[v] : 0.0;
        s.zmean[KK_MAXVAR + v] = (double)nn[v];
      }
    }

    // ---- right-looking Cholesky + forward substitution
    const int nri = (n + 7) >> 3, nci = (n + 15) >> 4;
    bool fail = false;
#pragma unroll
    for (int jb = 0; jb < CI; ++jb) {
      if (jb >= nci) break;
#pragma unroll 1
      for (int jj = 0; jj < 16; ++jj) {
        const int j = 16 * jb + jj;
        if (j >= n) break;
        const int buf = j & 1;
        double* cw = s.col[buf];
        // right-hand-side row j as it stands (its updates by columns < j are done)
        if (tid == j) {
#pragma unroll
          for (int k = 0; k < CB; ++k)
            if (k < C) s.yb[buf][k] = b[k];
        }
        if (pc == jj) {  // the eight owners of column j: lanes 8 (jj & 3) .. + 7 of warp jj / 4
          const unsigned grp = 0xffu << (8 * (jj & 3));
          const double dsel = (jj < 8) ? a[2 * jb][jb] : a[2 * jb + 1][jb];
          const double d = __shfl_sync(grp, dsel, 8 * (jj & 3) + (jj & 7));
          const double inv = d > 0.0 ? rsqrt(d) : 0.0;
          if (pr == (jj & 7)) {
            s.inv[buf] = inv;
            if (!(d > 0.0)) s.fail = 1;
          }
#pragma unroll
          for (int ri = 2 * jb; ri < RI; ++ri) {
            const int r = 8 * ri + pr;
            cw[pr * RIP + ri] = (r > j) ? a[ri][jb] * inv : 0.0;
          }
        }
        __syncthreads();
        if (s.fail) { fail = true; break; }
        const double inv = s.inv[buf];
        double y[CB];
#pragma unroll
        for (int k = 0; k < CB; ++k) y[k] = (k < C) ? s.yb[buf][k] * inv : 0.0;
        if (tid == j) {
#pragma unroll
          for (int k = 0; k < CB; ++k) b[k] = y[k];
        } else if (tid > j && tid < n) {
          const double lb = cw[(tid & 7) * RIP + (tid >> 3)];
#pragma unroll
          for (int k = 0; k < CB; ++k)
            if (k < C) b[k] = fma(-lb, y[k], b[k]);
        }
        double lc[CI], lr[RI];
#pragma unroll
        for (int ci = jb; ci < CI; ++ci) lc[ci] = cw[(pc & 7) * RIP + 2 * ci + (pc >> 3)];
#pragma unroll
        for (int ri = 2 * jb; ri < RI; ++ri) lr[ri] = cw[pr * RIP + ri];
#pragma unroll
        for (int ci = jb; ci < CI; ++ci) {
          if (ci >= nci) break;
#pragma unroll
          for (int ri = 2 * ci; ri < RI; ++ri) {
            if ((ri & 3) == 0 && ri >= nri) break;
            a[ri][ci] = fma(-lr[ri], lc[ci], a[ri][ci]);
          }
        }
      }
      if (fail) break;
    }
    if (fail) {
      if (tid == 0) {
        P.status[t] |= KK_ST_LDLT;
        const int p = atomicAdd(&P.counters[KK_CNT_FB], 1);
        P.fb_list[p] = t;
      }
      __syncthreads();
      continue;
    }

    // ---- G = Y^T Y over the forward-substituted columns (block reduction)
    {
      double g[NG];
      int e = 0;
#pragma unroll
      for (int ka = 0; ka < CB; ++ka)
#pragma unroll
        for (int kb = ka; kb < CB; ++kb) g[e++] = (ka < C && kb < C) ? warp_sum(b[ka] * b[kb]) : 0.0;
      if (lane == 0)
#pragma unroll
        for (int k = 0; k < NG; ++k) s.red[wid][k] = g[k];
    }
    __syncthreads();
    if (tid == 0) {
      int e = 0;
      for (int ka = 0; ka < CB; ++ka)
        for (int kb = ka; kb < CB; ++kb, ++e) {
          if (ka >= C || kb >= C) continue;
          const double g = s.red[0][e] + s.red[1][e] + s.red[2][e] + s.red[3][e];
          s.G[ka * C + kb] = g;
          s.G[kb * C + ka] = g;
        }
      int f = 0;
      if (C == 3 && P.pa == 1 && q == 1) finish_ok(P, t, s.G, &f);
      else finish_outputs(P, t, s.G, C, s.zmean, &f);
      if (f) {
        P.status[t] |= KK_ST_LDLT;
        const int p = atomicAdd(&P.counters[KK_CNT_FB], 1);
        P.fb_list[p] = t;
      } else {
        ++n_chol;
      }
    }
    __syncthreads();
  }
  if (tid == 0 && n_chol) atomicAdd(&P.counters[KK_CNT_CHOL], n_chol);
}

}  // namespace kk
