// kk_search.cu -- neighbour search for the kriging solve path.
//
// Replaces the reference's kd-tree + sector search (kriging.F90:490-666,
// 1093-1154; kriging_st.F90:467-686; kdtree2_maxidx.f90) with:
//   * a uniform grid over the search-space coordinates (counting sort into
//     CSR cells plus a summed-area table of cell counts), built on device;
//   * one warp per target: grow a box of cells until it holds K+1 points,
//     gather every point inside the ball that covers that box, then select
//     the K nearest by a histogram over squared distances refined by a
//     warp sort of the boundary bucket.  Distances are computed with the
//     reference's arithmetic, so the selected set equals the kd-tree's
//     whenever no two candidates tie at a selection boundary;
//   * targets whose boundary holds equal distances (or whose candidate
//     buffer overflows) run an exact replica of the kd-tree search and of
//     its heap tie-breaking on the device (k_search_kdtree).
#include <cuda_runtime.h>
#include <stdint.h>

#include "kk_device.cuh"
#include "kk_kernels.h"

namespace kk {

// ---------------------------------------------------------------------------
// grid build
// ---------------------------------------------------------------------------
__global__ void k_search_coords(KkSearch S, const double* __restrict__ x0, const double* __restrict__ x1,
                                const double* __restrict__ x2, const double* __restrict__ x3,
                                double* __restrict__ sc_unsorted, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* xs[4] = {x0, x1, x2, x3};
  double x[4], r[4];
  for (int d = 0; d < S.nlag; ++d) x[d] = xs[d][i];
  if (S.aniso) rotate_pt(S.rotmat, S.ndim, x, r);
  else for (int d = 0; d < S.ndim; ++d) r[d] = x[d];
  // time search coordinate t * time_at, kriging_st.F90:90-95
  if (S.st) r[S.nlag - 1] = dmul(x[S.nlag - 1], S.ta);
  for (int d = 0; d < S.grid.D; ++d) sc_unsorted[(size_t)d * n + i] = r[d];
}

__device__ __forceinline__ int cell_coord(const KkGrid& g, int d, double v) {
  double f = (v - g.lo[d]) * g.inv_h[d];
  int c = (int)floor(f);
  return c < 0 ? 0 : (c >= g.n[d] ? g.n[d] - 1 : c);
}

__global__ void k_cell_count(KkGrid g, const double* __restrict__ scu, int* __restrict__ cell_of,
                             int* __restrict__ count, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = 0, stride = 1;
  for (int d = 0; d < g.G; ++d) {
    c += cell_coord(g, d, scu[(size_t)g.gd[d] * n + i]) * stride;
    stride *= g.n[d];
  }
  cell_of[i] = c;
  atomicAdd(&count[c], 1);
}

// exclusive scan of cell counts (one block, chunked)
__global__ void k_scan_cells(const int* __restrict__ count, int* __restrict__ start, int ncell) {
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < ncell; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < ncell ? count[i] : 0;
    int s = v;
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane == 31) warp_tot[wid] = s;
    __syncthreads();
    if (wid == 0) {
      int w = lane < nw ? warp_tot[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      warp_tot[lane] = w;
    }
    __syncthreads();
    int excl = carry + (wid > 0 ? warp_tot[wid - 1] : 0) + s - v;
    if (i < ncell) start[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) start[ncell] = carry;
}

__global__ void k_scatter_points(KkGrid g, const double* __restrict__ scu, const int* __restrict__ cell_of,
                                 const int* __restrict__ start, int* __restrict__ cursor,
                                 double* __restrict__ sc, int* __restrict__ sidx, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = cell_of[i];
  int pos = start[c] + atomicAdd(&cursor[c], 1);
  for (int d = 0; d < g.D; ++d) sc[(size_t)d * n + pos] = scu[(size_t)d * n + i];
  sidx[pos] = i;
}

// Within each cell order points by original index so the sorted layout is
// deterministic (cells hold a handful of points).
__global__ void k_sort_cells(KkGrid g, const int* __restrict__ start, double* __restrict__ sc,
                             int* __restrict__ sidx, int ncell, int n) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int b = start[c], e = start[c + 1];
  for (int i = b + 1; i < e; ++i) {
    int key = sidx[i];
    double v[4];
    for (int d = 0; d < g.D; ++d) v[d] = sc[(size_t)d * n + i];
    int j = i - 1;
    while (j >= b && sidx[j] > key) {
      sidx[j + 1] = sidx[j];
      for (int d = 0; d < g.D; ++d) sc[(size_t)d * n + j + 1] = sc[(size_t)d * n + j];
      --j;
    }
    sidx[j + 1] = key;
    for (int d = 0; d < g.D; ++d) sc[(size_t)d * n + j + 1] = v[d];
  }
}

// summed-area table: sat[(z)(y)(x)] over (n0+1)(n1+1)(n2+1) with a zero border
__global__ void k_sat_fill(KkGrid g, const int* __restrict__ start, int* __restrict__ sat) {
  const int n0 = g.n[0], n1 = g.G > 1 ? g.n[1] : 1, n2 = g.G > 2 ? g.n[2] : 1;
  const long long tot = (long long)(n0 + 1) * (n1 + 1) * (n2 + 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    int x = (int)(q % (n0 + 1));
    long long r = q / (n0 + 1);
    int y = (int)(r % (n1 + 1));
    int z = (int)(r / (n1 + 1));
    int v = 0;
    if (x > 0 && (g.G < 2 || y > 0) && (g.G < 3 || z > 0)) {
      int cx = x - 1, cy = g.G > 1 ? y - 1 : 0, cz = g.G > 2 ? z - 1 : 0;
      int c = cx + n0 * (cy + n1 * cz);
      v = start[c + 1] - start[c];
    }
    sat[q] = v;
  }
}

__global__ void k_sat_pass(KkGrid g, int* __restrict__ sat, int axis) {
  const int n0 = g.n[0], n1 = g.G > 1 ? g.n[1] : 1, n2 = g.G > 2 ? g.n[2] : 1;
  const int e0 = n0 + 1, e1 = n1 + 1, e2 = n2 + 1;
  int len = axis == 0 ? e0 : (axis == 1 ? e1 : e2);
  long long lines = (long long)e0 * e1 * e2 / len;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < lines; l += (long long)gridDim.x * blockDim.x) {
    long long base, stride;
    if (axis == 0) { base = l * e0; stride = 1; }
    else if (axis == 1) { long long z = l / e0, x = l % e0; base = z * e0 * e1 + x; stride = e0; }
    else { base = l; stride = (long long)e0 * e1; }
    int acc = 0;
    for (int k = 0; k < len; ++k) { acc += sat[base + k * stride]; sat[base + k * stride] = acc; }
  }
}

// ---------------------------------------------------------------------------
// per-target search
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long sat_at(const KkGrid& g, int x, int y, int z) {
  const int e0 = g.n[0] + 1, e1 = (g.G > 1 ? g.n[1] : 1) + 1;
  return g.sat[(long long)x + (long long)e0 * ((long long)y + (long long)e1 * z)];
}

// count of points in the cell box [a, b] (inclusive, clipped)
// Points in the grid cells that lie entirely inside the ball of squared
// radius r2 around q (warp-wide sum; lanes take cell rows).  A lower bound
// on the points within the ball, so the K-th nearest distance is at most
// sqrt(r2) once it reaches K + 1.  Rounding is resolved towards counting
// fewer cells.
__device__ long long inner_count(const KkGrid& g, const double* qa, const double* q, double r2, int lane) {
#pragma unroll
  for (int d = 0; d < 4; ++d) {  // search dimensions without grid axis: their full extent
    if (d < g.D && !((g.gmask >> d) & 1)) {
      const double e = fmax(fabs(qa[d] - g.umin[d]), fabs(g.umax[d] - qa[d]));
      r2 -= e * e;
    }
  }
  if (!(r2 > 0.0)) return 0;
  r2 *= 1.0 - 1e-9;
  double eps[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) eps[d] = 1e-12 * (fabs(g.lo[d]) + g.n[d] * g.h[d]);
  const double r = sqrt(r2);
  int cnt = 0;
  if (g.G == 1) {
    if (lane == 0) {
      const int x0 = max(0, (int)ceil((q[0] - r + eps[0] - g.lo[0]) * g.inv_h[0]));
      const int x1 = min(g.n[0] - 1, (int)floor((q[0] + r - eps[0] - g.lo[0]) * g.inv_h[0]) - 1);
      if (x1 >= x0) cnt = __ldg(&g.cell_start[x1 + 1]) - __ldg(&g.cell_start[x0]);
    }
  } else {
    const int y0 = max(0, (int)floor((q[1] - r - g.lo[1]) * g.inv_h[1]));
    const int y1 = min(g.n[1] - 1, (int)floor((q[1] + r - g.lo[1]) * g.inv_h[1]));
    int z0 = 0, z1 = 0;
    if (g.G > 2) {
      z0 = max(0, (int)floor((q[2] - r - g.lo[2]) * g.inv_h[2]));
      z1 = min(g.n[2] - 1, (int)floor((q[2] + r - g.lo[2]) * g.inv_h[2]));
    }
    const int ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    if (ny > 0 && nz > 0) {
      for (int p = lane; p < ny * nz; p += 32) {
        const int y = y0 + p % ny, z = z0 + p / ny;
        const double yl = g.lo[1] + y * g.h[1];
        const double dy = fmax(fabs(q[1] - yl), fabs(yl + g.h[1] - q[1])) + eps[1];
        double rem = r2 - dy * dy;
        if (g.G > 2) {
          const double zl = g.lo[2] + z * g.h[2];
          const double dz = fmax(fabs(q[2] - zl), fabs(zl + g.h[2] - q[2])) + eps[2];
          rem -= dz * dz;
        }
        if (rem <= 0.0) continue;
        const double wx = sqrt(rem) - eps[0];
        const int x0 = max(0, (int)ceil((q[0] - wx - g.lo[0]) * g.inv_h[0]));
        const int x1 = min(g.n[0] - 1, (int)floor((q[0] + wx - g.lo[0]) * g.inv_h[0]) - 1);
        if (x1 < x0) continue;
        const int row = y * g.n[0] + z * g.n[0] * g.n[1];
        cnt += __ldg(&g.cell_start[row + x1 + 1]) - __ldg(&g.cell_start[row + x0]);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  return cnt;
}

__device__ __forceinline__ long long box_count(const KkGrid& g, const int* a, const int* b) {
  int x0 = a[0], x1 = b[0] + 1;
  if (g.G == 1) return sat_at(g, x1, 0, 0) - sat_at(g, x0, 0, 0);
  int y0 = a[1], y1 = b[1] + 1;
  if (g.G == 2)
    return sat_at(g, x1, y1, 0) - sat_at(g, x0, y1, 0) - sat_at(g, x1, y0, 0) + sat_at(g, x0, y0, 0);
  int z0 = a[2], z1 = b[2] + 1;
  return sat_at(g, x1, y1, z1) - sat_at(g, x0, y1, z1) - sat_at(g, x1, y0, z1) - sat_at(g, x1, y1, z0) +
         sat_at(g, x0, y0, z1) + sat_at(g, x0, y1, z0) + sat_at(g, x1, y0, z0) - sat_at(g, x0, y0, z0);
}

// squared search-space distance of sorted point j to q, with the reference's
// accumulation order sd = ((0 + d1^2) + d2^2) + ... (kdtree2_maxidx.f90:1547-1552)
__device__ __forceinline__ double dist2(const KkGrid& g, const double* q, int j) {
  double sd = 0.0;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    if (d < g.D) {
      double t = dsub(__ldg(&g.sc[(size_t)d * g.nobs + j]), q[d]);
      sd = dadd(sd, dmul(t, t));
    }
  }
  return sd;
}

struct WarpBuf {
  double* d2;    // [cap]
  int* idx;      // [cap] original observation index
  int* hist;     // [256]
  double* bd2;   // [bcap] boundary list
  int* bidx;     // [bcap]
  int* out;      // [ocap] selected indices
  double* outd;  // [ocap] selected distances
  signed char* sec;  // [cap] sector of each candidate
};

constexpr int NBIN = 256;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// bitonic sort of n (power of two, >= 32) (key, idx) pairs in shared memory by one warp
__device__ void warp_sort_pairs(double* key, int* idx, int n) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < n; i += 32) {
        int p = i ^ j;
        if (p > i) {
          bool up = ((i & k) == 0);
          double a = key[i], b = key[p];
          int ia = idx[i], ib = idx[p];
          bool gt = (a > b) || (a == b && ia > ib);
          if (gt == up) { key[i] = b; key[p] = a; idx[i] = ib; idx[p] = ia; }
        }
      }
      __syncwarp();
    }
  }
}

__device__ void warp_sort_ints(int* v, int n) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < n; i += 32) {
        int p = i ^ j;
        if (p > i) {
          bool up = ((i & k) == 0);
          int a = v[i], b = v[p];
          if ((a > b) == up) { v[i] = b; v[p] = a; }
        }
      }
      __syncwarp();
    }
  }
}

// Ascending bitonic sort of n2 = 32 or 64 ints held in registers, element i
// in lane i % 32, register i / 32 (v0, v1): compare-exchange across lanes by
// shuffle, across the two registers within a lane.
__device__ __forceinline__ void warp_sort_reg64(int& v0, int& v1, int n2) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= n2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j == 32) {  // partner is the other register of this lane
        const bool up = ((lane & k) == 0);
        const int lo = min(v0, v1), hi = max(v0, v1);
        v0 = up ? lo : hi;
        v1 = up ? hi : lo;
        continue;
      }
      const bool lower = (lane & j) == 0;
      const int o0 = __shfl_xor_sync(0xffffffffu, v0, j);
      const bool up0 = ((lane & k) == 0);
      v0 = (lower == up0) ? min(v0, o0) : max(v0, o0);
      if (n2 == 64) {
        const int o1 = __shfl_xor_sync(0xffffffffu, v1, j);
        const bool up1 = (((32 + lane) & k) == 0);
        v1 = (lower == up1) ? min(v1, o1) : max(v1, o1);
      }
    }
  }
}

// Select the K smallest squared distances among candidates [0, M) for which
// pred(j) holds; appends their (idx, d2) to out[*nout ...] when emit is set
// (out and outd then hold at least *nout + K entries).  Returns the K-th
// smallest value T in *T_out and sets *tie when a candidate outside the
// selection has distance exactly T.  Returns false when the boundary bucket
// overflows the boundary buffer.
template <class Pred>
__device__ bool warp_select(const WarpBuf& b, int M, int K, double dmax2, int bcap, Pred pred, bool emit,
                            int* nout, double* T_out, bool* tie) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < NBIN; i += 32) b.hist[i] = 0;
  __syncwarp();
  const double scale = dmax2 > 0.0 ? (double)NBIN / dmax2 : 0.0;
  for (int j = lane; j < M; j += 32) {
    if (!pred(j)) continue;
    int bin = (int)(b.d2[j] * scale);
    bin = bin < 0 ? 0 : (bin >= NBIN ? NBIN - 1 : bin);
    atomicAdd(&b.hist[bin], 1);
  }
  __syncwarp();
  // find the bucket holding the K-th smallest: each lane owns 8 bins
  int loc[8], s = 0;
  for (int q = 0; q < 8; ++q) { loc[q] = b.hist[lane * 8 + q]; s += loc[q]; }
  int incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  int excl = incl - s;
  unsigned hit = __ballot_sync(0xffffffffu, excl < K && incl >= K);
  int owner = __ffs(hit) - 1;
  int B = 0, cb = 0;
  if (lane == owner) {
    int acc = excl;
    for (int q = 0; q < 8; ++q) {
      if (acc + loc[q] >= K) { B = lane * 8 + q; cb = acc; break; }
      acc += loc[q];
    }
  }
  B = __shfl_sync(0xffffffffu, B, owner);
  cb = __shfl_sync(0xffffffffu, cb, owner);
  const int hB = b.hist[B];
  if (hB > bcap) return false;
  // pass 2: emit everything below bucket B, collect bucket B
  int nb = 0, no = *nout;
  for (int base = 0; base < M; base += 32) {
    int j = base + lane;
    int bin = -1;
    if (j < M && pred(j)) {
      bin = (int)(b.d2[j] * scale);
      bin = bin < 0 ? 0 : (bin >= NBIN ? NBIN - 1 : bin);
    }
    unsigned lo = __ballot_sync(0xffffffffu, bin >= 0 && bin < B);
    unsigned eq = __ballot_sync(0xffffffffu, bin == B);
    if (emit && bin >= 0 && bin < B) {
      int p = no + __popc(lo & lanemask_lt());
      b.out[p] = b.idx[j];
      b.outd[p] = b.d2[j];
    }
    if (bin == B) {
      int p = nb + __popc(eq & lanemask_lt());
      b.bd2[p] = b.d2[j];
      b.bidx[p] = b.idx[j];
    }
    no += __popc(lo);
    nb += __popc(eq);
  }
  __syncwarp();
  // sort the boundary bucket and take the first r = K - cb
  int np2 = 32;
  while (np2 < nb) np2 <<= 1;
  for (int i = nb + lane; i < np2; i += 32) { b.bd2[i] = 1.0e308; b.bidx[i] = 0x7fffffff; }
  __syncwarp();
  warp_sort_pairs(b.bd2, b.bidx, np2);
  const int r = K - cb;
  if (emit)
    for (int i = lane; i < r; i += 32) { b.out[no + i] = b.bidx[i]; b.outd[no + i] = b.bd2[i]; }
  double T = b.bd2[r - 1];
  *tie = (r < nb) && (b.bd2[r] == T);
  *T_out = T;
  *nout = no + r;
  __syncwarp();
  return true;
}

// Bitonic sort of (key, idx) pairs in shared memory by (idx >> 28, key,
// idx): the sector id rides in bits 28..30 of idx (observation indices are
// below 2^28 in sector mode).
__device__ void warp_sort_sec(double* key, int* idx, int n) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < n; i += 32) {
        int p = i ^ j;
        if (p > i) {
          bool up = ((i & k) == 0);
          double a = key[i], b = key[p];
          int ia = idx[i], ib = idx[p];
          int sa = ia >> 28, sb = ib >> 28;
          bool gt = (sa > sb) || (sa == sb && ((a > b) || (a == b && ia > ib)));
          if (gt == up) { key[i] = b; key[p] = a; idx[i] = ib; idx[p] = ia; }
        }
      }
      __syncwarp();
    }
  }
}

// Sector filter of apply_sector_filter (kriging.F90:1093-1154) in one pass:
// among the candidates j < nk (all within dmax2, sector sec[j] < nsec), the
// nmax nearest of every sector (all of them when fewer) are appended to
// out[*nout ...].  One histogram of nsec x (NBIN / nsec) distance buckets
// finds every sector's boundary bucket at once; the boundary buckets are
// sorted together by (sector, d2, idx).  *tie is set when a sector's cut
// falls between equal distances (the reference's heap order then decides:
// the caller takes the exact kd-tree path); returns false when the boundary
// buckets overflow bcap.
template <class Pred>
__device__ bool warp_select_sectors(const WarpBuf& b, int nk, Pred pred, int nsec, int nmax, double dmax2, int bcap,
                                    int* nout, bool* tie) {
  const int lane = threadIdx.x & 31;
  const int nbk = NBIN / nsec;                  // buckets per sector
  const int lps = nbk / 8;                      // lanes per sector (8 bins per lane)
  for (int i = lane; i < NBIN; i += 32) b.hist[i] = 0;
  __syncwarp();
  const double scale = dmax2 > 0.0 ? (double)nbk / dmax2 : 0.0;
  for (int j = lane; j < nk; j += 32) {
    if (!pred(j)) continue;
    int q = (int)(b.d2[j] * scale);
    q = q < 0 ? 0 : (q >= nbk ? nbk - 1 : q);
    atomicAdd(&b.hist[b.sec[j] * nbk + q], 1);
  }
  __syncwarp();
  // segmented inclusive scan: lane owns bins 8 lane .. 8 lane + 7
  int loc[8], sum = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) { loc[q] = b.hist[lane * 8 + q]; sum += loc[q]; }
  const int seg = lane % lps;
  int incl = sum;
  for (int o = 1; o < lps; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (seg >= o) incl += t;
  }
  const int excl = incl - sum;
  const int total = __shfl_sync(0xffffffffu, incl, (lane / lps) * lps + lps - 1);
  __syncwarp();
  // per sector: boundary bucket bs (nbk = none: the sector is taken whole)
  // and the count below it; kept in hist[NBIN - 32 ..] after the scan
  int* bsec = b.hist + NBIN - 32;   // [8] boundary bucket of each sector
  int* cbel = b.hist + NBIN - 24;   // [8] count below the boundary
  int* hb = b.hist + NBIN - 16;     // [8] size of the boundary bucket
  int* fill = b.hist + NBIN - 8;    // [8] boundary fill cursors
  const int sector = lane / lps;
  if (seg == 0 && total <= nmax) { bsec[sector] = nbk; cbel[sector] = total; hb[sector] = 0; }
  if (total > nmax && excl < nmax && incl >= nmax) {
    int acc = excl;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      if (acc + loc[q] >= nmax) {
        bsec[sector] = seg * 8 + q;
        cbel[sector] = acc;
        hb[sector] = loc[q];
        break;
      }
      acc += loc[q];
    }
  }
  __syncwarp();
  // boundary segments: offsets by sector
  int off[8];
  int nbt = 0;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    off[s] = nbt;
    if (s < nsec) nbt += hb[s];
  }
  if (nbt > bcap) return false;
  if (lane < 8) fill[lane] = 0;
  __syncwarp();
  // pass 2: emit everything below the boundary buckets, collect those buckets
  int no = *nout;
  for (int base = 0; base < nk; base += 32) {
    const int j = base + lane;
    int sj = 0, q = 0, bs = 0;
    const bool in = j < nk && pred(j);
    if (in) {
      sj = b.sec[j];
      q = (int)(b.d2[j] * scale);
      q = q < 0 ? 0 : (q >= nbk ? nbk - 1 : q);
      bs = bsec[sj];
    }
    const bool below = in && q < bs;
    const bool atb = in && q == bs;
    const unsigned lo = __ballot_sync(0xffffffffu, below);
    if (below) b.out[no + __popc(lo & lanemask_lt())] = b.idx[j];
    if (atb) {
      int o2 = 0;
#pragma unroll
      for (int s = 0; s < 8; ++s) if (s == sj) o2 = off[s];
      const int p = o2 + atomicAdd(&fill[sj], 1);
      b.bd2[p] = b.d2[j];
      b.bidx[p] = b.idx[j] | (sj << 28);
    }
    no += __popc(lo);
  }
  __syncwarp();
  bool t_any = false;
  if (nbt > 0) {
    int np2 = 32;
    while (np2 < nbt) np2 <<= 1;
    for (int i = nbt + lane; i < np2; i += 32) { b.bd2[i] = 1.0e308; b.bidx[i] = 0x7fffffff; }
    __syncwarp();
    warp_sort_sec(b.bd2, b.bidx, np2);
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      if (s >= nsec || hb[s] == 0) continue;
      const int r = nmax - cbel[s];
      for (int i = lane; i < r; i += 32) b.out[no + i] = b.bidx[off[s] + i] & 0x0fffffff;
      if (r < hb[s] && b.bd2[off[s] + r] == b.bd2[off[s] + r - 1]) t_any = true;
      no += r;
    }
  }
  *tie = t_any;
  *nout = no;
  __syncwarp();
  return true;
}

// Per-warp candidate buffers of k_search: CAP candidates {d2, idx, sector},
// ocap selected indices (and their distances when ocapd > 0), bcap
// boundary-bucket entries and the 256-bin histogram.  The plain k-nearest
// search keeps the K selected with their distances (ocap = ocapd, the next
// multiple of 32 above K, at most 320).  The sector search only needs the
// K-th distance of the first selection and keeps the 2^ndim * nmax sector
// picks (ocapd = 0).  The boundary buffer takes what is left of a quarter of
// the SM's shared memory, so that four 4-warp CTAs share an SM, when that
// leaves at least 128 entries; otherwise it holds 256 and three CTAs fit.  A
// target whose ball holds more than CAP points, or whose selection does not
// fit these buffers, takes the exact kd-tree path instead.
constexpr int KK_SEARCH_OCAP = 320;
constexpr int KK_SEARCH_BCAP = 256;
constexpr int KK_SMEM_PER_SM = 233472;  // 228 KB of shared memory per SM
constexpr int KK_SMEM_PER_CTA_RESERVED = 1024;
#ifndef KK_SEARCH_BISECT
#define KK_SEARCH_BISECT 5  // radius bisection steps
#endif
struct SearchLayout {
  int ocap, ocapd, bcap;
};
template <int CAP>
__host__ __device__ inline size_t search_smem_per_warp(const SearchLayout& L) {
  return sizeof(double) * (CAP + L.ocapd + L.bcap) + sizeof(int) * (CAP + L.ocap + L.bcap + 256) + CAP;
}
template <int CAP>
__host__ __device__ inline SearchLayout search_layout(const KkSearch& S) {
  SearchLayout L;
  if (S.mode == 2) {
    // at most KK_SEARCH_OCAP: a larger sector total takes the kd-tree path
    L.ocap = (((1 << S.ndim) * S.nmax + 1 + 31) / 32) * 32;
    if (L.ocap > KK_SEARCH_OCAP) L.ocap = KK_SEARCH_OCAP;
    L.ocapd = 0;
  } else {
    L.ocap = (S.K + 1 + 31) / 32 * 32;
    if (L.ocap > KK_SEARCH_OCAP) L.ocap = KK_SEARCH_OCAP;
    L.ocapd = L.ocap;
  }
  L.bcap = 0;
  const long long per_warp = (KK_SMEM_PER_SM / 4 - KK_SMEM_PER_CTA_RESERVED) / 4;
  const long long room = per_warp - (long long)search_smem_per_warp<CAP>(L);
  long long bcap = room / (long long)(sizeof(double) + sizeof(int));
  bcap = bcap / 16 * 16;
  L.bcap = (bcap >= 128) ? (int)(bcap < KK_SEARCH_BCAP ? bcap : KK_SEARCH_BCAP) : KK_SEARCH_BCAP;
  return L;
}

template <int CAP>
__global__ void __launch_bounds__(128) k_search(KkSearch S, int ntarget, const double* __restrict__ t0,
                                                const double* __restrict__ t1, const double* __restrict__ t2,
                                                const double* __restrict__ t3, const double* __restrict__ o0,
                                                const double* __restrict__ o1, const double* __restrict__ o2,
                                                const double* __restrict__ o3, int* __restrict__ nbr,
                                                int* __restrict__ nnear, int* __restrict__ status,
                                                int* __restrict__ redo_list, int* __restrict__ redo_count) {
  constexpr int WARPS = 4;
  const SearchLayout LY = search_layout<CAP>(S);
  const int BCAP = LY.bcap, OCAP = LY.ocap;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned char* base = smem_raw + (size_t)w * search_smem_per_warp<CAP>(LY);
  WarpBuf B;
  B.d2 = reinterpret_cast<double*>(base);
  B.outd = B.d2 + CAP;  // LY.ocapd entries (none in the sector layout)
  B.bd2 = B.outd + LY.ocapd;
  B.idx = reinterpret_cast<int*>(B.bd2 + BCAP);
  B.out = B.idx + CAP;
  B.bidx = B.out + OCAP;
  B.hist = B.bidx + BCAP;
  B.sec = reinterpret_cast<signed char*>(B.hist + NBIN);
  const KkGrid& g = S.grid;
  const double* ts[4] = {t0, t1, t2, t3};
  const double* os[4] = {o0, o1, o2, o3};

  for (int t = blockIdx.x * WARPS + w; t < ntarget; t += gridDim.x * WARPS) {
    double x[4] = {0.0, 0.0, 0.0, 0.0}, q[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < 4; ++d)
      if (d < S.nlag) x[d] = __ldg(&ts[d][t]);
    if (S.aniso) {
      rotate_pt(S.rotmat, S.ndim, x, q);
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (d < S.ndim) q[d] = x[d];
    }
    if (S.st) {
#pragma unroll
      for (int d = 1; d < 4; ++d)
        if (d == S.nlag - 1) q[d] = dmul(x[d], S.ta);
    }
    const int cvskip = S.cv ? t : -1;
    int st = 0;
    int nsel = 0;

    if (S.mode == 0) {
      // all observations (need_search = .false.): rotated_dists on the
      // difference (rotation.f90:193-218), maxdist filter
      for (int base = 0; base < S.nobs; base += 32) {
        int i = base + lane;
        bool keep = false;
        if (i < S.nobs && i != cvskip) {
          double diff[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
#pragma unroll
          for (int d = 0; d < 3; ++d)
            if (d < S.ndim) diff[d] = dsub(__ldg(&os[d][i]), S.st ? x[d] : q[d]);
          rotate_pt(S.rotmat, S.ndim, diff, r);
          double s = 0.0;
#pragma unroll
          for (int d = 0; d < 3; ++d)
            if (d < S.ndim) s = dadd(s, dmul(r[d], r[d]));
          if (S.st) {
            const double* ot = S.ndim == 1 ? o1 : (S.ndim == 2 ? o2 : o3);
            const double qt = S.nlag == 2 ? q[1] : (S.nlag == 3 ? q[2] : q[3]);
            double tt = dsub(dmul(__ldg(&ot[i]), S.ta), qt);
            s = dadd(s, dmul(tt, tt));
          }
          keep = s <= S.maxd2;
        }
        unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) nbr[(size_t)t * S.mmax + nsel + __popc(m & lanemask_lt())] = i;
        nsel += __popc(m);
      }
      if (lane == 0) { nnear[t] = nsel; status[t] = 0; }
      continue;
    }

    // ---- grow the cell box until it holds K+1 points (or all points) ----
    const int K = S.K;  // K < nobs here
    int c[4] = {0, 0, 0, 0}, a[4] = {0, 0, 0, 0}, bb[4] = {0, 0, 0, 0};
    // coordinates along the grid axes
    double qg[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (k < g.G) {
        const int d = g.gd[k];
        qg[k] = d == 0 ? q[0] : (d == 1 ? q[1] : (d == 2 ? q[2] : q[3]));
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (d < g.G) c[d] = cell_coord(g, d, qg[d]);
    // the smallest ring R whose box is the whole grid or holds K + 1 points
    // (both monotone in R): lane l tests R0 + l, 32 rings per round trip
    int R = -1;
    for (int R0 = 0; R < 0; R0 += 32) {
      const int Rl = R0 + lane;
      bool full = true;
      int al[3] = {0, 0, 0}, bl[3] = {0, 0, 0};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (d < g.G) {
          al[d] = max(0, c[d] - Rl);
          bl[d] = min(g.n[d] - 1, c[d] + Rl);
          if (al[d] > 0 || bl[d] < g.n[d] - 1) full = false;
        }
      }
      const bool ok = full || box_count(g, al, bl) >= (long long)K + 1;
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (m) R = R0 + __ffs(m) - 1;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d < g.G) {
        a[d] = max(0, c[d] - R);
        bb[d] = min(g.n[d] - 1, c[d] + R);
      }
    }
    // farthest corner of the box (every search dimension), with a margin
    double D2 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (k >= g.G) break;
      const double lo = (a[k] == 0) ? fmin(g.gumin[k], g.lo[k]) : g.lo[k] + a[k] * g.h[k];
      const double hi = (bb[k] == g.n[k] - 1) ? fmax(g.gumax[k], g.lo[k] + g.n[k] * g.h[k])
                                              : g.lo[k] + (bb[k] + 1) * g.h[k];
      const double e = fmax(fabs(qg[k] - lo), fabs(hi - qg[k]));
      D2 += e * e;
    }
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      if (d < g.D && !((g.gmask >> d) & 1)) {
        const double e = fmax(fabs(q[d] - g.umin[d]), fabs(g.umax[d] - q[d]));
        D2 += e * e;
      }
    }
    // tighten the radius: bisect for the smallest ball whose fully covered
    // cells already hold K + 1 points (the corner ball of the box can reach
    // far into a neighbouring cluster)
    {
      // lower bracket: a cell outside the ring-(R-1) box, which holds fewer
      // than K + 1 points, has its farthest corner at least R cell widths
      // away, so no smaller ball covers K + 1 points with whole cells (the
      // bracket only sets how fast the bisection closes: rhi stays a radius
      // whose covered cells hold K + 1 points)
      double hmin = g.h[0];
#pragma unroll
      for (int k = 1; k < 3; ++k)
        if (k < g.G) hmin = fmin(hmin, g.h[k]);
      double rhi = sqrt(D2), rlo = fmin(R * hmin * (1.0 - 1e-6), rhi);
      for (int it = 0; it < KK_SEARCH_BISECT; ++it) {
        const double mid = 0.5 * (rlo + rhi);
        if (inner_count(g, q, qg, mid * mid, lane) >= (long long)K + 1) rhi = mid;
        else rlo = mid;
      }
      D2 = fmin(D2, rhi * rhi);
    }
    D2 = D2 * (1.0 + 1e-9) + 1e-300;
    const double Dr = sqrt(D2);

    // ---- gather all points inside the ball of radius Dr ----
    int M = 0;
    bool overflow = false;
    int zlo = 0, zhi = 0, ylo = 0, yhi = 0;
    if (g.G > 2) {
      zlo = max(0, (int)floor((qg[2] - Dr - g.lo[2]) * g.inv_h[2]) - 1);
      zhi = min(g.n[2] - 1, (int)floor((qg[2] + Dr - g.lo[2]) * g.inv_h[2]) + 1);
    }
    if (g.G > 1) {
      ylo = max(0, (int)floor((qg[1] - Dr - g.lo[1]) * g.inv_h[1]) - 1);
      yhi = min(g.n[1] - 1, (int)floor((qg[1] + Dr - g.lo[1]) * g.inv_h[1]) + 1);
    }
    // cell rows (y, z) that can meet the ball: lanes take 32 rows at a time
    // and find each row's contiguous point range; the ranges of the group are
    // then gathered 32 points at a time (a lane finds its row by bisection
    // over the range starts), so short rows do not leave lanes idle
    {
      int* rstart = B.hist;       // [32] exclusive prefix of the range lengths
      int* rp0 = B.hist + 32;     // [32] first sorted point of each row's range
      const int ny = g.G > 1 ? yhi - ylo + 1 : 1;
      const int nz = g.G > 2 ? zhi - zlo + 1 : 1;
      const int nrows = (ny > 0 && nz > 0) ? ny * nz : 0;
      for (int rg = 0; rg < nrows && !overflow; rg += 32) {
        const int ridx = rg + lane;
        int p0 = 0, len = 0;
        if (ridx < nrows) {
          const int y = ylo + ridx % ny, z = zlo + ridx / ny;
          double dy2 = 0.0;
          if (g.G > 2) {
            double zl = g.lo[2] + z * g.h[2] - 1e-6 * g.h[2], zh = zl + 1.000002 * g.h[2];
            double dz = qg[2] < zl ? zl - qg[2] : (qg[2] > zh ? qg[2] - zh : 0.0);
            dy2 = dz * dz;
          }
          if (g.G > 1) {
            double yl = g.lo[1] + y * g.h[1] - 1e-6 * g.h[1], yh = yl + 1.000002 * g.h[1];
            double dy = qg[1] < yl ? yl - qg[1] : (qg[1] > yh ? qg[1] - yh : 0.0);
            dy2 += dy * dy;
          }
          if (dy2 <= D2) {
            double wx = sqrt(fmax(D2 - dy2, 0.0));
            int x0 = max(0, (int)floor((qg[0] - wx - g.lo[0]) * g.inv_h[0]) - 1);
            int x1 = min(g.n[0] - 1, (int)floor((qg[0] + wx - g.lo[0]) * g.inv_h[0]) + 1);
            int row = (g.G > 1 ? y : 0) * g.n[0] + (g.G > 2 ? z * g.n[0] * g.n[1] : 0);
            p0 = __ldg(&g.cell_start[row + x0]);
            len = __ldg(&g.cell_start[row + x1 + 1]) - p0;
          }
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t2 = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t2;
        }
        const int tot = __shfl_sync(0xffffffffu, incl, 31);
        rstart[lane] = incl - len;
        rp0[lane] = p0;
        __syncwarp();
        // two batches of 32 per round: every global load of both (coordinates,
        // original index) is issued before the first ballot
        for (int base = 0; base < tot; base += 64) {
          double d2v[2] = {0.0, 0.0};
          int oi[2] = {0, 0}, sec[2] = {0, 0};
          bool in[2] = {false, false};
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int i = base + 32 * u + lane;
            if (i < tot) {
              int k = 0;
#pragma unroll
              for (int step = 16; step > 0; step >>= 1)
                if (rstart[k + step] <= i) k += step;
              const int j = rp0[k] + (i - rstart[k]);
              // dist2 with the sector signs of the same differences
              double sd = 0.0;
#pragma unroll
              for (int d = 0; d < 4; ++d) {
                if (d < g.D) {
                  const double t = dsub(__ldg(&g.sc[(size_t)d * g.nobs + j]), q[d]);
                  sd = dadd(sd, dmul(t, t));
                  if (d < S.ndim && t < 0.0) sec[u] += 1 << d;
                }
              }
              d2v[u] = sd;
              in[u] = sd <= D2;
              oi[u] = __ldg(&g.sidx[j]);
            }
          }
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const unsigned m = __ballot_sync(0xffffffffu, in[u]);
            const int pos = M + __popc(m & lanemask_lt());
            if (in[u] && pos < CAP) {
              B.d2[pos] = d2v[u];
              B.idx[pos] = oi[u];
              if (S.mode == 2) B.sec[pos] = (signed char)sec[u];
            }
            M += __popc(m);
            if (M > CAP) overflow = true;
          }
        }
        __syncwarp();  // the next group reuses rstart / rp0
      }
    }
    __syncwarp();
    if (overflow || M < K || (S.mode != 2 && K >= OCAP)) {
      st |= KK_ST_OVERFLOW;
    } else {
      double T;
      bool tie = false;
      int nout = 0;
      // K nearest (kdtree2_n_nearest semantics: the K smallest distances)
      // the sector search keeps only the K-th distance T of this selection
      bool ok = warp_select(B, M, K, D2, BCAP, [](int) { return true; }, S.mode != 2, &nout, &T, &tie);
      if (!ok) st |= KK_ST_OVERFLOW;
      else if (tie && T <= S.maxd2) st |= KK_ST_TIE;
      if (!(st & (KK_ST_OVERFLOW | KK_ST_TIE))) {
        if (S.mode == 1) {
          // plain: drop the cross-validation target and apply maxdist
          for (int base = 0; base < nout; base += 32) {
            int i = base + lane;
            bool keep = i < nout && B.out[i] != cvskip && B.outd[i] <= S.maxd2;
            int v = keep ? B.out[i] : 0;
            unsigned m = __ballot_sync(0xffffffffu, keep);
            __syncwarp();
            if (keep) B.idx[nsel + __popc(m & lanemask_lt())] = v;
            nsel += __popc(m);
            __syncwarp();
          }
        } else {
          // sector filter (kriging.F90:1093-1154): within the K-set, the nmax
          // nearest of every sector among candidates within maxdist
          // the K-set is every candidate with distance <= T (no tie at T),
          // without the cross-validation target and points past maxdist
          const double* cd2 = B.d2;
          const int* cidx = B.idx;
          const double maxd2 = S.maxd2;
          auto inset = [=](int j) { return cd2[j] <= T && cd2[j] <= maxd2 && cidx[j] != cvskip; };
          const int nsec = 1 << S.ndim;
          int nfin = 0;
          bool ties = false;
          if (nsec * S.nmax >= OCAP || !warp_select_sectors(B, M, inset, nsec, S.nmax, T, BCAP, &nfin, &ties))
            st |= KK_ST_OVERFLOW;
          if (ties) st |= KK_ST_TIE;
          __syncwarp();
          for (int i = lane; i < nfin; i += 32) B.idx[i] = B.out[i];
          nsel = nfin;
          __syncwarp();
        }
      }
    }
    if (st & (KK_ST_OVERFLOW | KK_ST_TIE)) {
      if (lane == 0) {
        status[t] = st;
        nnear[t] = 0;
        int p = atomicAdd(redo_count, 1);
        redo_list[p] = t;
      }
      __syncwarp();
      continue;
    }
    // isort: ascending observation index (kriging_base.F90:3209-3211)
    int np2 = 32;
    while (np2 < nsel) np2 <<= 1;
    if (np2 <= 64) {
      // up to 64 indices: sorted in registers
      int v0 = lane < nsel ? B.idx[lane] : 0x7fffffff;
      int v1 = 32 + lane < nsel ? B.idx[32 + lane] : 0x7fffffff;
      warp_sort_reg64(v0, v1, np2);
      if (lane < nsel) nbr[(size_t)t * S.mmax + lane] = v0;
      if (32 + lane < nsel) nbr[(size_t)t * S.mmax + 32 + lane] = v1;
    } else {
      for (int i = nsel + lane; i < np2; i += 32) B.idx[i] = 0x7fffffff;
      __syncwarp();
      warp_sort_ints(B.idx, np2);
      for (int i = lane; i < nsel; i += 32) nbr[(size_t)t * S.mmax + i] = B.idx[i];
    }
    if (lane == 0) { nnear[t] = nsel; status[t] = 0; }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// exact kd-tree replica for tie / overflow targets (one thread per target).
// Its heap and visit order restate kdtree2 (M. Kennel 2004, Academic Free
// License 1.1), which the reference bundles as kdtree2_maxidx.f90.
// ---------------------------------------------------------------------------
struct KdHeapEntry {
  double dis;
  int idx;
  int pad;
};

__device__ double pq_insert(KdHeapEntry* a, int n, double dis, int idx) {
  int i = n;
  while (i > 1) {
    int ip = i / 2;
    double pd = a[ip].dis;
    if (dis > pd) { a[i] = a[ip]; i = ip; } else break;
  }
  a[i].dis = dis;
  a[i].idx = idx;
  return a[1].dis;
}

__device__ double pq_replace_max(KdHeapEntry* a, int N, double dis, int idx) {
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

__device__ void kd_heapsort(KdHeapEntry* a, int n) {
  if (n <= 1) return;
  int ileft = n / 2 + 1, iright = n;
  KdHeapEntry value;
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

// kdtree2_n_nearest (kdtree2_maxidx.f90:1043-1085) with search and
// process_terminal_node (1383-1612) unrolled onto an explicit stack; points
// with index >= maxn are skipped before their distance is taken (the
// _maxidx variants, kdtree2_maxidx.f90:1928-2110).
__device__ void kd_n_nearest(const KkTree& T, const double* qv, int nn, KdHeapEntry* heap, int maxn = 0x7fffffff) {
  struct Frame { int node; int phase; double dis; };
  Frame stack[192];
  int sp = 0;
  int nfound = 0;
  double ballsize = 1.7976931348623157e308;
  stack[sp++] = {T.root, 0, 0.0};
  while (sp > 0) {
    Frame f = stack[--sp];
    const int* ni = T.node_i + 5 * f.node;
    const int cut = ni[0], l = ni[1], u = ni[2], left = ni[3], right = ni[4];
    if (f.phase == 0) {
      if (!(left >= 0 && right >= 0)) {
        double bs = ballsize;
        for (int i = l; i <= u; ++i) {
          if (T.ind[i] >= maxn) continue;
          double sd = 0.0;
          bool skip = false;
          for (int k = 0; k < T.D; ++k) {
            double d = dsub(T.rdata[(size_t)i * T.D + k], qv[k]);
            sd = dadd(sd, dmul(d, d));
            if (sd > bs) { skip = true; break; }
          }
          if (skip) continue;
          int id = T.ind[i];
          if (nfound < nn) {
            ++nfound;
            double np = pq_insert(heap, nfound, sd, id);
            if (nfound == nn) bs = np;
          } else {
            bs = pq_replace_max(heap, nfound, sd, id);
          }
        }
        ballsize = bs;
        continue;
      }
      const double* nd = T.node_d + 3 * f.node;
      double qval = qv[cut];
      int closer;
      double dis;
      if (qval < nd[0]) {
        closer = left;
        double t = dsub(nd[2], qval);
        dis = dmul(t, t);
      } else {
        closer = right;
        double t = dsub(nd[1], qval);
        dis = dmul(t, t);
      }
      if (sp + 2 > 192) return;  // deeper than any tree built from int32 indices
      stack[sp++] = {f.node, 1, dis};
      stack[sp++] = {closer, 0, 0.0};
    } else {
      const double* nd = T.node_d + 3 * f.node;
      double qval = qv[cut];
      int farther = (qval < nd[0]) ? right : left;
      double dis = f.dis;
      double bs = ballsize;
      if (dis <= bs) {
        bool pruned = false;
        for (int i = 0; i < T.D; ++i) {
          if (i == cut) continue;
          double lo = T.box[(size_t)f.node * 2 * T.D + 2 * i], hi = T.box[(size_t)f.node * 2 * T.D + 2 * i + 1];
          double x = qv[i], e = 0.0;
          if (x > hi) { double t = dsub(x, hi); e = dmul(t, t); }
          else if (x < lo) { double t = dsub(lo, x); e = dmul(t, t); }
          dis = dadd(dis, e);
          if (dis > bs) { pruned = true; break; }
        }
        if (!pruned) stack[sp++] = {farther, 0, 0.0};
      }
    }
  }
}

__global__ void k_search_kdtree(KkSearch S, const int* __restrict__ list, const int* __restrict__ count,
                                const double* __restrict__ t0, const double* __restrict__ t1,
                                const double* __restrict__ t2, const double* __restrict__ t3,
                                const double* __restrict__ ox0, const double* __restrict__ ox1,
                                const double* __restrict__ ox2, int* __restrict__ nbr, int* __restrict__ nnear,
                                int* __restrict__ status, KdHeapEntry* __restrict__ heaps, int heap_stride) {
  const int n = *count;
  const double* ts[4] = {t0, t1, t2, t3};
  const double* os[3] = {ox0, ox1, ox2};
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x) {
    const int t = list[w];
    KdHeapEntry* h = heaps + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * heap_stride;
    double x[4], q[4];
    for (int d = 0; d < S.nlag; ++d) x[d] = ts[d][t];
    if (S.aniso) rotate_pt(S.rotmat, S.ndim, x, q);
    else for (int d = 0; d < S.ndim; ++d) q[d] = x[d];
    if (S.st) q[S.nlag - 1] = dmul(x[S.nlag - 1], S.ta);
    int nsel = 0;
    int* out = nbr + (size_t)t * S.mmax;
    const int cvskip = S.cv ? t : -1;
    if (S.mode == 2) {
      const int ncand = S.K;
      kd_n_nearest(S.tree, q, ncand, h);
      kd_heapsort(h, ncand);
      int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = 1; i <= ncand; ++i) {
        int idx = h[i].idx;
        if (idx == cvskip) continue;
        if (h[i].dis > S.maxd2) continue;
        double p[3], pr[3];
        for (int d = 0; d < S.ndim; ++d) p[d] = os[d][idx];
        if (S.aniso) rotate_pt(S.rotmat, S.ndim, p, pr);
        else for (int d = 0; d < S.ndim; ++d) pr[d] = p[d];
        double dx = dsub(pr[0], q[0]);
        double dy = S.ndim > 1 ? dsub(pr[1], q[1]) : 0.0;
        double dz = S.ndim == 3 ? dsub(pr[2], q[2]) : 0.0;
        int sec = (dx < 0.0 ? 1 : 0) + (dy < 0.0 ? 2 : 0) + (dz < 0.0 ? 4 : 0);
        if (cnt[sec] < S.nmax) { cnt[sec]++; out[nsel++] = idx; }
      }
    } else {
      kd_n_nearest(S.tree, q, S.K, h);
      for (int i = 1; i <= S.K; ++i)
        if (h[i].idx != cvskip && h[i].dis <= S.maxd2) out[nsel++] = h[i].idx;
    }
    // isort, kriging_base.F90:3510-3524
    for (int i = 1; i < nsel; ++i) {
      int tmp = out[i], j = i - 1;
      while (j >= 0 && out[j] > tmp) { out[j + 1] = out[j]; --j; }
      out[j + 1] = tmp;
    }
    nnear[t] = nsel;
  }
}

// Neighbours of the targets of a sequential simulation (search_neighbors,
// simulation branch, kriging.F90:524-612, and its closing maxdist filter,
// :660-661), one thread per target.  The observation set here is the nobs
// observations followed by the targets in visiting order, and target p may
// use the observations and the targets visited before it (indices < nobs +
// p).  Candidates: with sector search (S.mode 2) the min(nobs + p, S.K)
// nearest, sorted by distance (the tree is built with sort = sector_search,
// kriging.F90:378-381) and passed through the sector filter (at most nmax
// per sector, observations and targets alike, maxdist on both); otherwise
// the nmax nearest in heap order (kdtree2_n_nearest_maxidx), or all of them
// when nmax does not cut.  Then: the simulated members beyond maxdist go,
// the simulated members co-located with an observation member (relative
// tolerance 1e-6) go, and last the observation members beyond maxdist go.
// The list is the observation members ascending, then the simulated members
// in candidate order: the reference's matrix order.  heaps holds the
// candidates plus two entries per thread; a rejected candidate is marked by
// idx = -1.
__global__ void k_search_sgsim(KkSearch S, int ntarget, int nobs, const double* __restrict__ t0,
                               const double* __restrict__ t1, const double* __restrict__ t2,
                               const double* __restrict__ ox0, const double* __restrict__ ox1,
                               const double* __restrict__ ox2, int* __restrict__ nbr, int* __restrict__ nnear,
                               KdHeapEntry* __restrict__ heaps, int heap_stride) {
  const double* ts[3] = {t0, t1, t2};
  const double* os[3] = {ox0, ox1, ox2};
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  KdHeapEntry* h = heaps + (size_t)gt * heap_stride;
  for (int p = gt; p < ntarget; p += gridDim.x * blockDim.x) {
    double x[3] = {0.0, 0.0, 0.0}, q[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < S.ndim; ++d) x[d] = ts[d][p];
    if (S.aniso) rotate_pt(S.rotmat, S.ndim, x, q);
    else for (int d = 0; d < S.ndim; ++d) q[d] = x[d];
    int* out = nbr + (size_t)p * S.mmax;
    const int lim = nobs + p;
    const bool all = S.mode != 2 && S.nmax >= lim;
    // candidates h[1 .. nc]; with all, the simulated ones only (the
    // observations are 0 .. nobs - 1)
    int nc;
    if (S.mode == 2) {
      nc = min(lim, S.K);
      kd_n_nearest(S.tree, q, nc, h, lim);
      kd_heapsort(h, nc);
      int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = 1; i <= nc; ++i) {  // apply_sector_filter, kriging.F90:1093-1154
        const int idx = h[i].idx;
        bool take = h[i].dis <= S.maxd2;
        if (take) {
          double pt[3], pr[3];
          for (int d = 0; d < S.ndim; ++d) pt[d] = os[d][idx];
          if (S.aniso) rotate_pt(S.rotmat, S.ndim, pt, pr);
          else for (int d = 0; d < S.ndim; ++d) pr[d] = pt[d];
          const double dx = dsub(pr[0], q[0]);
          const double dy = S.ndim > 1 ? dsub(pr[1], q[1]) : 0.0;
          const double dz = S.ndim == 3 ? dsub(pr[2], q[2]) : 0.0;
          const int sec = (dx < 0.0 ? 1 : 0) + (dy < 0.0 ? 2 : 0) + (dz < 0.0 ? 4 : 0);
          take = cnt[sec] < S.nmax;
          if (take) cnt[sec]++;
        }
        if (!take) h[i].idx = -1;
      }
    } else if (!all) {
      nc = S.nmax;
      kd_n_nearest(S.tree, q, nc, h, lim);
    } else {
      nc = p;
      for (int j = 0; j < p; ++j) {  // rotated_dists of the raw centres (rotation.f90:193-218)
        double diff[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < S.ndim; ++d) diff[d] = dsub(os[d][nobs + j], q[d]);
        rotate_pt(S.rotmat, S.ndim, diff, r);
        double s2 = 0.0;
        for (int d = 0; d < S.ndim; ++d) s2 = dadd(s2, dmul(r[d], r[d]));
        h[1 + j].dis = s2;
        h[1 + j].idx = nobs + j;
      }
    }
    // the simulated members: maxdist (filter_by_maxlag, kriging_base.F90:2491-2505),
    // then co-location with an observation member (kriging.F90:584-609)
    for (int i = 1; i <= nc; ++i) {
      const int idx = h[i].idx;
      if (idx < nobs) continue;  // an observation, or rejected
      if (!(h[i].dis <= S.maxd2)) { h[i].idx = -1; continue; }
      bool dup = false;
      const int no_all = all ? nobs : nc;
      for (int o = 0; o < no_all && !dup; ++o) {
        const int io = all ? o : h[1 + o].idx;
        if (io < 0 || io >= nobs) continue;
        dup = true;
        for (int d = 0; d < S.ndim; ++d) {
          const double xo = os[d][io];
          if (fabs(os[d][idx] - xo) > 1.0e-6 * (1.0 + fabs(xo))) { dup = false; break; }
        }
      }
      if (dup) h[i].idx = -1;
    }
    // the observation members within maxdist (kriging.F90:660-661), ascending
    int no = 0;
    if (all) {
      for (int i = 0; i < nobs; ++i) {
        double diff[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < S.ndim; ++d) diff[d] = dsub(os[d][i], q[d]);
        rotate_pt(S.rotmat, S.ndim, diff, r);
        double s2 = 0.0;
        for (int d = 0; d < S.ndim; ++d) s2 = dadd(s2, dmul(r[d], r[d]));
        if (s2 <= S.maxd2) out[no++] = i;
      }
    } else {
      for (int i = 1; i <= nc; ++i) {
        const int idx = h[i].idx;
        if (idx >= 0 && idx < nobs && h[i].dis <= S.maxd2) out[no++] = idx;
      }
      // isort of the observation members (kriging_base.F90:3510-3524)
      for (int i = 1; i < no; ++i) {
        int tmp = out[i], j = i - 1;
        while (j >= 0 && out[j] > tmp) { out[j + 1] = out[j]; --j; }
        out[j + 1] = tmp;
      }
    }
    int k = no;
    for (int i = 1; i <= nc; ++i)
      if (h[i].idx >= nobs) out[k++] = h[i].idx;
    nnear[p] = k;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
void launch_search_coords(const KkSearch& S, const double* const* x, double* scu, int n, cudaStream_t st) {
  k_search_coords<<<(n + 255) / 256, 256, 0, st>>>(S, x[0], x[1], x[2], x[3], scu, n);
}

void launch_grid_build(const KkGrid& g, const double* scu, int* cell_of, int* count, int* start, int* cursor,
                       double* sc, int* sidx, int* sat, int n, cudaStream_t st) {
  long long ncell = 1;
  for (int d = 0; d < g.G; ++d) ncell *= g.n[d];
  cudaMemsetAsync(count, 0, sizeof(int) * ncell, st);
  cudaMemsetAsync(cursor, 0, sizeof(int) * ncell, st);
  k_cell_count<<<(n + 255) / 256, 256, 0, st>>>(g, scu, cell_of, count, n);
  k_scan_cells<<<1, 1024, 0, st>>>(count, start, (int)ncell);
  k_scatter_points<<<(n + 255) / 256, 256, 0, st>>>(g, scu, cell_of, start, cursor, sc, sidx, n);
  k_sort_cells<<<(int)((ncell + 255) / 256), 256, 0, st>>>(g, start, sc, sidx, (int)ncell, n);
  KkGrid g2 = g;
  g2.cell_start = start;
  k_sat_fill<<<1184, 256, 0, st>>>(g2, start, sat);
  for (int ax = 0; ax < g.G; ++ax) k_sat_pass<<<592, 256, 0, st>>>(g2, sat, ax);
}

void launch_search(const KkSearch& S, int ntarget, const double* const* tx, const double* const* ox, int* nbr,
                   int* nnear, int* status, int* redo_list, int* redo_count, int nsm, cudaStream_t st) {
  int blocks = (ntarget + 3) / 4;
  int cap_blocks = nsm * 8;
  if (blocks > cap_blocks) blocks = cap_blocks;
  if (blocks < 1) blocks = 1;
  const size_t smem = 4 * search_smem_per_warp<768>(search_layout<768>(S));
  static bool attr[64] = {false};  // per device: function attributes belong to a context
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr[dev]) {
    // the largest layout; smaller ones let more CTAs share an SM
    cudaFuncSetAttribute(k_search<768>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(4 * search_smem_per_warp<768>(SearchLayout{KK_SEARCH_OCAP, KK_SEARCH_OCAP, KK_SEARCH_BCAP})));
    cudaFuncSetAttribute(k_search<768>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (dev >= 0 && dev < 64) attr[dev] = true;
  }
  k_search<768><<<blocks, 128, smem, st>>>(S, ntarget, tx[0], tx[1], tx[2], tx[3], ox[0], ox[1], ox[2], ox[3], nbr,
                                        nnear, status, redo_list, redo_count);
}

void launch_search_kdtree(const KkSearch& S, const int* list, const int* count, const double* const* tx,
                          const double* const* ox, int* nbr, int* nnear, int* status, void* heaps,
                          int heap_stride, int nthreads, cudaStream_t st) {
  int blocks = (nthreads + 127) / 128;
  k_search_kdtree<<<blocks, 128, 0, st>>>(S, list, count, tx[0], tx[1], tx[2], tx[3], ox[0], ox[1], ox[2], nbr,
                                          nnear, status, reinterpret_cast<KdHeapEntry*>(heaps), heap_stride);
}

size_t kd_heap_entry_bytes() { return sizeof(KdHeapEntry); }

void launch_search_sgsim(const KkSearch& S, int ntarget, int nobs, const double* const* tx, const double* const* ox,
                         int* nbr, int* nnear, void* heaps, int heap_stride, int nthreads, cudaStream_t st) {
  const int blocks = (nthreads + 63) / 64;
  k_search_sgsim<<<blocks, 64, 0, st>>>(S, ntarget, nobs, tx[0], tx[1], tx[2], ox[0], ox[1], ox[2], nbr, nnear,
                                       static_cast<KdHeapEntry*>(heaps), heap_stride);
}

}  // namespace kk
