// kk_sgsim.cu -- the sequential part of a sequential Gaussian simulation.
//
// The reference simulates the targets one after another along a random path
// (solve_base with nsim > 0, kriging_base.F90:2055-2181): target p is kriged
// from the observations and the targets simulated before it, then drawn.  Its
// neighbour set, its kriging weights and its conditional variance depend on
// positions only, so they are computed for every target at once by the
// search and solve kernels (weights kept as in the weight store).  What stays
// sequential is the value: a dot product over the neighbours, some of which
// are earlier simulated values.  The host sorts the targets into dependency
// levels (a target's level is one above the highest level among its simulated
// neighbours); the targets of one level are independent and this kernel
// finishes them together, all realisations at once.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "kk_kernels.h"

namespace kk {

__device__ __forceinline__ double sim_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// estimate_block_base + sim_draw_base (kriging_base.F90:3446-3495,
// 2320-2327) for one variable: the observation part with its simple-kriging
// mean term, then the simulated part, then the draw; bounds last.  One warp
// per target, lanes over the neighbour rows.
__global__ void __launch_bounds__(256) k_sgsim_level(const __grid_constant__ SimParams S, const int* __restrict__ list,
                                                     int count) {
  const int lane = threadIdx.x & 31;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < count; it += nwarp) {
    const int p = __ldg(&list[it]);
    const int n = __ldg(&S.nnear[p]);
    const int* nb = S.nbr + (size_t)p * S.mmax;
    const double* w = S.w + (size_t)p * S.wstride;
    const double var = __ldg(&S.var[p]);
    const int target = __ldg(&S.path[p]) - 1;
    double avg = 0.0, tw = 0.0;
    for (int i = lane; i < n; i += 32) {
      const int idx = __ldg(&nb[i]);
      if (idx < S.nobs) {
        const double wt = __ldg(&w[i]);
        avg = fma(__ldg(&S.z[idx]), wt, avg);
        tw += wt;
      }
    }
    avg = sim_warp_sum(avg);
    tw = sim_warp_sum(tw);
    if (S.sk && S.sk_mean != 0.0) avg = avg + (1.0 - tw) * S.sk_mean;
    const double L = sqrt(var > 0.0 ? var : 0.0);
    for (int s = 0; s < S.nsim; ++s) {
      double dp = 0.0;
      for (int i = lane; i < n; i += 32) {
        const int idx = __ldg(&nb[i]);
        if (idx >= S.nobs) dp = fma(S.sim[(size_t)s * S.nb + (idx - S.nobs)], __ldg(&w[i]), dp);
      }
      dp = sim_warp_sum(dp);
      double v = avg + dp;
      v = v + L * __ldg(&S.sample[(size_t)p * S.nsim + s]);
      if (v < S.lo) v = S.lo;
      if (v > S.hi) v = S.hi;
      if (!(var == var) || n == 0) v = __longlong_as_double(0x7ff8000000000000ll);
      if (lane == 0) {
        S.sim[(size_t)s * S.nb + p] = v;
        S.out[(size_t)target * S.nsim + s] = v;
      }
    }
  }
}

void launch_sgsim_level(const SimParams& S, const int* list, int count, int nsm, cudaStream_t st) {
  if (count <= 0) return;
  const int blocks = std::max(1, std::min((count + 7) / 8, nsm * 8));
  k_sgsim_level<<<blocks, 256, 0, st>>>(S, list, count);
}

// Bounded wait of one position's publication: about 0.5 s at most.
#define KK_SIM_SPIN_LIMIT (1 << 22)

__device__ __forceinline__ int sim_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void sim_st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// All levels in one launch.  Warps pull positions in level order from a work
// counter.  A position's simulated neighbours sit at lower levels, so they
// were pulled earlier by warps that are running (the launch is cooperative:
// every block is resident), and the warp waits for each of them to be
// published (done[q], release / acquire at GPU scope; the values are read
// through L2).  A wait that runs past KK_SIM_SPIN_LIMIT sets *err, writes
// NaN and publishes anyway, so no warp waits on it for ever; the host then
// redoes the draws level by level.  Same arithmetic, in the same order, as
// k_sgsim_level.
__global__ void __launch_bounds__(256) k_sgsim_flow(const __grid_constant__ SimParams S, const int* __restrict__ order,
                                                    int count, int* __restrict__ done, int* __restrict__ work,
                                                    int* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(work, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= count) break;
    const int p = __ldg(&order[it]);
    const int n = __ldg(&S.nnear[p]);
    const int* nb = S.nbr + (size_t)p * S.mmax;
    const double* w = S.w + (size_t)p * S.wstride;
    const double var = __ldg(&S.var[p]);
    const int target = __ldg(&S.path[p]) - 1;
    double avg = 0.0, tw = 0.0;
    for (int i = lane; i < n; i += 32) {
      const int idx = __ldg(&nb[i]);
      if (idx < S.nobs) {
        const double wt = __ldg(&w[i]);
        avg = fma(__ldg(&S.z[idx]), wt, avg);
        tw += wt;
      }
    }
    avg = sim_warp_sum(avg);
    tw = sim_warp_sum(tw);
    if (S.sk && S.sk_mean != 0.0) avg = avg + (1.0 - tw) * S.sk_mean;
    const double L = sqrt(var > 0.0 ? var : 0.0);
    // wait for the simulated neighbours this lane reads below
    bool late = false;
    for (int i = lane; i < n; i += 32) {
      const int idx = __ldg(&nb[i]);
      if (idx >= S.nobs) {
        const int* f = done + (idx - S.nobs);
        int spins = 0;
        while (sim_ld_acquire(f) == 0) {
          if (++spins > KK_SIM_SPIN_LIMIT) { late = true; break; }
          __nanosleep(64);
        }
      }
    }
    late = __any_sync(0xffffffffu, late);
    for (int s = 0; s < S.nsim; ++s) {
      double dp = 0.0;
      for (int i = lane; i < n; i += 32) {
        const int idx = __ldg(&nb[i]);
        if (idx >= S.nobs) dp = fma(__ldcg(&S.sim[(size_t)s * S.nb + (idx - S.nobs)]), __ldg(&w[i]), dp);
      }
      dp = sim_warp_sum(dp);
      double v = avg + dp;
      v = v + L * __ldg(&S.sample[(size_t)p * S.nsim + s]);
      if (v < S.lo) v = S.lo;
      if (v > S.hi) v = S.hi;
      if (!(var == var) || n == 0 || late) v = __longlong_as_double(0x7ff8000000000000ll);
      if (lane == 0) {
        S.sim[(size_t)s * S.nb + p] = v;
        S.out[(size_t)target * S.nsim + s] = v;
      }
    }
    if (lane == 0) {
      if (late) atomicExch(err, 1);
      sim_st_release(done + p, 1);
    }
    __syncwarp();
  }
}

// One cooperative launch of k_sgsim_flow over the level-ordered positions;
// done (nb ints), work and err (one int each) must be zero.  False when the
// device cannot take a cooperative launch (the caller then launches the
// levels one by one).
bool launch_sgsim_flow(const SimParams& S, const int* order, int count, int* done, int* work, int* err, int nsm,
                       cudaStream_t st) {
  if (count <= 0) return true;
  int dev = 0, coop = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return false;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sgsim_flow, 256, 0) != cudaSuccess || per_sm < 1)
    return false;
  const int blocks = std::max(1, std::min(per_sm * nsm, (count + 7) / 8));
  void* args[] = {const_cast<SimParams*>(&S), const_cast<int**>(&order), &count, &done, &work, &err};
  return cudaLaunchCooperativeKernel((const void*)k_sgsim_flow, dim3(blocks), dim3(256), args, 0, st) == cudaSuccess;
}

}  // namespace kk
