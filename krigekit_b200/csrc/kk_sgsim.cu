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

}  // namespace kk
