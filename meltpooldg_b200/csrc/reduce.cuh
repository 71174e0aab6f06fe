// Block and grid reductions. A grid reduction writes one partial per CTA;
// the last CTA to finish (elected with an atomic counter) sums the partials
// in CTA order, so the result does not depend on CTA scheduling.
#pragma once

#include <cuda_runtime.h>

namespace mpdg {

// ---------------------------------------------------------------------------
// reductions: block sum, then the last CTA sums the per-CTA partials in order
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *red /* >= 32*NV */)
{
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) red[k * 32 + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = lane < nw ? red[k * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      v[k] = s;
    }
  }
}

// Returns true in thread 0 of the last CTA, with tot[] holding the grid sums.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double *partials, unsigned *counter,
                                         double (&tot)[NV])
{
  __shared__ double red[32 * NV];
  __shared__ int is_last;
  block_sum<NV>(v, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(size_t)k * gridDim.x + blockIdx.x] = v[k];
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double s[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    s[k] = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
      s[k] += __ldcg(partials + (size_t)k * gridDim.x + i);
  }
  block_sum<NV>(s, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) tot[k] = s[k];
    *counter = 0u;
    return true;
  }
  return false;
}

}  // namespace mpdg
