// reduce.cuh - deterministic block/grid reductions used inside kernels.
#pragma once
#include "internal.cuh"

namespace topo {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum NS values over the block; the result is valid in every thread.
template <int NS>
__device__ __forceinline__ void block_sum(double (&v)[NS]) {
  __shared__ double sh[NS][32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
#pragma unroll
  for (int s = 0; s < NS; ++s) v[s] = warp_sum(v[s]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) sh[s][wid] = v[s];
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double x = (lane < nw) ? sh[s][lane] : 0.0;
    v[s] = warp_sum(x);
  }
}

// Grid-wide deterministic reduction. Every block calls this with its thread
// values; partial sums go to red.partials[block*NS+s]. Returns true in the
// last block to arrive, where tot[] holds the grid totals summed in block
// order (so results do not depend on scheduling). The ticket is reset for the
// next kernel.
template <int NS>
__device__ __forceinline__ bool grid_sum(double (&v)[NS], RedWork red, double (&tot)[NS]) {
  __shared__ bool s_last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  block_sum<NS>(v);
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) red.partials[(size_t)bid * NS + s] = v[s];
    __threadfence();
    const unsigned t = atomicAdd(red.ticket, 1u);
    s_last = (t == nb - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double a = 0.0;
    for (unsigned b = tid; b < nb; b += nthr) a += __ldcg(red.partials + (size_t)b * NS + s);
    tot[s] = a;
  }
  block_sum<NS>(tot);
  if (tid == 0) *red.ticket = 0u;
  return true;
}

}  // namespace topo
