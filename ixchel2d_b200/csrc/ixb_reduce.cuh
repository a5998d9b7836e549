// ixb_reduce.cuh -- deterministic block and grid reductions of the
// convergence norms (fixed summation order, so results repeat bit for bit).
#pragma once
#include <cuda_runtime.h>

#include "ixb_device.cuh"

namespace ixb {

// ---------------------------------------------------------------------------
// reductions (fixed order: deterministic run to run)
// ---------------------------------------------------------------------------
static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

static __device__ double block_sum(double v) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    s = warp_sum(s);
  }
  return s;  // valid in thread 0
}

// Publish this CTA's partial; the last CTA to arrive sums all partials in
// CTA order (every thread of that CTA loads its share in one round trip)
// and stores sqrt(sum).  Returns true in every thread of that last CTA.
static __device__ bool finish_norm(const NormSlot& ns, double block_total) {
  __shared__ int is_last;
  if (threadIdx.x == 0) {
    ns.partials[blockIdx.x] = block_total;
    __threadfence();
    const unsigned prev = atomicAdd(ns.counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(ns.partials + i);
    s = block_sum(s);
    if (threadIdx.x == 0) {
      *ns.result = sqrt(s);
      *ns.counter = 0u;
    }
  }
  return is_last != 0;
}

// Two norms of one launch with a single arrival counter (a's): every CTA
// publishes both partials, and the last to arrive sums each in CTA order
// and stores both results before returning true (one counter round trip
// instead of two, and both norms final together).
static __device__ bool finish_norm2(const NormSlot& a, double total_a, const NormSlot& b, double total_b) {
  __shared__ int is_last;
  if (threadIdx.x == 0) {
    a.partials[blockIdx.x] = total_a;
    b.partials[blockIdx.x] = total_b;
    __threadfence();
    const unsigned prev = atomicAdd(a.counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    double sa = 0.0, sb = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
      sa += __ldcg(a.partials + i);
      sb += __ldcg(b.partials + i);
    }
    sa = block_sum(sa);
    sb = block_sum(sb);
    if (threadIdx.x == 0) {
      *a.result = sqrt(sa);
      *b.result = sqrt(sb);
      *a.counter = 0u;
    }
  }
  return is_last != 0;
}

// Per-instance norms of a batched launch.  Work item `item` (of instance
// `inst`, whose items are first .. first+count-1) publishes its partial;
// the last item of the instance to arrive sums the instance's partials in
// item order and stores sqrt(sum).  Called by all threads of the CTA.

static __device__ void finish_item_norm(const BatchNorm& bn, int inst, int first, int count, int item,
                                        double block_total) {
  __shared__ int is_last;
  if (threadIdx.x == 0) {
    bn.partials[item] = block_total;
    __threadfence();
    const unsigned prev = atomicAdd(bn.counter + inst, 1u);
    is_last = (prev == (unsigned)count - 1);
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) s += __ldcg(bn.partials + first + i);
    s = block_sum(s);
    if (threadIdx.x == 0) {
      bn.result[inst] = sqrt(s);
      bn.counter[inst] = 0u;
    }
  }
  __syncthreads();
}

}  // namespace ixb
