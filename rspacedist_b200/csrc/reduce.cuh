// reduce.cuh -- the fixed reduction tree used for every long FP64 sum.
//
// A sum over n terms is split into chunks of 4096: lane t (0..255) of chunk c
// accumulates terms 4096c + t + 256k (k = 0..15) with fma from zero; the 256
// lane sums fold by a shuffle tree inside each warp (offsets 16,8,4,2,1) and
// a tree over the eight warp sums (offsets 4,2,1).  Chunk sums are folded by
// one 256-thread block in the same way (lane t adds chunks t, t+256, ...).
// The order depends only on n, so results are reproducible run to run and
// equal to the CPU restatement of the same tree.
#pragma once
#include <cuda_runtime.h>

namespace rs {

constexpr int kTreeLanes = 256;
constexpr int kTreePerLane = 16;
constexpr int kTreeChunk = kTreeLanes * kTreePerLane;

// Folds the per-lane values of a 256-thread block; lane 0 returns the sum.
__device__ inline double tree_fold256(double v, double* ws /* smem[8] */) {
  const int t = threadIdx.x;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, off);
  if ((t & 31) == 0) ws[t >> 5] = v;
  __syncthreads();
  double w = 0.0;
  if (t < 32) {
    w = t < 8 ? ws[t] : 0.0;
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) w = w + __shfl_down_sync(0xffffffffu, w, off);
  }
  __syncthreads();
  return w;
}

inline long tree_chunks(long n) { return (n + kTreeChunk - 1) / kTreeChunk; }

}  // namespace rs
