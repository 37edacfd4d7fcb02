// Exclusive prefix sum of u32 counts on the device (bucket offsets for the
// MSM's counting sort, row pointers for the section-4 CSR build).
// Three launches: scan of 4096-entry tiles, scan of the tile sums by one
// block (looping with a running carry, so any size works), add tile bases.
// Replaces the reference's use of CUB DeviceScan::ExclusiveSum
// (include/msm_g1.cuh:774-811).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "runtime.hpp"

namespace zk {
namespace scan {
namespace {  // each translation unit gets its own kernel copies

constexpr int kTile = 4096;  // 1024 threads x 4

__device__ __forceinline__ uint32_t block_excl(uint32_t v, uint32_t* sm_warp, uint32_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t t = lane < nw ? sm_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) sm_warp[lane] = t;
  }
  __syncthreads();
  const uint32_t base = wid ? sm_warp[wid - 1] : 0;
  total = sm_warp[nw - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void __launch_bounds__(1024) k_tiles(uint32_t* __restrict__ a, size_t n,
                                                uint32_t* __restrict__ tiles) {
  __shared__ uint32_t sw[32];
  const size_t base = (size_t)blockIdx.x * kTile + threadIdx.x * 4;
  uint32_t v[4];
#pragma unroll
  for (int j = 0; j < 4; j++) v[j] = base + j < n ? a[base + j] : 0;
  uint32_t total;
  uint32_t run = block_excl(v[0] + v[1] + v[2] + v[3], sw, total);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if (base + j < n) a[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0) tiles[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_top(uint32_t* __restrict__ tiles, size_t nt) {
  __shared__ uint32_t sw[32];
  uint32_t carry = 0;
  for (size_t off = 0; off < nt; off += kTile) {
    const size_t base = off + threadIdx.x * 4;
    uint32_t v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] = base + j < nt ? tiles[base + j] : 0;
    uint32_t total;
    uint32_t run = block_excl(v[0] + v[1] + v[2] + v[3], sw, total) + carry;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (base + j < nt) tiles[base + j] = run;
      run += v[j];
    }
    carry += total;
  }
}

__global__ void k_add(uint32_t* __restrict__ a, uint32_t* __restrict__ copy, size_t n,
                      const uint32_t* __restrict__ tiles) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const uint32_t v = a[i] + tiles[i / kTile];
    a[i] = v;
    if (copy) copy[i] = v;
  }
}

inline size_t tile_count(size_t n) { return (n + kTile - 1) / kTile; }

// In-place exclusive scan of a[0..n); optional copy of the result; `tiles`
// needs tile_count(n) entries.
inline void exclusive(uint32_t* a, uint32_t* copy, size_t n, uint32_t* tiles, cudaStream_t st) {
  if (!n) return;
  const size_t nt = tile_count(n);
  k_tiles<<<(unsigned)nt, 1024, 0, st>>>(a, n, tiles);
  ZK_LAUNCHED();
  k_top<<<1, 1024, 0, st>>>(tiles, nt);
  ZK_LAUNCHED();
  k_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, copy, n, tiles);
  ZK_LAUNCHED();
}

}  // namespace
}  // namespace scan
}  // namespace zk
