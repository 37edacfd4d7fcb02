// Pippenger MSM on G1 / G2 for sm_100a.  See msm.hpp for the pipeline; the
// reference counterpart is include/msm_g1.cuh:271-926 and
// include/msm_g2.cuh:256-880.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "curve.cuh"
#include "host_field.hpp"
#include "msm.hpp"
#include "profile.hpp"
#include "scan.cuh"

namespace zk {
namespace {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr uint32_t kNeg = 0x80000000u;
constexpr int kRedT = 128;  // pairs per block in the bucket-reduction block passes

// ------------------------------------------------------------------ shape
struct Shape {
  size_t n;
  int c, W;              // window bits, scalar windows
  int Wk;                // bucket sets: W, or one per instance when windows share buckets
                         // (fixed bases)
  bool fixed;            // points carry precomputed 2^(c w) multiples (table of W*n records)
  int inst;              // fixed-base instances sharing the launch (1 otherwise)
  uint32_t B;            // buckets per set (2^(c-1))
  size_t entries;        // W*B + 1 scan entries (last = total)
  size_t records;        // W*n upper bound on sorted records
  int k0, k1, chunk;
  int levels;            // segmented-reduction levels (>= 1)
  size_t lvl_records[24];
  size_t lvl_blocks[24];
  int lvl_k[24];         // records per thread of each level
  size_t J;              // bucket-reduction level-1 chunks per window
};

// n: points (summed over instances for fixed-base multi-instance MSMs)
Shape make_shape(size_t n, bool g2, const MsmConfig& cfg, bool fixed = false, int inst = 1) {
  const int seg_t = g2 ? 64 : 128;
  Shape s{};
  s.n = n;
  s.inst = fixed ? inst : 1;
  s.c = cfg.c > 0 ? cfg.c : msm_default_c(n, g2);
  // the top window holds < c bits, so no carry leaves it; fixed-base MSMs
  // reduce scalars mod r first (254 bits)
  s.fixed = fixed;
  s.W = (fixed ? 254 : 256) / s.c + 1;
  s.Wk = fixed ? s.inst : s.W;
  s.B = 1u << (s.c - 1);
  s.entries = (size_t)s.Wk * s.B + 1;
  s.records = std::max<size_t>((size_t)s.W * n, 1);
  s.k0 = cfg.k0 > 0 ? cfg.k0 : msm_default_k0(n, fixed);
  s.k1 = cfg.k1;
  s.chunk = cfg.chunk > 0 ? cfg.chunk : msm_default_chunk(n, fixed, s.c);
  s.J = (s.B + s.chunk - 1) / s.chunk;
  size_t rec = s.records;
  int per_thread = s.k0;
  s.levels = 0;
  while (true) {
    // a level that fits one block spreads its records over every thread
    // (its depth is the per-thread run plus the block tree)
    if (s.levels > 0 && rec <= (size_t)seg_t * per_thread)
      per_thread = std::max<int>(2, (int)((rec + seg_t - 1) / seg_t));
    size_t per_block = (size_t)seg_t * per_thread;
    size_t blocks = (rec + per_block - 1) / per_block;
    s.lvl_records[s.levels] = rec;
    s.lvl_blocks[s.levels] = blocks;
    s.lvl_k[s.levels] = per_thread;
    s.levels++;
    if (blocks <= 1 || s.levels == 24) break;
    rec = 2 * blocks;
    per_thread = s.k1;
  }
  return s;
}

template <class F>
struct Layout {
  uint32_t* counts;   // entries (exclusive offsets after the scan), then the tile queue
  uint32_t* tileq;    // work-queue counter of the persistent level 0 (counts[entries])
  uint32_t* cursor;   // entries
  uint32_t* tiles;    // scan tile sums
  uint2* srec;        // records: (bucket key, point index | sign), one 8-byte store each
  xyzz<F>* buckets;   // W*B
  uint32_t* pkey[2];  // ping-pong partial records
  xyzz<F>* ppt[2];
  xyzz<F>* rrun[2];   // bucket-reduction (run, acc) pairs, ping-pong
  xyzz<F>* racc[2];
  xyzz<F>* outua;     // 2 * W: U_0..U_{W-1}, A_0..A_{W-1}
  size_t bytes;
};

template <class F>
Layout<F> carve(void* base, const Shape& s) {
  Layout<F> L{};
  Carver cv(base);
  L.counts = cv.take<uint32_t>(s.entries + 1);
  L.tileq = L.counts + s.entries;
  L.cursor = cv.take<uint32_t>(s.entries);
  L.tiles = cv.take<uint32_t>(scan::tile_count(s.entries) + 1);
  L.srec = cv.take<uint2>(s.records);
  L.buckets = cv.take<xyzz<F>>((size_t)s.Wk * s.B);
  size_t pmax[2] = {1, 1};
  for (int l = 1; l < s.levels; l++) pmax[l & 1] = std::max(pmax[l & 1], s.lvl_records[l]);
  for (int i = 0; i < 2; i++) {
    L.pkey[i] = cv.take<uint32_t>(pmax[i]);
    L.ppt[i] = cv.take<xyzz<F>>(pmax[i]);
  }
  const size_t j2 = (s.J + kRedT - 1) / kRedT;
  L.rrun[0] = cv.take<xyzz<F>>((size_t)s.Wk * s.J);
  L.racc[0] = cv.take<xyzz<F>>((size_t)s.Wk * s.J);
  L.rrun[1] = cv.take<xyzz<F>>((size_t)s.Wk * j2);
  L.racc[1] = cv.take<xyzz<F>>((size_t)s.Wk * j2);
  L.outua = cv.take<xyzz<F>>((size_t)s.Wk * 2);
  L.bytes = cv.off + 256;
  return L;
}

// --------------------------------------------------------------- digits
__device__ __forceinline__ void load_scalar(const uint64_t* sc, size_t i, uint32_t s[8]) {
  const uint4* p = reinterpret_cast<const uint4*>(sc) + 2 * i;
  uint4 a = __ldg(p), b = __ldg(p + 1);
  s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
  s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
}

// Pops the next c-bit window off a 256-bit scalar (s >>= c) and returns it.
__device__ __forceinline__ uint32_t pop_window(uint32_t s[8], int c) {
  const uint32_t v = s[0] & ((1u << c) - 1u);
#pragma unroll
  for (int i = 0; i < 7; i++) s[i] = __funnelshift_r(s[i], s[i + 1], c);
  s[7] >>= c;
  return v;
}

// Signed-digit recoding, digit in [-2^(c-1), 2^(c-1)]: the same digit set as
// the reference's g1_extractAllSigned (include/msm_g1.cuh:271-329).
// Returns the (window, bucket) key or kInvalid for a zero digit.
__device__ __forceinline__ uint32_t next_digit(uint32_t s[8], int c, uint32_t B, int w,
                                               uint32_t& carry, bool& neg) {
  uint32_t raw = pop_window(s, c) + carry;
  uint32_t mag;
  if (raw > B) {
    mag = (1u << c) - raw;
    carry = 1;
    neg = true;
  } else {
    mag = raw;
    carry = 0;
    neg = false;
  }
  return mag ? (uint32_t)w * B + (mag - 1) : kInvalid;
}

// k mod r for a 256-bit k (at most 5 subtractions of r < 2^254): fixed-base
// tables hold multiples of points of order r, so k and k mod r give the same
// sum, and the reduced scalar fits the tables' 254-bit window range.
__device__ __forceinline__ void reduce_mod_r(uint32_t s[8]) {
  for (int it = 0; it < 5; it++) {
    uint32_t d[8], bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
          "=r"(d[7]), "=r"(bw)
        : "r"(s[0]), "r"(s[1]), "r"(s[2]), "r"(s[3]), "r"(s[4]), "r"(s[5]), "r"(s[6]), "r"(s[7]),
          "n"(FrCfg::P0), "n"(FrCfg::P1), "n"(FrCfg::P2), "n"(FrCfg::P3), "n"(FrCfg::P4),
          "n"(FrCfg::P5), "n"(FrCfg::P6), "n"(FrCfg::P7));
    if (bw) return;  // s < r
#pragma unroll
    for (int q = 0; q < 8; q++) s[q] = d[q];
  }
}

// Scalar sources of one launch.  Windowed MSMs: one instance, key
// w * B + bucket, record value = point index.  Fixed-base MSMs: up to
// kMaxInst instances (grid.y), each with its own scalars and table; all
// windows of an instance share its bucket set, key = instance * B + bucket,
// and the record value names the instance's table entry (window w of point
// i: w * n + i).
constexpr int kMaxInst = 64;
struct ScalarSrc {
  const uint64_t* sc[kMaxInst];
  uint32_t n[kMaxInst];
};

template <bool kFixed>
__global__ void k_msm_hist(const __grid_constant__ ScalarSrc src, int c, int W, uint32_t B,
                           uint32_t* __restrict__ counts) {
  const int inst = blockIdx.y;
  const uint32_t n = src.n[inst];
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < n;
  uint32_t s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (active) load_scalar(src.sc[inst], i, s);
  if (kFixed) reduce_mod_r(s);
  const int lane = threadIdx.x & 31;
  uint32_t carry = 0;
  for (int w = 0; w < W; w++) {
    bool neg;
    uint32_t key = next_digit(s, c, B, kFixed ? inst : w, carry, neg);
    if (!active) key = kInvalid;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key != kInvalid && lane == __ffs(peers) - 1) atomicAdd(&counts[key], (uint32_t)__popc(peers));
  }
}

template <bool kFixed>
__global__ void k_msm_scatter(const __grid_constant__ ScalarSrc src, int c, int W, uint32_t B,
                              uint32_t* __restrict__ cursor, uint2* __restrict__ srec) {
  const int inst = blockIdx.y;
  const uint32_t n = src.n[inst];
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < n;
  uint32_t s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (active) load_scalar(src.sc[inst], i, s);
  if (kFixed) reduce_mod_r(s);
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  uint32_t carry = 0;
  for (int w = 0; w < W; w++) {
    bool neg;
    uint32_t key = next_digit(s, c, B, kFixed ? inst : w, carry, neg);
    if (!active) key = kInvalid;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (key != kInvalid && lane == leader) base = atomicAdd(&cursor[key], (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (key != kInvalid) {
      const uint32_t pos = base + __popc(peers & lt);
      const uint32_t idx = kFixed ? (uint32_t)((size_t)w * n + i) : (uint32_t)i;
      srec[pos] = make_uint2(key, idx | (neg ? kNeg : 0u));
    }
  }
}

// ------------------------------------------------- segmented reduction
// Node of the block-level segmented reduction: the partial sums of the first
// and last key-segments of a contiguous record range (one sum if the range
// holds a single segment).  Complete segments are written to their bucket as
// soon as they are known to be complete.  Nodes live in shared memory (one
// per thread) so the serial phase only keeps its running sum in registers.
template <class F>
struct __align__(16) SegNode {
  xyzz<F> f, l;
  uint32_t fk, lk;  // first / last key (fk == kInvalid: empty node)
  uint32_t single;
  uint32_t pad_;
};

template <class F>
constexpr int seg_threads() { return sizeof(F) == 32 ? 128 : 64; }

template <class F>
__device__ __forceinline__ void seg_merge(SegNode<F>& a, const SegNode<F>& b, xyzz<F>* buckets) {
  if (b.fk == kInvalid) return;
  if (a.fk == kInvalid) {
    a = b;
    return;
  }
  if (a.lk == b.fk) {
    const xyzz<F> j = xyzz_add(a.single ? a.f : a.l, b.f);
    if (a.single && b.single) {
      a.f = j;
    } else if (a.single) {
      a.f = j;
      a.l = b.l;
      a.single = 0;
    } else if (b.single) {
      a.l = j;
    } else {
      st_pod(&buckets[a.lk], j);
      a.l = b.l;
    }
    a.lk = b.lk;
  } else {
    if (!a.single) st_pod(&buckets[a.lk], a.l);
    if (!b.single) st_pod(&buckets[b.fk], b.f);
    a.l = b.single ? b.f : b.l;
    a.lk = b.lk;
    a.single = 0;
  }
}

// Closes the running segment `cur` (sum `acc`) of the thread's node.
template <class F>
__device__ __forceinline__ void seg_close(SegNode<F>& nd, const xyzz<F>& acc, uint32_t cur,
                                          xyzz<F>* buckets) {
  if (cur == kInvalid) return;
  if (nd.fk == kInvalid) {
    nd.fk = cur;
    nd.f = acc;
    nd.lk = cur;
    nd.single = 1;
  } else {
    // the previous last segment is now a middle segment: complete
    if (!nd.single) st_pod(&buckets[nd.lk], nd.l);
    nd.lk = cur;
    nd.l = acc;
    nd.single = 0;
  }
}

// Block tree over the per-thread nodes, then emit the block's boundary
// segments: complete ones go to their buckets, the others become partial
// records 2*block and 2*block+1 for the next level.
template <class F>
__device__ __forceinline__ void seg_block_finish(SegNode<F>* sm, uint32_t key_before,
                                                 uint32_t key_after, xyzz<F>* buckets,
                                                 uint32_t* okey, xyzz<F>* opt, size_t b) {
  constexpr int T = seg_threads<F>();
  const int t = threadIdx.x;
  __syncthreads();
  for (int s = 1; s < T; s <<= 1) {
    if ((t & (2 * s - 1)) == 0) seg_merge(sm[t], sm[t + s], buckets);
    __syncthreads();
  }
  if (t != 0) return;
  const SegNode<F>& r = sm[0];
  uint32_t hk = kInvalid, tk = kInvalid;
  if (r.fk != kInvalid) {
    const bool head = key_before == r.fk;
    if (r.single) {
      const bool tail = key_after == r.fk;
      if (!head && !tail) {
        st_pod(&buckets[r.fk], r.f);
      } else {
        hk = r.fk;
        st_pod(&opt[2 * b], r.f);
        if (tail) {
          tk = r.fk;
          st_pod(&opt[2 * b + 1], xyzz_inf<F>());
        }
      }
    } else {
      if (head) {
        hk = r.fk;
        st_pod(&opt[2 * b], r.f);
      } else {
        st_pod(&buckets[r.fk], r.f);
      }
      if (key_after == r.lk) {
        tk = r.lk;
        st_pod(&opt[2 * b + 1], r.l);
      } else {
        st_pod(&buckets[r.lk], r.l);
      }
    }
  }
  if (okey) {
    okey[2 * b] = hk;
    okey[2 * b + 1] = tk;
  }
}

// Where level 0 reads the points of its records.
template <class F>
struct PointSrc {
  const F* x;  // windowed: point i at x + i * stride, y likewise
  const F* y;
  uint32_t stride;
  int bshift;                 // fixed-base: instance = key >> bshift
  const F* table[kMaxInst];   // fixed-base: record r of an instance at table + 2 r (x, y)
};

// Level 0, one tile: records [b T K, (b + 1) T K) of the list sorted by
// (bucket key, point index | sign).
template <class F, bool kFixed>
__device__ __forceinline__ void accum0_tile(size_t b, SegNode<F>* sm,
                                            const uint2* __restrict__ srec, size_t total,
                                            const PointSrc<F>& src, int K,
                                            xyzz<F>* __restrict__ buckets,
                                            uint32_t* __restrict__ okey,
                                            xyzz<F>* __restrict__ opt) {
  constexpr int T = seg_threads<F>();
  SegNode<F>& nd = sm[threadIdx.x];
  nd.fk = nd.lk = kInvalid;
  nd.single = 1;
  const size_t bstart = b * T * K;
  const size_t bend = min(bstart + (size_t)T * K, total);
  uint32_t key_before = kInvalid, key_after = kInvalid;
  if (bstart < total) {
    key_before = bstart ? srec[bstart - 1].x : kInvalid;
    key_after = bend < total ? srec[bend].x : kInvalid;
    const size_t s = bstart + (size_t)threadIdx.x * K;
    const size_t e = min(s + K, bend);
    xyzz<F> acc = xyzz_inf<F>();
    uint32_t cur = kInvalid;
    for (size_t p = s; p < e; p++) {
      const uint2 rec = srec[p];
      const uint32_t key = rec.x;
      if (key != cur) {
        seg_close(nd, acc, cur, buckets);
        cur = key;
        acc = xyzz_inf<F>();
      }
      const uint32_t v = rec.y;
      const uint32_t idx = v & ~kNeg;
      F x, y;
      if (kFixed) {
        const F* t = src.table[key >> src.bshift];
        x = ld_pod(t + 2 * (size_t)idx);
        y = ld_pod(t + 2 * (size_t)idx + 1);
      } else {
        x = ld_pod(src.x + (size_t)idx * src.stride);
        y = ld_pod(src.y + (size_t)idx * src.stride);
      }
      if (!(fe_is_zero(x) && fe_is_zero(y))) {
        if (v & kNeg) y = fe_neg(y);
        acc = xyzz_madd(acc, x, y);
      }
    }
    seg_close(nd, acc, cur, buckets);
  }
  seg_block_finish(sm, key_before, key_after, buckets, okey, opt, b);
}

// One tile per block.  The G1 form takes 148 registers (three blocks per
// SM); capping it at 128 for four blocks spilled ~450 B a thread and ran
// ~1 % slower.  The G2 form is at the 255-register limit either way.
template <class F, bool kFixed>
__global__ void __launch_bounds__(seg_threads<F>()) k_msm_accum0(
    const uint2* __restrict__ srec, const uint32_t* __restrict__ total_p,
    const __grid_constant__ PointSrc<F> src, int K,
    xyzz<F>* __restrict__ buckets, uint32_t* __restrict__ okey, xyzz<F>* __restrict__ opt) {
  __shared__ SegNode<F> sm[seg_threads<F>()];
  accum0_tile<F, kFixed>(blockIdx.x, sm, srec, *total_p, src, K, buckets, okey, opt);
}

// Persistent form for multi-instance chains (several proofs' MSMs): a grid
// of as many blocks as the device holds at once, each claiming record tiles
// (instance, bucket range) from a device work queue until all `ntiles` are
// taken.  `queue` starts at zero.  Uncapped like the one-tile form (156
// registers, three G1 blocks per SM): fused batches ran ~2 % faster than
// with a 128-register cap.
template <class F, bool kFixed>
__global__ void __launch_bounds__(seg_threads<F>()) k_msm_accum0_queue(
    const uint2* __restrict__ srec, const uint32_t* __restrict__ total_p,
    const __grid_constant__ PointSrc<F> src, int K,
    xyzz<F>* __restrict__ buckets, uint32_t* __restrict__ okey, xyzz<F>* __restrict__ opt,
    uint32_t ntiles, uint32_t* __restrict__ queue) {
  __shared__ SegNode<F> sm[seg_threads<F>()];
  __shared__ uint32_t tile;
  const size_t total = *total_p;
  for (;;) {
    __syncthreads();  // the previous tile's outputs (thread 0) are written
    if (threadIdx.x == 0) tile = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t b = tile;
    if (b >= ntiles) return;
    accum0_tile<F, kFixed>(b, sm, srec, total, src, K, buckets, okey, opt);
  }
}

// Levels >= 1: records are (bucket key, XYZZ partial sum); kInvalid keys
// carry nothing and only ever separate different keys.
template <class F>
__global__ void __launch_bounds__(seg_threads<F>()) k_msm_accumN(
    const uint32_t* __restrict__ ikey, const xyzz<F>* __restrict__ ipt, size_t m, int K,
    xyzz<F>* __restrict__ buckets, uint32_t* __restrict__ okey, xyzz<F>* __restrict__ opt) {
  constexpr int T = seg_threads<F>();
  __shared__ SegNode<F> sm[T];
  SegNode<F>& nd = sm[threadIdx.x];
  nd.fk = nd.lk = kInvalid;
  nd.single = 1;
  const size_t bstart = (size_t)blockIdx.x * T * K;
  const size_t bend = min(bstart + (size_t)T * K, m);
  uint32_t key_before = kInvalid, key_after = kInvalid;
  if (bstart < m) {
    key_before = bstart ? ikey[bstart - 1] : kInvalid;
    key_after = bend < m ? ikey[bend] : kInvalid;
    const size_t s = bstart + (size_t)threadIdx.x * K;
    const size_t e = min(s + K, bend);
    xyzz<F> acc = xyzz_inf<F>();
    uint32_t cur = kInvalid;
    for (size_t p = s; p < e; p++) {
      const uint32_t key = ikey[p];
      if (key == kInvalid) continue;
      if (key != cur) {
        seg_close(nd, acc, cur, buckets);
        cur = key;
        acc = xyzz_inf<F>();
      }
      acc = xyzz_add(acc, ld_pod(ipt + p));
    }
    seg_close(nd, acc, cur, buckets);
  }
  seg_block_finish(sm, key_before, key_after, buckets, okey, opt, (size_t)blockIdx.x);
}

// dst[i] += src[i]: the buckets of two MSMs whose results are added, so one
// reduction yields the sum.
template <class F>
__global__ void __launch_bounds__(128) k_msm_bucket_add(xyzz<F>* __restrict__ dst,
                                                        const xyzz<F>* __restrict__ src,
                                                        size_t count) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  st_pod(&dst[i], xyzz_add(ld_pod(&dst[i]), ld_pod(&src[i])));
}

// ------------------------------------------------------ bucket reduction
// Window sums sum_b (b+1) S_b, without per-chunk scalar multiplications and
// without long serial chains above the first level.
//
// Level 1: thread per (window, chunk of L buckets) -> (run, acc) with
// run = sum S_b and acc = sum (i+1) S_{lo+i} (running sums from the top).
// Block passes: block per (window, segment of up to kRedT consecutive pairs,
// each covering 2^log_span buckets) -> run' = sum run_i and
// acc' = sum acc_i + 2^log_span * sum_i i run_i.  In the block,
// sum_i i run_i = sum_{i>=1} S_i with S_i = sum_{k>=i} run_k: a shared-memory
// suffix scan (log2 kRedT steps) and a tree reduction, so the depth is
// logarithmic.  The final pass (one segment per window) stops before the
// doublings and leaves U = sum_i i run_i and A = sum_i acc_i; the host forms
// the window sum A + 2^log_span U, where a serial doubling chain is cheap.
template <class F>
__global__ void __launch_bounds__(128) k_msm_reduce_l1(const xyzz<F>* __restrict__ buckets, int c,
                                                       int W, uint32_t B, uint32_t L, uint32_t J,
                                                       xyzz<F>* __restrict__ run_out,
                                                       xyzz<F>* __restrict__ acc_out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)W * J) return;
  const int w = (int)(t / J);
  const uint32_t j = (uint32_t)(t % J);
  const int nbits = 256 - w * c;
  const uint32_t Bw = nbits >= c ? B : (nbits <= 0 ? 1u : (1u << nbits));
  const uint32_t lo = j * L;
  xyzz<F> run = xyzz_inf<F>(), acc = xyzz_inf<F>();
  if (lo < Bw) {
    const uint32_t hi = min(lo + L, Bw);
    const xyzz<F>* bw = buckets + (size_t)w * B;
    for (uint32_t b = hi; b-- > lo;) {
      run = xyzz_add(run, ld_pod(bw + b));
      acc = xyzz_add(acc, run);
    }
  }
  st_pod(&run_out[t], run);
  st_pod(&acc_out[t], acc);
}

// block tree sum over the first `width` threads' values (a power of two;
// result valid in thread 0)
template <class F>
__device__ __forceinline__ xyzz<F> block_sum(xyzz<F> v, xyzz<F>* sm, int width) {
  const int i = threadIdx.x;
  sm[i] = v;
  __syncthreads();
  for (int s = width / 2; s > 0; s >>= 1) {
    if (i < s) sm[i] = xyzz_add(sm[i], sm[i + s]);
    __syncthreads();
  }
  const xyzz<F> r = sm[0];
  __syncthreads();
  return r;
}

// grid (segments, windows); out_u / out_a receive U and A of final passes.
// Depth: the scan and the trees run over the segment's width (the power of
// two covering its pairs), not the whole block.  When the doublings are few
// (always between passes, and in a final pass when log_span + 1 is below the
// tree depth) each thread folds 2^log_span S_i into its acc_i and one tree
// sums the result, instead of two trees and a serial doubling tail; a final
// pass then leaves U = infinity and the whole sum in A.
template <class F>
__global__ void __launch_bounds__(kRedT) k_msm_reduce_blk(
    const xyzz<F>* __restrict__ run_in, const xyzz<F>* __restrict__ acc_in, uint32_t Jin,
    int log_span, uint32_t Jout, xyzz<F>* __restrict__ run_out, xyzz<F>* __restrict__ acc_out,
    xyzz<F>* __restrict__ out_u, xyzz<F>* __restrict__ out_a) {
  __shared__ xyzz<F> sm[kRedT];
  const int w = blockIdx.y, i = threadIdx.x;
  const uint32_t idx = blockIdx.x * kRedT + i;
  const size_t base = (size_t)w * Jin;
  const uint32_t len = min((uint32_t)kRedT, Jin - blockIdx.x * kRedT);
  int width = 1, depth = 0;
  while (width < (int)len) {
    width <<= 1;
    depth++;
  }
  xyzz<F> r = idx < Jin ? ld_pod(run_in + base + idx) : xyzz_inf<F>();
  // inclusive suffix scan: r = S_i = sum_{k >= i} run_k within the segment
  sm[i] = r;
  __syncthreads();
  for (int off = 1; off < width; off <<= 1) {
    const xyzz<F> o = i + off < kRedT ? sm[i + off] : xyzz_inf<F>();
    __syncthreads();
    r = xyzz_add(r, o);
    sm[i] = r;
    __syncthreads();
  }
  const xyzz<F> total = sm[0];  // S_0 = sum of the segment's runs
  __syncthreads();
  const xyzz<F> acc = idx < Jin ? ld_pod(acc_in + base + idx) : xyzz_inf<F>();
  const size_t o = (size_t)w * Jout + blockIdx.x;
  if (Jout > 1 || log_span + 1 < depth) {
    xyzz<F> t = i >= 1 ? r : xyzz_inf<F>();
    for (int d = 0; d < log_span; d++) t = xyzz_dbl(t);
    const xyzz<F> s = block_sum<F>(xyzz_add(t, acc), sm, width);
    if (i != 0) return;
    if (Jout == 1) {
      st_pod(&out_u[w], xyzz_inf<F>());
      st_pod(&out_a[w], s);
    } else {
      st_pod(&run_out[o], total);
      st_pod(&acc_out[o], s);
    }
    return;
  }
  // final pass with many doublings: U and A separately, the host doubles U
  const xyzz<F> u = block_sum<F>(i >= 1 ? r : xyzz_inf<F>(), sm, width);
  const xyzz<F> a = block_sum<F>(acc, sm, width);
  if (i != 0) return;
  st_pod(&out_u[w], u);
  st_pod(&out_a[w], a);
}

// ------------------------------------------------------ fixed-base tables
// table record (w * n + i) = affine 2^(c w) P_i, stored (x, y) like a zkey
// section, for w < W = 254 / c + 1.  With these, all windows of a fixed-base
// MSM share one bucket set: one bucket reduction instead of W, and no
// doubling chain between windows.
//
// The affine conversions share inversions (Montgomery's trick): a thread
// doubles through kPreChunk windows, writing each multiple's X, Y into its
// table record and keeping ZZ, ZZZ and the running product of the ZZZs, then
// inverts that product once and walks back, so a chunk costs one inversion
// and ~7 products per record instead of one inversion per record.
constexpr int kPreChunk = 8;

template <class F>
__global__ void __launch_bounds__(128) k_msm_precompute(const F* __restrict__ px,
                                                        const F* __restrict__ py, uint32_t pstride,
                                                        size_t n, int c, int W,
                                                        F* __restrict__ table) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const F x = ld_pod(px + i * pstride), y = ld_pod(py + i * pstride);
  st_pod(table + 2 * i, x);
  st_pod(table + 2 * i + 1, y);
  const bool inf = fe_is_zero(x) && fe_is_zero(y);
  xyzz<F> acc;
  if (!inf) acc = xyzz<F>{x, y, fe_one_of<F>(), fe_one_of<F>()};
  for (int w0 = 1; w0 < W; w0 += kPreChunk) {
    const int cnt = min(kPreChunk, W - w0);
    F zz[kPreChunk], zzz[kPreChunk], pre[kPreChunk];
    F prod = fe_one_of<F>();
    for (int k = 0; k < cnt; k++) {
      const size_t rec = (size_t)(w0 + k) * n + i;
      if (!inf)
        for (int d = 0; d < c; d++) acc = xyzz_dbl(acc);
      // a multiple at infinity (only for points outside the order-r
      // subgroup) takes 1 in the product and is written as (0, 0)
      const bool at_inf = inf || xyzz_is_inf(acc);
      zz[k] = at_inf ? fe_zero_of<F>() : acc.zz;
      zzz[k] = at_inf ? fe_one_of<F>() : acc.zzz;
      prod = prod * zzz[k];
      pre[k] = prod;
      st_pod(table + 2 * rec, at_inf ? fe_zero_of<F>() : acc.x);
      st_pod(table + 2 * rec + 1, at_inf ? fe_zero_of<F>() : acc.y);
    }
    F inv = fe_inv(prod);  // 1 / (zzz_0 ... zzz_{cnt-1})
    for (int k = cnt - 1; k >= 0; k--) {
      const F zzzi = k ? inv * pre[k - 1] : inv;  // 1 / zzz_k
      inv = inv * zzz[k];
      if (fe_is_zero(zz[k])) continue;  // stored as (0, 0) already
      const size_t rec = (size_t)(w0 + k) * n + i;
      const F zi = zzzi * zz[k];  // ZZ / ZZZ = 1 / Z
      const F zzi = fe_sqr(zi);   // 1 / ZZ
      st_pod(table + 2 * rec, ld_pod(table + 2 * rec) * zzi);
      st_pod(table + 2 * rec + 1, ld_pod(table + 2 * rec + 1) * zzzi);
    }
  }
}


// Blocks of the persistent level 0 the device holds at once.
template <class F>
int queue_grid() {
  static const int g = [] {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_msm_accum0_queue<F, true>,
                                                      seg_threads<F>(), 0) != cudaSuccess) {
      (void)cudaGetLastError();
      per_sm = 1;
    }
    return std::max(1, per_sm) * device_sm_count();
  }();
  return g;
}

// The GPU part of one launch chain: a windowed MSM (inst = 1, points from
// ps.x / ps.y) or inst fixed-base MSMs of one window size sharing the chain
// (tables in ps.table).  n_max: the largest instance, n_total: their sum.
template <class F>
MsmResult msm_enqueue(const ScalarSrc& ss, const PointSrc<F>& ps, int inst, size_t n_max,
                      size_t n_total, void* scratch, size_t scratch_bytes, const MsmConfig& cfg,
                      cudaStream_t st, bool fixed, MsmMerge* merge_out = nullptr,
                      const MsmMerge* merge_in = nullptr) {
  constexpr bool g2 = sizeof(F) == 64;
  ZK_REQUIRE(n_max < (size_t(1) << 31), ZK_EINVAL, "msm: too many points (max 2^31 - 1)");
  ZK_REQUIRE(inst >= 1 && inst <= kMaxInst, ZK_EINVAL, "msm: 1..64 instances per launch");
  const Shape s = make_shape(n_total, g2, cfg, fixed, inst);
  ZK_REQUIRE(!fixed || (size_t)s.W * n_max < (size_t(1) << 31), ZK_EINVAL,
             "msm: fixed-base table too large (windows x points >= 2^31)");
  ZK_REQUIRE(s.c >= 4 && s.c <= 24, ZK_EINVAL, "msm: window size must be in [4, 24]");
  ZK_REQUIRE(s.records < (size_t(1) << 32) - 1, ZK_EINVAL, "msm: too many (point, window) records");
  ZK_REQUIRE(!fixed || (size_t)inst * s.B < kInvalid, ZK_EINVAL, "msm: too many buckets");
  Layout<F> L = carve<F>(scratch, s);
  ZK_REQUIRE(L.bytes <= scratch_bytes, ZK_EINVAL, "msm: scratch buffer too small");

  ZK_CUDA(cudaMemsetAsync(L.counts, 0, (s.entries + 1) * sizeof(uint32_t), st));
  ZK_CUDA(cudaMemsetAsync(L.buckets, 0, (size_t)s.Wk * s.B * sizeof(xyzz<F>), st));
  const int th = 256;
  const dim3 g((unsigned)((n_max + th - 1) / th), (unsigned)inst);
  if (n_max) {
    if (fixed)
      k_msm_hist<true><<<g, th, 0, st>>>(ss, s.c, s.W, s.B, L.counts);
    else
      k_msm_hist<false><<<g, th, 0, st>>>(ss, s.c, s.W, s.B, L.counts);
    ZK_LAUNCHED();
  }
  scan::exclusive(L.counts, L.cursor, s.entries, L.tiles, st);
  if (n_max) {
    if (fixed)
      k_msm_scatter<true><<<g, th, 0, st>>>(ss, s.c, s.W, s.B, L.cursor, L.srec);
    else
      k_msm_scatter<false><<<g, th, 0, st>>>(ss, s.c, s.W, s.B, L.cursor, L.srec);
    ZK_LAUNCHED();
  }
  const uint32_t* total_p = L.counts + (s.entries - 1);
  // level 0
  {
    uint32_t* ok = s.levels > 1 ? L.pkey[1] : nullptr;
    ProfScope prof(g2 ? kProfAccumG2 : kProfAccumG1, (double)n_total, st);
    if (fixed && inst > 1) {
      const unsigned grid = (unsigned)std::min<size_t>(s.lvl_blocks[0], queue_grid<F>());
      k_msm_accum0_queue<F, true><<<grid, seg_threads<F>(), 0, st>>>(
          L.srec, total_p, ps, s.k0, L.buckets, ok, L.ppt[1],
          (uint32_t)s.lvl_blocks[0], L.tileq);
    } else if (fixed)
      k_msm_accum0<F, true><<<(unsigned)s.lvl_blocks[0], seg_threads<F>(), 0, st>>>(
          L.srec, total_p, ps, s.k0, L.buckets, ok, L.ppt[1]);
    else
      k_msm_accum0<F, false><<<(unsigned)s.lvl_blocks[0], seg_threads<F>(), 0, st>>>(
          L.srec, total_p, ps, s.k0, L.buckets, ok, L.ppt[1]);
    ZK_LAUNCHED();
  }
  for (int l = 1; l < s.levels; l++) {
    const int in = l & 1, out = in ^ 1;
    uint32_t* ok = (l + 1 < s.levels) ? L.pkey[out] : nullptr;
    k_msm_accumN<F><<<(unsigned)s.lvl_blocks[l], seg_threads<F>(), 0, st>>>(
        L.pkey[in], L.ppt[in], s.lvl_records[l], s.lvl_k[l], L.buckets, ok, L.ppt[out]);
    ZK_LAUNCHED();
  }
  const size_t nbuckets = (size_t)s.Wk * s.B;
  if (merge_out && inst == 1) {
    // producer: the consumer reduces these buckets together with its own
    merge_out->buckets = L.buckets;
    merge_out->count = nbuckets;
    merge_out->c = s.c;
    merge_out->fixed = fixed;
    merge_out->g2 = g2;
    if (merge_out->ready) ZK_CUDA(cudaEventRecord(merge_out->ready, st));
    MsmResult none;
    none.c = s.c;
    return none;
  }
  if (merge_in) {
    ZK_REQUIRE(merge_in->buckets, ZK_EINTERNAL, "msm: merged MSM left no buckets");
    ZK_REQUIRE(inst == 1 && merge_in->count == nbuckets && merge_in->c == s.c &&
                   merge_in->fixed == fixed && merge_in->g2 == g2,
               ZK_EINTERNAL, "msm: merged bucket sets differ in shape");
    ZK_CUDA(cudaStreamWaitEvent(st, merge_in->ready, 0));
    k_msm_bucket_add<F><<<(unsigned)((nbuckets + 127) / 128), 128, 0, st>>>(
        L.buckets, static_cast<const xyzz<F>*>(merge_in->buckets), nbuckets);
    ZK_LAUNCHED();
  }
  int log_span = 0;
  {
    uint32_t J = (uint32_t)s.J;
    const uint32_t Lc = (uint32_t)s.chunk;
    while ((1u << log_span) < Lc) log_span++;
    const size_t tot = (size_t)s.Wk * J;
    k_msm_reduce_l1<F><<<(unsigned)((tot + 127) / 128), 128, 0, st>>>(
        L.buckets, s.fixed ? 0 : s.c, s.Wk, s.B, Lc, J, L.rrun[0], L.racc[0]);
    ZK_LAUNCHED();
    int cur = 0;
    for (;;) {
      const uint32_t Jout = (J + kRedT - 1) / kRedT;
      k_msm_reduce_blk<F><<<dim3(Jout, s.Wk), kRedT, 0, st>>>(
          L.rrun[cur], L.racc[cur], J, log_span, Jout, L.rrun[cur ^ 1], L.racc[cur ^ 1], L.outua,
          L.outua + s.Wk);
      ZK_LAUNCHED();
      if (Jout == 1) break;
      cur ^= 1;
      J = Jout;
      log_span += 7;  // kRedT = 2^7 pairs per block
    }
  }
  MsmResult res;
  res.d_data = L.outua;
  res.bytes = (size_t)2 * s.Wk * sizeof(xyzz<F>);
  res.windows = s.Wk;
  res.c = s.c;
  res.log_span = log_span;
  return res;
}

}  // namespace

// Defaults from autotuner runs (G1 and G2 agree within a few percent):
// window bits lg - 4 up to 2^16 points, then lg - 3 capped at 16 through
// 2^22 (a window's 2^15 buckets of XYZZ sums stay L2-resident), growing
// again by one per doubling beyond 2^22; records per accumulation thread 16
// up to 2^15 points, 32 up to 2^17, then 64 / 128 (fixed-base, below / from
// 2^20) or 128 / 256 (windowed, below / from 2^22); buckets per reduction
// thread 4 up to 2^16 points, 8 up to 2^18, then 16.  Small MSMs are bound
// by the depth of their dependent additions, so they get short per-thread
// runs.  Fixed-base sets of 2^19 or more buckets (windows of 20 bits and
// up) take 32 buckets per reduction thread: timed as whole 2^20 proofs,
// where four MSMs overlap, k0 128 / chunk 32 ran 23.3 ms against 24.8 ms
// for 64 / 16 (less reduction work beats a shorter chain there).
int msm_default_c(size_t n, bool g2) {
  (void)g2;
  int lg = 0;
  while ((size_t(1) << lg) < n) lg++;
  int c = lg <= 16 ? lg - 4 : std::min(lg - 3, 16 + std::max(0, lg - 22));
  if (c < 4) c = 4;
  if (c > 20) c = 20;
  return c;
}

int msm_effective_c(size_t n, bool g2, const MsmConfig& cfg) {
  return cfg.c > 0 ? cfg.c : msm_default_c(n, g2);
}

int msm_default_k0(size_t n, bool fixed) {
  int lg = 0;
  while ((size_t(1) << lg) < n) lg++;
  if (lg <= 15) return 16;
  if (lg <= 17) return 32;
  if (fixed) return lg <= 19 ? 64 : 128;
  return lg < 22 ? 128 : 256;
}

int msm_default_chunk(size_t n, bool fixed, int c) {
  if (fixed && c >= 20) return 32;
  int lg = 0;
  while ((size_t(1) << lg) < n) lg++;
  return lg <= 16 ? 4 : (lg <= 18 ? 8 : 16);
}

size_t msm_scratch_bytes(size_t n, bool g2, const MsmConfig& cfg) {
  const Shape s = make_shape(n, g2, cfg);
  if (g2) return carve<fp2_t>(nullptr, s).bytes;
  return carve<fp_t>(nullptr, s).bytes;
}

size_t msm_table_bytes(size_t n, bool g2, int c) {
  return (size_t)(254 / c + 1) * n * (g2 ? 128 : 64);
}

size_t msm_scratch_bytes_fixed(size_t n, bool g2, int c, const MsmConfig& cfg, int inst) {
  MsmConfig k = cfg;
  k.c = c;
  const Shape s = make_shape(n, g2, k, true, inst);
  if (g2) return carve<fp2_t>(nullptr, s).bytes;
  return carve<fp_t>(nullptr, s).bytes;
}

void msm_precompute(bool g2, const PointsView& pts, size_t n, int c, void* table, cudaStream_t st) {
  ZK_REQUIRE(c >= 4 && c <= 24, ZK_EINVAL, "msm table: window size must be in [4, 24]");
  if (!n) return;
  const int W = 254 / c + 1;
  const unsigned g = (unsigned)((n + 127) / 128);
  if (g2)
    k_msm_precompute<fp2_t><<<g, 128, 0, st>>>(reinterpret_cast<const fp2_t*>(pts.x),
                                               reinterpret_cast<const fp2_t*>(pts.y), pts.stride, n,
                                               c, W, reinterpret_cast<fp2_t*>(table));
  else
    k_msm_precompute<fp_t><<<g, 128, 0, st>>>(reinterpret_cast<const fp_t*>(pts.x),
                                              reinterpret_cast<const fp_t*>(pts.y), pts.stride, n,
                                              c, W, reinterpret_cast<fp_t*>(table));
  ZK_LAUNCHED();
}

namespace {
template <class F>
MsmResult enqueue_fixed_multi(int inst, const void* const* tables, const uint64_t* const* scalars,
                              const size_t* n, int c, void* scratch, size_t bytes,
                              const MsmConfig& cfg, cudaStream_t st, MsmMerge* merge_out = nullptr,
                              const MsmMerge* merge_in = nullptr) {
  ZK_REQUIRE(inst >= 1 && inst <= kMaxInst, ZK_EINVAL, "msm: 1..64 instances per launch");
  MsmConfig k = cfg;
  k.c = c;
  ScalarSrc ss{};
  PointSrc<F> ps{};
  ps.bshift = c - 1;
  size_t n_max = 0, n_total = 0;
  for (int i = 0; i < inst; i++) {
    ZK_REQUIRE(n[i] < (size_t(1) << 31), ZK_EINVAL, "msm: too many points (max 2^31 - 1)");
    ss.sc[i] = scalars[i];
    ss.n[i] = (uint32_t)n[i];
    ps.table[i] = reinterpret_cast<const F*>(tables[i]);
    n_max = std::max(n_max, n[i]);
    n_total += n[i];
  }
  return msm_enqueue<F>(ss, ps, inst, n_max, n_total, scratch, bytes, k, st, true, merge_out,
                       merge_in);
}

template <class F>
MsmResult enqueue_windowed(const PointsView& pts, const uint64_t* scalars, size_t n, void* scratch,
                           size_t bytes, const MsmConfig& cfg, cudaStream_t st,
                           MsmMerge* merge_out = nullptr, const MsmMerge* merge_in = nullptr) {
  ScalarSrc ss{};
  ss.sc[0] = scalars;
  ss.n[0] = (uint32_t)std::min(n, size_t(0xffffffffu));
  PointSrc<F> ps{};
  ps.x = reinterpret_cast<const F*>(pts.x);
  ps.y = reinterpret_cast<const F*>(pts.y);
  ps.stride = pts.stride;
  return msm_enqueue<F>(ss, ps, 1, n, n, scratch, bytes, cfg, st, false, merge_out, merge_in);
}
}  // namespace

MsmResult msm_enqueue_fixed(bool g2, const void* table, const uint64_t* scalars, size_t n, int c,
                            void* scratch, size_t bytes, const MsmConfig& cfg, cudaStream_t st,
                            MsmMerge* merge_out, const MsmMerge* merge_in) {
  if (g2)
    return enqueue_fixed_multi<fp2_t>(1, &table, &scalars, &n, c, scratch, bytes, cfg, st,
                                      merge_out, merge_in);
  return enqueue_fixed_multi<fp_t>(1, &table, &scalars, &n, c, scratch, bytes, cfg, st, merge_out,
                                   merge_in);
}

MsmResult msm_enqueue_fixed_multi(bool g2, int inst, const void* const* tables,
                                  const uint64_t* const* scalars, const size_t* n, int c,
                                  void* scratch, size_t bytes, const MsmConfig& cfg,
                                  cudaStream_t st) {
  if (g2) return enqueue_fixed_multi<fp2_t>(inst, tables, scalars, n, c, scratch, bytes, cfg, st);
  return enqueue_fixed_multi<fp_t>(inst, tables, scalars, n, c, scratch, bytes, cfg, st);
}

MsmResult msm_g1_enqueue(const PointsView& pts, const uint64_t* scalars, size_t n, void* scratch,
                         size_t bytes, const MsmConfig& cfg, cudaStream_t st, MsmMerge* merge_out,
                         const MsmMerge* merge_in) {
  return enqueue_windowed<fp_t>(pts, scalars, n, scratch, bytes, cfg, st, merge_out, merge_in);
}
MsmResult msm_g2_enqueue(const PointsView& pts, const uint64_t* scalars, size_t n, void* scratch,
                         size_t bytes, const MsmConfig& cfg, cudaStream_t st) {
  return enqueue_windowed<fp2_t>(pts, scalars, n, scratch, bytes, cfg, st);
}

namespace {
host::Fp fp_from_words(const uint32_t* w) {
  host::Fp r;
  memcpy(r.v, w, 32);
  return r;
}
host::Fp2 fp2_from_words(const uint32_t* q) { return host::Fp2{fp_from_words(q), fp_from_words(q + 8)}; }

// window w = A_w + 2^log_span U_w, then Horner over windows with c doublings
template <class T, class Load>
host::Xyzz<T> combine(const uint8_t* data, const MsmResult& r, size_t pt_bytes, Load load) {
  using P = host::Xyzz<T>;
  P acc = P::inf();
  for (int w = r.windows - 1; w >= 0; w--) {
    for (int i = 0; i < r.c && !acc.is_inf(); i++) acc = acc.dbl();
    P u = load(data + (size_t)w * pt_bytes);
    const P a = load(data + (size_t)(r.windows + w) * pt_bytes);
    for (int i = 0; i < r.log_span && !u.is_inf(); i++) u = u.dbl();
    acc = acc.add(u).add(a);
  }
  return acc;
}
}  // namespace

// instance i of a multi-instance result: its (U_i, A_i) as a one-window result
MsmResult gather_instance(const void* h_data, const MsmResult& r, int inst, size_t pt_bytes,
                          uint8_t* buf) {
  const uint8_t* d = reinterpret_cast<const uint8_t*>(h_data);
  memcpy(buf, d + (size_t)inst * pt_bytes, pt_bytes);
  memcpy(buf + pt_bytes, d + (size_t)(r.windows + inst) * pt_bytes, pt_bytes);
  MsmResult one = r;
  one.windows = 1;
  one.bytes = 2 * pt_bytes;
  return one;
}

bool msm_g1_combine_inst(const void* h_data, const MsmResult& r, int inst, uint64_t out[8]) {
  alignas(16) uint8_t buf[256];
  const MsmResult one = gather_instance(h_data, r, inst, 128, buf);
  return msm_g1_combine(buf, one, out);
}

bool msm_g2_combine_inst(const void* h_data, const MsmResult& r, int inst, uint64_t out[16]) {
  alignas(16) uint8_t buf[512];
  const MsmResult one = gather_instance(h_data, r, inst, 256, buf);
  return msm_g2_combine(buf, one, out);
}

host::Xyzz<host::Fp> msm_g1_combine_xyzz(const void* h_data, const MsmResult& r, int inst) {
  using P = host::Xyzz<host::Fp>;
  alignas(16) uint8_t buf[256];
  MsmResult one = r;
  if (inst >= 0) {
    one = gather_instance(h_data, r, inst, 128, buf);
    h_data = buf;
  }
  return combine<host::Fp>(reinterpret_cast<const uint8_t*>(h_data), one, 128,
                           [](const uint8_t* p) {
                             const uint32_t* q = reinterpret_cast<const uint32_t*>(p);
                             return P{fp_from_words(q), fp_from_words(q + 8), fp_from_words(q + 16),
                                      fp_from_words(q + 24)};
                           });
}

host::Xyzz<host::Fp2> msm_g2_combine_xyzz(const void* h_data, const MsmResult& r, int inst) {
  using P = host::Xyzz<host::Fp2>;
  alignas(16) uint8_t buf[512];
  MsmResult one = r;
  if (inst >= 0) {
    one = gather_instance(h_data, r, inst, 256, buf);
    h_data = buf;
  }
  return combine<host::Fp2>(reinterpret_cast<const uint8_t*>(h_data), one, 256,
                            [](const uint8_t* p) {
                              const uint32_t* q = reinterpret_cast<const uint32_t*>(p);
                              return P{fp2_from_words(q), fp2_from_words(q + 16),
                                       fp2_from_words(q + 32), fp2_from_words(q + 48)};
                            });
}

bool msm_g1_combine(const void* h_data, const MsmResult& r, uint64_t out[8]) {
  host::Fp x, y;
  const bool inf = msm_g1_combine_xyzz(h_data, r).to_affine(x, y);
  memcpy(out, x.v, 32);
  memcpy(out + 4, y.v, 32);
  return inf;
}

bool msm_g2_combine(const void* h_data, const MsmResult& r, uint64_t out[16]) {
  host::Fp2 x, y;
  const bool inf = msm_g2_combine_xyzz(h_data, r).to_affine(x, y);
  memcpy(out, x.c0.v, 32);
  memcpy(out + 4, x.c1.v, 32);
  memcpy(out + 8, y.c0.v, 32);
  memcpy(out + 12, y.c1.v, 32);
  return inf;
}

bool msm_g1_run(const PointsView& pts, const uint64_t* scalars, size_t n, DeviceBuffer& scratch,
                const MsmConfig& cfg, cudaStream_t st, uint64_t out[8]) {
  scratch.ensure(msm_scratch_bytes(n, false, cfg));
  const MsmResult r = msm_g1_enqueue(pts, scalars, n, scratch.ptr, scratch.cap, cfg, st);
  std::vector<uint8_t> h(r.bytes);
  ZK_CUDA(cudaMemcpyAsync(h.data(), r.d_data, r.bytes, cudaMemcpyDeviceToHost, st));
  ZK_CUDA(cudaStreamSynchronize(st));
  return msm_g1_combine(h.data(), r, out);
}

bool msm_g2_run(const PointsView& pts, const uint64_t* scalars, size_t n, DeviceBuffer& scratch,
                const MsmConfig& cfg, cudaStream_t st, uint64_t out[16]) {
  scratch.ensure(msm_scratch_bytes(n, true, cfg));
  const MsmResult r = msm_g2_enqueue(pts, scalars, n, scratch.ptr, scratch.cap, cfg, st);
  std::vector<uint8_t> h(r.bytes);
  ZK_CUDA(cudaMemcpyAsync(h.data(), r.d_data, r.bytes, cudaMemcpyDeviceToHost, st));
  ZK_CUDA(cudaStreamSynchronize(st));
  return msm_g2_combine(h.data(), r, out);
}

}  // namespace zk
