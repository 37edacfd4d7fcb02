// Fr NTT / INTT and the H-polynomial pipeline on sm_100a (see ntt.hpp).
// Reference counterparts: nttPrepare / twiddle builders
// (include/ntt_bn254.cuh:166-261), ntt_stockham_fwd/inv + ntt_scale
// (include/ntt_bn254.cuh:300-464), computeHPoly and its glue kernels
// (src/groth16.cu:174-183, 914-948, 1037-1128).
#include <cuda_runtime.h>

#include <vector>

#include "field.cuh"
#include "host_field.hpp"
#include "ntt.hpp"
#include "profile.hpp"
#include "runtime.hpp"

namespace zk {
namespace {

constexpr int kTile = 1024;       // elements per pass tile
constexpr int kPassThreads = 256;

using host::Fr;

// omega_{2^lg} in Montgomery form: 5^((r-1)/2^28) squared (28 - lg) times
Fr host_root(int lg) {
  uint64_t e[4];
  memcpy(e, host::FR_PARAMS.p, 32);
  e[0] -= 1;
  for (int i = 0; i < 28; i++) {
    e[0] = (e[0] >> 1) | (e[1] << 63);
    e[1] = (e[1] >> 1) | (e[2] << 63);
    e[2] = (e[2] >> 1) | (e[3] << 63);
    e[3] >>= 1;
  }
  Fr w = Fr::from_u64(5).pow(e);
  for (int i = lg; i < 28; i++) w = w.sqr();
  return w;
}

__global__ void k_tw_fill(fr_t* __restrict__ out, const fr_t* __restrict__ hi,
                          const fr_t* __restrict__ lo, int lo_bits, size_t n) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const fr_t a = fe_load<FrCfg>(hi, e >> lo_bits);
  const fr_t b = fe_load<FrCfg>(lo, e & ((size_t(1) << lo_bits) - 1));
  fe_store(out, e, a * b);
}

// arrays transformed by one pass launch (blockIdx.y): the three vectors of
// up to kMaxHBatch H polynomials of one size
constexpr int kMaxPassArrays = 3 * kMaxHBatch;
struct PassArgs {
  fr_t* in[kMaxPassArrays];
  fr_t* out[kMaxPassArrays];
};

// the vectors of up to kMaxHBatch H polynomials (blockIdx.y = polynomial)
struct HArgs {
  const fr_t* a[kMaxHBatch];
  const fr_t* b[kMaxHBatch];
  fr_t* c[kMaxHBatch];
  fr_t* h[kMaxHBatch];
};

// One pass: the stages on global index bits [lo, lo + k) for every
// sub-transform, in shared memory.  DIF runs the bits high -> low with
// butterflies (u + v, (u - v) w); DIT runs low -> high with (u + v w, u - v w).
// In both, the butterfly on bit b of pair (i, i + 2^b) uses
// w^((i mod 2^b) << (L - 1 - b)).  Stages go two at a time where they can
// (radix 4: a thread loads a quad of elements, runs both stages in registers
// and stores it back, one shared-memory round trip and one barrier for two
// stages); the butterflies of global bit 0 have w = 1 and skip the product.
struct NttSlots {
  const uint32_t* sm;
  int tile;
};

__device__ __forceinline__ fr_t sm_load(const uint32_t* sm, int tile, int slot) {
  fr_t x;
#pragma unroll
  for (int q = 0; q < 8; q++) x.v[q] = sm[q * tile + slot];
  return x;
}
__device__ __forceinline__ void sm_store(uint32_t* sm, int tile, int slot, const fr_t& x) {
#pragma unroll
  for (int q = 0; q < 8; q++) sm[q * tile + slot] = x.v[q];
}

// twiddle of the butterfly on local bit `bit` whose pair starts at local
// index j (only j mod 2^bit matters) in group g of the block
__device__ __forceinline__ fr_t ntt_twiddle(const fr_t* __restrict__ tw, int tw_shift, int L, int lo,
                                            int bit, int j, size_t gid) {
  const size_t lomask = (size_t(1) << lo) - 1;
  const size_t imod = ((size_t)(j & ((1 << bit) - 1)) << lo) | (gid & lomask);
  return fe_ldg<FrCfg>(tw, (imod << (L - 1 - (lo + bit))) << tw_shift);
}

template <bool DIT>
__device__ __forceinline__ void butterfly(fr_t& u, fr_t& v, const fr_t& w, bool trivial) {
  if (DIT) {
    if (!trivial) v = fe_mul_inline(v, w);
    const fr_t a = u + v;
    v = u - v;
    u = a;
  } else {
    const fr_t a = u + v;
    v = u - v;
    if (!trivial) v = fe_mul_inline(v, w);
    u = a;
  }
}

// Loads of values other blocks of the same launch may have written (the
// persistent H pipeline below) go around L1 (ld.global.cg); separate
// launches use plain loads.
template <bool CG>
__device__ __forceinline__ fr_t fr_load(const fr_t* base, size_t idx) {
  if (CG) {
    const uint4* q = reinterpret_cast<const uint4*>(base) + 2 * idx;
    const uint4 a = __ldcg(q), b = __ldcg(q + 1);
    return fr_t{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
  }
  return fe_load<FrCfg>(base, idx);
}

// One tile of a pass (block `blk` of the launch that runs this pass over
// the array in -> out).
template <bool DIT, bool CG>
__device__ __forceinline__ void pass_tile(const fr_t* in, fr_t* out, size_t blk,
                                          const fr_t* __restrict__ tw, int tw_shift, int L, int lo,
                                          int k, int log_g, uint32_t* sm) {
  const int tile = 1 << (k + log_g);
  const int G = 1 << log_g;
  const size_t gid0 = blk << log_g;
  const size_t lomask = (size_t(1) << lo) - 1;
  for (int e = threadIdx.x; e < tile; e += blockDim.x) {
    int j, g;
    if (lo == 0) {
      j = e & ((1 << k) - 1);
      g = e >> k;
    } else {
      g = e & (G - 1);
      j = e >> log_g;
    }
    const size_t gid = gid0 + g;
    const size_t idx = ((gid >> lo) << (lo + k)) | ((size_t)j << lo) | (gid & lomask);
    sm_store(sm, tile, (j << log_g) | g, fr_load<CG>(in, idx));
  }
  __syncthreads();
  for (int st = 0; st < k;) {
    if (st + 1 < k) {
      // two stages: DIT bits (b, b + 1) low first, DIF bits (b + 1, b) high first
      const int b = DIT ? st : (k - 2 - st);
      for (int qd = threadIdx.x; qd < tile / 4; qd += blockDim.x) {
        const int g = qd & (G - 1);
        const int jq = qd >> log_g;  // quad index over the k - 2 other bits
        const int jlo = jq & ((1 << b) - 1), jhi = jq >> b;
        const int j0 = (jhi << (b + 2)) | jlo;
        const int s00 = (j0 << log_g) | g;
        const int s01 = s00 | (1 << (b + log_g));
        const int s10 = s00 | (2 << (b + log_g));
        const int s11 = s01 | s10;
        const size_t gid = gid0 + g;
        fr_t x00 = sm_load(sm, tile, s00), x01 = sm_load(sm, tile, s01);
        fr_t x10 = sm_load(sm, tile, s10), x11 = sm_load(sm, tile, s11);
        const bool triv = lo + b == 0;  // bit 0 of the transform: w = 1
        // twiddles are loaded right before their butterflies (fewer live registers)
        auto low = [&] {
          const fr_t w = triv ? fr_t{} : ntt_twiddle(tw, tw_shift, L, lo, b, j0, gid);
          butterfly<DIT>(x00, x01, w, triv);
          butterfly<DIT>(x10, x11, w, triv);
        };
        auto high = [&] {
          butterfly<DIT>(x00, x10, ntt_twiddle(tw, tw_shift, L, lo, b + 1, j0, gid), false);
          butterfly<DIT>(x01, x11, ntt_twiddle(tw, tw_shift, L, lo, b + 1, j0 | (1 << b), gid),
                         false);
        };
        if (DIT) {
          low();
          high();
        } else {
          high();
          low();
        }
        sm_store(sm, tile, s00, x00);
        sm_store(sm, tile, s01, x01);
        sm_store(sm, tile, s10, x10);
        sm_store(sm, tile, s11, x11);
      }
      st += 2;
    } else {
      const int bit = DIT ? st : (k - 1 - st);
      for (int bf = threadIdx.x; bf < tile / 2; bf += blockDim.x) {
        const int g = bf & (G - 1);
        const int jb = bf >> log_g;
        const int jlo = jb & ((1 << bit) - 1), jhi = jb >> bit;
        const int j0 = (jhi << (bit + 1)) | jlo;
        const int s0 = (j0 << log_g) | g;
        const int s1 = s0 | (1 << (bit + log_g));
        const bool triv = lo + bit == 0;
        const fr_t w = triv ? fr_t{} : ntt_twiddle(tw, tw_shift, L, lo, bit, j0, gid0 + g);
        fr_t u = sm_load(sm, tile, s0), v = sm_load(sm, tile, s1);
        butterfly<DIT>(u, v, w, triv);
        sm_store(sm, tile, s0, u);
        sm_store(sm, tile, s1, v);
      }
      st += 1;
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < tile; e += blockDim.x) {
    int j, g;
    if (lo == 0) {
      j = e & ((1 << k) - 1);
      g = e >> k;
    } else {
      g = e & (G - 1);
      j = e >> log_g;
    }
    const size_t gid = gid0 + g;
    const size_t idx = ((gid >> lo) << (lo + k)) | ((size_t)j << lo) | (gid & lomask);
    fe_store(out, idx, sm_load(sm, tile, (j << log_g) | g));
  }
}

template <bool DIT>
__global__ void __launch_bounds__(kPassThreads) k_ntt_pass(PassArgs args, const fr_t* __restrict__ tw,
                                                           int tw_shift, int L, int lo, int k,
                                                           int log_g) {
  extern __shared__ uint32_t sm[];
  pass_tile<DIT, false>(args.in[blockIdx.y], args.out[blockIdx.y], blockIdx.x, tw, tw_shift, L, lo,
                        k, log_g, sm);
}

__global__ void k_bitrev(const fr_t* __restrict__ in, fr_t* __restrict__ out, int L, bool scale,
                         fr_t factor) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >> L) return;
  const size_t r = L ? (__brevll((unsigned long long)i) >> (64 - L)) : 0;
  fr_t x = fe_load<FrCfg>(in, i);
  if (scale) x = x * factor;
  fe_store(out, r, x);
}

// C = A * B elementwise
template <bool CG>
__device__ __forceinline__ void pointwise_elem(const fr_t* a, const fr_t* b, fr_t* c, size_t i) {
  fe_store(c, i, fr_load<CG>(a, i) * fr_load<CG>(b, i));
}

__global__ void k_pointwise_mul(const __grid_constant__ HArgs args, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i < n) pointwise_elem<false>(args.a[j], args.b[j], args.c[j], i);
}

// x[p] *= (1/N) omega_2n^rev(p) for coefficients held in bit-reversed order
// (the coset shift of src/groth16.cu:914-921 with the INTT scale folded in).
template <bool CG>
__device__ __forceinline__ void coset_elem(fr_t* a, size_t p, const fr_t* __restrict__ tw,
                                           int tw_shift, int L, const fr_t& c_even,
                                           const fr_t& c_odd) {
  const size_t e = L ? (__brevll((unsigned long long)p) >> (64 - L)) : 0;
  const size_t f = e >> 1;  // omega_2n^e = omega_2n^(e & 1) * omega_N^f
  const size_t half = L ? (size_t(1) << (L - 1)) : 1;
  fr_t t;
  if (f < half) {
    t = fe_ldg<FrCfg>(tw, f << tw_shift);
  } else {
    t = fe_neg(fe_ldg<FrCfg>(tw, (f - half) << tw_shift));  // omega_N^(N/2) = -1
  }
  fe_store(a, p, fr_load<CG>(a, p) * t * ((e & 1) ? c_odd : c_even));
}

__global__ void k_coset_scale(PassArgs args, const fr_t* __restrict__ tw, int tw_shift, int L,
                              fr_t c_even, fr_t c_odd) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >> L) return;
  coset_elem<false>(args.in[blockIdx.y], p, tw, tw_shift, L, c_even, c_odd);
}

// h = A*B - C, decoded to canonical (src/groth16.cu:935-948, 218-226), per
// polynomial
template <bool CG>
__device__ __forceinline__ void h_elem(const fr_t* a, const fr_t* b, const fr_t* c, fr_t* h, size_t i) {
  const fr_t v = fr_load<CG>(a, i) * fr_load<CG>(b, i) - fr_load<CG>(c, i);
  fe_store(h, i, fe_from_mont(v));
}

__global__ void k_h_final(const __grid_constant__ HArgs args, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i < n) h_elem<false>(args.a[j], args.b[j], args.c[j], args.h[j], i);
}

__global__ void k_fr_encode(const fr_t* __restrict__ in, fr_t* __restrict__ out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) fe_store(out, i, fe_to_mont(fe_load<FrCfg>(in, i)));
}
__global__ void k_fr_decode(const fr_t* __restrict__ in, fr_t* __restrict__ out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) fe_store(out, i, fe_from_mont(fe_load<FrCfg>(in, i)));
}

fr_t to_dev(const Fr& x) {
  fr_t r;
  memcpy(r.v, x.v, 32);
  return r;
}

// Bit ranges [lo, lo + k) covering [0, L) in near-equal pieces of at most
// maxbits (4..8) bits.
int split_passes(int L, int maxbits, int* lo, int* k) {
  const int np = (L + maxbits - 1) / maxbits;
  int at = 0;
  for (int i = 0; i < np; i++) {
    const int bits = (L - at) / (np - i);
    lo[i] = at;
    k[i] = bits;
    at += bits;
  }
  return np;
}

void run_pass(bool dit, const PassArgs& args, int count, const fr_t* tw, int tw_shift, int L, int lo,
              int k, cudaStream_t st) {
  const size_t groups = size_t(1) << (L - k);
  int log_g = 0;
  while ((1 << (log_g + 1 + k)) <= kTile && (size_t(1) << (log_g + 1)) <= groups &&
         (lo == 0 || log_g + 1 <= lo))
    log_g++;
  const size_t blocks = groups >> log_g;
  const size_t smem = (size_t)8 * 4 * (size_t(1) << (k + log_g));
  dim3 grid((unsigned)blocks, count);
  ProfScope prof(kProfNttPass, (double)count * (double)(size_t(1) << L), st);
  if (dit)
    k_ntt_pass<true><<<grid, kPassThreads, smem, st>>>(args, tw, tw_shift, L, lo, k, log_g);
  else
    k_ntt_pass<false><<<grid, kPassThreads, smem, st>>>(args, tw, tw_shift, L, lo, k, log_g);
  ZK_LAUNCHED();
}

// all DIF passes (high bit ranges first); first pass may be out of place
void dif(const PassArgs& first, const PassArgs& rest, int count, const fr_t* tw, int tw_shift, int L,
         int maxbits, cudaStream_t st) {
  int lo[8], k[8];
  const int np = split_passes(L, maxbits, lo, k);
  for (int i = np - 1; i >= 0; i--)
    run_pass(false, i == np - 1 ? first : rest, count, tw, tw_shift, L, lo[i], k[i], st);
}

void dit(const PassArgs& args, int count, const fr_t* tw, int tw_shift, int L, int maxbits,
         cudaStream_t st) {
  int lo[8], k[8];
  const int np = split_passes(L, maxbits, lo, k);
  for (int i = 0; i < np; i++) run_pass(true, args, count, tw, tw_shift, L, lo[i], k[i], st);
}

unsigned blocks_for(size_t n, int th = 256) { return (unsigned)((n + th - 1) / th); }

}  // namespace

void NttTables::ensure(int log_n, cudaStream_t st) {
  ZK_REQUIRE(log_n >= 0 && log_n <= kMaxLogN, ZK_EINVAL, "ntt: log_n out of range");
  const int need = log_n < 1 ? 1 : log_n;
  if (lmax >= need) return;
  const int lm = need;
  const size_t half = size_t(1) << (lm - 1);
  const int lo_bits = (lm - 1) < 12 ? (lm - 1) : 12;
  const size_t nlo = size_t(1) << lo_bits, nhi = half >> lo_bits;
  ZK_CUDA(cudaStreamSynchronize(st));
  fwd.ensure(half * 32);
  inv.ensure(half * 32);
  DeviceBuffer tmp;
  tmp.ensure((nlo + nhi) * 32 * 2);
  for (int dir = 0; dir < 2; dir++) {
    Fr w = host_root(lm);
    if (dir) w = w.inv();
    std::vector<Fr> lo_t(nlo), hi_t(nhi);
    lo_t[0] = Fr::one();
    for (size_t i = 1; i < nlo; i++) lo_t[i] = lo_t[i - 1] * w;
    Fr step = nlo ? lo_t[nlo - 1] * w : w;  // w^nlo
    hi_t[0] = Fr::one();
    for (size_t i = 1; i < nhi; i++) hi_t[i] = hi_t[i - 1] * step;
    char* base = tmp.as<char>() + dir * (nlo + nhi) * 32;
    // on st, so k_tw_fill is ordered after the copies: a blocking cudaMemcpy
    // from pageable memory may return before its DMA lands, and st does not
    // synchronize with the legacy default stream
    ZK_CUDA(cudaMemcpyAsync(base, hi_t.data(), nhi * 32, cudaMemcpyHostToDevice, st));
    ZK_CUDA(cudaMemcpyAsync(base + nhi * 32, lo_t.data(), nlo * 32, cudaMemcpyHostToDevice, st));
    fr_t* out = dir ? inv.as<fr_t>() : fwd.as<fr_t>();
    k_tw_fill<<<blocks_for(half), 256, 0, st>>>(out, reinterpret_cast<const fr_t*>(base),
                                                reinterpret_cast<const fr_t*>(base + nhi * 32),
                                                lo_bits, half);
    ZK_LAUNCHED();
  }
  ZK_CUDA(cudaStreamSynchronize(st));
  lmax = lm;
}

void ntt_inplace(NttTables& tw, uint64_t* a, int log_n, bool inverse, void* scratch,
                 cudaStream_t st) {
  ZK_REQUIRE(log_n >= 0 && log_n <= kMaxLogN, ZK_EINVAL, "ntt: log_n out of range");
  if (log_n == 0) return;
  tw.ensure(log_n, st);
  const int shift = tw.lmax - log_n;
  const fr_t* table = inverse ? tw.inv.as<fr_t>() : tw.fwd.as<fr_t>();
  fr_t* x = reinterpret_cast<fr_t*>(a);
  fr_t* s = reinterpret_cast<fr_t*>(scratch);
  PassArgs first{{x, nullptr, nullptr}, {s, nullptr, nullptr}};
  PassArgs rest{{s, nullptr, nullptr}, {s, nullptr, nullptr}};
  dif(first, rest, 1, table, shift, log_n, tw.pass_bits[log_n], st);
  const size_t n = size_t(1) << log_n;
  fr_t factor{};
  if (inverse) factor = to_dev(Fr::from_u64(n).inv());
  k_bitrev<<<blocks_for(n), 256, 0, st>>>(s, x, log_n, inverse, factor);
  ZK_LAUNCHED();
}

void hpoly_batch(NttTables& tw, int count, uint64_t* const* aw, uint64_t* const* bw,
                 uint64_t* const* cw, int log_n, uint64_t* const* h, cudaStream_t st) {
  ZK_REQUIRE(log_n >= 1 && log_n < kMaxLogN, ZK_EINVAL, "hpoly: log_n out of range");
  ZK_REQUIRE(count >= 1 && count <= kMaxHBatch, ZK_EINVAL, "hpoly: 1..16 polynomials per launch");
  tw.ensure(log_n, st);
  const size_t n = size_t(1) << log_n;
  const int shift = tw.lmax - log_n;
  HArgs ha{};
  PassArgs abc{};
  for (int j = 0; j < count; j++) {
    ha.a[j] = reinterpret_cast<const fr_t*>(aw[j]);
    ha.b[j] = reinterpret_cast<const fr_t*>(bw[j]);
    ha.c[j] = reinterpret_cast<fr_t*>(cw[j]);
    ha.h[j] = reinterpret_cast<fr_t*>(h[j]);
    abc.in[3 * j] = abc.out[3 * j] = reinterpret_cast<fr_t*>(aw[j]);
    abc.in[3 * j + 1] = abc.out[3 * j + 1] = reinterpret_cast<fr_t*>(bw[j]);
    abc.in[3 * j + 2] = abc.out[3 * j + 2] = reinterpret_cast<fr_t*>(cw[j]);
  }
  k_pointwise_mul<<<dim3(blocks_for(n), count), 256, 0, st>>>(ha, n);
  ZK_LAUNCHED();
  dif(abc, abc, 3 * count, tw.inv.as<fr_t>(), shift, log_n, tw.pass_bits[log_n], st);
  const Fr ninv = Fr::from_u64(n).inv();
  const Fr c_odd = ninv * host_root(log_n + 1);
  k_coset_scale<<<dim3(blocks_for(n), 3 * count), 256, 0, st>>>(abc, tw.fwd.as<fr_t>(), shift,
                                                                log_n, to_dev(ninv), to_dev(c_odd));
  ZK_LAUNCHED();
  dit(abc, 3 * count, tw.fwd.as<fr_t>(), shift, log_n, tw.pass_bits[log_n], st);
  k_h_final<<<dim3(blocks_for(n), count), 256, 0, st>>>(ha, n);
  ZK_LAUNCHED();
}

void hpoly(NttTables& tw, uint64_t* aw, uint64_t* bw, uint64_t* cw, int log_n, uint64_t* h,
           cudaStream_t st) {
  hpoly_batch(tw, 1, &aw, &bw, &cw, log_n, &h, st);
}

namespace {

struct HJobDev {
  fr_t *a, *b, *c, *h;
  fr_t c_even, c_odd;  // coset factors: 1/N and omega_2N / N
  uint32_t L, np, shift, elem_blocks;
  uint32_t pass_blocks[kMaxHPasses];  // tiles per array of pass i (bit ranges low -> high)
  uint8_t lo[kMaxHPasses], k[kMaxHPasses], log_g[kMaxHPasses];
};

struct HParams {
  const fr_t* tw_fwd;
  const fr_t* tw_inv;
  uint32_t njobs, nsteps, total;
  uint32_t off[kMaxHSteps * kMaxHJobs + 1];  // item prefix, step-major, then job
  HJobDev job[kMaxHJobs];
};

// work items of job J at step s (0: A*B, 1..np: DIF passes high -> low,
// np+1: coset, np+2..2np+1: DIT passes low -> high, 2np+2: h)
__host__ __device__ inline uint32_t h_items(const HJobDev& J, uint32_t s) {
  const uint32_t np = J.np;
  if (s == 0 || s == 2 * np + 2) return J.elem_blocks;
  if (s <= np) return 3 * J.pass_blocks[np - s];
  if (s == np + 1) return 3 * J.elem_blocks;
  if (s <= 2 * np + 1) return 3 * J.pass_blocks[s - np - 2];
  return 0;
}

constexpr long kHMaxSpins = long(1) << 25;  // x ~64 ns: about two seconds

__global__ void __launch_bounds__(kPassThreads) k_hpoly_persistent(const __grid_constant__ HParams p,
                                                                   uint32_t* sync) {
  extern __shared__ uint32_t sm[];
  __shared__ uint32_t s_job, s_step, s_local, s_stop;
  uint32_t* err = sync;
  uint32_t* queue = sync + 1;
  uint32_t* done = sync + 2;  // done[step * kMaxHJobs + job]
  const uint32_t nq = p.nsteps * p.njobs;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t t = atomicAdd(queue, 1u);
      s_stop = t >= p.total;
      if (t < p.total) {
        uint32_t lo = 0, hi = nq;  // largest q with off[q] <= t
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (p.off[mid] <= t) lo = mid;
          else hi = mid;
        }
        const uint32_t st = lo / p.njobs, jb = lo % p.njobs;
        s_step = st;
        s_job = jb;
        s_local = t - p.off[lo];
        if (st > 0) {
          // items are taken in step order, so every item of the previous
          // step was taken by a block that is running: the wait ends
          const uint32_t need = h_items(p.job[jb], st - 1);
          volatile uint32_t* d = done + (st - 1) * kMaxHJobs + jb;
          long spins = 0;
          while (*d < need) {
            if (++spins > kHMaxSpins || *(volatile uint32_t*)err) {
              atomicExch(err, 1u);
              s_stop = 1;
              break;
            }
            __nanosleep(64);
          }
          __threadfence();
        }
      }
    }
    __syncthreads();
    if (s_stop) return;
    const HJobDev& J = p.job[s_job];
    const uint32_t st = s_step, local = s_local, np = J.np;
    const size_t n = size_t(1) << J.L;
    if (st == 0) {
      const size_t i = (size_t)local * kPassThreads + threadIdx.x;
      if (i < n) pointwise_elem<true>(J.a, J.b, J.c, i);
    } else if (st <= np) {
      const uint32_t pi = np - st, nb = J.pass_blocks[pi];
      const uint32_t arr = local / nb;
      fr_t* x = arr == 0 ? J.a : (arr == 1 ? J.b : J.c);
      pass_tile<false, true>(x, x, local % nb, p.tw_inv, J.shift, J.L, J.lo[pi], J.k[pi],
                             J.log_g[pi], sm);
    } else if (st == np + 1) {
      const uint32_t arr = local / J.elem_blocks;
      fr_t* x = arr == 0 ? J.a : (arr == 1 ? J.b : J.c);
      const size_t i = (size_t)(local % J.elem_blocks) * kPassThreads + threadIdx.x;
      if (i < n) coset_elem<true>(x, i, p.tw_fwd, J.shift, J.L, J.c_even, J.c_odd);
    } else if (st <= 2 * np + 1) {
      const uint32_t pi = st - np - 2, nb = J.pass_blocks[pi];
      const uint32_t arr = local / nb;
      fr_t* x = arr == 0 ? J.a : (arr == 1 ? J.b : J.c);
      pass_tile<true, true>(x, x, local % nb, p.tw_fwd, J.shift, J.L, J.lo[pi], J.k[pi],
                            J.log_g[pi], sm);
    } else {
      const size_t i = (size_t)local * kPassThreads + threadIdx.x;
      if (i < n) h_elem<true>(J.a, J.b, J.c, J.h, i);
    }
    __syncthreads();  // every thread's writes of this item precede its count
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(done + st * kMaxHJobs + s_job, 1u);
    }
  }
}

// Blocks per SM the persistent H pipeline takes at most: it runs beside the
// MSM chains of the same group, so it leaves them room
#ifndef ZK_HPOLY_PER_SM
#define ZK_HPOLY_PER_SM 2
#endif
int hpoly_grid() {
  static const int g = [] {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hpoly_persistent, kPassThreads,
                                                      (size_t)8 * 4 * kTile) != cudaSuccess) {
      (void)cudaGetLastError();
      per_sm = 1;
    }
    per_sm = per_sm < 1 ? 1 : (per_sm > ZK_HPOLY_PER_SM ? ZK_HPOLY_PER_SM : per_sm);
    return per_sm * device_sm_count();
  }();
  return g;
}

}  // namespace

void hpoly_multi(NttTables& tw, int count, const HJob* jobs, uint32_t* sync, cudaStream_t st) {
  ZK_REQUIRE(count >= 1 && count <= kMaxHJobs, ZK_EINVAL, "hpoly: 1..32 jobs per launch");
  ZK_REQUIRE(sync, ZK_EINVAL, "hpoly: no synchronization words");
  int lmax = 1;
  for (int j = 0; j < count; j++) {
    ZK_REQUIRE(jobs[j].log_n >= 1 && jobs[j].log_n < kMaxLogN, ZK_EINVAL, "hpoly: log_n out of range");
    lmax = jobs[j].log_n > lmax ? jobs[j].log_n : lmax;
  }
  tw.ensure(lmax, st);
  static_assert(sizeof(HParams) < 32000, "kernel parameters must fit the 32 KB limit");
  HParams p{};
  p.tw_fwd = tw.fwd.as<fr_t>();
  p.tw_inv = tw.inv.as<fr_t>();
  p.njobs = (uint32_t)count;
  uint32_t nsteps = 0;
  double units = 0;
  for (int j = 0; j < count; j++) {
    HJobDev& J = p.job[j];
    const int L = jobs[j].log_n;
    const size_t n = size_t(1) << L;
    J.a = reinterpret_cast<fr_t*>(jobs[j].aw);
    J.b = reinterpret_cast<fr_t*>(jobs[j].bw);
    J.c = reinterpret_cast<fr_t*>(jobs[j].cw);
    J.h = reinterpret_cast<fr_t*>(jobs[j].h);
    J.L = (uint32_t)L;
    J.shift = (uint32_t)(tw.lmax - L);
    J.elem_blocks = (uint32_t)((n + kPassThreads - 1) / kPassThreads);
    int lo[8], k[8];
    const int np = split_passes(L, tw.pass_bits[L], lo, k);
    ZK_REQUIRE(np <= kMaxHPasses, ZK_EINVAL, "hpoly: too many passes");
    J.np = (uint32_t)np;
    for (int i = 0; i < np; i++) {
      const size_t groups = size_t(1) << (L - k[i]);
      int log_g = 0;
      while ((1 << (log_g + 1 + k[i])) <= kTile && (size_t(1) << (log_g + 1)) <= groups &&
             (lo[i] == 0 || log_g + 1 <= lo[i]))
        log_g++;
      J.lo[i] = (uint8_t)lo[i];
      J.k[i] = (uint8_t)k[i];
      J.log_g[i] = (uint8_t)log_g;
      J.pass_blocks[i] = (uint32_t)(groups >> log_g);
    }
    const Fr ninv = Fr::from_u64(n).inv();
    J.c_even = to_dev(ninv);
    J.c_odd = to_dev(ninv * host_root(L + 1));
    nsteps = nsteps > 2u * np + 3u ? nsteps : 2u * np + 3u;
    units += 6.0 * np * (double)n;
  }
  p.nsteps = nsteps;
  uint32_t total = 0;
  for (uint32_t st = 0; st < nsteps; st++)
    for (int j = 0; j < count; j++) {
      p.off[st * p.njobs + j] = total;
      total += h_items(p.job[j], st);
    }
  p.off[nsteps * p.njobs] = total;
  p.total = total;
  ZK_CUDA(cudaMemsetAsync(sync, 0, kHSyncWords * sizeof(uint32_t), st));
  const unsigned grid = (unsigned)(total < (uint32_t)hpoly_grid() ? total : hpoly_grid());
  ProfScope prof(kProfNttPass, units, st);
  k_hpoly_persistent<<<grid, kPassThreads, (size_t)8 * 4 * kTile, st>>>(p, sync);
  ZK_LAUNCHED();
}

void fr_encode(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t st) {
  if (!n) return;
  k_fr_encode<<<blocks_for(n), 256, 0, st>>>(reinterpret_cast<const fr_t*>(in),
                                             reinterpret_cast<fr_t*>(out), n);
  ZK_LAUNCHED();
}
void fr_decode(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t st) {
  if (!n) return;
  k_fr_decode<<<blocks_for(n), 256, 0, st>>>(reinterpret_cast<const fr_t*>(in),
                                             reinterpret_cast<fr_t*>(out), n);
  ZK_LAUNCHED();
}

}  // namespace zk
