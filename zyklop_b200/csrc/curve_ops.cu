// Batched fixed-base scalar multiplication k_i * G for the standard G1 / G2
// generators, with affine Montgomery output.  Used to build synthetic CRS
// points and seeded MSM bases on the device (the reference has no setup code:
// its CRS comes from snarkjs).
#include <cuda_runtime.h>

#include "context.hpp"
#include "curve.cuh"

namespace zk {
namespace {

__device__ __forceinline__ fp_t fp_c(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                     uint32_t a4, uint32_t a5, uint32_t a6, uint32_t a7) {
  return fp_t{{a0, a1, a2, a3, a4, a5, a6, a7}};
}

// generators in Montgomery form: G1 = (1, 2); G2 = the standard BN254
// generator (x = x0 + x1 u, y = y0 + y1 u)
__device__ __forceinline__ affine<fp_t> g1_gen() {
  return {fp_c(0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u, 0x7879462cu, 0x666ea36fu,
               0x9a07df2fu, 0x0e0a77c1u),
          fp_c(0x8b1e1b3au, 0xa6ba871bu, 0xeb8e167bu, 0x14f1d651u, 0xf0f28c58u, 0xccdd46deu,
               0x340fbe5eu, 0x1c14ef83u)};
}
__device__ __forceinline__ affine<fp2_t> g2_gen() {
  fp2_t x{fp_c(0x02bc2026u, 0x8e83b5d1u, 0x497b0172u, 0xdceb1935u, 0x97811adfu, 0xfbb82647u,
               0xaf96503bu, 0x19573841u),
          fp_c(0xa84c6140u, 0xafb4737du, 0x5802d8c4u, 0x6043dd5au, 0x52a02f86u, 0x09e950fcu,
               0x3aea7b6bu, 0x14fef083u)};
  fp2_t y{fp_c(0x886be9f6u, 0x619dfa9du, 0xf59e9b78u, 0xfe7fd297u, 0x231b7dfeu, 0xff9e1a62u,
               0xae9e4206u, 0x28fd7eebu),
          fp_c(0xc71856eeu, 0x64095b56u, 0x327d3cbbu, 0xdc57f922u, 0x33351076u, 0x55f935beu,
               0x93fd6482u, 0x0da4a0e6u)};
  return {x, y};
}

template <class F>
__device__ __forceinline__ affine<F> gen();
template <>
__device__ __forceinline__ affine<fp_t> gen<fp_t>() { return g1_gen(); }
template <>
__device__ __forceinline__ affine<fp2_t> gen<fp2_t>() { return g2_gen(); }

// k * G by left-to-right double-and-add over the 256-bit canonical scalar
template <class F>
__global__ void __launch_bounds__(128) k_mul_gen(const uint64_t* __restrict__ scalars, size_t n,
                                                 F* __restrict__ ox, F* __restrict__ oy) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4* sp = reinterpret_cast<const uint4*>(scalars) + 2 * i;
  const uint4 a = sp[0], b = sp[1];
  const uint32_t s[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  const affine<F> g = gen<F>();
  xyzz<F> acc = xyzz_inf<F>();
  for (int bit = 255; bit >= 0; bit--) {
    acc = xyzz_dbl(acc);
    if ((s[bit >> 5] >> (bit & 31)) & 1) acc = xyzz_madd(acc, g.x, g.y);
  }
  const affine<F> r = xyzz_to_affine(acc);
  st_pod(ox + i, r.x);
  st_pod(oy + i, r.y);
}

}  // namespace

void mul_generator(int group, const uint64_t* scalars, size_t n, uint64_t* px, uint64_t* py,
                   cudaStream_t st) {
  if (!n) return;
  const unsigned g = (unsigned)((n + 127) / 128);
  if (group == 1)
    k_mul_gen<fp_t><<<g, 128, 0, st>>>(scalars, n, reinterpret_cast<fp_t*>(px),
                                       reinterpret_cast<fp_t*>(py));
  else
    k_mul_gen<fp2_t><<<g, 128, 0, st>>>(scalars, n, reinterpret_cast<fp2_t*>(px),
                                        reinterpret_cast<fp2_t*>(py));
  ZK_LAUNCHED();
}

}  // namespace zk
