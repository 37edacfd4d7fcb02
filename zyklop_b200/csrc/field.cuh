// BN254 base field Fp and scalar field Fr on sm_100a.
//
// Elements are 8 x 32-bit little-endian limbs in Montgomery form with
// R = 2^256 — the same bytes as the reference's 4 x u64 limbs
// (include/fp_bn254.cuh:52-59, include/fr_bn254.cuh:40-49), so buffers cross
// the API unchanged.  Values are kept fully reduced in [0, m).
//
// Multiplication is CIOS Montgomery with 32-bit limbs: each of the 8 rows is
// two interleaved carry chains (even / odd limb products, mad.lo/madc.hi)
// followed by the reduction row against the modulus, whose limbs are PTX
// immediates.  Both BN254 moduli are below 2^254, so the 9-word accumulator
// never overflows and no tenth carry word is kept (t + a*b_i + m*p < 2^288).
// Replaces the reference's 4 x u64 CIOS fpMul / frMul
// (include/fp_bn254.cuh:187-277, include/fr_bn254.cuh:173-210).
#pragma once
#include <cstdint>

namespace zk {

struct FpCfg {
  static constexpr uint32_t P0 = 0xd87cfd47u, P1 = 0x3c208c16u, P2 = 0x6871ca8du, P3 = 0x97816a91u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t INV = 0xe4866389u;  // -p^-1 mod 2^32
  static constexpr uint32_t ONE[8] = {0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u,
                                      0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
  static constexpr uint32_t R2[8] = {0x538afa89u, 0xf32cfc5bu, 0xd44501fbu, 0xb5e71911u,
                                     0x0a417ff6u, 0x47ab1effu, 0xcab8351fu, 0x06d89f71u};
};

struct FrCfg {
  static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u, P3 = 0x2833e848u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t INV = 0xefffffffu;
  static constexpr uint32_t ONE[8] = {0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u,
                                      0x7879462eu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u};
  static constexpr uint32_t R2[8] = {0xae216da7u, 0x1bb8e645u, 0xe35c59e3u, 0x53fe3ab1u,
                                     0x53bb8085u, 0x8c49833du, 0x7f4e44a5u, 0x0216d0b1u};
};

template <class C>
struct fe {
  uint32_t v[8];
};

using fp_t = fe<FpCfg>;
using fr_t = fe<FrCfg>;

// ------------------------------------------------------------------ loads
template <class C>
__device__ __forceinline__ fe<C> fe_load(const void* base, size_t idx) {
  const uint4* p = reinterpret_cast<const uint4*>(base) + 2 * idx;
  uint4 a = p[0], b = p[1];
  return fe<C>{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}
template <class C>
__device__ __forceinline__ fe<C> fe_ldg(const void* base, size_t idx) {
  const uint4* p = reinterpret_cast<const uint4*>(base) + 2 * idx;
  uint4 a = __ldg(p), b = __ldg(p + 1);
  return fe<C>{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}
template <class C>
__device__ __forceinline__ void fe_store(void* base, size_t idx, const fe<C>& x) {
  uint4* p = reinterpret_cast<uint4*>(base) + 2 * idx;
  p[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
  p[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

template <class C>
__device__ __forceinline__ fe<C> fe_zero() {
  return fe<C>{{0, 0, 0, 0, 0, 0, 0, 0}};
}
template <class C>
__device__ __forceinline__ fe<C> fe_one() {
  return fe<C>{{C::ONE[0], C::ONE[1], C::ONE[2], C::ONE[3], C::ONE[4], C::ONE[5], C::ONE[6], C::ONE[7]}};
}
template <class C>
__device__ __forceinline__ bool fe_is_zero(const fe<C>& a) {
  return (a.v[0] | a.v[1] | a.v[2] | a.v[3] | a.v[4] | a.v[5] | a.v[6] | a.v[7]) == 0;
}
template <class C>
__device__ __forceinline__ bool fe_eq(const fe<C>& a, const fe<C>& b) {
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) d |= a.v[i] ^ b.v[i];
  return d == 0;
}

// ------------------------------------------------------------- reduction
// r = t - m if t >= m else t  (t < 2m)
template <class C>
__device__ __forceinline__ void fe_reduce_once(uint32_t* t) {
  uint32_t s0, s1, s2, s3, s4, s5, s6, s7, bw;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(s0), "=r"(s1), "=r"(s2), "=r"(s3), "=r"(s4), "=r"(s5), "=r"(s6), "=r"(s7), "=r"(bw)
      : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
        "n"(C::P0), "n"(C::P1), "n"(C::P2), "n"(C::P3), "n"(C::P4), "n"(C::P5), "n"(C::P6), "n"(C::P7));
  // bw == 0xffffffff when t < m (keep t)
  t[0] = bw ? t[0] : s0;
  t[1] = bw ? t[1] : s1;
  t[2] = bw ? t[2] : s2;
  t[3] = bw ? t[3] : s3;
  t[4] = bw ? t[4] : s4;
  t[5] = bw ? t[5] : s5;
  t[6] = bw ? t[6] : s6;
  t[7] = bw ? t[7] : s7;
}

// ---------------------------------------------------------------- add/sub
template <class C>
__device__ __forceinline__ fe<C> operator+(const fe<C>& a, const fe<C>& b) {
  fe<C> r;
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
        "=r"(r.v[6]), "=r"(r.v[7])
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
        "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
        "r"(b.v[6]), "r"(b.v[7]));
  fe_reduce_once<C>(r.v);
  return r;
}

template <class C>
__device__ __forceinline__ fe<C> operator-(const fe<C>& a, const fe<C>& b) {
  fe<C> r;
  uint32_t bw;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
        "=r"(r.v[6]), "=r"(r.v[7]), "=r"(bw)
      : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
        "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
        "r"(b.v[6]), "r"(b.v[7]));
  // add m back when the subtraction borrowed
  asm("add.cc.u32  %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %5, %13;\n\t"
      "addc.cc.u32 %6, %6, %14;\n\t"
      "addc.u32    %7, %7, %15;"
      : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]),
        "+r"(r.v[6]), "+r"(r.v[7])
      : "r"(bw & C::P0), "r"(bw & C::P1), "r"(bw & C::P2), "r"(bw & C::P3), "r"(bw & C::P4),
        "r"(bw & C::P5), "r"(bw & C::P6), "r"(bw & C::P7));
  return r;
}

template <class C>
__device__ __forceinline__ fe<C> fe_neg(const fe<C>& a) {
  return fe_zero<C>() - a;
}

template <class C>
__device__ __forceinline__ fe<C> fe_dbl(const fe<C>& a) {
  return a + a;
}

// ------------------------------------------------------------------- mul
// t[0..8] += x[0..7] * y  (t8 receives the top word; never overflows here)
#define ZK_ROW_EVEN(X0, X2, X4, X6, Y)                                                      \
  asm("mad.lo.cc.u32  %0, %9, %13, %0;\n\t"                                                 \
      "madc.hi.cc.u32 %1, %9, %13, %1;\n\t"                                                 \
      "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"                                                \
      "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"                                                \
      "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"                                                \
      "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"                                                \
      "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"                                                \
      "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"                                                \
      "addc.u32       %8, %8, 0;"                                                           \
      : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), \
        "+r"(t8)                                                                            \
      : "r"(X0), "r"(X2), "r"(X4), "r"(X6), "r"(Y))
#define ZK_ROW_ODD(X1, X3, X5, X7, Y)                                                       \
  asm("mad.lo.cc.u32  %0, %8, %12, %0;\n\t"                                                 \
      "madc.hi.cc.u32 %1, %8, %12, %1;\n\t"                                                 \
      "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"                                                 \
      "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"                                                 \
      "madc.lo.cc.u32 %4, %10, %12, %4;\n\t"                                                \
      "madc.hi.cc.u32 %5, %10, %12, %5;\n\t"                                                \
      "madc.lo.cc.u32 %6, %11, %12, %6;\n\t"                                                \
      "madc.hi.u32    %7, %11, %12, %7;"                                                    \
      : "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)      \
      : "r"(X1), "r"(X3), "r"(X5), "r"(X7), "r"(Y))
// t += m * modulus, modulus limbs as immediates
#define ZK_RED_EVEN(M)                                                                      \
  asm("mad.lo.cc.u32  %0, %13, %9, %0;\n\t"                                                 \
      "madc.hi.cc.u32 %1, %13, %9, %1;\n\t"                                                 \
      "madc.lo.cc.u32 %2, %13, %10, %2;\n\t"                                                \
      "madc.hi.cc.u32 %3, %13, %10, %3;\n\t"                                                \
      "madc.lo.cc.u32 %4, %13, %11, %4;\n\t"                                                \
      "madc.hi.cc.u32 %5, %13, %11, %5;\n\t"                                                \
      "madc.lo.cc.u32 %6, %13, %12, %6;\n\t"                                                \
      "madc.hi.cc.u32 %7, %13, %12, %7;\n\t"                                                \
      "addc.u32       %8, %8, 0;"                                                           \
      : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), \
        "+r"(t8)                                                                            \
      : "n"(C::P0), "n"(C::P2), "n"(C::P4), "n"(C::P6), "r"(M))
#define ZK_RED_ODD(M)                                                                       \
  asm("mad.lo.cc.u32  %0, %12, %8, %0;\n\t"                                                 \
      "madc.hi.cc.u32 %1, %12, %8, %1;\n\t"                                                 \
      "madc.lo.cc.u32 %2, %12, %9, %2;\n\t"                                                 \
      "madc.hi.cc.u32 %3, %12, %9, %3;\n\t"                                                 \
      "madc.lo.cc.u32 %4, %12, %10, %4;\n\t"                                                \
      "madc.hi.cc.u32 %5, %12, %10, %5;\n\t"                                                \
      "madc.lo.cc.u32 %6, %12, %11, %6;\n\t"                                                \
      "madc.hi.u32    %7, %12, %11, %7;"                                                    \
      : "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)      \
      : "n"(C::P1), "n"(C::P3), "n"(C::P5), "n"(C::P7), "r"(M))

// Fully unrolled product (~300 instructions).  Kernels with one or two
// products per loop body (NTT butterflies, SpMV, elementwise passes) call it
// directly.
template <class C>
__device__ __forceinline__ fe<C> fe_mul_inline(const fe<C>& a, const fe<C>& b) {
  uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0, t8 = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t bi = b.v[i];
    ZK_ROW_EVEN(a.v[0], a.v[2], a.v[4], a.v[6], bi);
    ZK_ROW_ODD(a.v[1], a.v[3], a.v[5], a.v[7], bi);
    const uint32_t m = t0 * C::INV;
    ZK_RED_EVEN(m);
    ZK_RED_ODD(m);
    // t0 is now zero: shift one word down
    t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = t6; t6 = t7; t7 = t8; t8 = 0;
  }
  fe<C> r{{t0, t1, t2, t3, t4, t5, t6, t7}};
  fe_reduce_once<C>(r.v);
  return r;
}

// Out-of-line product (arguments and result travel in registers).  Curve
// formulas use it through operator*: inlining every product of a mixed add,
// doubling and full add made the MSM kernels several times larger than the
// instruction cache (ncu: warps stalled on instruction fetch); one shared
// body per kernel keeps the hot loop resident.
template <class C>
__device__ __noinline__ fe<C> fe_mul_call(fe<C> a, fe<C> b) {
  return fe_mul_inline(a, b);
}

template <class C>
__device__ __forceinline__ fe<C> operator*(const fe<C>& a, const fe<C>& b) {
  return fe_mul_call<C>(a, b);
}

template <class C>
__device__ __forceinline__ fe<C> fe_sqr(const fe<C>& a) {
  return a * a;
}

// Montgomery encode / decode
template <class C>
__device__ __forceinline__ fe<C> fe_to_mont(const fe<C>& a) {
  const fe<C> r2{{C::R2[0], C::R2[1], C::R2[2], C::R2[3], C::R2[4], C::R2[5], C::R2[6], C::R2[7]}};
  return a * r2;
}
template <class C>
__device__ __forceinline__ fe<C> fe_from_mont(const fe<C>& a) {
  const fe<C> one{{1, 0, 0, 0, 0, 0, 0, 0}};
  return a * one;
}

// a^e for a small public exponent given as 8 x u32 limbs (square-and-multiply)
template <class C>
__device__ __forceinline__ fe<C> fe_pow(const fe<C>& a, const uint32_t* e) {
  fe<C> acc = fe_one<C>();
  for (int i = 255; i >= 0; i--) {
    acc = fe_sqr(acc);
    if ((e[i >> 5] >> (i & 31)) & 1) acc = acc * a;
  }
  return acc;
}

// Inverse by Fermat's little theorem (a^(m-2)); inv(0) = 0 like the reference's
// Bernstein-Yang inversion (include/fp_bn254.cuh:720-773).  Only used off the
// hot loops (window results, affine conversion of single points).
template <class C>
__device__ __forceinline__ fe<C> fe_inv(const fe<C>& a) {
  const uint32_t e[8] = {C::P0 - 2u, C::P1, C::P2, C::P3, C::P4, C::P5, C::P6, C::P7};
  return fe_pow(a, e);
}

// ------------------------------------------------------------------- Fp2
// Fp2 = Fp[u]/(u^2 + 1): c0 + c1 u, stored [c0, c1] like the reference
// (include/fp2_bn254.cuh:96-180).
struct fp2_t {
  fp_t c0, c1;
};

__device__ __forceinline__ fp2_t operator+(const fp2_t& a, const fp2_t& b) { return {a.c0 + b.c0, a.c1 + b.c1}; }
__device__ __forceinline__ fp2_t operator-(const fp2_t& a, const fp2_t& b) { return {a.c0 - b.c0, a.c1 - b.c1}; }
__device__ __forceinline__ fp2_t operator*(const fp2_t& a, const fp2_t& b) {
  // Karatsuba: 3 base-field multiplications
  fp_t t0 = a.c0 * b.c0, t1 = a.c1 * b.c1;
  fp_t t2 = (a.c0 + a.c1) * (b.c0 + b.c1);
  return {t0 - t1, t2 - t0 - t1};
}
__device__ __forceinline__ fp2_t fe_sqr(const fp2_t& a) {
  // (c0 + c1)(c0 - c1) + 2 c0 c1 u: 2 multiplications
  fp_t t = a.c0 * a.c1;
  return {(a.c0 + a.c1) * (a.c0 - a.c1), t + t};
}
__device__ __forceinline__ fp2_t fe_dbl(const fp2_t& a) { return {a.c0 + a.c0, a.c1 + a.c1}; }
__device__ __forceinline__ bool fe_is_zero(const fp2_t& a) { return fe_is_zero(a.c0) && fe_is_zero(a.c1); }
__device__ __forceinline__ fp2_t fe_neg(const fp2_t& a) { return {fe_neg(a.c0), fe_neg(a.c1)}; }
__device__ __forceinline__ fp2_t fe_inv(const fp2_t& a) {
  fp_t n = a.c0 * a.c0 + a.c1 * a.c1;
  fp_t ni = fe_inv(n);
  return {a.c0 * ni, fe_neg(a.c1) * ni};
}

template <class T>
__device__ __forceinline__ T fe_zero_of();
template <>
__device__ __forceinline__ fp_t fe_zero_of<fp_t>() { return fe_zero<FpCfg>(); }
template <>
__device__ __forceinline__ fp2_t fe_zero_of<fp2_t>() { return {fe_zero<FpCfg>(), fe_zero<FpCfg>()}; }
template <class T>
__device__ __forceinline__ T fe_one_of();
template <>
__device__ __forceinline__ fp_t fe_one_of<fp_t>() { return fe_one<FpCfg>(); }
template <>
__device__ __forceinline__ fp2_t fe_one_of<fp2_t>() { return {fe_one<FpCfg>(), fe_zero<FpCfg>()}; }

}  // namespace zk
