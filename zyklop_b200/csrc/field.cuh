// BN254 base field Fp and scalar field Fr on sm_100a.
//
// Elements are 8 x 32-bit little-endian limbs in Montgomery form with
// R = 2^256 — the same bytes as the reference's 4 x u64 limbs
// (include/fp_bn254.cuh:52-59, include/fr_bn254.cuh:40-49), so buffers cross
// the API unchanged.  Values are kept fully reduced in [0, m).
//
// Multiplication is separated Montgomery with 32-bit limbs: the 512-bit
// product comes from one level of Karatsuba over 128-bit halves (three 4 x 4
// limb schoolbook products, 96 multiply instructions instead of 128), then
// eight reduction rows against the modulus, whose limbs are PTX immediates,
// fold the low half and the high half is added at the end.  Each schoolbook
// or reduction row is two interleaved carry chains (even / odd limb
// products, mad.lo/madc.hi).  Both BN254 moduli are below 2^254, which bounds
// every intermediate (derivations at the functions).  The products are
// bit-identical to the reference's 4 x u64 CIOS fpMul / frMul
// (include/fp_bn254.cuh:187-277, include/fr_bn254.cuh:173-210): both return
// the unique a*b*R^-1 mod m in [0, m).
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

// r[0..7] = x[0..3] * y[0..3].  Row j adds x * y_j at limb j as an even
// chain (x0, x2) that also produces limb j+4 and an odd chain (x1, x3) that
// ends there: the partial product after row j is below 2^(32(j+5)), so the
// odd chain's last madc.hi never carries out.  Outputs are early-clobber:
// they are written while inputs are still being read.
__device__ __forceinline__ void mul_4x4(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3,
                                        uint32_t y0, uint32_t y1, uint32_t y2, uint32_t y3,
                                        uint32_t (&r)[8]) {
  asm("mul.lo.u32     %0, %8, %12;\n\t"
      "mul.hi.u32     %1, %8, %12;\n\t"
      "mul.lo.u32     %2, %10, %12;\n\t"
      "mul.hi.u32     %3, %10, %12;\n\t"
      "mad.lo.cc.u32  %1, %9, %12, %1;\n\t"
      "madc.hi.cc.u32 %2, %9, %12, %2;\n\t"
      "madc.lo.cc.u32 %3, %11, %12, %3;\n\t"
      "madc.hi.u32    %4, %11, %12, 0;\n\t"
      "mad.lo.cc.u32  %1, %8, %13, %1;\n\t"
      "madc.hi.cc.u32 %2, %8, %13, %2;\n\t"
      "madc.lo.cc.u32 %3, %10, %13, %3;\n\t"
      "madc.hi.cc.u32 %4, %10, %13, %4;\n\t"
      "addc.u32       %5, 0, 0;\n\t"
      "mad.lo.cc.u32  %2, %9, %13, %2;\n\t"
      "madc.hi.cc.u32 %3, %9, %13, %3;\n\t"
      "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"
      "madc.hi.u32    %5, %11, %13, %5;\n\t"
      "mad.lo.cc.u32  %2, %8, %14, %2;\n\t"
      "madc.hi.cc.u32 %3, %8, %14, %3;\n\t"
      "madc.lo.cc.u32 %4, %10, %14, %4;\n\t"
      "madc.hi.cc.u32 %5, %10, %14, %5;\n\t"
      "addc.u32       %6, 0, 0;\n\t"
      "mad.lo.cc.u32  %3, %9, %14, %3;\n\t"
      "madc.hi.cc.u32 %4, %9, %14, %4;\n\t"
      "madc.lo.cc.u32 %5, %11, %14, %5;\n\t"
      "madc.hi.u32    %6, %11, %14, %6;\n\t"
      "mad.lo.cc.u32  %3, %8, %15, %3;\n\t"
      "madc.hi.cc.u32 %4, %8, %15, %4;\n\t"
      "madc.lo.cc.u32 %5, %10, %15, %5;\n\t"
      "madc.hi.cc.u32 %6, %10, %15, %6;\n\t"
      "addc.u32       %7, 0, 0;\n\t"
      "mad.lo.cc.u32  %4, %9, %15, %4;\n\t"
      "madc.hi.cc.u32 %5, %9, %15, %5;\n\t"
      "madc.lo.cc.u32 %6, %11, %15, %6;\n\t"
      "madc.hi.u32    %7, %11, %15, %7;"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]),
        "=&r"(r[6]), "=&r"(r[7])
      : "r"(x0), "r"(x1), "r"(x2), "r"(x3), "r"(y0), "r"(y1), "r"(y2), "r"(y3));
}

// r[0..7] = x[0..3]^2: the six cross products once (positions 1-2, 3-4,
// 5-6 written directly, then x0 x2 + x1 x3 as one chain and x0 x3 as
// another), doubled, plus the four squares on the diagonal: 20 multiply
// instructions instead of 32.  The doubled cross sum is below 2^256.
__device__ __forceinline__ void sqr_4x4(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3,
                                        uint32_t (&r)[8]) {
  asm("mul.lo.u32     %1, %8, %9;\n\t"
      "mul.hi.u32     %2, %8, %9;\n\t"
      "mul.lo.u32     %3, %9, %10;\n\t"
      "mul.hi.u32     %4, %9, %10;\n\t"
      "mul.lo.u32     %5, %10, %11;\n\t"
      "mul.hi.u32     %6, %10, %11;\n\t"
      "mad.lo.cc.u32  %2, %8, %10, %2;\n\t"
      "madc.hi.cc.u32 %3, %8, %10, %3;\n\t"
      "madc.lo.cc.u32 %4, %9, %11, %4;\n\t"
      "madc.hi.cc.u32 %5, %9, %11, %5;\n\t"
      "addc.u32       %6, %6, 0;\n\t"
      "mad.lo.cc.u32  %3, %8, %11, %3;\n\t"
      "madc.hi.cc.u32 %4, %8, %11, %4;\n\t"
      "addc.cc.u32    %5, %5, 0;\n\t"
      "addc.cc.u32    %6, %6, 0;\n\t"
      "addc.u32       %7, 0, 0;\n\t"
      "add.cc.u32     %1, %1, %1;\n\t"
      "addc.cc.u32    %2, %2, %2;\n\t"
      "addc.cc.u32    %3, %3, %3;\n\t"
      "addc.cc.u32    %4, %4, %4;\n\t"
      "addc.cc.u32    %5, %5, %5;\n\t"
      "addc.cc.u32    %6, %6, %6;\n\t"
      "addc.u32       %7, %7, %7;\n\t"
      "mul.lo.u32     %0, %8, %8;\n\t"
      "mad.hi.cc.u32  %1, %8, %8, %1;\n\t"
      "madc.lo.cc.u32 %2, %9, %9, %2;\n\t"
      "madc.hi.cc.u32 %3, %9, %9, %3;\n\t"
      "madc.lo.cc.u32 %4, %10, %10, %4;\n\t"
      "madc.hi.cc.u32 %5, %10, %10, %5;\n\t"
      "madc.lo.cc.u32 %6, %11, %11, %6;\n\t"
      "madc.hi.u32    %7, %11, %11, %7;"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]),
        "=&r"(r[6]), "=&r"(r[7])
      : "r"(x0), "r"(x1), "r"(x2), "r"(x3));
}

// T[0..15] = a^2 for a < 2^255: aL^2 + 2 aL aH 2^128 + aH^2 2^256
// (20 + 32 + 20 = 72 multiply instructions instead of Karatsuba's 96).
__device__ __forceinline__ void fe_sqr_wide(const uint32_t (&a)[8], uint32_t (&T)[16]) {
  uint32_t lo[8], hi[8], x[8], x8;
  sqr_4x4(a[0], a[1], a[2], a[3], lo);
  sqr_4x4(a[4], a[5], a[6], a[7], hi);
  mul_4x4(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], x);
  asm("add.cc.u32  %0, %0, %0;\n\t"
      "addc.cc.u32 %1, %1, %1;\n\t"
      "addc.cc.u32 %2, %2, %2;\n\t"
      "addc.cc.u32 %3, %3, %3;\n\t"
      "addc.cc.u32 %4, %4, %4;\n\t"
      "addc.cc.u32 %5, %5, %5;\n\t"
      "addc.cc.u32 %6, %6, %6;\n\t"
      "addc.cc.u32 %7, %7, %7;\n\t"
      "addc.u32    %8, 0, 0;"
      : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]),
        "+r"(x[7]), "=r"(x8));
  T[0] = lo[0]; T[1] = lo[1]; T[2] = lo[2]; T[3] = lo[3];
  asm("add.cc.u32  %0, %12, %20;\n\t"
      "addc.cc.u32 %1, %13, %21;\n\t"
      "addc.cc.u32 %2, %14, %22;\n\t"
      "addc.cc.u32 %3, %15, %23;\n\t"
      "addc.cc.u32 %4, %16, %24;\n\t"
      "addc.cc.u32 %5, %17, %25;\n\t"
      "addc.cc.u32 %6, %18, %26;\n\t"
      "addc.cc.u32 %7, %19, %27;\n\t"
      "addc.cc.u32 %8, %29, %28;\n\t"
      "addc.cc.u32 %9, %30, 0;\n\t"
      "addc.cc.u32 %10, %31, 0;\n\t"
      "addc.u32    %11, %32, 0;"
      : "=r"(T[4]), "=r"(T[5]), "=r"(T[6]), "=r"(T[7]), "=r"(T[8]), "=r"(T[9]), "=r"(T[10]),
        "=r"(T[11]), "=r"(T[12]), "=r"(T[13]), "=r"(T[14]), "=r"(T[15])
      : "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(lo[7]), "r"(hi[0]), "r"(hi[1]), "r"(hi[2]),
        "r"(hi[3]), "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(x[5]), "r"(x[6]),
        "r"(x[7]), "r"(x8), "r"(hi[4]), "r"(hi[5]), "r"(hi[6]), "r"(hi[7]));
}

// T[0..15] = a * b for a, b < 2^255 (one Karatsuba level over 128-bit
// halves): T = lo + (mid - lo - hi) 2^128 + hi 2^256 with lo = aL bL,
// hi = aH bH, mid = (aL + aH)(bL + bH).  The half sums are 129-bit (carry
// bits ca, cb), so mid is the 4 x 4 product of their low limbs plus
// (ca sb + cb sa) 2^128 + ca cb 2^256, kept in nine limbs (mid < 2^258).
// Order keeps few values live: mid first, then lo folded into T[0..12], then
// hi added at 2^256 and subtracted at 2^128.  Every partial sum is a
// nonnegative part of the product (mid - lo >= hi), so no chain borrows out,
// and the largest, a b + hi 2^128 < 2^510 + 2^382, fits in 16 limbs (inputs
// near 2^256 would not: field elements and unreduced sums of two stay below
// 2^255).
__device__ __forceinline__ void fe_mul_wide(const uint32_t (&a)[8], const uint32_t (&b)[8],
                                            uint32_t (&T)[16]) {
  uint32_t sa0, sa1, sa2, sa3, ca, sb0, sb1, sb2, sb3, cb;
  asm("add.cc.u32  %0, %5, %9;\n\t"
      "addc.cc.u32 %1, %6, %10;\n\t"
      "addc.cc.u32 %2, %7, %11;\n\t"
      "addc.cc.u32 %3, %8, %12;\n\t"
      "addc.u32    %4, 0, 0;"
      : "=r"(sa0), "=r"(sa1), "=r"(sa2), "=r"(sa3), "=r"(ca)
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]));
  asm("add.cc.u32  %0, %5, %9;\n\t"
      "addc.cc.u32 %1, %6, %10;\n\t"
      "addc.cc.u32 %2, %7, %11;\n\t"
      "addc.cc.u32 %3, %8, %12;\n\t"
      "addc.u32    %4, 0, 0;"
      : "=r"(sb0), "=r"(sb1), "=r"(sb2), "=r"(sb3), "=r"(cb)
      : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
  uint32_t mid[8], m8;
  mul_4x4(sa0, sa1, sa2, sa3, sb0, sb1, sb2, sb3, mid);
  const uint32_t ma = 0u - ca, mb = 0u - cb;
  asm("add.cc.u32  %0, %0, %5;\n\t"
      "addc.cc.u32 %1, %1, %6;\n\t"
      "addc.cc.u32 %2, %2, %7;\n\t"
      "addc.cc.u32 %3, %3, %8;\n\t"
      "addc.u32    %4, 0, 0;"
      : "+r"(mid[4]), "+r"(mid[5]), "+r"(mid[6]), "+r"(mid[7]), "=r"(m8)
      : "r"(sb0 & ma), "r"(sb1 & ma), "r"(sb2 & ma), "r"(sb3 & ma));
  asm("add.cc.u32  %0, %0, %5;\n\t"
      "addc.cc.u32 %1, %1, %6;\n\t"
      "addc.cc.u32 %2, %2, %7;\n\t"
      "addc.cc.u32 %3, %3, %8;\n\t"
      "addc.u32    %4, %4, %9;"
      : "+r"(mid[4]), "+r"(mid[5]), "+r"(mid[6]), "+r"(mid[7]), "+r"(m8)
      : "r"(sa0 & mb), "r"(sa1 & mb), "r"(sa2 & mb), "r"(sa3 & mb), "r"(ca & cb));
  // lo: T[0..12] = lo + (mid - lo) 2^128
  uint32_t w[8];
  mul_4x4(a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3], w);
  asm("sub.cc.u32  %0, %0, %9;\n\t"
      "subc.cc.u32 %1, %1, %10;\n\t"
      "subc.cc.u32 %2, %2, %11;\n\t"
      "subc.cc.u32 %3, %3, %12;\n\t"
      "subc.cc.u32 %4, %4, %13;\n\t"
      "subc.cc.u32 %5, %5, %14;\n\t"
      "subc.cc.u32 %6, %6, %15;\n\t"
      "subc.cc.u32 %7, %7, %16;\n\t"
      "subc.u32    %8, %8, 0;"
      : "+r"(mid[0]), "+r"(mid[1]), "+r"(mid[2]), "+r"(mid[3]), "+r"(mid[4]), "+r"(mid[5]),
        "+r"(mid[6]), "+r"(mid[7]), "+r"(m8)
      : "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]));
  T[0] = w[0]; T[1] = w[1]; T[2] = w[2]; T[3] = w[3];
  asm("add.cc.u32  %0, %9, %13;\n\t"
      "addc.cc.u32 %1, %10, %14;\n\t"
      "addc.cc.u32 %2, %11, %15;\n\t"
      "addc.cc.u32 %3, %12, %16;\n\t"
      "addc.cc.u32 %4, %17, 0;\n\t"
      "addc.cc.u32 %5, %18, 0;\n\t"
      "addc.cc.u32 %6, %19, 0;\n\t"
      "addc.cc.u32 %7, %20, 0;\n\t"
      "addc.u32    %8, %21, 0;"
      : "=r"(T[4]), "=r"(T[5]), "=r"(T[6]), "=r"(T[7]), "=r"(T[8]), "=r"(T[9]), "=r"(T[10]),
        "=r"(T[11]), "=r"(T[12])
      : "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(mid[0]), "r"(mid[1]), "r"(mid[2]),
        "r"(mid[3]), "r"(mid[4]), "r"(mid[5]), "r"(mid[6]), "r"(mid[7]), "r"(m8));
  // hi: add at 2^256, subtract at 2^128
  mul_4x4(a[4], a[5], a[6], a[7], b[4], b[5], b[6], b[7], w);
  asm("add.cc.u32  %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %13, 0;\n\t"
      "addc.cc.u32 %6, %14, 0;\n\t"
      "addc.u32    %7, %15, 0;"
      : "+r"(T[8]), "+r"(T[9]), "+r"(T[10]), "+r"(T[11]), "+r"(T[12]), "=r"(T[13]), "=r"(T[14]),
        "=r"(T[15])
      : "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]));
  asm("sub.cc.u32  %0, %0, %12;\n\t"
      "subc.cc.u32 %1, %1, %13;\n\t"
      "subc.cc.u32 %2, %2, %14;\n\t"
      "subc.cc.u32 %3, %3, %15;\n\t"
      "subc.cc.u32 %4, %4, %16;\n\t"
      "subc.cc.u32 %5, %5, %17;\n\t"
      "subc.cc.u32 %6, %6, %18;\n\t"
      "subc.cc.u32 %7, %7, %19;\n\t"
      "subc.cc.u32 %8, %8, 0;\n\t"
      "subc.cc.u32 %9, %9, 0;\n\t"
      "subc.cc.u32 %10, %10, 0;\n\t"
      "subc.u32    %11, %11, 0;"
      : "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]), "+r"(T[8]), "+r"(T[9]), "+r"(T[10]),
        "+r"(T[11]), "+r"(T[12]), "+r"(T[13]), "+r"(T[14]), "+r"(T[15])
      : "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]));
}

// Montgomery reduction T * 2^-256 mod m for T < 2^256 * m (fully reduced
// result).  Eight rows fold the low half: starting from t = T_lo < 2^256, row i
// adds q_i * m (q_i = t_0 * (-m^-1) mod 2^32) and shifts one word down, so
// t < 2^256 + 2^32 m stays within nine words and ends at (T_lo + q m) / 2^256
// <= m.  Adding T_hi < m gives < 2m; one conditional subtraction finishes.
template <class C>
__device__ __forceinline__ fe<C> fe_redc(const uint32_t (&T)[16]) {
  uint32_t t0 = T[0], t1 = T[1], t2 = T[2], t3 = T[3], t4 = T[4], t5 = T[5], t6 = T[6], t7 = T[7];
  uint32_t t8 = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t m = t0 * C::INV;
    ZK_RED_EVEN(m);
    ZK_RED_ODD(m);
    t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = t6; t6 = t7; t7 = t8; t8 = 0;
  }
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
      : "r"(t0), "r"(t1), "r"(t2), "r"(t3), "r"(t4), "r"(t5), "r"(t6), "r"(t7), "r"(T[8]),
        "r"(T[9]), "r"(T[10]), "r"(T[11]), "r"(T[12]), "r"(T[13]), "r"(T[14]), "r"(T[15]));
  fe_reduce_once<C>(r.v);
  return r;
}

// Full product: a, b < m give T < m^2 < 2^256 * m / 4.
template <class C>
__device__ __forceinline__ fe<C> fe_mul_inline(const fe<C>& a, const fe<C>& b) {
  uint32_t T[16];
  fe_mul_wide(a.v, b.v, T);
  return fe_redc<C>(T);
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

// Out-of-line square (aL^2 + 2 aL aH 2^128 + aH^2 2^256, then REDC).
template <class C>
__device__ __noinline__ fe<C> fe_sqr_call(fe<C> a) {
  uint32_t T[16];
  fe_sqr_wide(a.v, T);
  return fe_redc<C>(T);
}

template <class C>
__device__ __forceinline__ fe<C> fe_sqr(const fe<C>& a) {
  return fe_sqr_call<C>(a);
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

// x[0..15] -= y[0..15]; the caller guarantees x >= y.
__device__ __forceinline__ void sub_16(uint32_t (&x)[16], const uint32_t (&y)[16]) {
  asm("sub.cc.u32  %0, %0, %16;\n\t"
      "subc.cc.u32 %1, %1, %17;\n\t"
      "subc.cc.u32 %2, %2, %18;\n\t"
      "subc.cc.u32 %3, %3, %19;\n\t"
      "subc.cc.u32 %4, %4, %20;\n\t"
      "subc.cc.u32 %5, %5, %21;\n\t"
      "subc.cc.u32 %6, %6, %22;\n\t"
      "subc.cc.u32 %7, %7, %23;\n\t"
      "subc.cc.u32 %8, %8, %24;\n\t"
      "subc.cc.u32 %9, %9, %25;\n\t"
      "subc.cc.u32 %10, %10, %26;\n\t"
      "subc.cc.u32 %11, %11, %27;\n\t"
      "subc.cc.u32 %12, %12, %28;\n\t"
      "subc.cc.u32 %13, %13, %29;\n\t"
      "subc.cc.u32 %14, %14, %30;\n\t"
      "subc.u32    %15, %15, %31;"
      : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]),
        "+r"(x[7]), "+r"(x[8]), "+r"(x[9]), "+r"(x[10]), "+r"(x[11]), "+r"(x[12]), "+r"(x[13]),
        "+r"(x[14]), "+r"(x[15])
      : "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]), "r"(y[4]), "r"(y[5]), "r"(y[6]), "r"(y[7]),
        "r"(y[8]), "r"(y[9]), "r"(y[10]), "r"(y[11]), "r"(y[12]), "r"(y[13]), "r"(y[14]),
        "r"(y[15]));
}

// y = x + p^2 (p the base-field modulus; every caller's x + p^2 < 2^512).
__device__ __forceinline__ void add_16_psq(const uint32_t (&x)[16], uint32_t (&y)[16]) {
  asm("add.cc.u32  %0, %16, 0x275d69b1;\n\t"
      "addc.cc.u32 %1, %17, 0x3b5458a2;\n\t"
      "addc.cc.u32 %2, %18, 0x09eac101;\n\t"
      "addc.cc.u32 %3, %19, 0xa602072d;\n\t"
      "addc.cc.u32 %4, %20, 0x6d96cadc;\n\t"
      "addc.cc.u32 %5, %21, 0x4a50189c;\n\t"
      "addc.cc.u32 %6, %22, 0x7a1242c8;\n\t"
      "addc.cc.u32 %7, %23, 0x04689e95;\n\t"
      "addc.cc.u32 %8, %24, 0x34c6b38d;\n\t"
      "addc.cc.u32 %9, %25, 0x26edfa5c;\n\t"
      "addc.cc.u32 %10, %26, 0x16375606;\n\t"
      "addc.cc.u32 %11, %27, 0xb00b8551;\n\t"
      "addc.cc.u32 %12, %28, 0x0348d21c;\n\t"
      "addc.cc.u32 %13, %29, 0x599a6f7c;\n\t"
      "addc.cc.u32 %14, %30, 0x763cbf9c;\n\t"
      "addc.u32    %15, %31, 0x0925c4b8;"
      : "=r"(y[0]), "=r"(y[1]), "=r"(y[2]), "=r"(y[3]), "=r"(y[4]), "=r"(y[5]), "=r"(y[6]),
        "=r"(y[7]), "=r"(y[8]), "=r"(y[9]), "=r"(y[10]), "=r"(y[11]), "=r"(y[12]), "=r"(y[13]),
        "=r"(y[14]), "=r"(y[15])
      : "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(x[5]), "r"(x[6]), "r"(x[7]),
        "r"(x[8]), "r"(x[9]), "r"(x[10]), "r"(x[11]), "r"(x[12]), "r"(x[13]), "r"(x[14]),
        "r"(x[15]));
}

// s = a + b without reduction (a, b < p give s < 2p < 2^255).
__device__ __forceinline__ void add_raw(const uint32_t (&a)[8], const uint32_t (&b)[8],
                                        uint32_t (&s)[8]) {
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]),
        "=r"(s[7])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
        "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
}

// (a0 + a1 u)(b0 + b1 u) with two reductions instead of three (Karatsuba over
// Fp2 on unreduced 512-bit products):
//   c0 = REDC(a0 b0 - a1 b1 + p^2),  c1 = REDC((a0 + a1)(b0 + b1) - a0 b0 - a1 b1).
// Both REDC arguments lie in [0, 2 p^2), below the 2^256 p / 2 that fe_redc
// needs (p < 2^254); adding p^2 changes nothing mod p.  Same result as three
// reduced products (the reference's fp2Mul, include/fp2_bn254.cuh:96-180).
// Out of line like fe_mul_call, so the curve formulas share one body.
static __device__ __noinline__ fp2_t fp2_mul_call(fp2_t a, fp2_t b) {
  uint32_t s[8], t[8], x[16], y[16], w[16];
  add_raw(a.c0.v, a.c1.v, s);
  add_raw(b.c0.v, b.c1.v, t);
  fe_mul_wide(s, t, x);
  fe_mul_wide(a.c0.v, b.c0.v, w);
  sub_16(x, w);
  add_16_psq(w, y);
  fe_mul_wide(a.c1.v, b.c1.v, w);
  sub_16(x, w);
  sub_16(y, w);
  return {fe_redc<FpCfg>(y), fe_redc<FpCfg>(x)};
}

__device__ __forceinline__ fp2_t operator*(const fp2_t& a, const fp2_t& b) {
  return fp2_mul_call(a, b);
}

// a b - c d in Fp with one reduction: REDC(a b + p^2 - c d), whose argument
// lies in (0, 2 p^2).  The Y coordinate of every XYZZ addition and doubling
// has this shape (Y3 = R (Q - X3) - Y1 PPP).
static __device__ __noinline__ fp_t fp_mul_sub_call(fp_t a, fp_t b, fp_t c, fp_t d) {
  uint32_t x[16], w[16];
  fe_mul_wide(a.v, b.v, w);
  add_16_psq(w, x);
  fe_mul_wide(c.v, d.v, w);
  sub_16(x, w);
  return fe_redc<FpCfg>(x);
}

__device__ __forceinline__ fp_t fe_mul_sub(const fp_t& a, const fp_t& b, const fp_t& c,
                                           const fp_t& d) {
  return fp_mul_sub_call(a, b, c, d);
}

// In Fp2 the same sharing (two reductions instead of four) keeps three
// 512-bit accumulators beside four Fp2 operands; the G2 kernels spilled and
// ran slower, so the Fp2 form stays two products and a subtraction.
__device__ __forceinline__ fp2_t fe_mul_sub(const fp2_t& a, const fp2_t& b, const fp2_t& c,
                                            const fp2_t& d) {
  return a * b - c * d;
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
