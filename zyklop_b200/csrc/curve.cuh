// Short-Weierstrass y^2 = x^3 + b (a = 0) group law for G1 (over Fp) and G2
// (over Fp2) on sm_100a.
//
// Bucket sums use extended-Jacobian "XYZZ" coordinates (x = X/ZZ, y = Y/ZZZ,
// ZZ^3 = ZZZ^2), EFD formulas madd-2008-s (8M+2S), add-2008-s (12M+2S),
// dbl-2008-s-1 and mdbl-2008-s-1.  The reference accumulates in plain
// Jacobian coordinates (pointMixedAdd 7M+4S, include/fp_bn254.cuh:931-977;
// point2JacAddMixed, include/fp2_bn254.cuh:224-403); both give the same
// group element, and every result leaves the library in affine form, where
// it is unique.  ZZ = ZZZ = 0 encodes the point at infinity, so an all-zero
// buffer is a valid array of empty buckets.
#pragma once
#include "field.cuh"

namespace zk {

template <class F>
struct __align__(16) xyzz {
  F x, y, zz, zzz;
};

template <class F>
struct affine {
  F x, y;
};

template <class F>
__device__ __forceinline__ xyzz<F> xyzz_inf() {
  return {fe_zero_of<F>(), fe_zero_of<F>(), fe_zero_of<F>(), fe_zero_of<F>()};
}

template <class F>
__device__ __forceinline__ bool xyzz_is_inf(const xyzz<F>& p) {
  return fe_is_zero(p.zz);
}

template <class F>
__device__ __forceinline__ F fe_triple(const F& a) {
  return fe_dbl(a) + a;
}

// dbl-2008-s-1 (a = 0)
template <class F>
__device__ __forceinline__ xyzz<F> xyzz_dbl(const xyzz<F>& p) {
  if (xyzz_is_inf(p)) return p;
  F u = fe_dbl(p.y);
  F v = fe_sqr(u);
  F w = u * v;
  F s = p.x * v;
  F m = fe_triple(fe_sqr(p.x));
  xyzz<F> r;
  r.x = fe_sqr(m) - fe_dbl(s);
  r.y = fe_mul_sub(m, s - r.x, w, p.y);
  r.zz = v * p.zz;
  r.zzz = w * p.zzz;
  return r;
}

// mdbl-2008-s-1: 2 * (x, y) for an affine point
template <class F>
__device__ __forceinline__ xyzz<F> xyzz_mdbl(const F& x, const F& y) {
  F u = fe_dbl(y);
  F v = fe_sqr(u);
  F w = u * v;
  F s = x * v;
  F m = fe_triple(fe_sqr(x));
  xyzz<F> r;
  r.x = fe_sqr(m) - fe_dbl(s);
  r.y = fe_mul_sub(m, s - r.x, w, y);
  r.zz = v;
  r.zzz = w;
  return r;
}

// p + (x, y) for an affine point that is not the point at infinity.  ZZ3
// and ZZZ3 are formed before X3 and Y3 so that ZZ1, ZZZ1 and PP die early
// (fewer live registers in the accumulation loops).
template <class F>
__device__ __forceinline__ xyzz<F> xyzz_madd(const xyzz<F>& p, const F& x, const F& y) {
  if (xyzz_is_inf(p)) return {x, y, fe_one_of<F>(), fe_one_of<F>()};
  F u2 = x * p.zz;
  F s2 = y * p.zzz;
  F pp_ = u2 - p.x;
  F rr = s2 - p.y;
  if (fe_is_zero(pp_)) {
    if (fe_is_zero(rr)) return xyzz_mdbl(x, y);
    return xyzz_inf<F>();
  }
  F pp = fe_sqr(pp_);
  F ppp = pp_ * pp;
  F q = p.x * pp;
  xyzz<F> r;
  r.zz = p.zz * pp;
  r.zzz = p.zzz * ppp;
  r.x = fe_sqr(rr) - ppp - fe_dbl(q);
  r.y = fe_mul_sub(rr, q - r.x, p.y, ppp);
  return r;
}

// add-2008-s
template <class F>
__device__ __forceinline__ xyzz<F> xyzz_add(const xyzz<F>& p, const xyzz<F>& q) {
  if (xyzz_is_inf(p)) return q;
  if (xyzz_is_inf(q)) return p;
  F u1 = p.x * q.zz;
  F u2 = q.x * p.zz;
  F s1 = p.y * q.zzz;
  F s2 = q.y * p.zzz;
  F pp_ = u2 - u1;
  F rr = s2 - s1;
  if (fe_is_zero(pp_)) {
    if (fe_is_zero(rr)) return xyzz_dbl(p);
    return xyzz_inf<F>();
  }
  F pp = fe_sqr(pp_);
  F ppp = pp_ * pp;
  F qq = u1 * pp;
  xyzz<F> r;
  r.zz = p.zz * q.zz * pp;
  r.zzz = p.zzz * q.zzz * ppp;
  r.x = fe_sqr(rr) - ppp - fe_dbl(qq);
  r.y = fe_mul_sub(rr, qq - r.x, s1, ppp);
  return r;
}

template <class F>
__device__ __forceinline__ xyzz<F> xyzz_neg(const xyzz<F>& p) {
  return {p.x, fe_neg(p.y), p.zz, p.zzz};
}

// affine conversion; (0, 0) for infinity like the reference
template <class F>
__device__ __forceinline__ affine<F> xyzz_to_affine(const xyzz<F>& p) {
  if (xyzz_is_inf(p)) return {fe_zero_of<F>(), fe_zero_of<F>()};
  F zzzi = fe_inv(p.zzz);            // 1/ZZZ
  F zi = zzzi * p.zz;                // ZZ/ZZZ = 1/Z
  F zzi = fe_sqr(zi);                // 1/ZZ
  return {p.x * zzi, p.y * zzzi};
}

// ---------------------------------------------------------- memory layout
// xyzz<fp_t> is 4 x 32 B, xyzz<fp2_t> is 8 x 32 B; both are moved as uint4s.
template <class T>
__device__ __forceinline__ T ld_pod(const T* p) {
  static_assert(sizeof(T) % 16 == 0, "16-byte multiple");
  T r;
  const uint4* s = reinterpret_cast<const uint4*>(p);
  uint4* d = reinterpret_cast<uint4*>(&r);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
  return r;
}
template <class T>
__device__ __forceinline__ void st_pod(T* p, const T& v) {
  static_assert(sizeof(T) % 16 == 0, "16-byte multiple");
  uint4* d = reinterpret_cast<uint4*>(p);
  const uint4* s = reinterpret_cast<const uint4*>(&v);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
}

}  // namespace zk
