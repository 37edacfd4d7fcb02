// Host-side BN254 arithmetic (4 x u64 Montgomery, R = 2^256) for the few
// serial steps that run on the CPU: combining an MSM's window sums (a chain of
// ~256 doublings, which is latency-bound and ~20x faster on one CPU core than
// on one GPU thread), affine conversion, Montgomery decoding for
// serialization, and the synthetic-circuit generator's scalar work.
//
// Same representation as the reference's host helpers (cpuFrMontMul,
// include/ntt_bn254.cuh:73-110) and its device field code.
#pragma once
#include <cstdint>
#include <cstring>

namespace zk {
namespace host {

typedef unsigned __int128 u128;

struct FieldParams {
  uint64_t p[4];
  uint64_t inv;  // -p^-1 mod 2^64
  uint64_t r2[4];
  uint64_t one[4];
};

inline constexpr FieldParams FP_PARAMS = {
    {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0x87d20782e4866389ULL,
    {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL},
    {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}};
inline constexpr FieldParams FR_PARAMS = {
    {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0xc2e1f593efffffffULL,
    {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL},
    {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL}};

template <const FieldParams& M>
struct F {
  uint64_t v[4];

  static F zero() { return F{{0, 0, 0, 0}}; }
  static F one() { return F{{M.one[0], M.one[1], M.one[2], M.one[3]}}; }
  static F from_raw(const uint64_t* x) {
    F r;
    memcpy(r.v, x, 32);
    return r;
  }
  static F from_u64(uint64_t x) { return F{{x, 0, 0, 0}}.to_mont(); }
  bool is_zero() const { return (v[0] | v[1] | v[2] | v[3]) == 0; }
  bool operator==(const F& o) const { return memcmp(v, o.v, 32) == 0; }
  bool operator!=(const F& o) const { return !(*this == o); }

  static uint64_t sub4(uint64_t* r, const uint64_t* a, const uint64_t* b) {
    u128 bw = 0;
    for (int i = 0; i < 4; i++) {
      u128 d = (u128)a[i] - b[i] - bw;
      r[i] = (uint64_t)d;
      bw = (d >> 64) & 1;
    }
    return (uint64_t)bw;
  }
  F operator+(const F& b) const {
    F r;
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
      c = (u128)v[i] + b.v[i] + (uint64_t)(c >> 64);
      r.v[i] = (uint64_t)c;
    }
    uint64_t s[4] = {0, 0, 0, 0};
    if (!sub4(s, r.v, M.p)) memcpy(r.v, s, 32);
    return r;
  }
  F operator-(const F& b) const {
    F r;
    if (sub4(r.v, v, b.v)) {
      u128 c = 0;
      for (int i = 0; i < 4; i++) {
        c = (u128)r.v[i] + M.p[i] + (uint64_t)(c >> 64);
        r.v[i] = (uint64_t)c;
      }
    }
    return r;
  }
  F operator-() const { return zero() - *this; }
  F operator*(const F& b) const {
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
      u128 c = 0;
      for (int j = 0; j < 4; j++) {
        c = (u128)v[i] * b.v[j] + t[j] + (uint64_t)(c >> 64);
        t[j] = (uint64_t)c;
      }
      c = (u128)t[4] + (uint64_t)(c >> 64);
      t[4] = (uint64_t)c;
      t[5] = (uint64_t)(c >> 64);
      uint64_t m = t[0] * M.inv;
      c = (u128)m * M.p[0] + t[0];
      for (int j = 1; j < 4; j++) {
        c = (u128)m * M.p[j] + t[j] + (uint64_t)(c >> 64);
        t[j - 1] = (uint64_t)c;
      }
      c = (u128)t[4] + (uint64_t)(c >> 64);
      t[3] = (uint64_t)c;
      t[4] = t[5] + (uint64_t)(c >> 64);
    }
    F r;
    uint64_t s[4] = {0, 0, 0, 0};
    if (t[4] || !sub4(s, t, M.p)) memcpy(r.v, s, 32);
    else memcpy(r.v, t, 32);
    return r;
  }
  F sqr() const { return *this * *this; }
  F dbl() const { return *this + *this; }
  F to_mont() const { return *this * F{{M.r2[0], M.r2[1], M.r2[2], M.r2[3]}}; }
  F from_mont() const { return *this * F{{1, 0, 0, 0}}; }
  F pow(const uint64_t* e, int nwords = 4) const {
    F acc = one();
    for (int i = nwords * 64 - 1; i >= 0; i--) {
      acc = acc.sqr();
      if ((e[i >> 6] >> (i & 63)) & 1) acc = acc * *this;
    }
    return acc;
  }
  F inv() const {
    uint64_t e[4] = {M.p[0] - 2, M.p[1], M.p[2], M.p[3]};
    return pow(e);
  }
};

using Fp = F<FP_PARAMS>;
using Fr = F<FR_PARAMS>;

struct Fp2 {
  Fp c0, c1;
  static Fp2 zero() { return {Fp::zero(), Fp::zero()}; }
  static Fp2 one() { return {Fp::one(), Fp::zero()}; }
  bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
  bool operator==(const Fp2& o) const { return c0 == o.c0 && c1 == o.c1; }
  Fp2 operator+(const Fp2& b) const { return {c0 + b.c0, c1 + b.c1}; }
  Fp2 operator-(const Fp2& b) const { return {c0 - b.c0, c1 - b.c1}; }
  Fp2 operator-() const { return {-c0, -c1}; }
  Fp2 operator*(const Fp2& b) const {
    Fp t0 = c0 * b.c0, t1 = c1 * b.c1;
    return {t0 - t1, (c0 + c1) * (b.c0 + b.c1) - t0 - t1};
  }
  Fp2 sqr() const { return *this * *this; }
  Fp2 dbl() const { return *this + *this; }
  Fp2 inv() const {
    Fp n = (c0.sqr() + c1.sqr()).inv();
    return {c0 * n, -(c1 * n)};
  }
};

// XYZZ point (same formulas as the device code, curve.cuh)
template <class T>
struct Xyzz {
  T x, y, zz, zzz;
  static Xyzz inf() { return {T::zero(), T::zero(), T::zero(), T::zero()}; }
  bool is_inf() const { return zz.is_zero(); }

  Xyzz dbl() const {
    if (is_inf()) return *this;
    T u = y.dbl(), v = u.sqr(), w = u * v, s = x * v;
    T m = x.sqr();
    m = m.dbl() + m;
    Xyzz r;
    r.x = m.sqr() - s.dbl();
    r.y = m * (s - r.x) - w * y;
    r.zz = v * zz;
    r.zzz = w * zzz;
    return r;
  }
  Xyzz add(const Xyzz& q) const {
    if (is_inf()) return q;
    if (q.is_inf()) return *this;
    T u1 = x * q.zz, u2 = q.x * zz, s1 = y * q.zzz, s2 = q.y * zzz;
    T p = u2 - u1, rr = s2 - s1;
    if (p.is_zero()) {
      if (rr.is_zero()) return dbl();
      return inf();
    }
    T pp = p.sqr(), ppp = p * pp, qq = u1 * pp;
    Xyzz r;
    r.x = rr.sqr() - ppp - qq.dbl();
    r.y = rr * (qq - r.x) - s1 * ppp;
    r.zz = zz * q.zz * pp;
    r.zzz = zzz * q.zzz * ppp;
    return r;
  }
  static Xyzz from_affine(const T& ax, const T& ay) {
    if (ax.is_zero() && ay.is_zero()) return inf();
    return {ax, ay, T::one(), T::one()};
  }
  // affine coordinates given zzzi = 1 / ZZZ (not at infinity)
  void to_affine_with(const T& zzzi, T& ax, T& ay) const {
    const T zi = zzzi * zz;  // ZZ / ZZZ = 1 / Z
    ax = x * zi.sqr();
    ay = y * zzzi;
  }
  // returns true for the point at infinity; (0,0) written then
  bool to_affine(T& ax, T& ay) const {
    if (is_inf()) {
      ax = T::zero();
      ay = T::zero();
      return true;
    }
    T zzzi = zzz.inv();
    T zi = zzzi * zz;
    T zzi = zi.sqr();
    ax = x * zzi;
    ay = y * zzzi;
    return false;
  }
};

// Inverts every nonzero v[i] in place with one field inversion in all
// (Montgomery's simultaneous-inversion trick: prefix products, one inverse,
// three products per value on the way back); zeros stay zero.
inline void batch_inv(Fp* v, size_t n) {
  if (!n) return;
  Fp* pre = new Fp[n];
  Fp acc = Fp::one();
  for (size_t i = 0; i < n; i++) {
    pre[i] = acc;
    if (!v[i].is_zero()) acc = acc * v[i];
  }
  Fp inv = acc.inv();
  for (size_t i = n; i-- > 0;) {
    if (v[i].is_zero()) continue;
    const Fp vi = v[i];
    v[i] = inv * pre[i];
    inv = inv * vi;
  }
  delete[] pre;
}

// Affine forms of G1 and G2 XYZZ points with a single shared inversion: the
// Fp inverses of every G1 point's ZZZ and of every G2 point's ZZZ norm
// (1 / z = conj(z) / (z0^2 + z1^2) in Fp2) come from one batch_inv.  Points
// at infinity give (0, 0) and inf[k] = true.  The reference inverts once per
// point (jacToAff with its BY inversion, include/fp_bn254.cuh:720-773).
inline void batch_to_affine(const Xyzz<Fp>* g1, size_t n1, Fp* x1, Fp* y1, bool* inf1,
                            const Xyzz<Fp2>* g2, size_t n2, Fp2* x2, Fp2* y2, bool* inf2) {
  Fp* d = new Fp[n1 + n2];
  for (size_t i = 0; i < n1; i++) d[i] = g1[i].is_inf() ? Fp::zero() : g1[i].zzz;
  for (size_t i = 0; i < n2; i++)
    d[n1 + i] = g2[i].is_inf() ? Fp::zero() : g2[i].zzz.c0.sqr() + g2[i].zzz.c1.sqr();
  batch_inv(d, n1 + n2);
  for (size_t i = 0; i < n1; i++) {
    inf1[i] = g1[i].is_inf();
    if (inf1[i]) x1[i] = y1[i] = Fp::zero();
    else g1[i].to_affine_with(d[i], x1[i], y1[i]);
  }
  for (size_t i = 0; i < n2; i++) {
    inf2[i] = g2[i].is_inf();
    if (inf2[i]) {
      x2[i] = y2[i] = Fp2::zero();
    } else {
      const Fp n = d[n1 + i];
      const Fp2 zi{g2[i].zzz.c0 * n, -(g2[i].zzz.c1 * n)};
      g2[i].to_affine_with(zi, x2[i], y2[i]);
    }
  }
  delete[] d;
}

}  // namespace host
}  // namespace zk
