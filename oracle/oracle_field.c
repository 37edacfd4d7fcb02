/*
 * CPU oracle — field arithmetic (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Fp / Fr Montgomery CIOS over 4 x 64-bit limbs with R = 2^256, restating the
 * reference's host-side formula cpuFrMontMul (include/ntt_bn254.cuh:73-110)
 * and its constants (include/fp_bn254.cuh:52-59, include/fr_bn254.cuh:40-49).
 * Inversion is Fermat's little theorem (a^(m-2)); the reference uses
 * Bernstein-Yang divsteps (include/fp_bn254.cuh:720-773) but both return the
 * unique inverse, and inv(0) = 0 in both.
 *
 * The Fp2/Fp6/Fp12 tower used by the pairing check has no reference
 * counterpart (the reference relies on snarkjs to verify proofs).
 */
#include "oracle_internal.h"

#include <string.h>

const fld ORC_FP = {
    {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0x87d20782e4866389ULL,
    {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL},
    {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL},
};
const fld ORC_FR = {
    {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0xc2e1f593efffffffULL,
    {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL},
    {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL},
};

static const fld* F(int which) { return which ? &ORC_FR : &ORC_FP; }

/* ---------------------------------------------------------------- 4x64 core */

int u256_geq(const uint64_t* a, const uint64_t* b) {
  for (int i = 3; i >= 0; i--) {
    if (a[i] > b[i]) return 1;
    if (a[i] < b[i]) return 0;
  }
  return 1;
}

int u256_is_zero(const uint64_t* a) { return (a[0] | a[1] | a[2] | a[3]) == 0; }

static inline uint64_t sub4(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  u128 borrow = 0;
  for (int i = 0; i < 4; i++) {
    u128 d = (u128)a[i] - b[i] - borrow;
    r[i] = (uint64_t)d;
    borrow = (d >> 64) & 1;
  }
  return (uint64_t)borrow;
}

static inline uint64_t add4(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  u128 c = 0;
  for (int i = 0; i < 4; i++) {
    c = (u128)a[i] + b[i] + (c >> 64);
    r[i] = (uint64_t)c;
  }
  return (uint64_t)(c >> 64);
}

void fm_mul(const fld* f, uint64_t* r, const uint64_t* a, const uint64_t* b) {
  /* CIOS: for each word of a, t += a_i * b, then t = (t + m*p) / 2^64 with
   * m = t_0 * (-p^-1) mod 2^64 (include/ntt_bn254.cuh:73-93). */
  uint64_t t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    u128 c = 0;
    for (int j = 0; j < 4; j++) {
      c = (u128)a[i] * b[j] + t[j] + (uint64_t)(c >> 64);
      t[j] = (uint64_t)c;
    }
    c = (u128)t[4] + (uint64_t)(c >> 64);
    t[4] = (uint64_t)c;
    t[5] = (uint64_t)(c >> 64);
    uint64_t m = t[0] * f->inv;
    c = (u128)m * f->p[0] + t[0];
    for (int j = 1; j < 4; j++) {
      c = (u128)m * f->p[j] + t[j] + (uint64_t)(c >> 64);
      t[j - 1] = (uint64_t)c;
    }
    c = (u128)t[4] + (uint64_t)(c >> 64);
    t[3] = (uint64_t)c;
    t[4] = t[5] + (uint64_t)(c >> 64);
  }
  /* final conditional subtraction (include/ntt_bn254.cuh:94-109) */
  uint64_t s[4];
  uint64_t borrow = sub4(s, t, f->p);
  if (t[4] || !borrow) memcpy(r, s, 32);
  else memcpy(r, t, 32);
}

void fm_add(const fld* f, uint64_t* r, const uint64_t* a, const uint64_t* b) {
  uint64_t t[4], s[4];
  uint64_t carry = add4(t, a, b);
  uint64_t borrow = sub4(s, t, f->p);
  if (carry || !borrow) memcpy(r, s, 32);
  else memcpy(r, t, 32);
}

void fm_sub(const fld* f, uint64_t* r, const uint64_t* a, const uint64_t* b) {
  uint64_t t[4];
  if (sub4(t, a, b)) add4(t, t, f->p);
  memcpy(r, t, 32);
}

void fm_neg(const fld* f, uint64_t* r, const uint64_t* a) {
  if (u256_is_zero(a)) { memset(r, 0, 32); return; }
  sub4(r, f->p, a);
}

void fm_pow(const fld* f, uint64_t* r, const uint64_t* base, const uint64_t* e, int nwords) {
  uint64_t acc[4], b[4];
  memcpy(acc, f->one, 32);
  memcpy(b, base, 32);
  for (int i = nwords * 64 - 1; i >= 0; i--) {
    fm_mul(f, acc, acc, acc);
    if ((e[i >> 6] >> (i & 63)) & 1) fm_mul(f, acc, acc, b);
  }
  memcpy(r, acc, 32);
}

void fm_inv(const fld* f, uint64_t* r, const uint64_t* a) {
  uint64_t e[4], two[4] = {2, 0, 0, 0};
  sub4(e, f->p, two);
  fm_pow(f, r, a, e, 4); /* 0^(p-2) = 0 */
}

void fm_encode(const fld* f, uint64_t* r, const uint64_t* a) { fm_mul(f, r, a, f->r2); }

void fm_decode(const fld* f, uint64_t* r, const uint64_t* a) {
  uint64_t one[4] = {1, 0, 0, 0};
  fm_mul(f, r, a, one);
}

void fm_from_u64(const fld* f, uint64_t* r, uint64_t v) {
  uint64_t t[4] = {v, 0, 0, 0};
  fm_encode(f, r, t);
}

/* -------------------------------------------------------------- exported */

void orc_f_mul(int w, uint64_t* r, const uint64_t* a, const uint64_t* b) { fm_mul(F(w), r, a, b); }
void orc_f_add(int w, uint64_t* r, const uint64_t* a, const uint64_t* b) { fm_add(F(w), r, a, b); }
void orc_f_sub(int w, uint64_t* r, const uint64_t* a, const uint64_t* b) { fm_sub(F(w), r, a, b); }
void orc_f_neg(int w, uint64_t* r, const uint64_t* a) { fm_neg(F(w), r, a); }
void orc_f_sqr(int w, uint64_t* r, const uint64_t* a) { fm_mul(F(w), r, a, a); }
void orc_f_inv(int w, uint64_t* r, const uint64_t* a) { fm_inv(F(w), r, a); }
void orc_f_inv_normal(int w, uint64_t* r, const uint64_t* a) {
  uint64_t t[4];
  fm_encode(F(w), t, a);
  fm_inv(F(w), t, t);
  fm_decode(F(w), r, t);
}
void orc_f_encode(int w, uint64_t* r, const uint64_t* a) { fm_encode(F(w), r, a); }
void orc_f_decode(int w, uint64_t* r, const uint64_t* a) { fm_decode(F(w), r, a); }
void orc_f_pow(int w, uint64_t* r, const uint64_t* base, const uint64_t* e) { fm_pow(F(w), r, base, e, 4); }

void orc_f_batch(int w, int op, uint64_t* r, const uint64_t* a, const uint64_t* b, size_t n) {
  const fld* f = F(w);
  for (size_t i = 0; i < n; i++) {
    uint64_t* ri = r + 4 * i;
    const uint64_t* ai = a + 4 * i;
    const uint64_t* bi = b ? b + 4 * i : NULL;
    switch (op) {
      case 0: fm_mul(f, ri, ai, bi); break;
      case 1: fm_add(f, ri, ai, bi); break;
      case 2: fm_sub(f, ri, ai, bi); break;
      case 3: fm_mul(f, ri, ai, ai); break;
      case 4: fm_neg(f, ri, ai); break;
      case 5: fm_inv(f, ri, ai); break;
      case 6: fm_encode(f, ri, ai); break;
      case 7: fm_decode(f, ri, ai); break;
      default: break;
    }
  }
}

/* ------------------------------------------------------------- Fp2 tower */
/* Fp2 = Fp[u]/(u^2 + 1); element = a0 + a1*u, 8 u64 [a0, a1]. */

void fp2_add(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  fm_add(&ORC_FP, r, a, b);
  fm_add(&ORC_FP, r + 4, a + 4, b + 4);
}
void fp2_sub(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  fm_sub(&ORC_FP, r, a, b);
  fm_sub(&ORC_FP, r + 4, a + 4, b + 4);
}
void fp2_neg(uint64_t* r, const uint64_t* a) {
  fm_neg(&ORC_FP, r, a);
  fm_neg(&ORC_FP, r + 4, a + 4);
}
void fp2_mul(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  uint64_t t0[4], t1[4], t2[4], t3[4];
  fm_mul(&ORC_FP, t0, a, b);         /* a0 b0 */
  fm_mul(&ORC_FP, t1, a + 4, b + 4); /* a1 b1 */
  fm_mul(&ORC_FP, t2, a, b + 4);     /* a0 b1 */
  fm_mul(&ORC_FP, t3, a + 4, b);     /* a1 b0 */
  fm_sub(&ORC_FP, r, t0, t1);
  fm_add(&ORC_FP, r + 4, t2, t3);
}
void fp2_sqr(uint64_t* r, const uint64_t* a) { fp2_mul(r, a, a); }
int fp2_is_zero(const uint64_t* a) { return u256_is_zero(a) && u256_is_zero(a + 4); }
void fp2_inv(uint64_t* r, const uint64_t* a) {
  /* 1/(a0 + a1 u) = (a0 - a1 u) / (a0^2 + a1^2) */
  uint64_t n0[4], n1[4], inv[4];
  fm_mul(&ORC_FP, n0, a, a);
  fm_mul(&ORC_FP, n1, a + 4, a + 4);
  fm_add(&ORC_FP, n0, n0, n1);
  fm_inv(&ORC_FP, inv, n0);
  uint64_t t[4];
  fm_mul(&ORC_FP, r, a, inv);
  fm_neg(&ORC_FP, t, a + 4);
  fm_mul(&ORC_FP, r + 4, t, inv);
}
/* multiply by xi = 9 + u */
static void fp2_mul_xi(uint64_t* r, const uint64_t* a) {
  uint64_t xi[8];
  fm_from_u64(&ORC_FP, xi, 9);
  fm_from_u64(&ORC_FP, xi + 4, 1);
  fp2_mul(r, a, xi);
}

/* Fp6 = Fp2[v]/(v^3 - xi); element = c0 + c1 v + c2 v^2, 24 u64. */
static void fp6_add(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  for (int i = 0; i < 3; i++) fp2_add(r + 8 * i, a + 8 * i, b + 8 * i);
}
static void fp6_sub(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  for (int i = 0; i < 3; i++) fp2_sub(r + 8 * i, a + 8 * i, b + 8 * i);
}
static void fp6_mul(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  /* schoolbook: c_k = sum_{i+j=k} a_i b_j + xi * sum_{i+j=k+3} a_i b_j */
  uint64_t acc[5][8];
  memset(acc, 0, sizeof(acc));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      uint64_t t[8];
      fp2_mul(t, a + 8 * i, b + 8 * j);
      fp2_add(acc[i + j], acc[i + j], t);
    }
  uint64_t t[8];
  fp2_mul_xi(t, acc[3]);
  fp2_add(r, acc[0], t);
  fp2_mul_xi(t, acc[4]);
  fp2_add(r + 8, acc[1], t);
  memcpy(r + 16, acc[2], 64);
}
/* multiply by v: (c0, c1, c2) -> (xi c2, c0, c1) */
static void fp6_mul_v(uint64_t* r, const uint64_t* a) {
  uint64_t t[8];
  fp2_mul_xi(t, a + 16);
  uint64_t c0[8], c1[8];
  memcpy(c0, a, 64);
  memcpy(c1, a + 8, 64);
  memcpy(r, t, 64);
  memcpy(r + 8, c0, 64);
  memcpy(r + 16, c1, 64);
}

/* Fp12 = Fp6[w]/(w^2 - v); element = d0 + d1 w, 48 u64. */
void fp12_mul(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  uint64_t t0[24], t1[24], t2[24], t3[24];
  fp6_mul(t0, a, b);
  fp6_mul(t1, a + 24, b + 24);
  fp6_mul(t2, a, b + 24);
  fp6_mul(t3, a + 24, b);
  fp6_mul_v(t1, t1);
  fp6_add(r, t0, t1);
  fp6_add(r + 24, t2, t3);
}
void fp12_one(uint64_t* r) {
  memset(r, 0, 48 * 8);
  memcpy(r, ORC_FP.one, 32);
}
int fp12_eq(const uint64_t* a, const uint64_t* b) { return memcmp(a, b, 48 * 8) == 0; }
void fp12_pow_words(uint64_t* r, const uint64_t* a, const uint64_t* e, int nwords) {
  uint64_t acc[48], base[48];
  fp12_one(acc);
  memcpy(base, a, sizeof(base));
  int top = nwords * 64 - 1;
  while (top > 0 && !((e[top >> 6] >> (top & 63)) & 1)) top--;
  for (int i = top; i >= 0; i--) {
    fp12_mul(acc, acc, acc);
    if ((e[i >> 6] >> (i & 63)) & 1) fp12_mul(acc, acc, base);
  }
  memcpy(r, acc, sizeof(acc));
}
/* (void) keep fp6_sub referenced for future use without warnings */
void orc_internal_fp6_sub(uint64_t* r, const uint64_t* a, const uint64_t* b) { fp6_sub(r, a, b); }
