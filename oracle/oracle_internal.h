/* Internal declarations shared by the oracle's C files (TEST INFRASTRUCTURE
 * ONLY; see oracle.h). */
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "oracle.h"

typedef unsigned __int128 u128;

typedef struct {
  uint64_t p[4];   /* modulus */
  uint64_t inv;    /* -p^-1 mod 2^64 */
  uint64_t r2[4];  /* 2^512 mod p */
  uint64_t one[4]; /* 2^256 mod p (Montgomery 1) */
} fld;

extern const fld ORC_FP;
extern const fld ORC_FR;

int u256_geq(const uint64_t* a, const uint64_t* b);
int u256_is_zero(const uint64_t* a);
void fm_mul(const fld* f, uint64_t* r, const uint64_t* a, const uint64_t* b);
void fm_add(const fld* f, uint64_t* r, const uint64_t* a, const uint64_t* b);
void fm_sub(const fld* f, uint64_t* r, const uint64_t* a, const uint64_t* b);
void fm_neg(const fld* f, uint64_t* r, const uint64_t* a);
void fm_pow(const fld* f, uint64_t* r, const uint64_t* base, const uint64_t* e, int nwords);
void fm_inv(const fld* f, uint64_t* r, const uint64_t* a);
void fm_encode(const fld* f, uint64_t* r, const uint64_t* a);
void fm_decode(const fld* f, uint64_t* r, const uint64_t* a);
void fm_from_u64(const fld* f, uint64_t* r, uint64_t v);

void fp2_add(uint64_t* r, const uint64_t* a, const uint64_t* b);
void fp2_sub(uint64_t* r, const uint64_t* a, const uint64_t* b);
void fp2_neg(uint64_t* r, const uint64_t* a);
void fp2_mul(uint64_t* r, const uint64_t* a, const uint64_t* b);
void fp2_sqr(uint64_t* r, const uint64_t* a);
void fp2_inv(uint64_t* r, const uint64_t* a);
int fp2_is_zero(const uint64_t* a);

void fp12_mul(uint64_t* r, const uint64_t* a, const uint64_t* b);
void fp12_one(uint64_t* r);
int fp12_eq(const uint64_t* a, const uint64_t* b);
void fp12_pow_words(uint64_t* r, const uint64_t* a, const uint64_t* e, int nwords);

/* Jacobian points used by the MSM: G1 uses 4-limb coordinates, G2 8-limb. */
typedef struct { uint64_t x[4], y[4], z[4]; } g1j;
typedef struct { uint64_t x[8], y[8], z[8]; } g2j;

void g1j_set_inf(g1j* p);
void g1j_dbl(g1j* r, const g1j* p);
void g1j_add(g1j* r, const g1j* p, const g1j* q);
void g1j_add_aff(g1j* r, const g1j* p, const uint64_t* qx, const uint64_t* qy);
int g1j_to_aff(uint64_t* out, const g1j* p);
void g2j_set_inf(g2j* p);
void g2j_dbl(g2j* r, const g2j* p);
void g2j_add(g2j* r, const g2j* p, const g2j* q);
void g2j_add_aff(g2j* r, const g2j* p, const uint64_t* qx, const uint64_t* qy);
int g2j_to_aff(uint64_t* out, const g2j* p);
