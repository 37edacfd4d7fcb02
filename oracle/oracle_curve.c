/*
 * CPU oracle — G1/G2 group law and Pippenger MSM (TEST INFRASTRUCTURE ONLY;
 * see oracle.h).
 *
 * MSM semantics follow the reference's msm_g1 / msm_g2_device
 * (include/msm_g1.cuh:714-926, include/msm_g2.cuh:669-854): SoA affine
 * Montgomery points where (0,0) is the point at infinity and is skipped,
 * canonical integer scalars, affine Montgomery result.  The bucket method here
 * uses unsigned c-bit digits and a running-sum window reduction; the
 * reference uses signed digits (include/msm_g1.cuh:271-329).  Both compute the
 * same group element, and the affine result is unique.
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

/* ------------------------------------------------------------ G1 (Fp) */
static void g1_fadd(uint64_t* r, const uint64_t* a, const uint64_t* b) { fm_add(&ORC_FP, r, a, b); }
static void g1_fsub(uint64_t* r, const uint64_t* a, const uint64_t* b) { fm_sub(&ORC_FP, r, a, b); }
static void g1_fmul(uint64_t* r, const uint64_t* a, const uint64_t* b) { fm_mul(&ORC_FP, r, a, b); }
static void g1_finv(uint64_t* r, const uint64_t* a) { fm_inv(&ORC_FP, r, a); }
#define PT g1j
#define PFX g1j_
#define W 4
#define FADD g1_fadd
#define FSUB g1_fsub
#define FMUL g1_fmul
#define FINV g1_finv
#define FZERO(a) u256_is_zero(a)
#define FONE (ORC_FP.one)
#include "oracle_curve_tmpl.h"
#undef PT
#undef PFX
#undef W
#undef FADD
#undef FSUB
#undef FMUL
#undef FINV
#undef FZERO
#undef FONE

/* ------------------------------------------------------------ G2 (Fp2) */
static uint64_t FP2_ONE[8];
static void g2_init_one(void) {
  if (FP2_ONE[0] == 0) {
    uint64_t t[8] = {0};
    memcpy(t, ORC_FP.one, 32);
    memcpy(FP2_ONE, t, 64);
  }
}
#define PT g2j
#define PFX g2j_
#define W 8
#define FADD fp2_add
#define FSUB fp2_sub
#define FMUL fp2_mul
#define FINV fp2_inv
#define FZERO(a) fp2_is_zero(a)
#define FONE (g2_init_one(), FP2_ONE)
#include "oracle_curve_tmpl.h"
#undef PT
#undef PFX
#undef W
#undef FADD
#undef FSUB
#undef FMUL
#undef FINV
#undef FZERO
#undef FONE

/* ------------------------------------------------------------ exported */

static void g1_from_aff(g1j* r, const uint64_t* a) {
  g1j_set_inf(r);
  g1j_add_aff(r, r, a, a + 4);
}
static void g2_from_aff(g2j* r, const uint64_t* a) {
  g2j_set_inf(r);
  g2j_add_aff(r, r, a, a + 8);
}

int orc_g1_add(uint64_t* r, const uint64_t* p, const uint64_t* q) {
  g1j a;
  g1_from_aff(&a, p);
  g1j_add_aff(&a, &a, q, q + 4);
  return g1j_to_aff(r, &a);
}

int orc_g2_add(uint64_t* r, const uint64_t* p, const uint64_t* q) {
  g2j a;
  g2_from_aff(&a, p);
  g2j_add_aff(&a, &a, q, q + 8);
  return g2j_to_aff(r, &a);
}

int orc_g1_mul(uint64_t* r, const uint64_t* p, const uint64_t* k) {
  g1j acc;
  g1j_set_inf(&acc);
  for (int i = 255; i >= 0; i--) {
    g1j_dbl(&acc, &acc);
    if ((k[i >> 6] >> (i & 63)) & 1) g1j_add_aff(&acc, &acc, p, p + 4);
  }
  return g1j_to_aff(r, &acc);
}

int orc_g2_mul(uint64_t* r, const uint64_t* p, const uint64_t* k) {
  g2j acc;
  g2j_set_inf(&acc);
  for (int i = 255; i >= 0; i--) {
    g2j_dbl(&acc, &acc);
    if ((k[i >> 6] >> (i & 63)) & 1) g2j_add_aff(&acc, &acc, p, p + 8);
  }
  return g2j_to_aff(r, &acc);
}

int orc_g1_on_curve(const uint64_t* p) {
  if (u256_is_zero(p) && u256_is_zero(p + 4)) return 1;
  uint64_t l[4], rr[4], b[4];
  fm_mul(&ORC_FP, l, p + 4, p + 4);
  fm_mul(&ORC_FP, rr, p, p);
  fm_mul(&ORC_FP, rr, rr, p);
  fm_from_u64(&ORC_FP, b, 3);
  fm_add(&ORC_FP, rr, rr, b);
  return memcmp(l, rr, 32) == 0;
}

/* twist coefficient b' = 3 / (9 + u) */
static void g2_b(uint64_t* b) {
  uint64_t xi[8], three[8] = {0};
  fm_from_u64(&ORC_FP, xi, 9);
  fm_from_u64(&ORC_FP, xi + 4, 1);
  fm_from_u64(&ORC_FP, three, 3);
  fp2_inv(xi, xi);
  fp2_mul(b, three, xi);
}

int orc_g2_on_curve(const uint64_t* p) {
  if (fp2_is_zero(p) && fp2_is_zero(p + 8)) return 1;
  uint64_t l[8], rr[8], b[8];
  fp2_mul(l, p + 8, p + 8);
  fp2_mul(rr, p, p);
  fp2_mul(rr, rr, p);
  g2_b(b);
  fp2_add(rr, rr, b);
  return memcmp(l, rr, 64) == 0;
}

void orc_g1_generator(uint64_t* r) {
  fm_from_u64(&ORC_FP, r, 1);
  fm_from_u64(&ORC_FP, r + 4, 2);
}

void orc_g2_generator(uint64_t* r) {
  /* standard BN254 G2 generator (x = x0 + x1 u, y = y0 + y1 u), canonical */
  static const uint64_t g[16] = {
      0x46debd5cd992f6edULL, 0x674322d4f75edaddULL, 0x426a00665e5c4479ULL, 0x1800deef121f1e76ULL,
      0x97e485b7aef312c2ULL, 0xf1aa493335a9e712ULL, 0x7260bfb731fb5d25ULL, 0x198e9393920d483aULL,
      0x4ce6cc0166fa7daaULL, 0xe3d1e7690c43d37bULL, 0x4aab71808dcb408fULL, 0x12c85ea5db8c6debULL,
      0x55acdadcd122975bULL, 0xbc4b313370b38ef3ULL, 0xec9e99ad690c3395ULL, 0x090689d0585ff075ULL};
  for (int i = 0; i < 4; i++) fm_encode(&ORC_FP, r + 4 * i, g + 4 * i);
}

/* ------------------------------------------------------------ Pippenger */

static int pick_c(size_t n) {
  int c = 1;
  while (((size_t)1 << (c + 3)) < n && c < 16) c++;
  return c;
}

static uint32_t digit_at(const uint64_t* k, int bit, int c) {
  uint32_t v = 0;
  for (int b = 0; b < c && bit + b < 256; b++) v |= (uint32_t)((k[(bit + b) >> 6] >> ((bit + b) & 63)) & 1) << b;
  return v;
}

int orc_msm_g1(const uint64_t* px, const uint64_t* py, const uint64_t* sc, size_t n,
               uint64_t* out, int threads) {
  const int c = pick_c(n);
  const int nw = (256 + c - 1) / c;
  const size_t nb = ((size_t)1 << c) - 1;
  g1j* win = (g1j*)malloc(sizeof(g1j) * nw);
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
  for (int w = 0; w < nw; w++) {
    g1j* bk = (g1j*)malloc(sizeof(g1j) * nb);
    for (size_t b = 0; b < nb; b++) g1j_set_inf(&bk[b]);
    for (size_t i = 0; i < n; i++) {
      uint32_t d = digit_at(sc + 4 * i, w * c, c);
      if (d) g1j_add_aff(&bk[d - 1], &bk[d - 1], px + 4 * i, py + 4 * i);
    }
    g1j run, acc;
    g1j_set_inf(&run);
    g1j_set_inf(&acc);
    for (size_t b = nb; b-- > 0;) {
      g1j_add(&run, &run, &bk[b]);
      g1j_add(&acc, &acc, &run);
    }
    win[w] = acc;
    free(bk);
  }
  g1j res;
  g1j_set_inf(&res);
  for (int w = nw - 1; w >= 0; w--) {
    for (int i = 0; i < c; i++) g1j_dbl(&res, &res);
    g1j_add(&res, &res, &win[w]);
  }
  free(win);
  return g1j_to_aff(out, &res);
}

int orc_msm_g2(const uint64_t* px, const uint64_t* py, const uint64_t* sc, size_t n,
               uint64_t* out, int threads) {
  const int c = pick_c(n);
  const int nw = (256 + c - 1) / c;
  const size_t nb = ((size_t)1 << c) - 1;
  g2j* win = (g2j*)malloc(sizeof(g2j) * nw);
  if (threads <= 0) threads = omp_get_max_threads();
  g2_init_one();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
  for (int w = 0; w < nw; w++) {
    g2j* bk = (g2j*)malloc(sizeof(g2j) * nb);
    for (size_t b = 0; b < nb; b++) g2j_set_inf(&bk[b]);
    for (size_t i = 0; i < n; i++) {
      uint32_t d = digit_at(sc + 4 * i, w * c, c);
      if (d) g2j_add_aff(&bk[d - 1], &bk[d - 1], px + 8 * i, py + 8 * i);
    }
    g2j run, acc;
    g2j_set_inf(&run);
    g2j_set_inf(&acc);
    for (size_t b = nb; b-- > 0;) {
      g2j_add(&run, &run, &bk[b]);
      g2j_add(&acc, &acc, &run);
    }
    win[w] = acc;
    free(bk);
  }
  g2j res;
  g2j_set_inf(&res);
  for (int w = nw - 1; w >= 0; w--) {
    for (int i = 0; i < c; i++) g2j_dbl(&res, &res);
    g2j_add(&res, &res, &win[w]);
  }
  free(win);
  return g2j_to_aff(out, &res);
}
