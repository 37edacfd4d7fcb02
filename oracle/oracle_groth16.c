/*
 * CPU oracle — NTT, H polynomial, section-4 SpMV, Groth16 prove, pairing
 * check (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Follows the reference prover step by step:
 *   NTT convention       include/ntt_bn254.cuh:190-261, 300-464
 *                        (natural-order DFT, omega_N = 5^((r-1)/N), inverse
 *                        scaled by 1/N)
 *   SpMV                 src/groth16.cu:144-167, 737-809
 *   H polynomial         src/groth16.cu:1037-1090
 *   proof assembly       src/groth16.cu:1143-1397 (no blinding; the optional
 *                        r/s blinding below is the standard Groth16 form the
 *                        reference omits)
 *   zkey / wtns layout   src/zkey_utils.cpp:19-51, src/wtns_utils.cpp:13-26,
 *                        src/binfile_utils.cpp:15-178
 * The pairing is an ate pairing (loop length 6x^2) with a plain final
 * exponentiation; the reference has no pairing code.
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

/* ------------------------------------------------------------------ NTT */

static void fr_root(int log_n, uint64_t* w) {
  /* omega_28 = 5^((r-1)/2^28), then square down to the requested order */
  uint64_t five[4], e[4];
  fm_from_u64(&ORC_FR, five, 5);
  memcpy(e, ORC_FR.p, 32);
  e[0] -= 1;
  for (int i = 0; i < 28; i++) { /* e >>= 1 (r-1 is divisible by 2^28) */
    e[0] = (e[0] >> 1) | (e[1] << 63);
    e[1] = (e[1] >> 1) | (e[2] << 63);
    e[2] = (e[2] >> 1) | (e[3] << 63);
    e[3] >>= 1;
  }
  fm_pow(&ORC_FR, w, five, e, 4);
  for (int i = log_n; i < 28; i++) fm_mul(&ORC_FR, w, w, w);
}

static size_t bitrev(size_t x, int bits) {
  size_t r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

void orc_ntt(uint64_t* a, int log_n, int inverse, int threads) {
  const size_t n = (size_t)1 << log_n;
  if (threads <= 0) threads = omp_get_max_threads();
  if (log_n == 0) return;
  for (size_t i = 0; i < n; i++) {
    size_t j = bitrev(i, log_n);
    if (i < j) {
      uint64_t t[4];
      memcpy(t, a + 4 * i, 32);
      memcpy(a + 4 * i, a + 4 * j, 32);
      memcpy(a + 4 * j, t, 32);
    }
  }
  uint64_t w[4];
  fr_root(log_n, w);
  if (inverse) fm_inv(&ORC_FR, w, w);
  /* tw[k] = w^k for k < n/2 */
  uint64_t* tw = (uint64_t*)malloc(32 * (n / 2));
  memcpy(tw, ORC_FR.one, 32);
  for (size_t k = 1; k < n / 2; k++) fm_mul(&ORC_FR, tw + 4 * k, tw + 4 * (k - 1), w);
  for (int s = 1; s <= log_n; s++) {
    const size_t len = (size_t)1 << s, half = len >> 1, stride = n / len;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (size_t idx = 0; idx < n / 2; idx++) {
      size_t blk = idx / half, j = idx % half;
      uint64_t* u = a + 4 * (blk * len + j);
      uint64_t* v = u + 4 * half;
      uint64_t t[4];
      fm_mul(&ORC_FR, t, v, tw + 4 * (j * stride));
      fm_sub(&ORC_FR, v, u, t);
      fm_add(&ORC_FR, u, u, t);
    }
  }
  free(tw);
  if (inverse) {
    uint64_t ninv[4], nn[4];
    fm_from_u64(&ORC_FR, nn, (uint64_t)n);
    fm_inv(&ORC_FR, ninv, nn);
#pragma omp parallel for num_threads(threads)
    for (size_t i = 0; i < n; i++) fm_mul(&ORC_FR, a + 4 * i, a + 4 * i, ninv);
  }
}

void orc_hpoly(const uint64_t* aw, const uint64_t* bw, int log_n, uint64_t* h, int threads) {
  const size_t n = (size_t)1 << log_n;
  if (threads <= 0) threads = omp_get_max_threads();
  uint64_t* A = (uint64_t*)malloc(32 * n);
  uint64_t* B = (uint64_t*)malloc(32 * n);
  uint64_t* C = (uint64_t*)malloc(32 * n);
  memcpy(A, aw, 32 * n);
  memcpy(B, bw, 32 * n);
  /* 1. Cw = Aw * Bw (src/groth16.cu:1059-1060) */
#pragma omp parallel for num_threads(threads)
  for (size_t i = 0; i < n; i++) fm_mul(&ORC_FR, C + 4 * i, A + 4 * i, B + 4 * i);
  /* 2. inverse NTTs */
  orc_ntt(A, log_n, 1, threads);
  orc_ntt(B, log_n, 1, threads);
  orc_ntt(C, log_n, 1, threads);
  /* 3. coset shift by omega_2n^i (src/groth16.cu:914-921, 1069-1076) */
  uint64_t w2[4];
  fr_root(log_n + 1, w2);
  uint64_t* pw = (uint64_t*)malloc(32 * n);
  memcpy(pw, ORC_FR.one, 32);
  for (size_t i = 1; i < n; i++) fm_mul(&ORC_FR, pw + 4 * i, pw + 4 * (i - 1), w2);
#pragma omp parallel for num_threads(threads)
  for (size_t i = 0; i < n; i++) {
    fm_mul(&ORC_FR, A + 4 * i, A + 4 * i, pw + 4 * i);
    fm_mul(&ORC_FR, B + 4 * i, B + 4 * i, pw + 4 * i);
    fm_mul(&ORC_FR, C + 4 * i, C + 4 * i, pw + 4 * i);
  }
  free(pw);
  /* 4. forward NTTs */
  orc_ntt(A, log_n, 0, threads);
  orc_ntt(B, log_n, 0, threads);
  orc_ntt(C, log_n, 0, threads);
  /* 5. h = A*B - C, 6. decode to canonical (src/groth16.cu:935-948, 218-226) */
#pragma omp parallel for num_threads(threads)
  for (size_t i = 0; i < n; i++) {
    uint64_t t[4];
    fm_mul(&ORC_FR, t, A + 4 * i, B + 4 * i);
    fm_sub(&ORC_FR, t, t, C + 4 * i);
    fm_decode(&ORC_FR, h + 4 * i, t);
  }
  free(A);
  free(B);
  free(C);
}

void orc_spmv(const uint8_t* entries, size_t n_entries, const uint64_t* witness,
              uint32_t n_vars, uint32_t domain, uint64_t* aw, uint64_t* bw) {
  memset(aw, 0, 32 * (size_t)domain);
  memset(bw, 0, 32 * (size_t)domain);
  for (size_t k = 0; k < n_entries; k++) {
    const uint8_t* e = entries + 44 * k;
    uint32_t mat, row, sig;
    uint64_t val[4], prod[4];
    memcpy(&mat, e, 4);
    memcpy(&row, e + 4, 4);
    memcpy(&sig, e + 8, 4);
    memcpy(val, e + 12, 32);
    if (row >= domain || sig >= n_vars || mat > 1) continue;
    /* frMul(coef * R^2, w) = coef * w * R: Montgomery without an encode pass */
    fm_mul(&ORC_FR, prod, val, witness + 4 * (size_t)sig);
    uint64_t* dst = (mat == 0 ? aw : bw) + 4 * (size_t)row;
    fm_add(&ORC_FR, dst, dst, prod);
  }
}

/* --------------------------------------------------------- BinFile parse */

typedef struct {
  const uint8_t* base;
  size_t len;
  uint32_t nsec;
  uint32_t type[64];
  const uint8_t* start[64];
  uint64_t size[64];
} binfile;

static int bf_open(binfile* f, const uint8_t* data, size_t len, const char* magic) {
  if (len < 12 || memcmp(data, magic, 4) != 0) return -1;
  uint32_t ns;
  memcpy(&ns, data + 8, 4);
  size_t pos = 12;
  f->base = data;
  f->len = len;
  f->nsec = 0;
  for (uint32_t i = 0; i < ns; i++) {
    if (pos + 12 > len) return -2;
    uint32_t t;
    uint64_t s;
    memcpy(&t, data + pos, 4);
    memcpy(&s, data + pos + 4, 8);
    pos += 12;
    if (pos + s > len) return -3;
    if (f->nsec < 64) {
      f->type[f->nsec] = t;
      f->start[f->nsec] = data + pos;
      f->size[f->nsec] = s;
      f->nsec++;
    }
    pos += s;
  }
  return 0;
}

static const uint8_t* bf_section(const binfile* f, uint32_t id, uint64_t* size) {
  for (uint32_t i = 0; i < f->nsec; i++)
    if (f->type[i] == id) {
      if (size) *size = f->size[i];
      return f->start[i];
    }
  return NULL;
}

typedef struct {
  uint32_t n_vars, n_public, domain_raw, domain;
  int log_n;
  const uint64_t *alpha1, *beta1, *beta2, *gamma2, *delta1, *delta2;
  const uint8_t* coefs;
  uint32_t n_coefs;
  const uint64_t *ic, *a, *b1, *b2, *c, *h;
} zkey_view;

static int zkey_parse(zkey_view* z, binfile* f, const uint8_t* data, size_t len) {
  if (bf_open(f, data, len, "zkey")) return -10;
  uint64_t sz;
  const uint8_t* s1 = bf_section(f, 1, &sz);
  if (!s1 || sz < 4) return -11;
  uint32_t proto;
  memcpy(&proto, s1, 4);
  if (proto != 1) return -12;
  const uint8_t* s2 = bf_section(f, 2, &sz);
  if (!s2) return -13;
  uint32_t n8q, n8r;
  memcpy(&n8q, s2, 4);
  if (n8q != 32) return -14;
  memcpy(&n8r, s2 + 4 + 32, 4);
  if (n8r != 32) return -15;
  const uint8_t* p = s2 + 4 + 32 + 4 + 32;
  memcpy(&z->n_vars, p, 4);
  memcpy(&z->n_public, p + 4, 4);
  memcpy(&z->domain_raw, p + 8, 4);
  p += 12;
  z->alpha1 = (const uint64_t*)p;
  z->beta1 = (const uint64_t*)(p + 64);
  z->beta2 = (const uint64_t*)(p + 128);
  z->gamma2 = (const uint64_t*)(p + 256);
  z->delta1 = (const uint64_t*)(p + 384);
  z->delta2 = (const uint64_t*)(p + 448);
  z->domain = 1;
  z->log_n = 0;
  while (z->domain < z->domain_raw) { z->domain <<= 1; z->log_n++; }
  const uint8_t* s4 = bf_section(f, 4, &sz);
  if (!s4) return -16;
  memcpy(&z->n_coefs, s4, 4);
  if (4 + 44ull * z->n_coefs > sz) return -17;
  z->coefs = s4 + 4;
  z->ic = (const uint64_t*)bf_section(f, 3, NULL);
  z->a = (const uint64_t*)bf_section(f, 5, NULL);
  z->b1 = (const uint64_t*)bf_section(f, 6, NULL);
  z->b2 = (const uint64_t*)bf_section(f, 7, NULL);
  z->c = (const uint64_t*)bf_section(f, 8, NULL);
  z->h = (const uint64_t*)bf_section(f, 9, NULL);
  if (!z->a || !z->b2 || !z->c || !z->h) return -18;
  return 0;
}

static int wtns_parse(const uint8_t* data, size_t len, const uint64_t** w, uint32_t* nv) {
  binfile f;
  if (bf_open(&f, data, len, "wtns")) return -20;
  uint64_t sz;
  const uint8_t* s1 = bf_section(&f, 1, &sz);
  if (!s1) return -21;
  uint32_t n8;
  memcpy(&n8, s1, 4);
  if (n8 != 32) return -22;
  memcpy(nv, s1 + 4 + 32, 4);
  const uint8_t* s2 = bf_section(&f, 2, &sz);
  if (!s2 || sz < 32ull * *nv) return -23;
  *w = (const uint64_t*)s2;
  return 0;
}

/* split AoS points into SoA (G1: limbs = 4, G2: limbs = 8) with an optional
 * leading point */
static void soa(const uint64_t* aos, size_t n, int limbs, const uint64_t* lead,
                uint64_t** px, uint64_t** py) {
  size_t tot = n + (lead ? 1 : 0);
  *px = (uint64_t*)malloc(8 * limbs * tot);
  *py = (uint64_t*)malloc(8 * limbs * tot);
  size_t o = 0;
  if (lead) {
    memcpy(*px, lead, 8 * limbs);
    memcpy(*py, lead + limbs, 8 * limbs);
    o = 1;
  }
  for (size_t i = 0; i < n; i++) {
    memcpy(*px + limbs * (i + o), aos + 2 * limbs * i, 8 * limbs);
    memcpy(*py + limbs * (i + o), aos + 2 * limbs * i + limbs, 8 * limbs);
  }
}

static int prove_core(const uint8_t* zkey, size_t zkey_len, const uint8_t* wtns, size_t wtns_len,
                      const uint64_t* rb, const uint64_t* sb, uint64_t* proof, uint64_t* aw_out,
                      uint64_t* bw_out, uint64_t* h_out, int threads) {
  binfile f;
  zkey_view z;
  int rc = zkey_parse(&z, &f, zkey, zkey_len);
  if (rc) return rc;
  const uint64_t* w;
  uint32_t nw;
  rc = wtns_parse(wtns, wtns_len, &w, &nw);
  if (rc) return rc;
  if (nw < z.n_vars) return -30;
  const uint32_t n = z.domain, m1 = z.n_vars, l = z.n_public;
  uint64_t* aw = (uint64_t*)malloc(32 * (size_t)n);
  uint64_t* bw = (uint64_t*)malloc(32 * (size_t)n);
  uint64_t* h = (uint64_t*)malloc(32 * (size_t)n);
  orc_spmv(z.coefs, z.n_coefs, w, m1, n, aw, bw);
  if (aw_out) memcpy(aw_out, aw, 32 * (size_t)n);
  if (bw_out) memcpy(bw_out, bw, 32 * (size_t)n);
  orc_hpoly(aw, bw, z.log_n, h, threads);
  if (h_out) memcpy(h_out, h, 32 * (size_t)n);
  if (!proof) goto done;
  {
    /* d_we = [1 || w] (src/groth16.cu:1316-1326) */
    uint64_t* we = (uint64_t*)malloc(32 * ((size_t)m1 + 1));
    memset(we, 0, 32);
    we[0] = 1;
    memcpy(we + 4, w, 32 * (size_t)m1);
    uint64_t *px, *py;
    /* pi_A = MSM_G1([alpha1, A_0..], [1, w]) (src/groth16.cu:1330-1339) */
    soa(z.a, m1, 4, z.alpha1, &px, &py);
    uint64_t pa[8], pb[16], pc[8], ph[8];
    orc_msm_g1(px, py, we, m1 + 1, pa, threads);
    free(px);
    free(py);
    /* pi_B = MSM_G2([beta2, B2_0..], [1, w]) (src/groth16.cu:1341-1355) */
    soa(z.b2, m1, 8, z.beta2, &px, &py);
    orc_msm_g2(px, py, we, m1 + 1, pb, threads);
    free(px);
    free(py);
    /* pi_C = MSM_G1(C, w[l+1..]) + MSM_G1(H, h) (src/groth16.cu:1357-1389) */
    const uint32_t nc = m1 - l - 1;
    soa(z.c, nc, 4, NULL, &px, &py);
    orc_msm_g1(px, py, we + 4 * ((size_t)l + 2), nc, pc, threads);
    free(px);
    free(py);
    soa(z.h, n, 4, NULL, &px, &py);
    orc_msm_g1(px, py, h, n, ph, threads);
    free(px);
    free(py);
    orc_g1_add(pc, pc, ph);
    if (rb && sb) {
      /* A += r delta1; B += s delta2;
       * C += s A + r B1 - r s delta1, B1 = beta1 + sum w_i B1_i + s delta1 */
      uint64_t t1[8], t2[16], b1[8], rs[4], nrs[4];
      orc_g1_mul(t1, z.delta1, rb);
      orc_g1_add(pa, pa, t1);
      orc_g2_mul(t2, z.delta2, sb);
      orc_g2_add(pb, pb, t2);
      soa(z.b1, m1, 4, z.beta1, &px, &py);
      orc_msm_g1(px, py, we, m1 + 1, b1, threads);
      free(px);
      free(py);
      orc_g1_mul(t1, z.delta1, sb);
      orc_g1_add(b1, b1, t1);
      orc_g1_mul(t1, pa, sb);
      orc_g1_add(pc, pc, t1);
      orc_g1_mul(t1, b1, rb);
      orc_g1_add(pc, pc, t1);
      uint64_t re[4], se[4];
      fm_encode(&ORC_FR, re, rb);
      fm_encode(&ORC_FR, se, sb);
      fm_mul(&ORC_FR, rs, re, se);
      fm_neg(&ORC_FR, rs, rs);
      fm_decode(&ORC_FR, nrs, rs);
      orc_g1_mul(t1, z.delta1, nrs);
      orc_g1_add(pc, pc, t1);
    }
    memcpy(proof, pa, 64);
    memcpy(proof + 8, pb, 128);
    memcpy(proof + 24, pc, 64);
    free(we);
  }
done:
  free(aw);
  free(bw);
  free(h);
  return 0;
}

int orc_prove(const uint8_t* zkey, size_t zkey_len, const uint8_t* wtns, size_t wtns_len,
              const uint64_t* r_blind, const uint64_t* s_blind, uint64_t* proof, int threads) {
  return prove_core(zkey, zkey_len, wtns, wtns_len, r_blind, s_blind, proof, NULL, NULL, NULL,
                    threads);
}

int orc_prove_intermediates(const uint8_t* zkey, size_t zkey_len, const uint8_t* wtns,
                            size_t wtns_len, uint64_t* aw, uint64_t* bw, uint64_t* h, int threads) {
  return prove_core(zkey, zkey_len, wtns, wtns_len, NULL, NULL, NULL, aw, bw, h, threads);
}

/* --------------------------------------------------------------- pairing */

/* (p^12 - 1) / r, little-endian 64-bit words */
static const uint64_t FINAL_EXP[44] = {
    0x86964b64ca86f120ULL, 0x40a4efb7e54523a4ULL, 0x837fa97896e84abbULL, 0x361102b6b9b2b918ULL,
    0xc0de81def35692daULL, 0xbe04c7e8a6c3c760ULL, 0xd766f9c9d570bb7fULL, 0xc230974d83561841ULL,
    0x5bba1668c3be69a3ULL, 0x7f3811c410526294ULL, 0x29baee7ddadda71cULL, 0xbf813b8d145da900ULL,
    0x641bbadf423f9a2cULL, 0xa80bb4ea44eacc5eULL, 0xcd65664814fde37cULL, 0x4a0364b9580291d2ULL,
    0xee93dfb10826f0ddULL, 0x6b42db8dc5514724ULL, 0xbb10cf430b0f3785ULL, 0x40494e406f804216ULL,
    0x55cfe107acf3aafbULL, 0x2088ec80e0ebae87ULL, 0x846a3ed011a337a0ULL, 0x48a45a4a1e3a5195ULL,
    0xe5664568dfc50e16ULL, 0xab6a41294c0cc4ebULL, 0x82d0d602d268c7daULL, 0x6668449aed3cc48aULL,
    0x5062cd0fb2015dfcULL, 0x7f2940a8b1ddb3d1ULL, 0x77f5b63a2a226448ULL, 0xfef0781361e443aeULL,
    0xf977870e88d5c6c8ULL, 0x790364a61f676baaULL, 0x5887e72eceaddea3ULL, 0x1377e563a09a1b70ULL,
    0x0c54efee1bd8c3b2ULL, 0x3ec3d15ad524d8f7ULL, 0xdaf15466b2383a5dULL, 0xe1e30a73bb94fec0ULL,
    0x6a1c71015f3f7be2ULL, 0x842d43bf6369b1ffULL, 0x20fddadf107d20bcULL, 0x0000002f4b6dc970ULL};
/* ate loop length T = t - 1 = 6 x^2, x = 4965661367192848881 */
static const uint64_t ATE_T[2] = {0xf83e9682e87cfd46ULL, 0x6f4d8248eeb859fbULL};

/* line through twist points with slope lam, anchored at (xr, yr), evaluated
 * at P = (xp, yp):  yp + (-lam xp) w + (lam xr - yr) w^3 */
static void line_eval(uint64_t* l, const uint64_t* lam, const uint64_t* xr, const uint64_t* yr,
                      const uint64_t* xp, const uint64_t* yp) {
  memset(l, 0, 48 * 8);
  memcpy(l, yp, 32); /* d0.c0.a0 */
  uint64_t xpe[8] = {0}, t[8];
  memcpy(xpe, xp, 32);
  fp2_mul(t, lam, xpe);
  fp2_neg(l + 24, t); /* d1.c0 */
  fp2_mul(t, lam, xr);
  fp2_sub(l + 32, t, yr); /* d1.c1 */
}

void orc_pairing(uint64_t* out, const uint64_t* P, const uint64_t* Q) {
  int pinf = u256_is_zero(P) && u256_is_zero(P + 4);
  int qinf = fp2_is_zero(Q) && fp2_is_zero(Q + 8);
  if (pinf || qinf) { fp12_one(out); return; }
  uint64_t f[48], l[48];
  fp12_one(f);
  uint64_t xr[8], yr[8];
  memcpy(xr, Q, 64);
  memcpy(yr, Q + 8, 64);
  int top = 127;
  while (!((ATE_T[top >> 6] >> (top & 63)) & 1)) top--;
  for (int i = top - 1; i >= 0; i--) {
    /* doubling step: lam = 3 x^2 / (2 y) */
    uint64_t lam[8], t[8], u[8], x3[8], y3[8];
    fp2_mul(t, xr, xr);
    fp2_add(u, t, t);
    fp2_add(t, u, t);
    fp2_add(u, yr, yr);
    fp2_inv(u, u);
    fp2_mul(lam, t, u);
    line_eval(l, lam, xr, yr, P, P + 4);
    fp12_mul(f, f, f);
    fp12_mul(f, f, l);
    fp2_mul(x3, lam, lam);
    fp2_sub(x3, x3, xr);
    fp2_sub(x3, x3, xr);
    fp2_sub(t, xr, x3);
    fp2_mul(y3, lam, t);
    fp2_sub(y3, y3, yr);
    memcpy(xr, x3, 64);
    memcpy(yr, y3, 64);
    if ((ATE_T[i >> 6] >> (i & 63)) & 1) {
      /* addition step with Q: lam = (yq - yr) / (xq - xr) */
      fp2_sub(t, Q + 8, yr);
      fp2_sub(u, Q, xr);
      fp2_inv(u, u);
      fp2_mul(lam, t, u);
      line_eval(l, lam, xr, yr, P, P + 4);
      fp12_mul(f, f, l);
      fp2_mul(x3, lam, lam);
      fp2_sub(x3, x3, xr);
      fp2_sub(x3, x3, Q);
      fp2_sub(t, xr, x3);
      fp2_mul(y3, lam, t);
      fp2_sub(y3, y3, yr);
      memcpy(xr, x3, 64);
      memcpy(yr, y3, 64);
    }
  }
  fp12_pow_words(out, f, FINAL_EXP, 44);
}

int orc_verify(const uint8_t* zkey, size_t zkey_len, const uint64_t* proof,
               const uint64_t* publics, uint32_t n_public) {
  binfile f;
  zkey_view z;
  int rc = zkey_parse(&z, &f, zkey, zkey_len);
  if (rc) return rc;
  if (!z.ic || n_public != z.n_public) return -40;
  if (!orc_g1_on_curve(proof) || !orc_g2_on_curve(proof + 8) || !orc_g1_on_curve(proof + 24))
    return 0;
  uint64_t vkx[8], t[8];
  memcpy(vkx, z.ic, 64);
  for (uint32_t i = 0; i < n_public; i++) {
    orc_g1_mul(t, z.ic + 8 * (i + 1), publics + 4 * i);
    orc_g1_add(vkx, vkx, t);
  }
  uint64_t lhs[48], r1[48], r2[48], r3[48];
  orc_pairing(lhs, proof, proof + 8);
  orc_pairing(r1, z.alpha1, z.beta2);
  orc_pairing(r2, vkx, z.gamma2);
  orc_pairing(r3, proof + 24, z.delta2);
  fp12_mul(r1, r1, r2);
  fp12_mul(r1, r1, r3);
  return fp12_eq(lhs, r1) ? 1 : 0;
}
