/*
 * CPU oracle for the BN254 Groth16 prove path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * prover's arithmetic (Julienbxl/Zyklop) used as the checker for the CUDA
 * library: only the tests, the smoke check and the benchmark's CPU-baseline
 * leg may load it.  Nothing in the product links or calls it.
 *
 * Conventions (identical to the reference):
 *   - field elements are 4 x u64 little-endian limbs;
 *   - Montgomery form uses R = 2^256 for both Fp and Fr
 *     (include/fp_bn254.cuh:52-59, include/fr_bn254.cuh:40-49);
 *   - G1 affine points are (x[4], y[4]) Montgomery Fp, (0,0) = infinity
 *     (include/msm_g1.cuh:232-245);
 *   - G2 affine points are (x.a0, x.a1, y.a0, y.a1), 16 u64 Montgomery;
 *   - MSM scalars are canonical Fr integers (include/msm_g1.cuh:271-329).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- fields (which = 0: Fp base field, 1: Fr scalar field) ---------------- */
void orc_f_mul(int which, uint64_t* r, const uint64_t* a, const uint64_t* b);
void orc_f_add(int which, uint64_t* r, const uint64_t* a, const uint64_t* b);
void orc_f_sub(int which, uint64_t* r, const uint64_t* a, const uint64_t* b);
void orc_f_neg(int which, uint64_t* r, const uint64_t* a);
void orc_f_sqr(int which, uint64_t* r, const uint64_t* a);
/* inverse of a Montgomery element (0 -> 0) */
void orc_f_inv(int which, uint64_t* r, const uint64_t* a);
/* inverse of a canonical element, result canonical (0 -> 0) */
void orc_f_inv_normal(int which, uint64_t* r, const uint64_t* a);
void orc_f_encode(int which, uint64_t* r, const uint64_t* a);
void orc_f_decode(int which, uint64_t* r, const uint64_t* a);
/* Montgomery base^e, e a 4-limb canonical integer */
void orc_f_pow(int which, uint64_t* r, const uint64_t* base, const uint64_t* e);
/* batched element-wise ops over n elements (op: 0 mul, 1 add, 2 sub, 3 sqr,
 * 4 neg, 5 inv, 6 encode, 7 decode); b may be NULL for unary ops */
void orc_f_batch(int which, int op, uint64_t* r, const uint64_t* a, const uint64_t* b, size_t n);

/* ---- curves -------------------------------------------------------------- */
/* G1 affine add of two Montgomery points; returns 1 if the result is infinity */
int orc_g1_add(uint64_t* r, const uint64_t* p, const uint64_t* q);
/* k * P for an affine Montgomery point and canonical scalar k */
int orc_g1_mul(uint64_t* r, const uint64_t* p, const uint64_t* k);
int orc_g2_add(uint64_t* r, const uint64_t* p, const uint64_t* q);
int orc_g2_mul(uint64_t* r, const uint64_t* p, const uint64_t* k);
/* On-curve test (infinity counts as on the curve). */
int orc_g1_on_curve(const uint64_t* p);
int orc_g2_on_curve(const uint64_t* p);
/* Generators, affine Montgomery. */
void orc_g1_generator(uint64_t* r);
void orc_g2_generator(uint64_t* r);

/* Pippenger MSM, reference semantics (SoA inputs, (0,0) points skipped).
 * px,py: n x 4 (G1) or n x 8 (G2) u64; scalars n x 4 canonical.
 * out: affine Montgomery (8 or 16 u64).  Returns 1 for infinity.
 * threads <= 0 uses every OpenMP thread. */
int orc_msm_g1(const uint64_t* px, const uint64_t* py, const uint64_t* sc, size_t n,
               uint64_t* out, int threads);
int orc_msm_g2(const uint64_t* px, const uint64_t* py, const uint64_t* sc, size_t n,
               uint64_t* out, int threads);

/* ---- polynomials ---------------------------------------------------------- */
/* In-place natural-order NTT of 2^log_n Montgomery Fr elements; inverse scales
 * by 1/N.  Root: omega_N = 5^((r-1)/N). */
void orc_ntt(uint64_t* a, int log_n, int inverse, int threads);
/* H evaluations on the odd coset: Aw, Bw (Montgomery) -> h (canonical),
 * following src/groth16.cu:1037-1090.  Aw and Bw are not modified. */
void orc_hpoly(const uint64_t* aw, const uint64_t* bw, int log_n, uint64_t* h, int threads);
/* Section-4 SpMV (src/groth16.cu:144-167, 737-809): entries = raw 44-byte
 * records, witness canonical; Aw/Bw Montgomery, domain-sized. */
void orc_spmv(const uint8_t* entries, size_t n_entries, const uint64_t* witness,
              uint32_t n_vars, uint32_t domain, uint64_t* aw, uint64_t* bw);

/* ---- Groth16 -------------------------------------------------------------- */
/* Prove from in-memory zkey and wtns images.  r_blind / s_blind (canonical Fr)
 * may be NULL for the reference's unblinded proof.  proof: pi_A[8], pi_B[16],
 * pi_C[8] affine Montgomery.  Returns 0 or a negative error. */
int orc_prove(const uint8_t* zkey, size_t zkey_len, const uint8_t* wtns, size_t wtns_len,
              const uint64_t* r_blind, const uint64_t* s_blind, uint64_t* proof, int threads);
/* Optional intermediates of orc_prove (any pointer may be NULL): aw, bw
 * Montgomery (domain), h canonical (domain). */
int orc_prove_intermediates(const uint8_t* zkey, size_t zkey_len, const uint8_t* wtns,
                            size_t wtns_len, uint64_t* aw, uint64_t* bw, uint64_t* h, int threads);

/* Ate pairing e(P, Q) in Fp12 (12 Fp elements, Montgomery, tower
 * Fp2[u]/(u^2+1), Fp6 = Fp2[v]/(v^3-(9+u)), Fp12 = Fp6[w]/(w^2-v)). */
void orc_pairing(uint64_t* out12x4, const uint64_t* p_g1, const uint64_t* q_g2);
/* Groth16 verification e(A,B) == e(alpha,beta) e(vk_x,gamma) e(C,delta)
 * from a zkey image (verification key in sections 2 and 3) and public
 * signals (canonical).  Returns 1 if valid, 0 if not, negative on error. */
int orc_verify(const uint8_t* zkey, size_t zkey_len, const uint64_t* proof,
               const uint64_t* publics, uint32_t n_public);

#ifdef __cplusplus
}
#endif
