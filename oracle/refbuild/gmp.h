/* Minimal stand-in for <gmp.h>, used only to compile the reference prover's
 * zkey/wtns header readers (src/zkey_utils.hpp:16-18, src/wtns_utils.hpp:13),
 * which keep the field primes in mpz_t values that nothing on the proving path
 * reads.  Only the four names those readers touch are provided; mpz_import
 * keeps nothing. */
#pragma once
#include <stddef.h>
typedef struct { int alloc_; int size_; void* d_; } zk_stub_mpz_struct;
typedef zk_stub_mpz_struct mpz_t[1];
static inline void mpz_init(mpz_t x) { x->alloc_ = 0; x->size_ = 0; x->d_ = 0; }
static inline void mpz_clear(mpz_t x) { (void)x; }
static inline void mpz_import(mpz_t rop, size_t count, int order, size_t size,
                              int endian, size_t nails, const void* op) {
  (void)rop; (void)count; (void)order; (void)size; (void)endian; (void)nails; (void)op;
}
