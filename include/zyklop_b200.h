/*
 * zyklop_b200 — C ABI of the B200 (sm_100a) Groth16 / BN254 prover library.
 *
 * Plain pointers and sizes only.  Every entry point returns a status code
 * (ZK_OK on success) and never exits the process; zk_last_error() gives the
 * calling thread's message for the last failure.  Field elements are
 * 4 x u64 little-endian limbs (the reference's layout); "Montgomery" means
 * x * 2^256 mod m, as in the reference.
 *
 * Each declaration names the reference interface it replaces
 * (Julienbxl/Zyklop, file:line).
 */
#ifndef ZYKLOP_B200_H
#define ZYKLOP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define ZK_OK 0
#define ZK_EINVAL 1     /* bad argument or size                        */
#define ZK_ECUDA 2      /* CUDA runtime error                          */
#define ZK_ENOMEM 3     /* device or host allocation failed            */
#define ZK_EIO 4        /* file could not be opened / read             */
#define ZK_EFORMAT 5    /* malformed zkey / wtns                       */
#define ZK_EWITNESS 6   /* witness shorter than the circuit needs      */
#define ZK_ETIMEOUT 7   /* a bounded wait gave up                      */
#define ZK_EINTERNAL 8  /* unexpected internal failure                 */
#define ZK_ENOTSUP 9    /* unsupported parameter                       */
#define ZK_ECANCELED 10 /* request dropped before it started           */

typedef struct zk_ctx zk_ctx;

/* Library version string. */
const char* zk_version(void);

/* Message of the calling thread's last failure ("" if none). */
const char* zk_last_error(void);

/* A context owns one CUDA stream, the device scratch arena and the cached NTT
 * twiddle tables for one device.  Calls on one context are serialized; use
 * one context per host thread for concurrency.  Passing ctx = NULL to any
 * entry point uses a per-device default context (current device).  A
 * context's own stream is a blocking stream: its work starts after work the
 * caller queued on the legacy default stream (the stream the reference uses
 * for everything), so device buffers written there are ready; use
 * zk_ctx_set_stream to run on another stream instead.
 * Replaces the reference's global state (g_ntt_* statics,
 * include/ntt_bn254.cuh:50-53; implicit device 0 and legacy stream). */
int zk_ctx_create(int device, zk_ctx** out);
int zk_ctx_destroy(zk_ctx* ctx);
/* Synchronize the context's stream. */
int zk_ctx_sync(zk_ctx* ctx);
/* Use the caller's CUDA stream (a cudaStream_t) as the context stream.  Every
 * proof on the context starts after the work already queued on that stream
 * and finishes before work queued after it, so events recorded there bracket
 * whole proofs.  Only for contexts from zk_ctx_create. */
int zk_ctx_set_stream(zk_ctx* ctx, void* stream);
/* Device buffers come from a per-device stream-ordered pool that keeps freed
 * blocks for reuse (loading and freeing circuits then costs no driver
 * mapping work).  This returns the pool's unused blocks on the context's
 * device to the driver. */
int zk_release_cached_memory(zk_ctx* ctx);

/* Allocations the library has made in this process so far (device blocks
 * and their bytes, pinned host buffers), and the reserved / in-use bytes of
 * its memory pool on `device` (0 when that device has none yet).  For
 * checking that a call allocates nothing.  No reference counterpart. */
typedef struct {
  uint64_t device_allocations;
  uint64_t device_allocated_bytes;
  uint64_t pinned_allocations;
  uint64_t pool_reserved_bytes;
  uint64_t pool_used_bytes;
} zk_memory_stats_t;
int zk_memory_stats(int device, zk_memory_stats_t* out);

/* ---- measurement ----------------------------------------------------------- */
/* Number of kernels this library has launched in the process so far. */
int zk_launch_count(uint64_t* out);
/* Kernel timing: while on, the hot kernels are bracketed by CUDA events on the
 * stream they run on.  zk_ctx_profile waits for them, returns per-kind totals
 * (milliseconds, launches, work units) and clears the record.  Kinds: 0 = G1
 * bucket accumulation (units: MSM points), 1 = G2 bucket accumulation
 * (points), 2 = NTT passes (elements), 3 = section-4 SpMV (coefficients).
 * Replaces the reference's env-gated cudaEvent phase timers (ZK_G1_DEBUG,
 * ZK_G2_DEBUG, ZK_HPIPE_DEBUG: include/msm_g1.cuh:78-227,
 * include/msm_g2.cuh:118-200, src/groth16.cu:951-1022). */
#define ZK_PROF_KINDS 4
typedef struct {
  double ms[ZK_PROF_KINDS];
  double launches[ZK_PROF_KINDS];
  double units[ZK_PROF_KINDS];
} zk_profile;
int zk_ctx_set_profiling(zk_ctx* ctx, int on);
int zk_ctx_profile(zk_ctx* ctx, zk_profile* out);
/* Measured carry-chain IMAD throughput of the device (mad.lo.cc / madc.hi.cc,
 * the field multiplication's instruction mix), in 10^12 ops/s: the
 * denominator of the MSM roofline.  No reference counterpart. */
int zk_imad_probe(zk_ctx* ctx, double* tiops);
/* The same measurement for kind 0 (carry chains, = zk_imad_probe) or kind 1
 * (independent mad.lo / mad.hi streams without carries: the integer pipe's
 * rate when no carry flag serializes the instructions).  No reference
 * counterpart. */
int zk_int_probe(zk_ctx* ctx, int kind, double* tiops);

/* ---- field primitives (device pointers, n elements of 4 x u64) ----------- */
#define ZK_FIELD_FP 0
#define ZK_FIELD_FR 1
#define ZK_OP_MUL 0     /* Montgomery product                        */
#define ZK_OP_ADD 1
#define ZK_OP_SUB 2
#define ZK_OP_SQR 3
#define ZK_OP_NEG 4
#define ZK_OP_INV 5     /* Montgomery inverse (0 -> 0)               */
#define ZK_OP_ENCODE 6  /* canonical -> Montgomery                   */
#define ZK_OP_DECODE 7  /* Montgomery -> canonical                   */
/* out[i] = op(a[i], b[i]); b is ignored by unary ops.  Replaces the
 * reference's device field functions exercised by its unit tests:
 * fpMul/fpSqr/fpAdd/fpSub/fpNeg/fpInv (include/fp_bn254.cuh:87-775) and
 * frMul/frAdd/frSub/frNeg/frInv/frMontEncode/Decode
 * (include/fr_bn254.cuh:191-321). */
int zk_field_op(zk_ctx* ctx, int field, int op, uint64_t* d_out, const uint64_t* d_a,
                const uint64_t* d_b, size_t n);

/* ---- NTT ----------------------------------------------------------------- */
/* In-place natural-order NTT of 2^log_n Montgomery Fr elements on the device;
 * inverse != 0 gives the inverse scaled by 1/N.  omega_N = 5^((r-1)/N).
 * Replaces nttPrepare / ntt / nttDestroy (include/ntt_bn254.cuh:190-281,
 * 418-464); no prepare call is needed (tables are cached per context). */
int zk_ntt(zk_ctx* ctx, uint64_t* d_a, uint32_t log_n, int inverse);

/* H evaluations h[j] = (A*B - C)(omega_2n^(2j+1)), canonical, from
 * d_aw = A.w and d_bw = B.w (Montgomery, 2^log_n each; both are
 * overwritten).  Replaces computeHPoly (src/groth16.cu:1037-1128). */
int zk_hpoly(zk_ctx* ctx, uint64_t* d_aw, uint64_t* d_bw, uint32_t log_n, uint64_t* d_h);

/* ---- MSM ------------------------------------------------------------------ */
/* sum_i k_i * P_i on G1.  d_px, d_py: n x 4 u64 affine Montgomery (SoA,
 * (0,0) = infinity); d_scalars: n x 4 u64 canonical integers.
 * h_out: x[4], y[4] affine Montgomery ((0,0) for infinity); *is_inf set if
 * not NULL.  Blocks until the result is on the host.
 * Replaces msm_g1 (include/msm_g1.cuh:918-926). */
int zk_msm_g1(zk_ctx* ctx, const uint64_t* d_px, const uint64_t* d_py, const uint64_t* d_scalars,
              size_t n, uint64_t* h_out, int* is_inf);

/* Same on G2: d_px, d_py n x 8 u64 ([a0, a1] per coordinate); h_out 16 u64
 * (x.a0, x.a1, y.a0, y.a1).  Replaces msm_g2_device
 * (include/msm_g2.cuh:669-854). */
int zk_msm_g2(zk_ctx* ctx, const uint64_t* d_px, const uint64_t* d_py, const uint64_t* d_scalars,
              size_t n, uint64_t* h_out, int* is_inf);

/* G1 MSM that allocates nothing, for callers that cannot call cudaMalloc (a
 * plugin inside a host application that has given all device memory to its
 * own pool allocator, or a latency-critical loop that cannot take
 * cudaMalloc's implicit device synchronization).  Same inputs and result as
 * zk_msm_g1, on the caller's `stream` (a cudaStream_t; NULL = default
 * stream); blocks until the result is on the host.  Its scratch is a fixed
 * 24 MiB __device__ array, so n is limited to 65536 points (larger n returns
 * ZK_EINVAL).  CUDA loads a library's device code lazily, so that array
 * takes device memory when a device first runs this call (which also looks
 * up the array's address), not when the library loads: make one warm-up
 * call on each device before the host application's pool claims the
 * device's memory (if the array cannot be placed, the call fails with
 * ZK_ENOMEM and says so).  The call synchronizes its stream, so it cannot
 * run while that stream is being captured into a CUDA graph (ZK_ENOTSUP).
 * All calls share the array: calls that overlap on the GPU race, so
 * serialize them.  No counterpart in the reference. */
int zk_msm_g1_noalloc(const uint64_t* d_px, const uint64_t* d_py, const uint64_t* d_scalars,
                      size_t n, uint64_t* h_out, int* is_inf, void* stream);

/* Fixed-base MSM: precompute once for a resident set of n points of prime
 * order r (group 1: n x 4 u64 coordinates, group 2: n x 8), then run MSMs
 * against it with any scalars (reduced mod r).  c = 0 picks the window size.
 * The table holds (254/c + 1) multiples per point.  zk_msm_table_run takes up
 * to n scalars (missing ones count as zero) and returns the same affine
 * result as zk_msm_g1 / zk_msm_g2 on those points.  No reference
 * counterpart (the reference recomputes every window from the bases). */
typedef struct zk_msm_table zk_msm_table;
int zk_msm_table_create(zk_ctx* ctx, int group, const uint64_t* d_px, const uint64_t* d_py,
                        size_t n, int c, zk_msm_table** out);
int zk_msm_table_run(zk_msm_table* t, const uint64_t* d_scalars, size_t n, uint64_t* h_out,
                     int* is_inf);
int zk_msm_table_free(zk_msm_table* t);

/* Pippenger parameters for subsequent MSMs on this context (group 1 or 2):
 * window bits c (0 = automatic), records per thread k0 (0 = by size) / k1,
 * and the fan-in `chunk` (a power of two, 0 = by size, and for fixed-base
 * MSMs by window bits) of the first bucket-reduction level.
 * Replaces the reference's compile-time
 * MSM_G1_C_BITS / C_BITS and ZK_G1_* / ZK_G2_* environment knobs
 * (include/msm_g1.cuh:45-117, include/msm_g2.cuh:39-116). */
int zk_msm_set_config(zk_ctx* ctx, int group, int c, int k0, int k1, int chunk);

/* Device scratch bytes an MSM of n points needs under the current config. */
int zk_msm_scratch_bytes(zk_ctx* ctx, int group, size_t n, size_t* bytes);

/* ---- Groth16 proving ------------------------------------------------------- */
/* A circuit is a zkey made resident on the device: CRS points (sections 5-9,
 * kept in their AoS zkey layout), A/B matrices as CSR built on the GPU from
 * section 4, and the verification-key points.  It belongs to the context it
 * was loaded on.  No reference counterpart: the reference re-reads the zkey in
 * every groth16Prove call (src/groth16.cu:1143-1293). */
typedef struct zk_circuit zk_circuit;
int zk_circuit_load_file(zk_ctx* ctx, const char* zkey_path, zk_circuit** out);
int zk_circuit_load_mem(zk_ctx* ctx, const uint8_t* zkey, size_t len, zk_circuit** out);
int zk_circuit_free(zk_circuit* c);
int zk_circuit_info(const zk_circuit* c, uint32_t* n_vars, uint32_t* n_public, uint32_t* domain);

/* Builds fixed-base tables for the circuit's point sets: for each point P
 * and window w < 254/c + 1 the multiple 2^(c w) P, kept resident (W times the
 * points' memory).  Later proofs then sort every (point, window) digit into
 * one shared bucket set: one bucket reduction per MSM instead of one per
 * window and no doubling chain, with larger windows (fewer additions).
 * c_g1 / c_g2: window bits (0 = default for the size).  Proofs are
 * unchanged bit for bit.  A resident-CRS format for repeated proofs of one
 * circuit; the reference has no counterpart. */
int zk_circuit_precompute(zk_circuit* c, int c_g1, int c_g2);

/* Proves with a witness of n_witness >= nVars canonical Fr values (wtns
 * section 2 layout).  r, s: canonical Fr blinding scalars, or both NULL for
 * the reference's unblinded proof (which is then bit-identical to the
 * reference's).  proof: pi_A[8], pi_B[16], pi_C[8] u64, affine Montgomery,
 * the layout of the reference's Groth16Proof (include/groth16.cuh:69-73).
 * Replaces the proving part of groth16Prove (src/groth16.cu:1177-1389).
 * zk_prove takes a host witness, zk_prove_device a device one. */
int zk_prove(zk_circuit* c, const uint64_t* h_witness, size_t n_witness, const uint64_t* r,
             const uint64_t* s, uint64_t* proof);
int zk_prove_device(zk_circuit* c, const uint64_t* d_witness, size_t n_witness, const uint64_t* r,
                    const uint64_t* s, uint64_t* proof);
/* Proves `count` jobs: circuits[i] (all loaded on `ctx`) with witnesses[i]
 * (n_witness[i] values; host memory, or device memory if on_device != 0),
 * writing proofs + 32 * i.  Up to `inflight` (1..16) proofs are on the GPU at
 * once, each on its own workspace and streams, so one proof's serial tail
 * (window combination, blinding) overlaps the next proofs' kernels.  r, s:
 * count x 4 u64 blinding scalars, or both NULL.  Every proof equals the one
 * zk_prove gives for the same job.  No reference counterpart (the reference
 * proves one file pair per process). */
int zk_prove_batch(zk_ctx* ctx, size_t count, zk_circuit* const* circuits,
                   const uint64_t* const* witnesses, const size_t* n_witness, int on_device,
                   const uint64_t* r, const uint64_t* s, uint64_t* proofs, int inflight);
/* When on, each workspace captures a proof's device pipeline (about 60
 * kernels and copies across 5 streams) into a CUDA graph the first time it
 * proves a circuit and replays it afterwards; in fused batches (mode 2),
 * each group's device pipeline (its MSM chains, SpMVs and H pipelines) is
 * captured the first time that group of jobs comes and replayed when it
 * comes again.  Results are unchanged. */
int zk_ctx_set_graphs(zk_ctx* ctx, int on);
/* How zk_prove_batch runs: mode 1 = in-flight pipelines (up to `inflight`
 * proofs at once, each with its own workspace and streams); mode 2 = fused
 * groups: proofs over circuits with fixed-base tables (zk_circuit_precompute)
 * are grouped by table window bits, up to `group` per group, and each group
 * runs three multi-instance MSM launch chains (every job's A and C, every
 * job's B2, every job's H) whose bucket accumulation is a persistent kernel
 * pulling (instance, bucket-range) tiles from a device work queue, per-job
 * SpMVs, and every job's H pipeline (of any sizes) in one persistent launch
 * pulling (job, step, tile) items from a device work queue; two groups
 * alternate so host combination overlaps GPU work; mode 0 (default) = fused
 * when every circuit has tables, else in-flight.  Results never change. */
int zk_ctx_set_batch_mode(zk_ctx* ctx, int mode, int group);
/* Streams a proof spreads its MSMs over (1..5; 0 = the default 5, or the
 * ZYKLOP_PROVE_STREAMS environment variable).  With 1 the MSMs run back to
 * back, so per-kernel timings (zk_ctx_profile) are not shared with other
 * kernels of the same proof.  Results never change. */
int zk_ctx_set_prove_streams(zk_ctx* ctx, int n);

/* Autotuning.  Each call times candidate settings on seeded synthetic inputs
 * (points k_i * G, scalars of the given distribution: 0 uniform in Fr, 1 the
 * circom-like mix of bits and small integers) on the context's stream, checks
 * that every candidate gives the same result, and records the fastest in the
 * context for (group, log_n, dist).  Later MSMs and proofs of that size and
 * distribution use it unless zk_msm_set_config set an explicit window.
 * Results never change.  No reference counterpart (the reference fixes its
 * window sizes and bucket tiers at compile time, include/msm_g1.cuh:714-926). */
typedef struct {
  int c;         /* window bits (windowed MSMs) */
  int k0;        /* sorted records per accumulation thread (bucket split threshold) */
  int k1;        /* partial records per thread in later levels */
  int chunk;     /* buckets per thread in the bucket reduction */
  int table_c;   /* fixed-base table window bits (zk_autotune_table_c) */
  int pass_bits; /* largest NTT pass radix, 2^pass_bits (zk_autotune_ntt) */
  double ms;     /* time of the chosen setting */
} zk_tune_result;
/* Windowed (fixed_c = 0) or fixed-base (fixed_c = table window bits) MSM of
 * 2^log_n points: window bits, split threshold and reduction chunk. */
int zk_autotune_msm(zk_ctx* ctx, int group, int log_n, int dist, int fixed_c, zk_tune_result* out);
/* Fixed-base table window bits for 2^log_n points, tables no larger than
 * max_table_bytes (0: no cap); used by zk_circuit_precompute(c, 0, 0). */
int zk_autotune_table_c(zk_ctx* ctx, int group, int log_n, int dist, size_t max_table_bytes,
                        zk_tune_result* out);
/* NTT pass radix for the H pipeline at 2^log_n points. */
int zk_autotune_ntt(zk_ctx* ctx, int log_n, zk_tune_result* out);
/* The context's tuned settings as text (one entry per line), and back; an
 * import replaces entries with the same key.  *len receives the text length;
 * buf may be NULL to query it. */
int zk_tune_export(zk_ctx* ctx, char* buf, size_t cap, size_t* len);
int zk_tune_import(zk_ctx* ctx, const char* text);
/* Scalar distribution hint for zk_msm_g1 / zk_msm_g2 / zk_msm_table_run on
 * this context (0 uniform, 1 skewed). */
int zk_ctx_set_scalar_dist(zk_ctx* ctx, int dist);
/* A circuit's witness distribution: -1 detects it from each host witness
 * (the default), 0 / 1 fix it. */
int zk_circuit_set_scalar_dist(zk_circuit* c, int dist);

/* Proof server: continuous batching over resident circuits.  A worker thread
 * keeps up to max_inflight proofs on the GPU, each in its own workspace with
 * its own streams; queued requests are admitted (in the order
 * zk_server_set_policy picks) as soon as a workspace is free and the device
 * has room for its buffers plus reserve_bytes (admission by free memory), so
 * a request that arrives while others run overlaps with them.  Each proof equals the one zk_prove gives
 * for the same job.  The witness buffer and the circuit must stay valid until
 * zk_server_wait returns for that ticket.  No reference counterpart (the
 * reference proves one file pair per process). */
typedef struct zk_server zk_server;
int zk_server_create(zk_ctx* ctx, int max_inflight, size_t reserve_bytes, zk_server** out);
/* Queues one proof; r and s (4 u64 each) are blinding scalars or both NULL. */
int zk_server_submit(zk_server* srv, zk_circuit* c, const uint64_t* h_witness, size_t n_witness,
                     const uint64_t* r, const uint64_t* s, uint64_t* ticket);
/* Waits for a ticket (timeout_ms < 0: no limit; ZK_ETIMEOUT when it runs out,
 * the ticket stays valid), writes the 32-u64 proof and the time from submit
 * to completion.  A failed proof returns its error code; the ticket is then
 * released either way. */
int zk_server_wait(zk_server* srv, uint64_t ticket, int timeout_ms, uint64_t* proof,
                   double* latency_ms);
int zk_server_stats(zk_server* srv, uint64_t* completed, uint64_t* failed,
                    uint64_t* peak_inflight, uint64_t* admission_waits);
/* Admission order: policy 0 = arrival order; policy 1 (the default) = the
 * smallest circuit among the first 64 queued requests, except that a request
 * queued for longer than max_wait_ms (default 500) goes first. */
int zk_server_set_policy(zk_server* srv, int policy, int max_wait_ms);
/* Drops every request still queued (not yet on the GPU); waiting on one of
 * them returns ZK_ECANCELED.  Proofs already in flight finish normally. */
int zk_server_cancel_queued(zk_server* srv, uint64_t* n_cancelled);
/* Finishes every queued proof, then stops the worker and frees the server. */
int zk_server_destroy(zk_server* srv);

/* Unblinded proof that also copies out A.w, B.w (Montgomery, domain x 4 u64)
 * and h (canonical, domain x 4 u64) into host buffers (any may be NULL).
 * For checking the pipeline's intermediates. */
int zk_prove_intermediates(zk_circuit* c, const uint64_t* h_witness, size_t n_witness,
                           uint64_t* aw, uint64_t* bw, uint64_t* h, uint64_t* proof);

/* Every intermediate of an unblinded proof, for comparing the pipeline step
 * by step with the reference prover's own (src/groth16.cu:1143-1397).  The
 * caller sets the buffer pointers it wants (host memory, domain x 4 u64
 * each; NULL skips) and the call fills them and the MSM results:
 *   aw, bw       A.w, B.w (Montgomery), readAndComputeMVM's outputs
 *                (src/groth16.cu:737-861);
 *   ea, eb, ec   A, B and C = A.B evaluated on the odd coset
 *                omega_2n^(2j+1) (Montgomery, natural order), the buffers
 *                computeHPoly leaves after its forward NTTs
 *                (src/groth16.cu:1037-1128);
 *   h            h_j = (A.B - C)(omega_2n^(2j+1)), canonical;
 *   msm_*        the four MSM results, affine Montgomery: A (alpha1
 *                included), B2 (beta2 included), the C part and the H part
 *                of pi_C (src/groth16.cu:1329-1389); inf[k] = 1 where a
 *                result is the point at infinity.
 * The proof is the same as zk_prove's. */
typedef struct {
  uint64_t* aw;
  uint64_t* bw;
  uint64_t* ea;
  uint64_t* eb;
  uint64_t* ec;
  uint64_t* h;
  uint64_t msm_a[8];
  uint64_t msm_b2[16];
  uint64_t msm_c[8];
  uint64_t msm_h[8];
  int32_t inf[4];
} zk_prove_trace;
int zk_prove_traced(zk_circuit* c, const uint64_t* h_witness, size_t n_witness,
                    zk_prove_trace* trace, uint64_t* proof);

/* One-shot proof from zkey + wtns files / in-memory images (the circuit is
 * loaded, used and released inside the call).  Replaces
 * groth16Prove(const char*, const char*, Groth16Proof&)
 * (include/groth16.cuh:119-123, src/groth16.cu:1143-1397). */
int zk_groth16_prove_files(zk_ctx* ctx, const char* zkey_path, const char* wtns_path,
                           uint64_t* proof);
int zk_groth16_prove_mem(zk_ctx* ctx, const uint8_t* zkey, size_t zkey_len, const uint8_t* wtns,
                         size_t wtns_len, uint64_t* proof);

/* Same fields as the reference's Groth16ZkeyHeader (include/groth16.cuh:79-86). */
typedef struct {
  uint32_t n_constraints; /* zkey domainSize field */
  uint32_t n_vars;
  uint32_t n_public;
  uint32_t domain_size;   /* next power of two >= n_constraints */
  int32_t log_domain;
  uint64_t prime[4];      /* BN254 scalar field modulus */
} zk_zkey_header;
/* Replaces groth16ReadZkeyHeader (include/groth16.cuh:177-180). */
int zk_read_zkey_header(const char* zkey_path, zk_zkey_header* hdr);

/* snarkjs JSON text of a proof, the reference's exact format; needs
 * out_size >= ~1100.  Replaces groth16ProofToSnarkjsJson
 * (include/groth16.cuh:149-153, src/groth16.cu:1467-1502). */
int zk_proof_to_json(const uint64_t* proof, char* out, size_t out_size);
/* 256-byte EVM calldata (A.x, A.y, B.x.a1, B.x.a0, B.y.a1, B.y.a0, C.x, C.y,
 * big-endian canonical).  Replaces groth16ProofToCalldata
 * (include/groth16.cuh:163-167, src/groth16.cu:1509-1557). */
int zk_proof_to_calldata(const uint64_t* proof, uint8_t* out, size_t out_size);
/* public.json text (w[1..n_public] in decimal) from a wtns file.  Replaces
 * writePublicJson (src/main.cu:28-110). */
int zk_public_json(const char* wtns_path, uint32_t n_public, char* out, size_t out_size);

/* ---- setup helpers --------------------------------------------------------- */
/* d_px[i], d_py[i] = k_i * G (affine Montgomery) for the standard generator of
 * G1 (group 1; 4 u64 per coordinate) or G2 (group 2; 8 u64), k_i canonical
 * (n x 4 u64).  No reference counterpart: the reference's CRS points come
 * from snarkjs; this builds seeded synthetic CRS points and MSM bases. */
int zk_mul_generator(zk_ctx* ctx, int group, const uint64_t* d_scalars, size_t n, uint64_t* d_px,
                     uint64_t* d_py);

/* Seeded synthetic Groth16 circuit + CRS, written as snarkjs-layout .zkey and
 * .wtns files (sections 1-9; wtns version 2).  domain = 2^log_domain holds
 * 2^log_domain - n_public - 1 multiplication gates plus the n_public + 1
 * public-input rows; each gate's A and B rows have nnz_min..nnz_max nonzeros
 * on earlier variables.  witness_kind 0: uniform Fr inputs, gate outputs are
 * the products; 1: circom-like values (55% in {0,1}, 15% below 2^64, 30%
 * uniform).  The CRS comes from toxic waste derived from `seed`.  No
 * reference counterpart (the reference's circuits come from circom/snarkjs). */
typedef struct {
  uint32_t log_domain;
  uint32_t n_public;
  uint32_t n_private_inputs;
  uint32_t nnz_min;
  uint32_t nnz_max;
  uint32_t witness_kind;
  uint64_t seed;
} zk_synth_params;
int zk_synth_circuit(zk_ctx* ctx, const zk_synth_params* params, const char* zkey_path,
                     const char* wtns_path);

#ifdef __cplusplus
}
#endif

#endif /* ZYKLOP_B200_H */
