// Groth16 prover: device-resident circuit + proving pipeline.
//
// Replaces groth16Prove (src/groth16.cu:1143-1397).  The same algebra:
//   pi_A = MSM_G1([alpha1, A_0..A_m], [1, w_0..w_m])
//   pi_B = MSM_G2([beta2, B2_0..B2_m], [1, w_0..w_m])
//   pi_C = MSM_G1(C, w_{l+1..m}) + MSM_G1(H, h)
// with h from the section-4 SpMV and the coset H pipeline, and optional
// blinding r, s (which the reference omits): A += r delta1, B += s delta2,
// C += s A + r B1 - r s delta1 with B1 = beta1 + sum w_i B1_i + s delta1.
//
// What changes is the organisation: the circuit (CSR matrices built on the
// GPU from the raw section-4 bytes, CRS points in their zkey AoS layout) is
// uploaded once and stays resident; a proof uploads only its witness; the
// four MSMs run concurrently on their own streams while SpMV -> H -> MSM_H
// runs on a fifth, instead of the reference's sequential, allocating calls.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "context.hpp"
#include "zkey.hpp"

struct zk_circuit {
  zk_ctx* ctx = nullptr;
  uint64_t id = 0;  // unique per loaded circuit (keys captured graphs)
  uint32_t m1 = 0, l = 0, n = 0;  // nVars, nPublic, domain
  int log_n = 0;
  uint32_t n_coefs = 0;
  uint64_t alpha1[8], beta1[8], beta2[16], gamma2[16], delta1[8], delta2[16];
  std::vector<uint64_t> ic;  // (l + 1) x 8, empty if the zkey has no section 3
  bool has_b1 = false;
  // witness scalar distribution (keys autotuned MSM settings); detected from
  // host witnesses unless set explicitly
  int dist = 0;
  bool dist_auto = true;
  // CRS points, AoS (x, y) records; A / B1 / B2 carry alpha1 / beta1 / beta2
  // as record 0, like the reference's extended buffers (src/groth16.cu:1199-1227)
  zk::DeviceBuffer pts_a, pts_b1, pts_b2, pts_c, pts_h;
  // CSR of the A and B matrices: row pointers (n + 1), signal ids, coef * R^2
  zk::DeviceBuffer row[2], sig[2], val[2];
  // optional fixed-base tables (window multiples) of the point sets above,
  // window bits per group (0: not built)
  int tab_c[2] = {0, 0};
  zk::DeviceBuffer tab_a, tab_b1, tab_b2, tab_c_pts, tab_h;
};

struct zk_msm_table {
  zk_ctx* ctx = nullptr;
  int group = 1, c = 0;
  size_t n = 0;
  zk::DeviceBuffer table;
};

namespace zk {

// Loads a circuit from a parsed zkey (uploads and builds the CSR on the
// context's stream; blocks until done).
zk_circuit* circuit_load(zk_ctx* ctx, const BinFile& zkey);

struct ProveIntermediates {
  uint64_t* aw = nullptr;  // host, domain x 4 (Montgomery A.w)
  uint64_t* bw = nullptr;  // host, domain x 4 (Montgomery B.w)
  uint64_t* h = nullptr;   // host, domain x 4 (canonical h)
  // host, domain x 4: A, B and C = A.B evaluated on the odd coset
  // omega_2n^(2j+1) (Montgomery, natural order), the H pipeline's last NTT
  uint64_t* ea = nullptr;
  uint64_t* eb = nullptr;
  uint64_t* ec = nullptr;
  // filled when the proof finishes: each MSM's own result (affine
  // Montgomery; A includes alpha1, B2 beta2) and whether it is infinity
  uint64_t msm_a[8] = {}, msm_b2[16] = {}, msm_c[8] = {}, msm_h[8] = {};
  int inf[4] = {};
};

// Builds fixed-base tables for every point set of the circuit (c_g1 / c_g2
// window bits; 0 picks the default for the set's size).
void circuit_precompute(zk_circuit* c, int c_g1, int c_g2);

// Default window bits of a fixed-base MSM over n points.
int msm_fixed_default_c(size_t n, bool g2);

// Proves with a witness of >= m1 canonical Fr values (host or device memory).
// r / s: canonical Fr blinding scalars or nullptr (reference behaviour).
void prove(zk_circuit* c, const uint64_t* witness, size_t n_witness, bool witness_on_device,
           const uint64_t* r, const uint64_t* s, uint64_t proof[32], ProveIntermediates* dbg);

// One-shot unblinded proof from a parsed zkey and a host witness, without a
// resident circuit: each CRS point set is uploaded on the stream of the MSM
// that reads it and that MSM starts at once, so the upload of the rest
// overlaps the MSMs already running; B1 (used only for blinding) is not
// uploaded.  The same result as circuit_load + prove.
void prove_oneshot(zk_ctx* ctx, const BinFile& zkey, const uint64_t* witness, size_t n_witness,
                   uint64_t proof[32]);

// Proves `count` jobs (circuits of one context, witnesses host or device)
// with up to `inflight` proofs on the GPU at once, each on its own workspace
// and streams; the host combination of one proof overlaps the GPU work of the
// next ones.  rs / ss: count x 4 u64 blinding scalars or both null.
void prove_batch(zk_ctx* ctx, size_t count, zk_circuit* const* cs, const uint64_t* const* wits,
                 const size_t* nwits, bool on_device, const uint64_t* rs, const uint64_t* ss,
                 uint64_t* proofs, int inflight);

// Fused batches: jobs whose circuits hold fixed-base tables are grouped by
// table window bits; each group of up to `group` proofs runs as one launch
// chain per stage (witness staging, SpMV and H per job, then one
// multi-instance G1 MSM over every job's A / C / H (/ B1) and one over every
// job's B2), and two group workspaces alternate so one group's host
// combination overlaps the next group's GPU work.
void prove_batch_fused(zk_ctx* ctx, size_t count, zk_circuit* const* cs,
                       const uint64_t* const* wits, const size_t* nwits, bool on_device,
                       const uint64_t* rs, const uint64_t* ss, uint64_t* proofs, int group);

// Pieces shared by the single, in-flight and fused paths.
void check_job(zk_circuit* c, const uint64_t* witness, size_t n_witness, bool blind);
void note_witness(zk_circuit* c, const uint64_t* witness, bool on_device);
// A.w, B.w (Montgomery, domain entries each) from we = [1 || w] on `st`.
void spmv_enqueue(zk_circuit* c, const uint64_t* we, uint64_t* aw, uint64_t* bw, cudaStream_t st);
// pi_A, pi_B, pi_C in XYZZ coordinates, before the affine conversion.
struct ProofXyzz {
  host::Xyzz<host::Fp> a, c;
  host::Xyzz<host::Fp2> b;
};
// pi_A, pi_B, pi_C from the MSM sums: a = A (alpha1 included), b = B2
// (beta2 included), c = the C part plus the H part; b1 (the B1 MSM), r and s
// are null for the unblinded proof.
ProofXyzz assemble_proof(const zk_circuit* c, const host::Xyzz<host::Fp>& a,
                         const host::Xyzz<host::Fp2>& b, const host::Xyzz<host::Fp>& c_plus_h,
                         const host::Xyzz<host::Fp>* b1, const uint64_t* r, const uint64_t* s);
// Affine proofs (pi_A[8], pi_B[16], pi_C[8] u64 Montgomery) of n assembled
// proofs with one field inversion for all of them.
void proofs_to_affine(const ProofXyzz* p, size_t n, uint64_t* const* out);

uint64_t next_circuit_id();

}  // namespace zk
