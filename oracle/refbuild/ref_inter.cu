// Harness that runs the reference prover's own pipeline steps one by one and
// hands back every intermediate, so tests can compare them bit for bit with
// the library's.  The reference translation unit src/groth16.cu is included
// unmodified (its steps are `static`, so they are reachable only from inside
// that unit); nothing here computes anything itself.  Test infrastructure,
// compiled for sm_100a by oracle/refbuild/Makefile.
//
// Steps called, in groth16Prove's order (src/groth16.cu:1143-1397):
//   nttPrepare                 include/ntt_bn254.cuh:190-261
//   readWitness                src/groth16.cu:867-893
//   readAndComputeMVM          src/groth16.cu:737-861   -> A.w, B.w
//   computeHPoly               src/groth16.cu:1037-1128 -> coset evaluations, h
//   readAndUnpackG1/G2Chunked  src/groth16.cu:563-681   -> SoA CRS points
//   msm_g1 / msm_g2_device     include/msm_g1.cuh:918, include/msm_g2.cuh:669
#include "groth16.cu"

namespace {

void copy_out(uint64_t* dst, const uint64_t* d_src, size_t n) {
  if (dst) G16_CUDA_CHECK(cudaMemcpy(dst, d_src, n * 32, cudaMemcpyDeviceToHost));
}

void g1_out(const FpPointAff& p, uint64_t* out) {
  memcpy(out, p.X, 32);
  memcpy(out + 4, p.Y, 32);
}

}  // namespace

extern "C" {

// Intermediates of the reference's unblinded proof of (zkey, wtns); any output
// may be NULL.  aw, bw: A.w and B.w (Montgomery, domain x 4 u64) as
// readAndComputeMVM leaves them; ea, eb, ec: the coset evaluations of A, B and
// C = A.B that computeHPoly leaves in its three buffers (Montgomery, natural
// order); h: its canonical output.  msm: the four MSM results, affine
// Montgomery: A (8 u64, alpha1 included), B2 (16), C part (8), H part (8).
// inf[4]: 1 where that MSM result is the point at infinity.
int zkref_intermediates(const char* zkey_path, const char* wtns_path, uint64_t* aw, uint64_t* bw,
                        uint64_t* ea, uint64_t* eb, uint64_t* ec, uint64_t* h, uint64_t* msm_a,
                        uint64_t* msm_b2, uint64_t* msm_c, uint64_t* msm_h, int* inf) {
  BinFileUtils::BinFile zkey(zkey_path, "zkey", 1);
  auto zkh = ZKeyUtils::loadHeader(&zkey);
  uint32_t n = 1;
  int ld = 0;
  while (n < (uint32_t)zkh->domainSize) {
    n <<= 1;
    ld++;
  }
  const uint32_t m1 = zkh->nVars, l = zkh->nPublic;
  nttPrepare(ld + 1);
  std::vector<uint64_t> w = readWitness(wtns_path, m1);

  uint64_t *d_Aw, *d_Bw, *d_Cw, *d_h;
  readAndComputeMVM(zkey, w, m1, n, &d_Aw, &d_Bw);
  copy_out(aw, d_Aw, n);
  copy_out(bw, d_Bw, n);
  G16_CUDA_CHECK(cudaMalloc(&d_Cw, (size_t)n * 32));
  G16_CUDA_CHECK(cudaMalloc(&d_h, (size_t)n * 32));
  G16_CUDA_CHECK(cudaMemset(d_Cw, 0, (size_t)n * 32));
  G16_CUDA_CHECK(cudaMemset(d_h, 0, (size_t)n * 32));
  computeHPoly(d_Aw, d_Bw, d_Cw, ld, d_h, nullptr);
  G16_CUDA_CHECK(cudaDeviceSynchronize());
  copy_out(ea, d_Aw, n);
  copy_out(eb, d_Bw, n);
  copy_out(ec, d_Cw, n);
  copy_out(h, d_h, n);

  // CRS points: A and B2 lead with alpha1 / beta2 under the scalar 1
  const uint32_t m1e = m1 + 1, nc = m1 - l - 1;
  uint64_t *ax, *ay, *bx, *by, *cx, *cy, *hx, *hy, *we;
  G16_CUDA_CHECK(cudaMalloc(&ax, (size_t)m1e * 32));
  G16_CUDA_CHECK(cudaMalloc(&ay, (size_t)m1e * 32));
  G16_CUDA_CHECK(cudaMalloc(&bx, (size_t)m1e * 64));
  G16_CUDA_CHECK(cudaMalloc(&by, (size_t)m1e * 64));
  G16_CUDA_CHECK(cudaMalloc(&cx, (size_t)(nc ? nc : 1) * 32));
  G16_CUDA_CHECK(cudaMalloc(&cy, (size_t)(nc ? nc : 1) * 32));
  G16_CUDA_CHECK(cudaMalloc(&hx, (size_t)n * 32));
  G16_CUDA_CHECK(cudaMalloc(&hy, (size_t)n * 32));
  const uint64_t* alpha1 = (const uint64_t*)zkh->vk_alpha1;
  const uint64_t* beta2 = (const uint64_t*)zkh->vk_beta2;
  G16_CUDA_CHECK(cudaMemcpy(ax, alpha1, 32, cudaMemcpyHostToDevice));
  G16_CUDA_CHECK(cudaMemcpy(ay, alpha1 + 4, 32, cudaMemcpyHostToDevice));
  G16_CUDA_CHECK(cudaMemcpy(bx, beta2, 64, cudaMemcpyHostToDevice));
  G16_CUDA_CHECK(cudaMemcpy(by, beta2 + 8, 64, cudaMemcpyHostToDevice));
  cudaStream_t st;
  G16_CUDA_CHECK(cudaStreamCreate(&st));
  readAndUnpackG1Chunked(zkey, 5, m1, ax + 4, ay + 4, st);
  readAndUnpackG2Chunked(zkey, 7, m1, bx + 8, by + 8, st);
  readAndUnpackG1Chunked(zkey, 8, nc, cx, cy, st);
  readAndUnpackG1Chunked(zkey, 9, n, hx, hy, st);
  G16_CUDA_CHECK(cudaStreamSynchronize(st));
  G16_CUDA_CHECK(cudaStreamDestroy(st));

  G16_CUDA_CHECK(cudaMalloc(&we, (size_t)m1e * 32));
  const uint64_t one[4] = {1, 0, 0, 0};
  G16_CUDA_CHECK(cudaMemcpy(we, one, 32, cudaMemcpyHostToDevice));
  G16_CUDA_CHECK(cudaMemcpy(we + 4, w.data(), (size_t)m1 * 32, cudaMemcpyHostToDevice));

  FpPointAff ra, rc, rh;
  Fp2PointAff rb;
  msm_g1(ax, ay, we, (int)m1e, ra);
  msm_g2_device(bx, by, we, (int)m1e, rb);
  msm_g1(cx, cy, we + (size_t)(l + 2) * 4, (int)nc, rc);
  msm_g1(hx, hy, d_h, (int)n, rh);
  if (msm_a) g1_out(ra, msm_a);
  if (msm_b2) {
    memcpy(msm_b2, rb.X, 64);
    memcpy(msm_b2 + 8, rb.Y, 64);
  }
  if (msm_c) g1_out(rc, msm_c);
  if (msm_h) g1_out(rh, msm_h);
  if (inf) {
    inf[0] = ra.infinity ? 1 : 0;
    inf[1] = rb.infinity ? 1 : 0;
    inf[2] = rc.infinity ? 1 : 0;
    inf[3] = rh.infinity ? 1 : 0;
  }

  for (uint64_t* p : {ax, ay, bx, by, cx, cy, hx, hy, we, d_Aw, d_Bw, d_Cw, d_h}) cudaFree(p);
  nttDestroy();
  return 0;
}

// computeHPoly (src/groth16.cu:1037-1128) on device buffers of 2^log_n
// Montgomery values: d_aw, d_bw are overwritten with the odd-coset
// evaluations of A and B, d_cw (scratch) with C's, and d_h receives h
// (canonical).  Three coset INTT / NTT pairs.
int zkref_hpoly_device(uint64_t* d_aw, uint64_t* d_bw, uint64_t* d_cw, int log_n, uint64_t* d_h) {
  nttPrepare(log_n + 1);
  computeHPoly(d_aw, d_bw, d_cw, log_n, d_h, nullptr);
  const cudaError_t e = cudaDeviceSynchronize();
  nttDestroy();
  return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
