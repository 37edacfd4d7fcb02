// Seeded synthetic R1CS circuits with a matching Groth16 CRS, written as
// snarkjs-layout .zkey / .wtns files.  The reference ships no zkeys (its
// benchmark circuits need circom + snarkjs + a ptau download); these stand in
// for them with the shapes of the benchmark configurations.
//
// Circuit (domain n = 2^log_domain, l public inputs, k private inputs):
//   w_0 = 1, w_1..w_l public, w_{l+1}..w_{l+k} private inputs, then one
//   output variable per gate.  Gate row i: A and B rows with nnz in
//   [nnz_min, nnz_max] on random earlier variables with random nonzero
//   coefficients; C row = 1 * w_out(i).  Then l + 1 public rows
//   A[nG + s][s] = 1 (the snarkjs convention that binds public inputs), so
//   nG = n - l - 1 gates fill the domain exactly.
// Witness kinds: 0 "uniform": inputs uniform in Fr, w_out = (A.w)(B.w);
//   1 "circom": every variable is drawn from {0,1} (55%), [0, 2^64) (15%) or
//   Fr (30%) and the last B coefficient of each gate is solved so that
//   (A.w)(B.w) = w_out.
// CRS (toxic waste tau, alpha, beta, gamma, delta from the seed):
//   A_i = u_i(tau) G1, B1_i = v_i(tau) G1, B2_i = v_i(tau) G2,
//   C_i = (beta u_i + alpha v_i + w_i)(tau) / delta G1   (i > l),
//   IC_i = (beta u_i + alpha v_i + w_i)(tau) / gamma G1  (i <= l),
//   H_j = L^{2n}_{2j+1}(tau) / delta G1: the odd-index Lagrange basis of the
//   size-2n domain, which is what the prover's h_odd evaluations
//   (src/groth16.cu:1024-1090) pair with.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "capi_util.hpp"
#include "host_field.hpp"
#include "runtime.hpp"

namespace zk {
void mul_generator(int group, const uint64_t* scalars, size_t n, uint64_t* px, uint64_t* py,
                   cudaStream_t st);

namespace {

using host::Fr;

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto& v : s) {  // splitmix64 seeding
      x += 0x9e3779b97f4a7c15ULL;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      v = z ^ (z >> 31);
    }
  }
  uint64_t next() {  // xoshiro256**
    const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t below(uint64_t n) { return next() % n; }
  double unit() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  // uniform canonical element of Fr (rejection sampling on 254 bits)
  Fr fr_canon() {
    for (;;) {
      Fr x{{next(), next(), next(), next() & 0x3fffffffffffffffULL}};
      uint64_t t[4];
      if (Fr::sub4(t, x.v, host::FR_PARAMS.p)) return x;
    }
  }
  Fr fr_mont_nonzero() {
    for (;;) {
      Fr x = fr_canon();
      if (!x.is_zero()) return x.to_mont();
    }
  }
};

Fr root_of_unity(int lg) {  // omega_{2^lg} = 5^((r-1)/2^28)^(2^(28-lg)), Montgomery
  uint64_t e[4];
  memcpy(e, host::FR_PARAMS.p, 32);
  e[0] -= 1;
  for (int i = 0; i < 28; i++) {
    e[0] = (e[0] >> 1) | (e[1] << 63);
    e[1] = (e[1] >> 1) | (e[2] << 63);
    e[2] = (e[2] >> 1) | (e[3] << 63);
    e[3] >>= 1;
  }
  Fr w = Fr::from_u64(5).pow(e);
  for (int i = lg; i < 28; i++) w = w.sqr();
  return w;
}

void batch_inverse(std::vector<Fr>& v) {
  std::vector<Fr> pre(v.size());
  Fr acc = Fr::one();
  for (size_t i = 0; i < v.size(); i++) {
    pre[i] = acc;
    acc = acc * v[i];
  }
  Fr inv = acc.inv();
  for (size_t i = v.size(); i-- > 0;) {
    const Fr t = inv * pre[i];
    inv = inv * v[i];
    v[i] = t;
  }
}

// Lagrange basis of the size-M domain at tau: L_k = (tau^M - 1)/M * w^k/(tau - w^k)
// for the indices k = first + step * j, j < count.
std::vector<Fr> lagrange(const Fr& tau, int lg, size_t first, size_t step, size_t count) {
  const Fr w = root_of_unity(lg);
  const uint64_t M = uint64_t(1) << lg;
  Fr tm = tau;
  for (int i = 0; i < lg; i++) tm = tm.sqr();
  const Fr zf = (tm - Fr::one()) * Fr::from_u64(M).inv();
  uint64_t e[4] = {first, 0, 0, 0}, es[4] = {step, 0, 0, 0};
  Fr wk = w.pow(e), ws = w.pow(es);
  std::vector<Fr> num(count), den(count);
  for (size_t j = 0; j < count; j++) {
    num[j] = zf * wk;
    den[j] = tau - wk;
    wk = wk * ws;
  }
  batch_inverse(den);
  for (size_t j = 0; j < count; j++) num[j] = num[j] * den[j];
  return num;
}

struct Entry {
  uint32_t row, sig;
  Fr coef;  // Montgomery
};

void put32(std::vector<uint8_t>& b, uint32_t v) {
  const size_t o = b.size();
  b.resize(o + 4);
  memcpy(&b[o], &v, 4);
}
void put64(std::vector<uint8_t>& b, uint64_t v) {
  const size_t o = b.size();
  b.resize(o + 8);
  memcpy(&b[o], &v, 8);
}
void put_bytes(std::vector<uint8_t>& b, const void* p, size_t n) {
  const size_t o = b.size();
  b.resize(o + n);
  memcpy(&b[o], p, n);
}
size_t begin_section(std::vector<uint8_t>& b, uint32_t type) {
  put32(b, type);
  put64(b, 0);
  return b.size();
}
void end_section(std::vector<uint8_t>& b, size_t start) {
  const uint64_t sz = b.size() - start;
  memcpy(&b[start - 8], &sz, 8);
}

// k_i * G on the device for canonical scalars, AoS (x, y) records appended to `out`
void points(int group, const std::vector<Fr>& canon, cudaStream_t st, std::vector<uint8_t>& out) {
  const size_t n = canon.size(), w = group == 1 ? 4 : 8;
  if (!n) return;
  const size_t chunk = size_t(1) << 22;
  DeviceBuffer dsc, dx, dy;
  dsc.ensure(32 * std::min(n, chunk));
  dx.ensure(8 * w * std::min(n, chunk));
  dy.ensure(8 * w * std::min(n, chunk));
  std::vector<uint64_t> hx(w * std::min(n, chunk)), hy(w * std::min(n, chunk));
  for (size_t off = 0; off < n; off += chunk) {
    const size_t cnt = std::min(chunk, n - off);
    ZK_CUDA(cudaMemcpyAsync(dsc.ptr, canon[off].v, 32 * cnt, cudaMemcpyHostToDevice, st));
    mul_generator(group, dsc.as<uint64_t>(), cnt, dx.as<uint64_t>(), dy.as<uint64_t>(), st);
    ZK_CUDA(cudaMemcpyAsync(hx.data(), dx.ptr, 8 * w * cnt, cudaMemcpyDeviceToHost, st));
    ZK_CUDA(cudaMemcpyAsync(hy.data(), dy.ptr, 8 * w * cnt, cudaMemcpyDeviceToHost, st));
    ZK_CUDA(cudaStreamSynchronize(st));
    const size_t o = out.size();
    out.resize(o + 16 * w * cnt);
    uint8_t* d = &out[o];
    for (size_t i = 0; i < cnt; i++) {
      memcpy(d + 16 * w * i, &hx[w * i], 8 * w);
      memcpy(d + 16 * w * i + 8 * w, &hy[w * i], 8 * w);
    }
  }
}

void write_file(const std::string& path, const std::vector<uint8_t>& b) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) throw Error(ZK_EIO, "cannot write " + path);
  const size_t wr = fwrite(b.data(), 1, b.size(), f);
  fclose(f);
  if (wr != b.size()) throw Error(ZK_EIO, "short write to " + path);
}

}  // namespace

void synth_circuit(zk_ctx* ctx, const zk_synth_params& P, const char* zkey_path,
                   const char* wtns_path) {
  ZK_REQUIRE(P.log_domain >= 2 && P.log_domain <= 24, ZK_EINVAL, "synth: log_domain in [2, 24]");
  const uint32_t n = 1u << P.log_domain, l = P.n_public, k = P.n_private_inputs;
  ZK_REQUIRE(l + 2 < n, ZK_EINVAL, "synth: too many public inputs for the domain");
  ZK_REQUIRE(P.nnz_min >= 1 && P.nnz_max >= P.nnz_min && P.nnz_max <= 16, ZK_EINVAL,
             "synth: nnz range must satisfy 1 <= nnz_min <= nnz_max <= 16");
  ZK_REQUIRE(P.witness_kind <= 1, ZK_EINVAL, "synth: witness_kind is 0 or 1");
  const uint32_t nG = n - l - 1;
  const uint64_t m1 = 1ull + l + k + nG;
  ZK_REQUIRE(m1 < (1ull << 31), ZK_EINVAL, "synth: too many variables");
  Rng rng(P.seed);
  const Fr one = Fr::one();

  // ---- witness values (Montgomery while building)
  std::vector<Fr> w(m1);
  auto draw = [&](bool circom) -> Fr {
    if (!circom) return rng.fr_canon().to_mont();
    const double u = rng.unit();
    if (u < 0.55) return Fr::from_u64(rng.below(2));
    if (u < 0.70) return Fr::from_u64(rng.next());
    return rng.fr_canon().to_mont();
  };
  const bool circom = P.witness_kind == 1;
  w[0] = one;
  for (uint64_t i = 1; i <= (uint64_t)l + k; i++) w[i] = draw(circom);
  const uint64_t out0 = 1ull + l + k;
  if (circom)
    for (uint64_t i = out0; i < m1; i++) w[i] = draw(true);

  // ---- R1CS rows
  std::vector<Entry> A, B;
  A.reserve((size_t)nG * P.nnz_max + l + 1);
  B.reserve((size_t)nG * P.nnz_max);
  std::vector<uint32_t> solve_at;      // circom: index in B of the solved entry per gate
  std::vector<Fr> a_val, need;         // circom: A.w, and B.w target minus partial
  std::vector<Fr> inv_in;              // values to invert
  const uint32_t span = P.nnz_max - P.nnz_min + 1;
  for (uint32_t g = 0; g < nG; g++) {
    const uint64_t avail = out0 + g;  // earlier variables
    const uint32_t na = P.nnz_min + (uint32_t)rng.below(span);
    const uint32_t nb = P.nnz_min + (uint32_t)rng.below(span);
    Fr a = Fr::zero();
    for (int tries = 0;; tries++) {
      const size_t mark = A.size();
      a = Fr::zero();
      for (uint32_t j = 0; j < na; j++) {
        const uint32_t v = (uint32_t)rng.below(avail);
        const Fr cf = rng.fr_mont_nonzero();
        A.push_back({g, v, cf});
        a = a + cf * w[v];
      }
      if (!circom || !a.is_zero() || tries > 8) {
        if (circom && a.is_zero()) {  // fall back to the constant-one variable
          const Fr cf = rng.fr_mont_nonzero();
          A.push_back({g, 0, cf});
          a = a + cf;
        }
        break;
      }
      A.resize(mark);
    }
    Fr b = Fr::zero();
    for (uint32_t j = 0; j < nb; j++) {
      uint32_t v = (uint32_t)rng.below(avail);
      if (circom && j + 1 == nb) {
        for (int t = 0; t < 8 && w[v].is_zero(); t++) v = (uint32_t)rng.below(avail);
        if (w[v].is_zero()) v = 0;
        solve_at.push_back((uint32_t)B.size());
        B.push_back({g, v, Fr::zero()});
        continue;
      }
      const Fr cf = rng.fr_mont_nonzero();
      B.push_back({g, v, cf});
      b = b + cf * w[v];
    }
    if (circom) {
      a_val.push_back(a);
      need.push_back(b);  // partial B.w so far
      inv_in.push_back(a);
      inv_in.push_back(w[B.back().sig]);
    } else {
      w[out0 + g] = a * b;
    }
  }
  if (circom) {
    batch_inverse(inv_in);
    for (uint32_t g = 0; g < nG; g++) {
      // (a)(b_partial + c w_x) = w_out  =>  c = (w_out / a - b_partial) / w_x
      const Fr c = (w[out0 + g] * inv_in[2 * g] - need[g]) * inv_in[2 * g + 1];
      B[solve_at[g]].coef = c;
    }
  }
  for (uint32_t s = 0; s <= l; s++) A.push_back({nG + s, s, one});  // public rows

  // ---- QAP at tau
  const Fr tau = rng.fr_mont_nonzero(), alpha = rng.fr_mont_nonzero(),
           beta = rng.fr_mont_nonzero(), gamma = rng.fr_mont_nonzero(),
           delta = rng.fr_mont_nonzero();
  const std::vector<Fr> L = lagrange(tau, (int)P.log_domain, 0, 1, n);
  std::vector<Fr> u(m1, Fr::zero()), v(m1, Fr::zero()), cw(m1, Fr::zero());
  for (const Entry& e : A) u[e.sig] = u[e.sig] + e.coef * L[e.row];
  for (const Entry& e : B) v[e.sig] = v[e.sig] + e.coef * L[e.row];
  for (uint32_t g = 0; g < nG; g++) cw[out0 + g] = cw[out0 + g] + L[g];
  const Fr gi = gamma.inv(), di = delta.inv();
  std::vector<Fr> sA(m1), sB(m1), sC, sIC;
  for (uint64_t i = 0; i < m1; i++) {
    sA[i] = u[i].from_mont();
    sB[i] = v[i].from_mont();
    const Fr q = beta * u[i] + alpha * v[i] + cw[i];
    if (i <= l) sIC.push_back((q * gi).from_mont());
    else sC.push_back((q * di).from_mont());
  }
  std::vector<Fr> sH = lagrange(tau, (int)P.log_domain + 1, 1, 2, n);
  for (auto& x : sH) x = (x * di).from_mont();

  // ---- zkey
  zk_ctx* c = resolve_ctx(ctx);
  cudaStream_t st = c->stream;
  std::vector<uint8_t> z;
  z.reserve(64 + 1200 + 44 * (A.size() + B.size()) + 64 * (4 * m1 + n) + 128 * m1);
  put_bytes(z, "zkey", 4);
  put32(z, 1);
  put32(z, 9);
  size_t s = begin_section(z, 1);
  put32(z, 1);
  end_section(z, s);
  s = begin_section(z, 2);
  put32(z, 32);
  put_bytes(z, host::FP_PARAMS.p, 32);
  put32(z, 32);
  put_bytes(z, host::FR_PARAMS.p, 32);
  put32(z, (uint32_t)m1);
  put32(z, l);
  put32(z, n);
  const std::vector<Fr> vk1 = {alpha.from_mont(), beta.from_mont(), delta.from_mont()};
  const std::vector<Fr> vk2 = {beta.from_mont(), gamma.from_mont(), delta.from_mont()};
  std::vector<uint8_t> p1, p2;
  points(1, vk1, st, p1);
  points(2, vk2, st, p2);
  put_bytes(z, &p1[0], 64);     // alpha1
  put_bytes(z, &p1[64], 64);    // beta1
  put_bytes(z, &p2[0], 128);    // beta2
  put_bytes(z, &p2[128], 128);  // gamma2
  put_bytes(z, &p1[128], 64);   // delta1
  put_bytes(z, &p2[256], 128);  // delta2
  end_section(z, s);
  s = begin_section(z, 3);
  points(1, sIC, st, z);
  end_section(z, s);
  s = begin_section(z, 4);
  put32(z, (uint32_t)(A.size() + B.size()));
  for (int m = 0; m < 2; m++)
    for (const Entry& e : (m ? B : A)) {
      put32(z, (uint32_t)m);
      put32(z, e.row);
      put32(z, e.sig);
      const Fr stored = e.coef.to_mont();  // coef * R^2 (F3)
      put_bytes(z, stored.v, 32);
    }
  end_section(z, s);
  s = begin_section(z, 5);
  points(1, sA, st, z);
  end_section(z, s);
  s = begin_section(z, 6);
  points(1, sB, st, z);
  end_section(z, s);
  s = begin_section(z, 7);
  points(2, sB, st, z);
  end_section(z, s);
  s = begin_section(z, 8);
  points(1, sC, st, z);
  end_section(z, s);
  s = begin_section(z, 9);
  points(1, sH, st, z);
  end_section(z, s);
  write_file(zkey_path, z);
  std::vector<uint8_t>().swap(z);

  // ---- wtns (version 2, canonical values)
  std::vector<uint8_t> wt;
  wt.reserve(64 + 32 * m1);
  put_bytes(wt, "wtns", 4);
  put32(wt, 2);
  put32(wt, 2);
  s = begin_section(wt, 1);
  put32(wt, 32);
  put_bytes(wt, host::FR_PARAMS.p, 32);
  put32(wt, (uint32_t)m1);
  end_section(wt, s);
  s = begin_section(wt, 2);
  for (uint64_t i = 0; i < m1; i++) {
    const Fr x = w[i].from_mont();
    put_bytes(wt, x.v, 32);
  }
  end_section(wt, s);
  write_file(wtns_path, wt);
}

}  // namespace zk

extern "C" int zk_synth_circuit(zk_ctx* ctx, const zk_synth_params* params, const char* zkey_path,
                                const char* wtns_path) {
  ZK_API_BEGIN
  ZK_REQUIRE(params && zkey_path && wtns_path, ZK_EINVAL, "zk_synth_circuit: NULL argument");
  zk::synth_circuit(ctx, *params, zkey_path, wtns_path);
  ZK_API_END
}
