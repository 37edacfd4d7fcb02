// Proof and public-signal serialization on the host.
//
// Output formats are the reference's, character for character:
//   proof JSON  groth16ProofToSnarkjsJson (src/groth16.cu:1467-1502)
//   calldata    groth16ProofToCalldata (src/groth16.cu:1509-1557)
//   public.json writePublicJson (src/main.cu:28-110)
// The reference decodes Montgomery coordinates with one-element GPU kernel
// launches (src/groth16.cu:1432-1465); here decoding is host arithmetic.
#include <cstdio>
#include <cstring>
#include <string>

#include "host_field.hpp"
#include "runtime.hpp"
#include "serialize.hpp"

namespace zk {

std::string dec_string(const uint64_t v[4]) {
  uint64_t n[4];
  memcpy(n, v, 32);
  char tmp[96];
  int len = 0;
  do {
    uint64_t rem = 0;
    for (int i = 3; i >= 0; i--) {
      const unsigned __int128 d = ((unsigned __int128)rem << 64) | n[i];
      n[i] = (uint64_t)(d / 10);
      rem = (uint64_t)(d % 10);
    }
    tmp[len++] = (char)('0' + rem);
  } while (n[0] | n[1] | n[2] | n[3]);
  std::string s(len, '0');
  for (int i = 0; i < len; i++) s[i] = tmp[len - 1 - i];
  return s;
}

static std::string fp_dec(const uint64_t* mont) {
  const host::Fp x = host::Fp::from_raw(mont).from_mont();
  return dec_string(x.v);
}

std::string proof_json(const uint64_t proof[32]) {
  const uint64_t* a = proof;
  const uint64_t* b = proof + 8;
  const uint64_t* c = proof + 24;
  char buf[2048];
  snprintf(buf, sizeof(buf),
           "{\n"
           " \"pi_a\": [\"%s\",\"%s\",\"1\"],\n"
           " \"pi_b\": [[\"%s\",\"%s\"],[\"%s\",\"%s\"],[\"1\",\"0\"]],\n"
           " \"pi_c\": [\"%s\",\"%s\",\"1\"],\n"
           " \"protocol\": \"groth16\",\n"
           " \"curve\": \"bn128\"\n"
           "}",
           fp_dec(a).c_str(), fp_dec(a + 4).c_str(), fp_dec(b).c_str(), fp_dec(b + 4).c_str(),
           fp_dec(b + 8).c_str(), fp_dec(b + 12).c_str(), fp_dec(c).c_str(), fp_dec(c + 4).c_str());
  return buf;
}

static void be32(const uint64_t* mont, uint8_t* out) {
  const host::Fp x = host::Fp::from_raw(mont).from_mont();
  for (int i = 0; i < 4; i++) {
    const uint64_t v = x.v[3 - i];
    for (int j = 0; j < 8; j++) out[i * 8 + j] = (uint8_t)(v >> ((7 - j) * 8));
  }
}

void proof_calldata(const uint64_t proof[32], uint8_t out[256]) {
  // A.x, A.y, B.x.a1, B.x.a0, B.y.a1, B.y.a0, C.x, C.y, big-endian canonical
  be32(proof, out);
  be32(proof + 4, out + 32);
  be32(proof + 12, out + 64);
  be32(proof + 8, out + 96);
  be32(proof + 20, out + 128);
  be32(proof + 16, out + 160);
  be32(proof + 24, out + 192);
  be32(proof + 28, out + 224);
}

std::string public_json(const uint64_t* values, uint32_t n_public) {
  std::string s = "[\n";
  for (uint32_t i = 0; i < n_public; i++) {
    s += " \"" + dec_string(values + 4 * (size_t)i) + "\"";
    s += (i + 1 < n_public) ? ",\n" : "\n";
  }
  s += "]\n";
  return s;
}

}  // namespace zk
