// snarkjs BinFile readers (see zkey.hpp).
#include "zkey.hpp"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstring>

#include "runtime.hpp"

namespace zk {

namespace {
const uint64_t kP[4] = {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL,
                        0x30644e72e131a029ULL};
const uint64_t kR[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL,
                        0x30644e72e131a029ULL};

uint32_t rd32(const uint8_t* p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}
uint64_t rd64(const uint8_t* p) {
  uint64_t v;
  memcpy(&v, p, 8);
  return v;
}
[[noreturn]] void bad(const std::string& m) { throw Error(ZK_EFORMAT, m); }
}  // namespace

std::unique_ptr<BinFile> BinFile::open(const std::string& path, const char* magic,
                                       uint32_t max_version) {
  std::unique_ptr<BinFile> f(new BinFile());
  f->fd_ = ::open(path.c_str(), O_RDONLY);
  if (f->fd_ < 0) throw Error(ZK_EIO, "cannot open " + path + ": " + strerror(errno));
  struct stat st;
  if (fstat(f->fd_, &st) != 0) throw Error(ZK_EIO, "cannot stat " + path);
  f->len_ = (size_t)st.st_size;
  if (f->len_ == 0) bad(path + ": empty file");
  f->map_ = mmap(nullptr, f->len_, PROT_READ, MAP_PRIVATE, f->fd_, 0);
  if (f->map_ == MAP_FAILED) {
    f->map_ = nullptr;
    throw Error(ZK_EIO, "cannot map " + path);
  }
  madvise(f->map_, f->len_, MADV_SEQUENTIAL);
  f->base_ = reinterpret_cast<const uint8_t*>(f->map_);
  f->parse(magic, max_version);
  return f;
}

std::unique_ptr<BinFile> BinFile::wrap(const void* data, size_t len, const char* magic,
                                       uint32_t max_version) {
  if (!data) throw Error(ZK_EINVAL, "NULL file image");
  std::unique_ptr<BinFile> f(new BinFile());
  f->base_ = reinterpret_cast<const uint8_t*>(data);
  f->len_ = len;
  f->parse(magic, max_version);
  return f;
}

BinFile::~BinFile() {
  if (map_) munmap(map_, len_);
  if (fd_ >= 0) ::close(fd_);
}

void BinFile::parse(const char* magic, uint32_t max_version) {
  if (len_ < 12) bad("file is too short");
  if (memcmp(base_, magic, 4) != 0) bad(std::string("invalid file type, expected ") + magic);
  const uint32_t version = rd32(base_ + 4);
  if (version > max_version) bad("unsupported file version " + std::to_string(version));
  const uint32_t ns = rd32(base_ + 8);
  uint64_t pos = 12;
  for (uint32_t i = 0; i < ns; i++) {
    if (pos + 12 > len_) bad("truncated section table");
    const uint32_t t = rd32(base_ + pos);
    const uint64_t s = rd64(base_ + pos + 4);
    pos += 12;
    if (s > len_ - pos) bad("section " + std::to_string(i) + " runs past the end of the file");
    secs_.push_back({t, pos, s});
    pos += s;
  }
}

const uint8_t* BinFile::section(uint32_t type, uint64_t* size) const {
  for (const Sec& s : secs_)
    if (s.type == type) {
      if (size) *size = s.size;
      return base_ + s.off;
    }
  if (size) *size = 0;
  return nullptr;
}

ZkeyView parse_zkey(const BinFile& f) {
  ZkeyView z;
  uint64_t sz;
  const uint8_t* s1 = f.section(1, &sz);
  if (!s1 || sz < 4) bad("zkey: missing header section 1");
  if (rd32(s1) != 1) bad("zkey file is not groth16");
  const uint8_t* s2 = f.section(2, &sz);
  if (!s2 || sz < 4 + 32 + 4 + 32 + 12 + 6 * 64) bad("zkey: missing or short section 2");
  if (rd32(s2) != 32) bad("zkey: base field is not 32 bytes");
  if (memcmp(s2 + 4, kP, 32) != 0) bad("zkey: base field is not BN254");
  if (rd32(s2 + 36) != 32) bad("zkey: scalar field is not 32 bytes");
  if (memcmp(s2 + 40, kR, 32) != 0) bad("zkey: scalar field is not BN254");
  const uint8_t* p = s2 + 72;
  z.n_vars = rd32(p);
  z.n_public = rd32(p + 4);
  z.domain_raw = rd32(p + 8);
  p += 12;
  if (sz < (uint64_t)(p - s2) + 2 * 64 + 2 * 128 + 64 + 128) bad("zkey: section 2 too short");
  z.alpha1 = reinterpret_cast<const uint64_t*>(p);
  z.beta1 = reinterpret_cast<const uint64_t*>(p + 64);
  z.beta2 = reinterpret_cast<const uint64_t*>(p + 128);
  z.gamma2 = reinterpret_cast<const uint64_t*>(p + 256);
  z.delta1 = reinterpret_cast<const uint64_t*>(p + 384);
  z.delta2 = reinterpret_cast<const uint64_t*>(p + 448);
  if (z.n_vars < z.n_public + 1) bad("zkey: nVars < nPublic + 1");
  if (z.domain_raw == 0 || z.domain_raw > (1u << 27)) bad("zkey: domain size out of range");
  z.domain = 1;
  z.log_n = 0;
  while (z.domain < z.domain_raw) {
    z.domain <<= 1;
    z.log_n++;
  }
  const uint8_t* s4 = f.section(4, &sz);
  if (!s4 || sz < 4) bad("zkey: missing section 4");
  z.n_coefs = rd32(s4);
  if (4 + 44ull * z.n_coefs > sz) bad("zkey: section 4 shorter than its entry count");
  z.coefs = s4 + 4;
  const uint64_t m1 = z.n_vars, nc = (uint64_t)z.n_vars - z.n_public - 1;
  auto need = [&](uint32_t id, uint64_t bytes, bool required) -> const uint64_t* {
    uint64_t s;
    const uint8_t* d = f.section(id, &s);
    if (!d) {
      if (required) bad("zkey: missing section " + std::to_string(id));
      return nullptr;
    }
    if (s < bytes) bad("zkey: section " + std::to_string(id) + " is too short");
    return reinterpret_cast<const uint64_t*>(d);
  };
  z.ic = need(3, 64ull * (z.n_public + 1), false);
  z.a = need(5, 64 * m1, true);
  z.b1 = need(6, 64 * m1, false);
  z.b2 = need(7, 128 * m1, true);
  z.c = need(8, 64 * nc, true);
  z.h = need(9, 64ull * z.domain, true);
  return z;
}

WtnsView parse_wtns(const BinFile& f) {
  WtnsView w;
  uint64_t sz;
  const uint8_t* s1 = f.section(1, &sz);
  if (!s1 || sz < 40) bad("wtns: missing or short section 1");
  if (rd32(s1) != 32) bad("wtns: field element size is not 32 bytes");
  if (memcmp(s1 + 4, kR, 32) != 0) bad("wtns: field is not the BN254 scalar field");
  w.n_vars = rd32(s1 + 36);
  const uint8_t* s2 = f.section(2, &sz);
  if (!s2) bad("wtns: missing section 2");
  if (sz < 32ull * w.n_vars) bad("wtns: section 2 shorter than nVars values");
  w.values = reinterpret_cast<const uint64_t*>(s2);
  return w;
}

}  // namespace zk
