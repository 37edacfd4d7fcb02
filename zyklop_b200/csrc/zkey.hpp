// snarkjs BinFile readers for .zkey (Groth16) and .wtns files.
//
// Same format contract as the reference's readers (src/binfile_utils.cpp:
// 15-178, src/zkey_utils.cpp:19-51, src/wtns_utils.cpp:13-26) and layout
// facts as the reference code reads them:
//   file     = magic[4] | version u32 | nSections u32 | {type u32, size u64, data}*
//   zkey §1  = protocol u32 (1 = Groth16)
//   zkey §2  = n8q u32, q, n8r u32, r, nVars u32, nPublic u32, domainSize u32,
//              alpha1 G1, beta1 G1, beta2 G2, gamma2 G2, delta1 G1, delta2 G2
//   zkey §3  = IC points (nPublic + 1) G1       §4 = nCoefs u32, 44-byte entries
//   zkey §5  = A (nVars) G1   §6 = B1 (nVars) G1   §7 = B2 (nVars) G2
//   zkey §8  = C (nVars - nPublic - 1) G1        §9 = H (domain) G1
//   wtns §1  = n8 u32, prime, nVars u32;  §2 = nVars x n8-byte values
// Points are affine Montgomery, G2 as (x.a0, x.a1, y.a0, y.a1).  The domain
// is the next power of two >= domainSize, as in src/groth16.cu:1155-1160.
// Unlike the reference, every size is checked against the file and a bad
// file is reported as ZK_EFORMAT instead of an uncaught exception / exit.
#pragma once
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace zk {

class BinFile {
 public:
  // Maps a file read-only (throws ZK_EIO / ZK_EFORMAT).
  static std::unique_ptr<BinFile> open(const std::string& path, const char* magic,
                                       uint32_t max_version);
  // Wraps caller memory (not copied; must outlive the BinFile).
  static std::unique_ptr<BinFile> wrap(const void* data, size_t len, const char* magic,
                                       uint32_t max_version);
  ~BinFile();
  BinFile(const BinFile&) = delete;
  BinFile& operator=(const BinFile&) = delete;

  // First section of this type, or nullptr (size 0) if absent.
  const uint8_t* section(uint32_t type, uint64_t* size) const;
  const uint8_t* data() const { return base_; }
  size_t size() const { return len_; }

 private:
  BinFile() = default;
  void parse(const char* magic, uint32_t max_version);
  const uint8_t* base_ = nullptr;
  size_t len_ = 0;
  void* map_ = nullptr;
  int fd_ = -1;
  struct Sec {
    uint32_t type;
    uint64_t off, size;
  };
  std::vector<Sec> secs_;
};

struct ZkeyView {
  uint32_t n_vars = 0, n_public = 0, domain_raw = 0, domain = 0;
  int log_n = 0;
  const uint64_t *alpha1 = nullptr, *beta1 = nullptr, *beta2 = nullptr, *gamma2 = nullptr,
                 *delta1 = nullptr, *delta2 = nullptr;
  const uint8_t* coefs = nullptr;  // n_coefs x 44 bytes
  uint32_t n_coefs = 0;
  const uint64_t* ic = nullptr;    // (n_public + 1) x 8 u64, may be null
  const uint64_t* a = nullptr;     // n_vars x 8 u64
  const uint64_t* b1 = nullptr;    // n_vars x 8 u64, may be null
  const uint64_t* b2 = nullptr;    // n_vars x 16 u64
  const uint64_t* c = nullptr;     // (n_vars - n_public - 1) x 8 u64
  const uint64_t* h = nullptr;     // domain x 8 u64
};

ZkeyView parse_zkey(const BinFile& f);

struct WtnsView {
  uint32_t n_vars = 0;
  const uint64_t* values = nullptr;  // n_vars x 4 u64 canonical
};

WtnsView parse_wtns(const BinFile& f);

}  // namespace zk
