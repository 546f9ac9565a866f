// Host-side LDPCA ladder: load the compact ladder file, expand the per-code
// tables, compute the GF(2) inverse of the full-rate matrix, upload.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "dvc_types.h"

namespace dvc {

struct LadderHost {
  int n = 0, e = 0, period = 0, num_codes = 0, invh_words = 0;
  std::vector<int> jc, bpp, idx, synd_len, row_ptr;
  std::vector<float> code_rate;
  std::vector<uint16_t> ir, row_edge, pos, rid;
  std::vector<uint8_t> crc_tab;
  std::vector<uint32_t> invh;
  std::vector<int> ir_full;  // full-rate rows (the encoder's parity-check matrix)
  std::vector<uint16_t> ir_full16;
};

// Reads every ladder in `path` (layout documented in ladders/ladders.py).
bool load_ladders(const std::string &path, std::vector<LadderHost> &out, std::string &err);
// GF(2) inverse of the full-rate matrix, cached in `cache_path` when given.
bool ladder_inverse(LadderHost &L, const std::string &cache_path, std::string &err);

// Device copy; owns its allocations.
struct LadderGpu {
  LadderDev dev{};
  std::vector<void *> allocs;
  bool upload(const LadderHost &L, std::string &err);
  void release();
};

uint8_t crc8_bytes(const uint8_t *p, int n);

}  // namespace dvc
