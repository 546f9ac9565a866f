// LDPCA ladder loading and device upload.  See ladder.h.
#include "ladder.h"

#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

namespace dvc {

static uint8_t g_crc_table[256];
static bool g_crc_ready = false;

// CRC-8 with polynomial x^8 + x^2 + x + 1, initial value 0, no final xor
// (the reference's crc8.h:20-67); the byte table is generated from the polynomial.
uint8_t crc8_bytes(const uint8_t *p, int n) {
  if (!g_crc_ready) {
    for (int b = 0; b < 256; b++) {
      uint8_t c = (uint8_t)b;
      for (int k = 0; k < 8; k++) c = (uint8_t)((c & 0x80) ? ((c << 1) ^ 0x07) : (c << 1));
      g_crc_table[b] = c;
    }
    g_crc_ready = true;
  }
  uint8_t crc = 0;
  for (int i = 0; i < n; i++) crc = g_crc_table[crc ^ p[i]];
  return crc;
}

static bool rd(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

bool load_ladders(const std::string &path, std::vector<LadderHost> &out, std::string &err) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open ladder file " + path;
    return false;
  }
  char magic[4];
  uint32_t ver = 0, nl = 0;
  if (!rd(f, magic, 4) || memcmp(magic, "LDLA", 4) != 0 || !rd(f, &ver, 4) || ver != 1 || !rd(f, &nl, 4)) {
    fclose(f);
    err = "bad ladder file header in " + path;
    return false;
  }
  for (uint32_t l = 0; l < nl; l++) {
    uint32_t hdr[4];
    if (!rd(f, hdr, 16)) break;
    LadderHost L;
    L.n = (int)hdr[0];
    L.e = (int)hdr[1];
    L.period = (int)hdr[2];
    L.num_codes = (int)hdr[3];
    std::vector<uint16_t> jc16(L.n + 1), ir16(L.e);
    if (!rd(f, jc16.data(), 2 * jc16.size()) || !rd(f, ir16.data(), 2 * ir16.size())) break;
    L.jc.assign(jc16.begin(), jc16.end());
    L.ir_full.assign(ir16.begin(), ir16.end());
    L.ir_full16 = ir16;
    L.bpp.resize(L.num_codes);
    L.idx.assign((size_t)L.num_codes * L.period, 0);
    for (int c = 0; c < L.num_codes; c++) {
      uint16_t b;
      if (!rd(f, &b, 2)) {
        fclose(f);
        err = "truncated ladder file";
        return false;
      }
      L.bpp[c] = b;
      std::vector<uint16_t> tmp(b);
      if (!rd(f, tmp.data(), 2 * (size_t)b)) {
        fclose(f);
        err = "truncated ladder file";
        return false;
      }
      for (int k = 0; k < b; k++) L.idx[(size_t)c * L.period + k] = tmp[k];
    }
    // expand the per-code rows: row of edge e in code c is the first kept
    // accumulated-syndrome position >= its full-rate row
    L.synd_len.resize(L.num_codes);
    L.code_rate.resize(L.num_codes);
    L.ir.resize((size_t)L.num_codes * L.e);
    L.row_ptr.assign((size_t)L.num_codes * (L.n + 1), 0);
    L.row_edge.resize((size_t)L.num_codes * L.e);
    for (int c = 0; c < L.num_codes; c++) {
      const int b = L.bpp[c];
      const int m = (L.n / L.period) * b;
      L.synd_len[c] = m;
      L.code_rate[c] = (float)m / (float)L.n;  // ReadLdpcaLadderFile_LdpcaDecoder.cpp:182-183
      std::vector<int> bounds(m);
      for (int k = 0; k < m; k++) bounds[k] = L.idx[(size_t)c * L.period + k % b] + (k / b) * L.period;
      int *rp = &L.row_ptr[(size_t)c * (L.n + 1)];
      for (int e = 0; e < L.e; e++) {
        int r = (int)(std::lower_bound(bounds.begin(), bounds.end(), L.ir_full[e]) - bounds.begin());
        if (r >= m) {
          fclose(f);
          err = "ladder expansion out of range";
          return false;
        }
        L.ir[(size_t)c * L.e + e] = (uint16_t)r;
        rp[r + 1]++;
      }
      for (int r = 0; r < m; r++) rp[r + 1] += rp[r];
      for (int r = m; r < L.n; r++) rp[r + 1] = rp[r];
      std::vector<int> fill(rp, rp + m);
      for (int e = 0; e < L.e; e++) {
        const int r = L.ir[(size_t)c * L.e + e];
        L.row_edge[(size_t)c * L.e + fill[r]++] = (uint16_t)e;
      }
    }
    // the decoder kernel takes every column to have degree 3 (edge e = 3k + i)
    // and stages the per-code index arrays with 16-byte copies
    for (int k = 0; k <= L.n; k++)
      if (L.jc[k] != 3 * k) {
        fclose(f);
        err = "ladder with a column degree other than 3";
        return false;
      }
    if (L.e % 8 != 0 || L.e > 65535) {
      fclose(f);
      err = "ladder edge count not a multiple of 8 or above 65535";
      return false;
    }
    // row-order positions: pos[e] and the row of each position
    L.pos.resize((size_t)L.num_codes * L.e);
    L.rid.resize((size_t)L.num_codes * L.e);
    for (int c = 0; c < L.num_codes; c++)
      for (int p = 0; p < L.e; p++) {
        const int e = L.row_edge[(size_t)c * L.e + p];
        L.pos[(size_t)c * L.e + e] = (uint16_t)p;
        L.rid[(size_t)c * L.e + p] = L.ir[(size_t)c * L.e + e];
      }
    // CRC-8 is linear over GF(2) for a fixed message length (zero initial
    // value, no final xor), so the CRC of a bitplane is the xor of the CRCs
    // of its single set bits.
    L.crc_tab.resize(L.n);
    std::vector<uint8_t> msg(L.n / 8, 0);
    for (int i = 0; i < L.n; i++) {
      msg[i >> 3] = (uint8_t)(0x80 >> (i & 7));
      L.crc_tab[i] = crc8_bytes(msg.data(), L.n / 8);
      msg[i >> 3] = 0;
    }
    out.push_back(std::move(L));
  }
  fclose(f);
  if (out.empty()) {
    err = "no ladders in " + path;
    return false;
  }
  return true;
}

bool ladder_inverse(LadderHost &L, const std::string &cache_path, std::string &err) {
  const int n = L.n;
  L.invh_words = (n + 31) / 32;
  const size_t total = (size_t)n * L.invh_words;
  // the cache carries n and a checksum of the full-rate matrix it inverts
  uint64_t sig = 1469598103934665603ull;
  for (int v : L.ir_full) sig = (sig ^ (uint64_t)v) * 1099511628211ull;
  for (int v : L.jc) sig = (sig ^ (uint64_t)v) * 1099511628211ull;
  if (!cache_path.empty()) {
    FILE *f = fopen(cache_path.c_str(), "rb");
    if (f) {
      uint64_t hdr[2] = {0, 0};
      L.invh.resize(total);
      bool ok = rd(f, hdr, 16) && hdr[0] == (uint64_t)n && hdr[1] == sig && rd(f, L.invh.data(), 4 * total);
      fclose(f);
      if (ok) return true;
    }
  }
  const int w2 = (2 * n + 63) / 64;
  std::vector<uint64_t> a((size_t)n * w2, 0);
  for (int col = 0; col < n; col++)
    for (int e = L.jc[col]; e < L.jc[col + 1]; e++) {
      const int r = L.ir_full[e];
      a[(size_t)r * w2 + (col >> 6)] ^= 1ull << (col & 63);
    }
  for (int r = 0; r < n; r++) a[(size_t)r * w2 + ((n + r) >> 6)] |= 1ull << ((n + r) & 63);
  std::vector<uint64_t> tmp(w2);
  for (int col = 0; col < n; col++) {
    const int wi = col >> 6;
    const uint64_t bit = 1ull << (col & 63);
    int p = -1;
    for (int r = col; r < n; r++)
      if (a[(size_t)r * w2 + wi] & bit) {
        p = r;
        break;
      }
    if (p < 0) {
      err = "full-rate parity-check matrix is singular";
      return false;
    }
    if (p != col) {
      std::swap_ranges(a.begin() + (size_t)p * w2, a.begin() + (size_t)(p + 1) * w2, a.begin() + (size_t)col * w2);
    }
    const uint64_t *pr = &a[(size_t)col * w2];
    for (int r = 0; r < n; r++) {
      if (r == col) continue;
      uint64_t *rr = &a[(size_t)r * w2];
      if (rr[wi] & bit)
        for (int w = wi; w < w2; w++) rr[w] ^= pr[w];
    }
  }
  L.invh.assign(total, 0u);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      const int c = n + i;
      if ((a[(size_t)j * w2 + (c >> 6)] >> (c & 63)) & 1ull) L.invh[(size_t)j * L.invh_words + (i >> 5)] |= 1u << (i & 31);
    }
  if (!cache_path.empty()) {
    std::string tmpname = cache_path + ".tmp";
    FILE *f = fopen(tmpname.c_str(), "wb");
    if (f) {
      uint64_t hdr[2] = {(uint64_t)n, sig};
      fwrite(hdr, 8, 2, f);
      fwrite(L.invh.data(), 4, total, f);
      fclose(f);
      rename(tmpname.c_str(), cache_path.c_str());
    }
  }
  return true;
}

template <class T>
static bool put(std::vector<void *> &allocs, const std::vector<T> &v, const T **dst, std::string &err) {
  void *p = nullptr;
  const size_t bytes = v.size() * sizeof(T);
  if (cudaMalloc(&p, bytes ? bytes : 4) != cudaSuccess) {
    err = "cudaMalloc failed for ladder tables";
    return false;
  }
  allocs.push_back(p);
  if (bytes && cudaMemcpy(p, v.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    err = "cudaMemcpy failed for ladder tables";
    return false;
  }
  *dst = (const T *)p;
  return true;
}

bool LadderGpu::upload(const LadderHost &L, std::string &err) {
  dev.n = L.n;
  dev.e = L.e;
  dev.period = L.period;
  dev.num_codes = L.num_codes;
  dev.invh_words = L.invh_words;
  return put(allocs, L.jc, &dev.jc, err) && put(allocs, L.bpp, &dev.bpp, err) && put(allocs, L.idx, &dev.idx, err) &&
         put(allocs, L.synd_len, &dev.synd_len, err) && put(allocs, L.code_rate, &dev.code_rate, err) &&
         put(allocs, L.row_ptr, &dev.row_ptr, err) && put(allocs, L.pos, &dev.pos, err) &&
         put(allocs, L.rid, &dev.rid, err) && put(allocs, L.ir_full16, &dev.ir_full, err) &&
         put(allocs, L.crc_tab, &dev.crc_tab, err) && put(allocs, L.invh, &dev.invh, err);
}

void LadderGpu::release() {
  for (void *p : allocs) cudaFree(p);
  allocs.clear();
}

}  // namespace dvc
