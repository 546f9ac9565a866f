// Intra blocks of WZ frames (IntraMode 1): host decoder of the reference's
// intra bitstream.
//
// The reference codes the 4x4 blocks of intra 8x8 blocks H.264-style
// (DvcDec/src/intra.cpp:187-268, vlc.cpp:423-761): CAVLC coefficients
// (coeff_token, trailing-one signs, levels with an adaptive suffix length,
// total_zeros, run_before; the coeff_token table chosen by the predicted
// number of non-zero coefficients of the left and upper intra blocks),
// de-quantisation ROUND(c * 2^((QP-4)/6) * 64 pre-scale) in double, the 4x4
// integer inverse transform with a final >> 6, and DC prediction from the
// neighbouring pixels of left / upper blocks that are themselves intra.
// The bitstream is one bit string for the whole sequence: every intra 4x4
// block of every frame, frames in decoding order, blocks in raster order.
//
// The VLC tables are the standard's (ITU-T H.264 tables 9-5, 9-7 and 9-10,
// luma 4x4); they are written here as code strings and turned into prefix
// codes at first use, where they are checked to be prefix-free.  The decoder
// reads through a 64-bit window of the stream: symbols by direct lookup on
// its next 10 bits (a binary search for the coeff_tokens longer than that),
// level prefixes by counting leading zeros; only the coded coefficients are
// de-quantised, and a block whose only coefficient is the DC skips the
// transform (its 16 outputs all equal DC >> 6).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dvc_b200.h"

namespace {

// coeff_token, 0 <= nC < 2, 2 <= nC < 4, 4 <= nC < 8: code of
// (TrailingOnes t, TotalCoeff c) at [c][t] ("" where t > c)
const char *kCoeffToken[3][17][4] = {
    {{"1", "", "", ""},
     {"000101", "01", "", ""},
     {"00000111", "000100", "001", ""},
     {"000000111", "00000110", "0000101", "00011"},
     {"0000000111", "000000110", "00000101", "000011"},
     {"00000000111", "0000000110", "000000101", "0000100"},
     {"0000000001111", "00000000110", "0000000101", "00000100"},
     {"0000000001011", "0000000001110", "00000000101", "000000100"},
     {"0000000001000", "0000000001010", "0000000001101", "0000000100"},
     {"00000000001111", "00000000001110", "0000000001001", "00000000100"},
     {"00000000001011", "00000000001010", "00000000001101", "0000000001100"},
     {"000000000001111", "000000000001110", "00000000001001", "00000000001100"},
     {"000000000001011", "000000000001010", "000000000001101", "00000000001000"},
     {"0000000000001111", "000000000000001", "000000000001001", "000000000001100"},
     {"0000000000001011", "0000000000001110", "0000000000001101", "000000000001000"},
     {"0000000000000111", "0000000000001010", "0000000000001001", "0000000000001100"},
     {"0000000000000100", "0000000000000110", "0000000000000101", "0000000000001000"}},
    {{"11", "", "", ""},
     {"001011", "10", "", ""},
     {"000111", "00111", "011", ""},
     {"0000111", "001010", "001001", "0101"},
     {"00000111", "000110", "000101", "0100"},
     {"00000100", "0000110", "0000101", "00110"},
     {"000000111", "00000110", "00000101", "001000"},
     {"00000001111", "000000110", "000000101", "000100"},
     {"00000001011", "00000001110", "00000001101", "0000100"},
     {"000000001111", "00000001010", "00000001001", "000000100"},
     {"000000001011", "000000001110", "000000001101", "00000001100"},
     {"000000001000", "000000001010", "000000001001", "00000001000"},
     {"0000000001111", "0000000001110", "0000000001101", "000000001100"},
     {"0000000001011", "0000000001010", "0000000001001", "0000000001100"},
     {"0000000000111", "00000000001011", "0000000000110", "0000000001000"},
     {"00000000001001", "00000000001000", "00000000001010", "0000000000001"},
     {"00000000000111", "00000000000110", "00000000000101", "00000000000100"}},
    {{"1111", "", "", ""},
     {"001111", "1110", "", ""},
     {"001011", "01111", "1101", ""},
     {"001000", "01100", "01110", "1100"},
     {"0001111", "01010", "01011", "1011"},
     {"0001011", "01000", "01001", "1010"},
     {"0001001", "001110", "001101", "1001"},
     {"0001000", "001010", "001001", "1000"},
     {"00001111", "0001110", "0001101", "01101"},
     {"00001011", "00001110", "0001010", "001100"},
     {"000001111", "00001010", "00001101", "0001100"},
     {"000001011", "000001110", "00001001", "00001100"},
     {"000001000", "000001010", "000001101", "00001000"},
     {"0000001101", "000000111", "000001001", "000001100"},
     {"0000001001", "0000001100", "0000001011", "0000001010"},
     {"0000000101", "0000001000", "0000000111", "0000000110"},
     {"0000000001", "0000000100", "0000000011", "0000000010"}}};

// total_zeros for TotalCoeff 1..15 (index tc-1), value = position in the list
const char *kTotalZeros[15][16] = {
    {"1", "011", "010", "0011", "0010", "00011", "00010", "000011", "000010", "0000011", "0000010", "00000011",
     "00000010", "000000011", "000000010", "000000001"},
    {"111", "110", "101", "100", "011", "0101", "0100", "0011", "0010", "00011", "00010", "000011", "000010", "000001",
     "000000"},
    {"0101", "111", "110", "101", "0100", "0011", "100", "011", "0010", "00011", "00010", "000001", "00001", "000000"},
    {"00011", "111", "0101", "0100", "110", "101", "100", "0011", "011", "0010", "00010", "00001", "00000"},
    {"0101", "0100", "0011", "111", "110", "101", "100", "011", "0010", "00001", "0001", "00000"},
    {"000001", "00001", "111", "110", "101", "100", "011", "010", "0001", "001", "000000"},
    {"000001", "00001", "101", "100", "011", "11", "010", "0001", "001", "000000"},
    {"000001", "0001", "00001", "011", "11", "10", "010", "001", "000000"},
    {"000001", "000000", "0001", "11", "10", "001", "01", "00001"},
    {"00001", "00000", "001", "11", "10", "01", "0001"},
    {"0000", "0001", "001", "010", "1", "011"},
    {"0000", "0001", "01", "1", "001"},
    {"000", "001", "1", "01"},
    {"00", "01", "1"},
    {"0", "1"}};

// run_before for zerosLeft 1..6 and > 6 (index min(zerosLeft, 7) - 1)
const char *kRunBefore[7][15] = {{"1", "0"},
                                 {"1", "01", "00"},
                                 {"11", "10", "01", "00"},
                                 {"11", "10", "01", "001", "000"},
                                 {"11", "10", "011", "010", "001", "000"},
                                 {"11", "000", "001", "011", "010", "101", "100"},
                                 {"111", "110", "101", "100", "011", "010", "001", "0001", "00001", "000001",
                                  "0000001", "00000001", "000000001", "0000000001", "00000000001"}};

// zig-zag scan (DvcDec/src/global.cpp:36-41)
const int kZigzag[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};

struct Code {
  int len;
  uint32_t bits;
  int sym;
};
using Table = std::vector<Code>;

// a prefix code of length len covers the 16-bit values [lo, hi) whose top
// len bits are the code: a symbol is found by one binary search on the next 16
// bits of the stream
struct Interval {
  uint32_t lo, hi;
  int len, sym;
};
using Intervals = std::vector<Interval>;

// direct lookup on the next `bits` bits of the stream: entry = sym << 8 | len
// for every value whose top bits are a code of at most `bits` bits, 0 for the
// rest (a longer code, found by the binary search, or no code at all)
struct Lut {
  int bits = 0;
  std::vector<uint32_t> e;
};

constexpr int kLutMaxBits = 10;

struct Tables {
  Table coeff[3], total_zeros[15], run_before[7];
  Intervals coeff_iv[3], total_zeros_iv[15], run_before_iv[7];
  Lut coeff_lut[3], total_zeros_lut[15], run_before_lut[7];
  bool ok = true;
};

Lut lut(const Table &t) {
  Lut L;
  for (const Code &c : t) L.bits = std::max(L.bits, c.len);
  L.bits = std::min(L.bits, kLutMaxBits);
  L.e.assign((size_t)1 << L.bits, 0u);
  for (const Code &c : t) {
    if (c.len > L.bits) continue;
    const uint32_t lo = c.bits << (L.bits - c.len), hi = (c.bits + 1) << (L.bits - c.len);
    for (uint32_t v = lo; v < hi; v++) L.e[v] = ((uint32_t)c.sym << 8) | (uint32_t)c.len;
  }
  return L;
}

Intervals intervals(const Table &t) {
  Intervals v;
  for (const Code &c : t)
    v.push_back(Interval{c.bits << (16 - c.len), (c.bits + 1) << (16 - c.len), c.len, c.sym});
  std::sort(v.begin(), v.end(), [](const Interval &a, const Interval &b) { return a.lo < b.lo; });
  return v;
}

void add(Table &t, const char *s, int sym) {
  if (!s || !*s) return;
  Code c{(int)strlen(s), 0u, sym};
  for (const char *p = s; *p; p++) c.bits = (c.bits << 1) | (uint32_t)(*p == '1');
  t.push_back(c);
}

bool prefix_free(const Table &t) {
  for (size_t i = 0; i < t.size(); i++)
    for (size_t j = 0; j < t.size(); j++) {
      if (i == j || t[i].len > t[j].len) continue;
      if ((t[j].bits >> (t[j].len - t[i].len)) == t[i].bits) return false;
    }
  return true;
}

const Tables &tables() {
  static Tables T;
  static std::once_flag once;
  std::call_once(once, [] {
    for (int v = 0; v < 3; v++) {
      for (int c = 0; c <= 16; c++)
        for (int t = 0; t < 4; t++) add(T.coeff[v], kCoeffToken[v][c][t], c * 4 + t);
      T.ok = T.ok && prefix_free(T.coeff[v]);
      T.coeff_iv[v] = intervals(T.coeff[v]);
      T.coeff_lut[v] = lut(T.coeff[v]);
    }
    for (int i = 0; i < 15; i++) {
      for (int z = 0; z < 16; z++) add(T.total_zeros[i], kTotalZeros[i][z], z);
      T.ok = T.ok && prefix_free(T.total_zeros[i]);
      T.total_zeros_iv[i] = intervals(T.total_zeros[i]);
      T.total_zeros_lut[i] = lut(T.total_zeros[i]);
    }
    for (int i = 0; i < 7; i++) {
      for (int r = 0; r < 15; r++) add(T.run_before[i], kRunBefore[i][r], r);
      T.ok = T.ok && prefix_free(T.run_before[i]);
      T.run_before_iv[i] = intervals(T.run_before[i]);
      T.run_before_lut[i] = lut(T.run_before[i]);
    }
  });
  return T;
}

// MSB-first reader over a 64-bit window: window() holds the stream's bits from
// pos on (at least 57 of them), zeros past the end; consuming bits past the
// end marks the read bad
struct Bits {
  const uint8_t *d;
  size_t nbits, pos;
  bool bad = false;
  uint64_t window() const {
    const size_t byte = pos >> 3, nbytes = nbits >> 3;
    uint64_t w = 0;
    if (byte + 8 <= nbytes) {
      memcpy(&w, d + byte, 8);
      w = __builtin_bswap64(w);
    } else {
      for (size_t i = 0; i < 8 && byte + i < nbytes; i++) w |= (uint64_t)d[byte + i] << (56 - 8 * i);
    }
    return w << (pos & 7);
  }
  void skip(int n) {
    pos += (size_t)n;
    if (pos > nbits) bad = true;
  }
  // the next n bits (1 <= n <= 32)
  uint32_t read(int n) {
    const uint32_t v = (uint32_t)(window() >> (64 - n));
    skip(n);
    return v;
  }
  int bit() { return (int)read(1); }
  // one symbol of a prefix code: the lookup table, else the binary search
  // over the next 16 bits
  int vlc(const Lut &L, const Intervals &t) {
    const uint64_t w = window();
    const uint32_t e = L.e[(size_t)(w >> (64 - L.bits))];
    if (e) {
      skip((int)(e & 0xFF));
      return bad ? -1 : (int)(e >> 8);
    }
    const uint32_t v = (uint32_t)(w >> 48);
    size_t a = 0, b = t.size();
    while (a < b) {  // the last interval starting at or below v
      const size_t m = (a + b) / 2;
      if (t[m].lo <= v) a = m + 1;
      else b = m;
    }
    if (a == 0 || v >= t[a - 1].hi) {
      bad = true;
      return -1;
    }
    skip(t[a - 1].len);
    return bad ? -1 : t[a - 1].sym;
  }
};

struct Frame {
  int w, h, b4w, b4h, b8w;
  const uint8_t *mode;  // 8x8 block modes
  bool intra(int bx, int by) const { return mode[(by >> 1) * b8w + (bx >> 1)] == 1; }
};

// the coefficients of one block: level lev[k] at block position at[k] (the
// zig-zag scan mapped to raster order), k < the returned total coefficient
// count; -1 on a bitstream error
int read_coeffs(Bits &bs, const Tables &T, const Frame &F, int bx, int by, int *nnz, int at[16], int lev[16]) {
  int nc = 0, cnt = 0;
  if (bx > 0 && F.intra(bx - 1, by)) {
    nc += nnz[by * F.b4w + bx - 1];
    cnt++;
  }
  if (by > 0 && F.intra(bx, by - 1)) {
    nc += nnz[(by - 1) * F.b4w + bx];
    cnt++;
  }
  if (cnt == 2) nc = (nc + 1) >> 1;
  int total, t1;
  if (nc >= 8) {  // 6-bit fixed-length coeff_token
    const uint32_t v = bs.read(6);
    if (v == 3) {
      total = 0;
      t1 = 0;
    } else {
      total = (int)(v >> 2) + 1;
      t1 = (int)(v & 3);
      if (t1 > total) return -1;
    }
  } else {
    const int cls = nc < 2 ? 0 : nc < 4 ? 1 : 2;
    const int sym = bs.vlc(T.coeff_lut[cls], T.coeff_iv[cls]);
    if (sym < 0) return -1;
    total = sym >> 2;
    t1 = sym & 3;
  }
  nnz[by * F.b4w + bx] = total;
  if (total == 0) return 0;
  int level[16], run[16] = {0};
  // trailing ones, highest frequency first
  for (int k = total - 1; k >= total - t1; k--) level[k] = bs.bit() ? -1 : 1;
  int suffix_len = (total > 10 && t1 < 3) ? 1 : 0;
  for (int k = total - 1 - t1; k >= 0; k--) {
    // level_prefix: the zeros before the next 1 (at most 25 here, which keeps
    // the prefix, its 1 and a suffix of prefix - 3 bits inside the window)
    const uint64_t w = bs.window();
    const int prefix = w ? __builtin_clzll(w) : 64;
    if (prefix > 25) return -1;
    bs.skip(prefix + 1);
    int code = (std::min(15, prefix) << suffix_len);
    const int ssize = (prefix == 14 && suffix_len == 0) ? 4 : (prefix >= 15 ? prefix - 3 : suffix_len);
    if (ssize > 0) code += (int)bs.read(ssize);
    if (prefix >= 15 && suffix_len == 0) code += 15;
    if (prefix >= 16) code += (1 << (prefix - 3)) - 4096;  // escapes beyond 15 (Level_VLC0/VLCN vlc.cpp:231-364)
    if (k == total - 1 - t1 && t1 < 3) code += 2;
    const int v = (code % 2 == 0) ? (code + 2) >> 1 : (-code - 1) >> 1;
    level[k] = v;
    if (suffix_len == 0) suffix_len = 1;
    const int a = v < 0 ? -v : v;
    if (a > (3 << (suffix_len - 1)) && suffix_len < 6) suffix_len++;
    if (k == total - 1 - t1 && a > 3) suffix_len = 2;
  }
  int zeros = 0;
  if (total < 16) {
    zeros = bs.vlc(T.total_zeros_lut[total - 1], T.total_zeros_iv[total - 1]);
    if (zeros < 0) return -1;
  }
  int left = zeros, i = total - 1;
  while (left > 0 && i > 0) {
    const int rb = std::min(left, 7) - 1;
    const int r = bs.vlc(T.run_before_lut[rb], T.run_before_iv[rb]);
    if (r < 0 || r > left) return -1;
    run[i] = r;
    left -= r;
    i--;
  }
  run[i] = left;
  int pos = 0;
  for (int k = 0; k < total; k++) {
    pos += run[k];
    if (pos > 15) return -1;
    at[k] = kZigzag[pos];
    lev[k] = level[k];
    pos++;
  }
  return bs.bad ? -1 : total;
}

// H.264 4x4 inverse transform with the final division by 64 (intra.cpp:35-77)
void inverse44(int *b) {
  int t[16];
  for (int c = 0; c < 4; c++) {
    const int x0 = b[c], x1 = b[4 + c], x2 = b[8 + c], x3 = b[12 + c];
    t[c] = x0 + x1 + x2 + (x3 >> 1);
    t[4 + c] = x0 + (x1 >> 1) - x2 - x3;
    t[8 + c] = x0 - (x1 >> 1) - x2 + x3;
    t[12 + c] = x0 - x1 + x2 - (x3 >> 1);
  }
  for (int r = 0; r < 4; r++) {
    const int y0 = t[4 * r], y1 = t[4 * r + 1], y2 = t[4 * r + 2], y3 = t[4 * r + 3];
    b[4 * r] = y0 + y1 + y2 + (y3 >> 1);
    b[4 * r + 1] = y0 + (y1 >> 1) - y2 - y3;
    b[4 * r + 2] = y0 - (y1 >> 1) - y2 + y3;
    b[4 * r + 3] = y0 - y1 + y2 - (y3 >> 1);
  }
  for (int i = 0; i < 16; i++) b[i] >>= 6;
}

int round_half_away(double x) { return x >= 0.0 ? (int)(x + 0.5) : -(int)(-x + 0.5); }  // defines.h:23

// ---- encoder side: the exact inverse of read_coeffs

struct BitWriter {
  uint8_t *d;
  size_t nbits, pos;
  bool over = false;
  void bit(int b) {
    if (pos >= nbits) {
      over = true;
      return;
    }
    const uint8_t m = (uint8_t)(0x80u >> (pos & 7));
    if (b) d[pos >> 3] |= m;
    else d[pos >> 3] &= (uint8_t)~m;
    pos++;
  }
  void put(uint32_t v, int n) {
    for (int i = n - 1; i >= 0; i--) bit((int)((v >> i) & 1u));
  }
  bool vlc(const Table &t, int sym) {
    for (const Code &c : t)
      if (c.sym == sym) {
        put(c.bits, c.len);
        return true;
      }
    return false;
  }
};

// coefficients coeff[16] (raster positions of the 4x4 block) as CAVLC; false
// when a value is outside what the syntax can carry
bool write_coeffs(BitWriter &bw, const Frame &F, int bx, int by, std::vector<int> &nnz, const int coeff[16]) {
  const Tables &T = tables();
  int nc = 0, cnt = 0;
  if (bx > 0 && F.intra(bx - 1, by)) {
    nc += nnz[by * F.b4w + bx - 1];
    cnt++;
  }
  if (by > 0 && F.intra(bx, by - 1)) {
    nc += nnz[(by - 1) * F.b4w + bx];
    cnt++;
  }
  if (cnt == 2) nc = (nc + 1) >> 1;
  int level[16], pos[16], total = 0;
  for (int p = 0; p < 16; p++) {
    const int v = coeff[kZigzag[p]];
    if (v) {
      level[total] = v;
      pos[total] = p;
      total++;
    }
  }
  int t1 = 0;
  for (int k = total - 1; k >= 0 && t1 < 3 && (level[k] == 1 || level[k] == -1); k--) t1++;
  nnz[by * F.b4w + bx] = total;
  if (nc >= 8) {
    bw.put(total == 0 ? 3u : (uint32_t)(((total - 1) << 2) | t1), 6);
  } else if (!bw.vlc(T.coeff[nc < 2 ? 0 : nc < 4 ? 1 : 2], total * 4 + t1)) {
    return false;
  }
  if (total == 0) return true;
  for (int k = total - 1; k >= total - t1; k--) bw.bit(level[k] < 0 ? 1 : 0);
  int suffix_len = (total > 10 && t1 < 3) ? 1 : 0;
  for (int k = total - 1 - t1; k >= 0; k--) {
    const int v = level[k];
    int code = v > 0 ? 2 * v - 2 : -2 * v - 1;
    if (k == total - 1 - t1 && t1 < 3) code -= 2;
    if (suffix_len == 0) {
      if (code < 14) {
        bw.put(1u, code + 1);
      } else if (code < 30) {
        bw.put(1u, 15);
        bw.put((uint32_t)(code - 14), 4);
      } else {
        if (code - 30 >= 4096) return false;
        bw.put(1u, 16);
        bw.put((uint32_t)(code - 30), 12);
      }
    } else if (code < (15 << suffix_len)) {
      bw.put(1u, (code >> suffix_len) + 1);
      bw.put((uint32_t)(code & ((1 << suffix_len) - 1)), suffix_len);
    } else {
      if (code - (15 << suffix_len) >= 4096) return false;
      bw.put(1u, 16);
      bw.put((uint32_t)(code - (15 << suffix_len)), 12);
    }
    int sl = suffix_len == 0 ? 1 : suffix_len;
    const int a = v < 0 ? -v : v;
    if (a > (3 << (sl - 1)) && sl < 6) sl++;
    if (k == total - 1 - t1 && a > 3) sl = 2;
    suffix_len = sl;
  }
  if (total < 16) {
    const int zeros = pos[total - 1] + 1 - total;
    if (!bw.vlc(T.total_zeros[total - 1], zeros)) return false;
    int left = zeros;
    for (int i = total - 1; i > 0 && left > 0; i--) {
      const int run = pos[i] - pos[i - 1] - 1;
      if (!bw.vlc(T.run_before[std::min(left, 7) - 1], run)) return false;
      left -= run;
    }
  }
  return true;
}

}  // namespace

namespace {

// DC prediction from the reconstructed intra neighbours of block (bx, by)
int dc_pred(const Frame &F, const uint8_t *recon, int bx, int by) {
  const int top = by * 4, left = bx * 4, width = F.w;
  const bool up = by > 0 && F.intra(bx, by - 1), lf = bx > 0 && F.intra(bx - 1, by);
  int s = 0;
  if (up)
    for (int j = 0; j < 4; j++) s += recon[(top - 1) * width + left + j];
  if (lf)
    for (int i = 0; i < 4; i++) s += recon[(top + i) * width + left - 1];
  return (up && lf) ? (s + 4) >> 3 : (up || lf) ? (s + 2) >> 2 : 128;
}

}  // namespace

extern "C" int dvc_intra_encode_frame(const uint8_t *ori, int width, int height, int intra_qp, const uint8_t *mode,
                                      uint8_t *stream, size_t stream_bytes, size_t *bit_offset, uint8_t *recon,
                                      int *block_bits) {
  if (!ori || !stream || !bit_offset || !mode || !recon ||
      !((width == 176 && height == 144) || (width == 352 && height == 288)) || intra_qp < 0 || intra_qp > 51)
    return DVC_E_ARG;
  if (!tables().ok) return DVC_E_DATA;
  Frame F{width, height, width / 4, height / 4, width / 8, mode};
  BitWriter bw{stream, stream_bytes * 8, *bit_offset};
  // the decoder's de-quantisation scale, computed the same way
  const double qstep = pow(2.0, ((double)intra_qp - 4.0) / 6.0);
  const double a2 = 0.25, b2 = 0.4, ab = 0.5 * sqrt(0.4);
  const double pre[16] = {a2, ab, a2, ab, ab, b2, ab, b2, a2, ab, a2, ab, ab, b2, ab, b2};
  // forward normalisation of the core transform: a^2, ab/2, b^2/4 (a = 1/2, b = sqrt(2/5))
  const double ea = 0.25, eb = 0.1, eab = 0.25 * sqrt(0.4);
  const double ef[16] = {ea, eab, ea, eab, eab, eb, eab, eb, ea, eab, ea, eab, eab, eb, eab, eb};
  std::vector<int> nnz((size_t)F.b4w * F.b4h, 0);
  for (int by = 0; by < F.b4h; by++)
    for (int bx = 0; bx < F.b4w; bx++) {
      if (!F.intra(bx, by)) continue;
      const int top = by * 4, left = bx * 4;
      const int pred = dc_pred(F, recon, bx, by);
      int x[16], t[16], coeff[16], blk[16];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) x[4 * i + j] = (int)ori[(top + i) * width + left + j] - pred;
      // core transform rows then columns: Cf X Cf^T
      for (int i = 0; i < 4; i++) {
        const int *r = x + 4 * i;
        t[4 * i] = r[0] + r[1] + r[2] + r[3];
        t[4 * i + 1] = 2 * r[0] + r[1] - r[2] - 2 * r[3];
        t[4 * i + 2] = r[0] - r[1] - r[2] + r[3];
        t[4 * i + 3] = r[0] - 2 * r[1] + 2 * r[2] - r[3];
      }
      for (int j = 0; j < 4; j++) {
        const int c0 = t[j], c1 = t[4 + j], c2 = t[8 + j], c3 = t[12 + j];
        x[j] = c0 + c1 + c2 + c3;
        x[4 + j] = 2 * c0 + c1 - c2 - 2 * c3;
        x[8 + j] = c0 - c1 - c2 + c3;
        x[12 + j] = c0 - 2 * c1 + 2 * c2 - c3;
      }
      // quantisation with a one-third rounding offset, as intra coders use
      for (int i = 0; i < 16; i++) {
        const double y = (double)x[i] * ef[i] / qstep;
        const int q = (int)(fabs(y) + 1.0 / 3.0);
        coeff[i] = y < 0 ? -q : q;
      }
      const size_t before = bw.pos;
      if (!write_coeffs(bw, F, bx, by, nnz, coeff)) return DVC_E_ARG;
      if (block_bits) block_bits[by * F.b4w + bx] = (int)(bw.pos - before);
      // the decoder's reconstruction, so that later blocks predict from it
      for (int i = 0; i < 16; i++) blk[i] = round_half_away((double)coeff[i] * qstep * (pre[i] * 64.0));
      inverse44(blk);
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
          const int v = blk[4 * i + j] + pred;
          recon[(top + i) * width + left + j] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
  if (bw.over) return DVC_E_ARG;
  *bit_offset = bw.pos;
  return DVC_OK;
}

extern "C" int dvc_intra_decode_frame(const uint8_t *stream, size_t stream_bytes, size_t *bit_offset, int width,
                                      int height, int intra_qp, const uint8_t *mode, uint8_t *recon) {
  if (!stream || !bit_offset || !mode || !recon || !((width == 176 && height == 144) || (width == 352 && height == 288)) ||
      intra_qp < 0 || intra_qp > 51)
    return DVC_E_ARG;
  const Tables &T = tables();
  if (!T.ok) return DVC_E_DATA;
  Frame F{width, height, width / 4, height / 4, width / 8, mode};
  Bits bs{stream, stream_bytes * 8, *bit_offset};
  // de-quantisation scale: Qstep * 64 * pre-scale (intra.cpp:214, transform.cpp:12-52)
  const double qstep = pow(2.0, ((double)intra_qp - 4.0) / 6.0);
  const double a2 = 0.25, b2 = 0.4, ab = 0.5 * sqrt(0.4);
  const double pre[16] = {a2, ab, a2, ab, ab, b2, ab, b2, a2, ab, a2, ab, ab, b2, ab, b2};
  double pre64[16];
  for (int i = 0; i < 16; i++) pre64[i] = pre[i] * 64.0;
  std::vector<int> nnz((size_t)F.b4w * F.b4h, 0);
  for (int by = 0; by < F.b4h; by++)
    for (int bx = 0; bx < F.b4w; bx++) {
      if (!F.intra(bx, by)) continue;
      int at[16], lev[16];
      const int total = read_coeffs(bs, T, F, bx, by, nnz.data(), at, lev);
      if (total < 0) return DVC_E_DATA;
      // DC prediction from intra neighbours (intra.cpp:120-184)
      const int top = by * 4, left = bx * 4;
      const bool up = by > 0 && F.intra(bx, by - 1), lf = bx > 0 && F.intra(bx - 1, by);
      int s = 0;
      if (up)
        for (int j = 0; j < 4; j++) s += recon[(top - 1) * width + left + j];
      if (lf)
        for (int i = 0; i < 4; i++) s += recon[(top + i) * width + left - 1];
      const int pred = (up && lf) ? (s + 4) >> 3 : (up || lf) ? (s + 2) >> 2 : 128;
      // de-quantisation of the coded coefficients (the others stay 0)
      int blk[16] = {0};
      bool dc_only = true;
      for (int k = 0; k < total; k++) {
        blk[at[k]] = round_half_away((double)lev[k] * qstep * pre64[at[k]]);
        dc_only = dc_only && at[k] == 0;
      }
      if (dc_only) {  // no residual, or a lone DC: all 16 outputs of the transform equal blk[0] >> 6
        const int v = (blk[0] >> 6) + pred;
        const int c = v < 0 ? 0 : v > 255 ? 255 : v;
        for (int i = 0; i < 4; i++) memset(recon + (size_t)(top + i) * width + left, c, 4);
        continue;
      }
      inverse44(blk);
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
          const int v = blk[4 * i + j] + pred;
          recon[(top + i) * width + left + j] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
  *bit_offset = bs.pos;
  return DVC_OK;
}
