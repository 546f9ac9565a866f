// JBIG (ITU-T T.82) decoder for the 8x8 skip / intra mode maps of the WZ
// bitstream.
//
// The reference encoder codes each map with JBIG-KIT (DvcEnc/src/sJBIG.cpp,
// wzbitstream.cpp:28-44): one bit plane, no resolution reduction (D = 0),
// one stripe of the whole map, options TPDON | DPON (which only concern
// resolution-reduced layers, so neither applies), maximum AT offset 8, and it
// writes the coded stripe without the 20-byte header; the decoder rebuilds
// that header (DvcDec/src/wzbitstream.cpp:38-66).  Decoding the lowest
// resolution layer of such a stream needs:
//
//  * the QM arithmetic decoder with the 113-state probability estimation table
//    of the standard (shared by T.82 and T.81), one state and MPS per context;
//  * the three-line template: three pixels of line y-2 (x-1..x+1), five of
//    line y-1 (x-2..x+2) and two of line y (the adaptive pixel at its default
//    place x-2, and x-1); pixels outside the map are 0;
//  * the stripe's protected coded data: 0xFF 0x00 is a 0xFF byte, 0xFF and any
//    other byte is a marker that ends the data, after which the decoder reads
//    zero bytes; SDNORM (0xFF 0x02) or SDRST (0xFF 0x03) closes the stripe.
//
// The encoder (dvc_jbig_encode_mode_map) writes the same form: the coded
// stripe of the map with the same template and options, closed by SDNORM.
//
// An adaptive-template move (ATMOVE marker) is refused: the reference encoder
// does not emit one for maps of these sizes (none in thousands of maps coded
// by it), and a stream that had one would decode wrongly here.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/dvc_b200.h"

namespace {

// T.82 Table 24 / T.81 Table D.3: Qe, next state after LPS and after MPS, MPS switch
const uint16_t kQe[113] = {
    0x5A1D, 0x2586, 0x1114, 0x080B, 0x03D8, 0x01DA, 0x00E5, 0x006F, 0x0036, 0x001A, 0x000D, 0x0006, 0x0003, 0x0001,
    0x5A7F, 0x3F25, 0x2CF2, 0x207C, 0x17B9, 0x1182, 0x0CEF, 0x09A1, 0x072F, 0x055C, 0x0406, 0x0303, 0x0240, 0x01B1,
    0x0144, 0x00F5, 0x00B7, 0x008A, 0x0068, 0x004E, 0x003B, 0x002C, 0x5AE1, 0x484C, 0x3A0D, 0x2EF1, 0x261F, 0x1F33,
    0x19A8, 0x1518, 0x1177, 0x0E74, 0x0BFB, 0x09F8, 0x0861, 0x0706, 0x05CD, 0x04DE, 0x040F, 0x0363, 0x02D4, 0x025C,
    0x01F8, 0x01A4, 0x0160, 0x0125, 0x00F6, 0x00CB, 0x00AB, 0x008F, 0x5B12, 0x4D04, 0x412C, 0x37D8, 0x2FE8, 0x293C,
    0x2379, 0x1EDF, 0x1AA9, 0x174E, 0x1424, 0x119C, 0x0F6B, 0x0D51, 0x0BB6, 0x0A40, 0x5832, 0x4D1C, 0x438E, 0x3BDD,
    0x34EE, 0x2EAE, 0x299A, 0x2516, 0x5570, 0x4CA9, 0x44D9, 0x3E22, 0x3824, 0x32B4, 0x2E17, 0x56A8, 0x4F46, 0x47E5,
    0x41CF, 0x3C3D, 0x375E, 0x5231, 0x4C0F, 0x4639, 0x415E, 0x5627, 0x50E7, 0x4B85, 0x5597, 0x504F, 0x5A10, 0x5522,
    0x59EB};
const uint8_t kNextLps[113] = {
    1,  14, 16, 18, 20, 23, 25, 28, 30, 33, 35, 9,  10, 12, 15, 36, 38, 39, 40, 42, 43, 45, 46,  48,  49,  51,  52,  54,
    56, 57, 59, 60, 62, 63, 32, 33, 37, 64, 65, 67, 68, 69, 70, 72, 73, 74, 75, 77, 78, 79, 48,  50,  50,  51,  52,  53,
    54, 55, 56, 57, 58, 59, 61, 61, 65, 80, 81, 82, 83, 84, 86, 87, 87, 72, 72, 74, 74, 75, 77,  77,  80,  88,  89,  90,
    91, 92, 93, 86, 88, 95, 96, 97, 99, 99, 93, 95, 101, 102, 103, 104, 99, 105, 106, 107, 103, 105, 108, 109, 110, 111,
    110, 112, 112};
const uint8_t kNextMps[113] = {
    1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 13, 15, 16, 17,  18, 19,  20,  21,  22,  23,  24,  25,  26,  27,
    28, 29, 30, 31, 32, 33, 34, 35, 9,  37, 38, 39, 40, 41, 42, 43, 44,  45, 46,  47,  48,  49,  50,  51,  52,  53,  54,
    55, 56, 57, 58, 59, 60, 61, 62, 63, 32, 65, 66, 67, 68, 69, 70, 71,  72, 73,  74,  75,  76,  77,  78,  79,  48,  81,
    82, 83, 84, 85, 86, 87, 71, 89, 90, 91, 92, 93, 94, 86, 96, 97, 98,  99, 100, 93,  102, 103, 104, 99,  106, 107, 103,
    109, 107, 111, 109, 111};
const uint8_t kSwitch[113] = {1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                              0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                              0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0,
                              0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 1};

// QM decoder over the protected coded data of one stripe
struct QmDecoder {
  const uint8_t *d;
  size_t len, pos = 0;
  bool ended = false;  // a marker was reached: zero bytes from here on
  uint32_t c = 0, a = 0x10000;
  int ct = 0;
  uint8_t st[1024] = {0}, mps[1024] = {0};

  void byte_in() {
    uint32_t b = 0;
    if (!ended && pos < len) {
      b = d[pos];
      if (b == 0xFF) {
        if (pos + 1 < len && d[pos + 1] == 0x00) {
          pos += 2;
        } else {
          ended = true;
          b = 0;
        }
      } else {
        pos++;
      }
    }
    c += b << 8;
  }
  void init(const uint8_t *data, size_t n) {
    d = data;
    len = n;
    byte_in();
    c <<= 8;
    byte_in();
    c <<= 8;
    ct = 0;
    a = 0x10000;
  }
  void renorm() {
    do {
      if (ct == 0) {
        byte_in();
        ct = 8;
      }
      a <<= 1;
      c <<= 1;
      ct--;
    } while (a < 0x8000);
  }
  int decode(int cx) {
    const int s = st[cx], m = mps[cx];
    const uint32_t q = kQe[s];
    a -= q;
    int bit;
    if ((c >> 16) < a) {
      if (a >= 0x8000) return m;
      // MPS path below half: conditional exchange
      if (a < q) {
        bit = 1 - m;
        if (kSwitch[s]) mps[cx] = (uint8_t)(1 - m);
        st[cx] = kNextLps[s];
      } else {
        bit = m;
        st[cx] = kNextMps[s];
      }
    } else {
      c -= a << 16;
      if (a < q) {
        bit = m;
        st[cx] = kNextMps[s];
      } else {
        bit = 1 - m;
        if (kSwitch[s]) mps[cx] = (uint8_t)(1 - m);
        st[cx] = kNextLps[s];
      }
      a = q;
    }
    renorm();
    return bit;
  }
};

// QM encoder (T.82 6.8): the interval register C holds, from bit 27 down, a
// carry bit, the 8 bits of the next output byte, 3 spacer bits and the 16
// bits aligned with A.  Output bytes are held back one at a time (`buffer`)
// and runs of 0xFF are only counted (`stacked`), so that a carry out of C can
// still propagate into them; every 0xFF written is followed by a 0x00 stuff
// byte.
struct QmEncoder {
  std::vector<uint8_t> out;
  uint32_t c = 0, a = 0x10000;
  int ct = 11, stacked = 0, buffer = -1;
  uint8_t st[1024] = {0}, mps[1024] = {0};

  void put(int b) {
    out.push_back((uint8_t)b);
    if (b == 0xFF) out.push_back(0x00);
  }
  void byte_out() {
    const uint32_t t = c >> 19;
    if (t > 0xFF) {  // carry: the held byte grows by one, the stacked 0xFF become 0x00
      if (buffer >= 0) put(buffer + 1);
      for (; stacked > 0; stacked--) out.push_back(0x00);
      buffer = (int)(t & 0xFF);
    } else if (t == 0xFF) {
      stacked++;
    } else {
      if (buffer >= 0) put(buffer);
      for (; stacked > 0; stacked--) put(0xFF);
      buffer = (int)t;
    }
    c &= 0x7FFFF;
  }
  void renorm() {
    do {
      a <<= 1;
      c <<= 1;
      if (--ct == 0) {
        byte_out();
        ct = 8;
      }
    } while (a < 0x8000);
  }
  // the upper sub-interval of size Qe belongs to the LPS unless A - Qe < Qe,
  // in which case the two sub-intervals swap (conditional exchange)
  void encode(int cx, int pix) {
    const int s = st[cx];
    const uint32_t q = kQe[s];
    a -= q;
    if (pix == mps[cx]) {
      if (a >= 0x8000) return;
      if (a < q) {
        c += a;
        a = q;
      }
      st[cx] = kNextMps[s];
    } else {
      if (a >= q) {
        c += a;
        a = q;
      }
      if (kSwitch[s]) mps[cx] = (uint8_t)(1 - mps[cx]);
      st[cx] = kNextLps[s];
    }
    renorm();
  }
  // pick the value in [C, C + A) with the most trailing zero bits, write out
  // what is left, and drop final bytes that are 0x00 (a decoder reads zeros
  // past the end of the data)
  void flush() {
    const uint32_t t = (a - 1 + c) & 0xFFFF0000u;
    c = t < c ? t + 0x8000 : t;
    c <<= ct;
    if (c & 0xF8000000u) {
      if (buffer >= 0) put(buffer + 1);
      if (c & 0x7FFF800u)
        for (; stacked > 0; stacked--) out.push_back(0x00);
    } else {
      if (buffer >= 0) put(buffer);
      for (; stacked > 0; stacked--) put(0xFF);
    }
    if (c & 0x7FFF800u) {
      put((int)((c >> 19) & 0xFF));
      if (c & 0x7F800u) put((int)((c >> 11) & 0xFF));
    }
  }
};

}  // namespace

extern "C" int dvc_jbig_encode_mode_map(const uint8_t *map, int w, int h, uint8_t *out, size_t cap, size_t *len) {
  if (!map || !out || !len || w <= 0 || h <= 0 || w > 4096 || h > 4096) return DVC_E_ARG;
  QmEncoder q;
  const int W = w + 4;
  std::vector<uint8_t> r2(W, 0), r1(W, 0), r0(W, 0);
  for (int y = 0; y < h; y++) {
    std::fill(r0.begin(), r0.end(), 0);
    for (int x = 0; x < w; x++) {
      const int X = x + 2;
      const int cx = (r2[X - 1] << 9) | (r2[X] << 8) | (r2[X + 1] << 7) | (r1[X - 2] << 6) | (r1[X - 1] << 5) |
                     (r1[X] << 4) | (r1[X + 1] << 3) | (r1[X + 2] << 2) | (r0[X - 2] << 1) | r0[X - 1];
      const int pix = map[(size_t)y * w + x] ? 1 : 0;
      q.encode(cx, pix);
      r0[X] = (uint8_t)pix;
    }
    r2.swap(r1);
    r1.swap(r0);
  }
  q.flush();
  q.out.push_back(0xFF);  // SDNORM closes the stripe
  q.out.push_back(0x02);
  *len = q.out.size();
  if (q.out.size() > cap) return DVC_E_ARG;
  memcpy(out, q.out.data(), q.out.size());
  return DVC_OK;
}

extern "C" int dvc_jbig_decode_mode_map(const uint8_t *data, size_t len, int w, int h, uint8_t *map, size_t *used) {
  if (!data || !map || w <= 0 || h <= 0 || w > 4096 || h > 4096) return DVC_E_ARG;
  // end of the protected data: the first 0xFF not followed by 0x00
  size_t end = 0;
  while (end < len && !(data[end] == 0xFF && end + 1 < len && data[end + 1] != 0x00)) end += data[end] == 0xFF ? 2 : 1;
  if (end + 1 >= len) return DVC_E_DATA;  // no closing marker: truncated
  const uint8_t marker = data[end + 1];
  if (marker != 0x02 && marker != 0x03) return DVC_E_DATA;  // ATMOVE, COMMENT, NEWLEN or ABORT
  QmDecoder q;
  q.init(data, end);
  // rows y-2, y-1, y with two zero columns on either side
  const int W = w + 4;
  std::vector<uint8_t> r2(W, 0), r1(W, 0), r0(W, 0);
  for (int y = 0; y < h; y++) {
    std::fill(r0.begin(), r0.end(), 0);
    for (int x = 0; x < w; x++) {
      const int X = x + 2;
      const int cx = (r2[X - 1] << 9) | (r2[X] << 8) | (r2[X + 1] << 7) | (r1[X - 2] << 6) | (r1[X - 1] << 5) |
                     (r1[X] << 4) | (r1[X + 1] << 3) | (r1[X + 2] << 2) | (r0[X - 2] << 1) | r0[X - 1];
      r0[X] = (uint8_t)q.decode(cx);
      map[(size_t)y * w + x] = r0[X];
    }
    r2.swap(r1);
    r1.swap(r0);
  }
  if (used) *used = end + 2;
  return DVC_OK;
}
