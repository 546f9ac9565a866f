// Test driver: random and damaged inputs for the library's host-side coders,
// built with AddressSanitizer / UndefinedBehaviorSanitizer by
// tests/test_host_fuzz.py.  Every input sits in a heap block of exactly its
// size, so a read past its end is reported.  Modes:
//   intra_dec  random bit strings under random intra maps -> decoded or refused
//   intra_enc  random frames, maps and IntraQP -> encoded (or, in the small
//              buffers some cases get, refused with DVC_E_ARG) and decoded back
//              to the encoder's reconstruction
//   jbig_dec   encoded mode maps, cut or with a flipped bit, and random bytes
// Exit status 0 when every call behaves; a sanitizer report aborts the run.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <random>
#include <string>
#include <vector>

#include "../include/dvc_b200.h"

static int intra_dec(int n_iter) {
  std::mt19937_64 rng(1);
  for (int t = 0; t < n_iter; t++) {
    const int w = (t & 1) ? 176 : 352, h = (t & 1) ? 144 : 288;
    const size_t n = 1 + rng() % 600;
    uint8_t *d = (uint8_t *)malloc(n);
    for (size_t i = 0; i < n; i++) d[i] = (t % 3) ? (uint8_t)rng() : (uint8_t)((t % 7) ? 0 : 0xFF);
    std::vector<uint8_t> mode((w / 8) * (h / 8)), rec(w * h);
    const double p = (rng() % 1000) / 1000.0;
    for (auto &m : mode) m = ((rng() % 1000) / 1000.0 < p) ? 1 : 0;
    size_t off = rng() % 8;
    const int rc = dvc_intra_decode_frame(d, n, &off, w, h, (int)(rng() % 52), mode.data(), rec.data());
    free(d);
    if (rc == DVC_OK && off > 8 * n) return fprintf(stderr, "offset past the end\n"), 1;
    if (rc != DVC_OK && rc != DVC_E_DATA) return fprintf(stderr, "status %d\n", rc), 1;
  }
  return 0;
}

static int intra_enc(int n_iter) {
  std::mt19937_64 rng(3);
  for (int t = 0; t < n_iter; t++) {
    const int w = (t & 1) ? 176 : 352, h = (t & 1) ? 144 : 288;
    std::vector<uint8_t> ori(w * h), mode((w / 8) * (h / 8)), rec(w * h), dec(w * h);
    for (int i = 0; i < w * h; i++)
      ori[i] = t % 3 == 0 ? (uint8_t)rng() : t % 3 == 1 ? (uint8_t)((i % w) * 255 / w) : (uint8_t)((rng() % 8) ? 0 : 255);
    const double p = (rng() % 1000) / 1000.0;
    for (auto &m : mode) m = ((rng() % 1000) / 1000.0 < p) ? 1 : 0;
    const size_t cap = (t % 5 == 0) ? 1 + rng() % 2000 : (size_t)1 << 20;
    uint8_t *buf = (uint8_t *)calloc(cap, 1);
    std::vector<int> bits((w / 4) * (h / 4));
    const size_t off0 = rng() % 8;
    size_t off = off0;
    const int qp = (int)(rng() % 52);
    const int rc = dvc_intra_encode_frame(ori.data(), w, h, qp, mode.data(), buf, cap, &off, rec.data(), bits.data());
    int bad = 0;
    if (rc == DVC_OK) {
      size_t o2 = off0;
      if (dvc_intra_decode_frame(buf, cap, &o2, w, h, qp, mode.data(), dec.data()) != DVC_OK || o2 != off) bad = 1;
      for (int i = 0; i < w * h && !bad; i++)
        if (mode[(i / w / 8) * (w / 8) + (i % w) / 8] && dec[i] != rec[i]) bad = 2;
    } else if (rc != DVC_E_ARG || cap >= ((size_t)1 << 20)) {  // refused only for lack of room
      bad = 3;
    }
    free(buf);
    if (bad) return fprintf(stderr, "case %d: %s\n", t, bad == 3 ? "unexpected status" : "round trip differs"), 1;
  }
  return 0;
}

static int jbig_dec(int n_iter) {
  std::mt19937_64 rng(2);
  for (int t = 0; t < n_iter; t++) {
    const int w = (t & 1) ? 22 : 44, h = (t & 1) ? 18 : 36;
    std::vector<uint8_t> mp(w * h), out(w * h);
    size_t n;
    uint8_t *d;
    if (t % 2 == 0) {  // a real stream of a random map, then cut or with a bit flipped
      const double p = (rng() % 1000) / 1000.0;
      for (auto &m : mp) m = ((rng() % 1000) / 1000.0 < p) ? 1 : 0;
      std::vector<uint8_t> buf(4096);
      size_t len = 0;
      if (dvc_jbig_encode_mode_map(mp.data(), w, h, buf.data(), buf.size(), &len) != DVC_OK)
        return fprintf(stderr, "encoder refused a map\n"), 1;
      n = (rng() % 4 == 0) ? rng() % (len + 1) : len;
      if (n == 0) n = 1;
      d = (uint8_t *)malloc(n);
      memcpy(d, buf.data(), n);
      if (rng() % 3 == 0) d[rng() % n] ^= (uint8_t)(1u << (rng() % 8));
    } else {
      n = 1 + rng() % 300;
      d = (uint8_t *)malloc(n);
      for (size_t i = 0; i < n; i++) d[i] = (uint8_t)rng();
    }
    size_t used = 0;
    const int rc = dvc_jbig_decode_mode_map(d, n, w, h, out.data(), &used);
    free(d);
    if (rc == DVC_OK && used > n) return fprintf(stderr, "used past the end\n"), 1;
    if (rc != DVC_OK && rc != DVC_E_DATA) return fprintf(stderr, "status %d\n", rc), 1;
  }
  return 0;
}

int main(int argc, char **argv) {
  const std::string mode = argc > 1 ? argv[1] : "";
  const int n = argc > 2 ? atoi(argv[2]) : 1000;
  if (mode == "intra_dec") return intra_dec(n);
  if (mode == "intra_enc") return intra_enc(n);
  if (mode == "jbig_dec") return jbig_dec(n);
  fprintf(stderr, "usage: fuzz_host intra_dec|intra_enc|jbig_dec [iterations]\n");
  return 2;
}
