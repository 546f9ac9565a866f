// Host-side builder and loader of the tables that make the device float
// functions in exact_libm.h return the C library's bits (see that header for
// the method).  The tables are derived from the C library that the reference
// decoder links on this host, by calling it over each input domain:
//
//   logf   every positive float up to 10001: hash of (input, result) pairs
//          where the library differs from xl_logf_base;
//   expf   every float in [-104, -0]: hash of the differing pairs;
//   tanhf  y1 = first float with tanhf(y) == 1 (checked to stay 1 above it);
//   phi    -logf(tanhf(y)) for every y in [2^-31, y1), the belief-propagation
//          magnitude, as one direct table (dvc_phi_build; not stored in the
//          file, rebuilt in about a second when a context starts).
//
// The file starts with the C library's version string; a loader that finds a
// different version (or no file) rebuilds the tables.
#include "libm_tables.h"

#include <gnu/libc-version.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
#include <vector>

#include "exact_libm.h"

namespace {

struct Pair { uint32_t key, val; };

// Small tables of the table-driven base functions (exact_libm.h), computed in
// extended precision: 2^(j/32); per mantissa bin of [1, 2) (128 bins) the
// reciprocal of the bin centre and the log of the centre.  The bins touching 1
// (the first) and 2 (the last, folded) use the exact centres 1 and 2.
void make_small(XlmSmallTables &t) {
  for (int j = 0; j < 32; j++) t.exp2j[j] = (double)exp2l((long double)j / 32.0L);
  const long double sqrt2 = sqrtl(2.0L), ln2 = logl(2.0L);
  for (int i = 0; i < 128; i++) {
    long double c = 1.0L + ((long double)i + 0.5L) / 128.0L;
    if (i == 0) c = 1.0L;
    if (i == 127) c = 2.0L;
    const double invc = (double)(1.0L / c);
    const int fold = c >= sqrt2 ? 1 : 0;
    t.invc[i] = invc;
    t.efold[i] = fold;
    // log of the exact reciprocal actually used, so log m = -log(invc) + log1p(m*invc - 1)
    long double lc = -logl((long double)invc);
    if (fold) lc -= ln2;
    t.logc[i] = (double)lc;
  }
}

XlSmall view(const XlmSmallTables &t) { return XlSmall{t.exp2j, t.invc, t.logc, t.efold}; }

int hw_threads() {
  unsigned n = std::thread::hardware_concurrency();
  return n ? (int)n : 4;
}

template <class F>
void parallel_ranges(uint64_t lo, uint64_t hi_incl, int threads, F fn) {
  const uint64_t n = hi_incl - lo + 1;
  const uint64_t chunk = (n + threads - 1) / threads;
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; t++) {
    uint64_t a = lo + chunk * t;
    if (a > hi_incl) break;
    uint64_t b = std::min(hi_incl, a + chunk - 1);
    ts.emplace_back([=]() { fn(t, a, b); });
  }
  for (auto &th : ts) th.join();
}

uint32_t hash_slot(uint32_t key, int log2cap) { return (key * 0x9E3779B1u) >> (32 - log2cap); }

void build_hash(const std::vector<Pair> &pairs, std::vector<uint32_t> &table, uint32_t &cap) {
  int lg = 4;
  while ((1ull << lg) < pairs.size() * 2 + 16) lg++;
  cap = 1u << lg;
  table.assign((size_t)cap * 2, 0xFFFFFFFFu);
  for (const Pair &p : pairs) {
    uint32_t s = hash_slot(p.key, lg);
    while (table[2 * s] != 0xFFFFFFFFu) s = (s + 1) & (cap - 1);
    table[2 * s] = p.key;
    table[2 * s + 1] = p.val;
  }
}


}  // namespace

extern "C" int dvc_libm_build(const char *path, int threads, char *err, int errlen) {
  if (threads <= 0) threads = hw_threads();
  std::vector<std::vector<Pair>> parts(threads);
  XlmSmallTables small;
  make_small(small);
  const XlSmall sv = view(small);

  // ---- logf over (0, 10001]
  parallel_ranges(XL_LOG_LO, XL_LOG_HI, threads, [&](int t, uint64_t a, uint64_t b) {
    auto &v = parts[t];
    for (uint64_t u = a; u <= b; u++) {
      const float x = xl_bitsf((uint32_t)u);
      const float g = logf(x), m = xl_logf_base(x, sv);
      if (xl_fbits(g) != xl_fbits(m)) v.push_back({(uint32_t)u, xl_fbits(g)});
    }
  });
  std::vector<Pair> logp;
  for (auto &v : parts) { logp.insert(logp.end(), v.begin(), v.end()); v.clear(); }

  // ---- expf over [-104, -0], and the largest midpoint distance of an
  //      exception whose result is a normal float
  std::vector<uint32_t> tie(threads, 0);
  parallel_ranges(XL_EXP_LO, XL_EXP_HI, threads, [&](int t, uint64_t a, uint64_t b) {
    auto &v = parts[t];
    for (uint64_t u = a; u <= b; u++) {
      const float x = xl_bitsf((uint32_t)u);
      const double d = xl_exp_d((double)x, sv);
      const float g = expf(x), m = xl_expf_base(x, sv);
      if (xl_fbits(g) != xl_fbits(m)) {
        v.push_back({(uint32_t)u, xl_fbits(g)});
        if (d >= 0x1p-126) tie[t] = std::max(tie[t], xl_tie_dist(d));
      }
    }
  });
  const uint32_t exp_tie = *std::max_element(tie.begin(), tie.end());
  std::vector<Pair> expp;
  for (auto &v : parts) { expp.insert(expp.end(), v.begin(), v.end()); v.clear(); }

  // ---- tanh threshold y1: smallest float y with tanhf(y) == 1
  uint32_t y1 = xl_fbits(8.0f);
  while (tanhf(xl_bitsf(y1)) != 1.0f) y1++;
  for (uint32_t u = y1; u <= xl_fbits(64.0f); u += 997)
    if (tanhf(xl_bitsf(u)) != 1.0f) {
      snprintf(err, errlen, "tanhf not 1 above its threshold at %08x", u);
      return -2;
    }
  const float big[] = {64.0f, 1e3f, 1e10f, 3e38f};
  for (float v : big)
    if (tanhf(v) != 1.0f) {
      snprintf(err, errlen, "tanhf(%g) != 1", (double)v);
      return -2;
    }

  // below y1 the phi table covers [2^-31, y1); -logf(1) must be -0 above it
  if (xl_fbits(-logf(1.0f)) != 0x80000000u) {
    snprintf(err, errlen, "-logf(1) is not -0");
    return -2;
  }

  std::vector<uint32_t> log_tab, exp_tab;
  uint32_t log_cap = 0, exp_cap = 0;
  build_hash(logp, log_tab, log_cap);
  build_hash(expp, exp_tab, exp_cap);

  XlmHeader h;
  memset(&h, 0, sizeof h);
  memcpy(h.magic, XLM_MAGIC, 8);
  snprintf(h.libc, sizeof h.libc, "%s", gnu_get_libc_version());
  h.log_cap = log_cap;
  h.log_count = (uint32_t)logp.size();
  h.exp_cap = exp_cap;
  h.exp_count = (uint32_t)expp.size();
  h.tanh_ylo = XL_TANH_YLO;
  h.tanh_y1 = y1;
  h.exp_tie = exp_tie;
  std::string tmp = std::string(path) + ".tmp";
  FILE *f = fopen(tmp.c_str(), "wb");
  if (!f) {
    snprintf(err, errlen, "cannot write %s", tmp.c_str());
    return -4;
  }
  fwrite(&h, sizeof h, 1, f);
  fwrite(log_tab.data(), 4, log_tab.size(), f);
  fwrite(exp_tab.data(), 4, exp_tab.size(), f);
  fwrite(&small, sizeof small, 1, f);
  fclose(f);
  if (rename(tmp.c_str(), path) != 0) {
    snprintf(err, errlen, "cannot rename %s", tmp.c_str());
    return -4;
  }
  return 0;
}

int dvc_libm_load(const char *path, XlmHost *out, char *err, int errlen) {
  FILE *f = fopen(path, "rb");
  if (!f) {
    snprintf(err, errlen, "no table file %s", path);
    return -1;
  }
  XlmHeader h;
  if (fread(&h, sizeof h, 1, f) != 1 || memcmp(h.magic, XLM_MAGIC, 8) != 0) {
    fclose(f);
    snprintf(err, errlen, "bad table header in %s", path);
    return -2;
  }
  if (strcmp(h.libc, gnu_get_libc_version()) != 0) {
    fclose(f);
    snprintf(err, errlen, "tables built for C library %s, running %s", h.libc, gnu_get_libc_version());
    return -3;
  }
  out->hdr = h;
  out->log_tab.resize((size_t)h.log_cap * 2);
  out->exp_tab.resize((size_t)h.exp_cap * 2);
  bool ok = fread(out->log_tab.data(), 4, out->log_tab.size(), f) == out->log_tab.size() &&
            fread(out->exp_tab.data(), 4, out->exp_tab.size(), f) == out->exp_tab.size() &&
            fread(&out->small, sizeof out->small, 1, f) == 1;
  fclose(f);
  if (!ok) {
    snprintf(err, errlen, "truncated table file %s", path);
    return -2;
  }
  return 0;
}

void dvc_phi_build(float *out, uint32_t ylo, uint32_t y1, int threads) {
  if (threads <= 0) threads = hw_threads();
  parallel_ranges(ylo, (uint64_t)y1 - 1, threads, [&](int, uint64_t a, uint64_t b) {
    for (uint64_t u = a; u <= b; u++) out[u - ylo] = -logf(tanhf(xl_bitsf((uint32_t)u)));
  });
}
