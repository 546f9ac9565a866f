// Host-side builder and loader of the correction tables that make the device
// float functions in exact_libm.h return the C library's bits (see that
// header for the method).  The tables are derived from the C library that the
// reference decoder links on this host, by calling it over each input domain:
//
//   logf   every positive float up to 10001: hash of (input, result) pairs
//          where the library differs from xl_logf_base;
//   expf   every float in [-104, -0]: hash of the differing pairs;
//   expm1f arguments +-2y of every tanh argument y in [2^-31, y1): a bitmap over
//          y marking where the library's expm1f differs from xl_expm1f_base
//          (the library's value is then the neighbour toward the double value);
//   tanhf  y1 = first float with tanhf(y) == 1; the builder checks that below
//          y1 tanhf equals the expm1f formula bit for bit.
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

float tanh_formula(float y, float e) {
  // glibc-equivalent evaluation order, float arithmetic
  if (y >= 1.0f) return 1.0f - 2.0f / (e + 2.0f);
  return -e / (e + 2.0f);
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

  // ---- expf over [-104, -0]
  parallel_ranges(XL_EXP_LO, XL_EXP_HI, threads, [&](int t, uint64_t a, uint64_t b) {
    auto &v = parts[t];
    for (uint64_t u = a; u <= b; u++) {
      const float x = xl_bitsf((uint32_t)u);
      const float g = expf(x), m = xl_expf_base(x, sv);
      if (xl_fbits(g) != xl_fbits(m)) v.push_back({(uint32_t)u, xl_fbits(g)});
    }
  });
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

  // ---- expm1f bitmap over y in [ylo, y1) and the tanh identity check
  const uint32_t ylo = XL_TANH_YLO;
  const uint64_t ny = (uint64_t)y1 - ylo;
  std::vector<uint32_t> bitmap((ny + 31) / 32, 0u);
  std::atomic<long long> bad_identity(0), em1_count(0);
  std::atomic<uint32_t> first_bad(0);
  std::vector<std::vector<Pair>> esc_parts(threads);
  // threads write disjoint 32-aligned word ranges
  const uint64_t words = bitmap.size();
  parallel_ranges(0, words - 1, threads, [&](int tid, uint64_t wa, uint64_t wb) {
    long long cnt = 0;
    for (uint64_t wi = wa; wi <= wb; wi++) {
      uint32_t word = 0;
      for (int bit = 0; bit < 32; bit++) {
        const uint64_t i = wi * 32 + bit;
        if (i >= ny) break;
        const float y = xl_bitsf((uint32_t)(ylo + i));
        const float a = (y >= 1.0f) ? 2.0f * y : -2.0f * y;
        const float g = expm1f(a);
        const float m = xl_expm1f_base(a, sv);
        if (xl_fbits(g) != xl_fbits(m)) {
          if (xl_fbits(xl_step_toward(m, xl_expm1_d((double)a, sv))) != xl_fbits(g))
            esc_parts[tid].push_back({ylo + (uint32_t)i, xl_fbits(g)});
          word |= 1u << bit;
          cnt++;
        }
        if (xl_fbits(tanhf(y)) != xl_fbits(tanh_formula(y, g))) {
          bad_identity++;
          first_bad = ylo + (uint32_t)i;
        }
      }
      bitmap[wi] = word;
    }
    em1_count += cnt;
  });
  if (bad_identity.load()) {
    snprintf(err, errlen, "tanh identity failures %lld (first y bits %08x)", bad_identity.load(), first_bad.load());
    return -3;
  }
  std::vector<Pair> escp;
  for (auto &v : esc_parts) escp.insert(escp.end(), v.begin(), v.end());

  std::vector<uint32_t> log_tab, exp_tab, esc_tab;
  uint32_t log_cap = 0, exp_cap = 0, esc_cap = 0;
  build_hash(logp, log_tab, log_cap);
  build_hash(expp, exp_tab, exp_cap);
  build_hash(escp, esc_tab, esc_cap);

  XlmHeader h;
  memset(&h, 0, sizeof h);
  memcpy(h.magic, XLM_MAGIC, 8);
  snprintf(h.libc, sizeof h.libc, "%s", gnu_get_libc_version());
  h.log_cap = log_cap;
  h.log_count = (uint32_t)logp.size();
  h.exp_cap = exp_cap;
  h.exp_count = (uint32_t)expp.size();
  h.tanh_ylo = ylo;
  h.tanh_y1 = y1;
  h.em1_words = (uint32_t)bitmap.size();
  h.em1_count = (uint32_t)em1_count.load();
  h.esc_cap = esc_cap;
  h.esc_count = (uint32_t)escp.size();
  std::string tmp = std::string(path) + ".tmp";
  FILE *f = fopen(tmp.c_str(), "wb");
  if (!f) {
    snprintf(err, errlen, "cannot write %s", tmp.c_str());
    return -4;
  }
  fwrite(&h, sizeof h, 1, f);
  fwrite(log_tab.data(), 4, log_tab.size(), f);
  fwrite(exp_tab.data(), 4, exp_tab.size(), f);
  fwrite(bitmap.data(), 4, bitmap.size(), f);
  fwrite(esc_tab.data(), 4, esc_tab.size(), f);
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
  out->em1_bitmap.resize(h.em1_words);
  out->esc_tab.resize((size_t)h.esc_cap * 2);
  bool ok = fread(out->log_tab.data(), 4, out->log_tab.size(), f) == out->log_tab.size() &&
            fread(out->exp_tab.data(), 4, out->exp_tab.size(), f) == out->exp_tab.size() &&
            fread(out->em1_bitmap.data(), 4, out->em1_bitmap.size(), f) == out->em1_bitmap.size() &&
            fread(out->esc_tab.data(), 4, out->esc_tab.size(), f) == out->esc_tab.size() &&
            fread(&out->small, sizeof out->small, 1, f) == 1;
  fclose(f);
  if (!ok) {
    snprintf(err, errlen, "truncated table file %s", path);
    return -2;
  }
  return 0;
}
