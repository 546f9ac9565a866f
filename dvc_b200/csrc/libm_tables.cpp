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
//          magnitude (dvc_phi_build, packed by dvc_phi_pack; not stored in the
//          file, rebuilt in about two seconds when a context starts).
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

bool dvc_phi_pack(const float *phi, uint32_t ylo, uint32_t y1, int threads, PhiPacked &out, char *err, int errlen) {
  if (threads <= 0) threads = hw_threads();
  const uint32_t B = 1u << XL_PHI_BINADE_BITS;
  if ((ylo & (B - 1)) != 0 || y1 <= ylo) {
    snprintf(err, errlen, "phi table range [%08x, %08x) does not start a binade", ylo, y1);
    return false;
  }
  const uint64_t n = (uint64_t)y1 - ylo;
  const int nb = (int)((n + B - 1) / B);
  auto bits = [&](uint64_t i) { return xl_fbits(phi[i]); };
  std::atomic<int> next{0};
  auto pool = [&](auto fn) {
    next = 0;
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++)
      ts.emplace_back([&]() {
        for (int b; (b = next.fetch_add(1)) < nb;) fn(b);
      });
    for (auto &th : ts) th.join();
  };
  // per binade: the smallest feasible layout.  Delta: G entries per record
  // hold fields of W = 96 / G bits, so a group's span (bits(v_0) - bits of its
  // last value, which needs the binade to be non-increasing) must stay below
  // 2^W.  Split: every group may change value at most twice; G = 2 always fits.
  std::vector<uint32_t> fmt(nb);
  std::vector<uint64_t> nrec(nb);
  pool([&](int b) {
    const uint64_t a = (uint64_t)b * B, e = std::min<uint64_t>(n, a + B), len = e - a;
    std::vector<uint32_t> pre(len);  // changes in (a, a + t]
    bool mono = true;
    uint32_t c = 0;
    pre[0] = 0;
    for (uint64_t t = 1; t < len; t++) {
      const uint32_t u0 = bits(a + t - 1), u1 = bits(a + t);
      c += u1 != u0;
      if (u1 > u0) mono = false;
      pre[t] = c;
    }
    uint64_t best = ~0ull;
    for (uint32_t G = 2; G <= 255; G++) {
      const uint32_t W = 96 / G;
      const uint64_t recs = (len + G - 1) / G;
      uint64_t dmax = 0, rmax = 0;
      for (uint64_t g0 = 0; g0 < len; g0 += G) {
        const uint64_t g1 = std::min<uint64_t>(len, g0 + G) - 1;
        dmax = std::max<uint64_t>(dmax, (uint64_t)bits(a + g0) - bits(a + g1));
        rmax = std::max<uint64_t>(rmax, pre[g1] - pre[g0]);
      }
      if (G >= 4 && G <= 32 && mono && dmax <= ((1ull << W) - 1) && recs * 16 < best) {
        best = recs * 16;
        fmt[b] = G | (W << 8);
        nrec[b] = recs;
      }
      if (rmax <= 2 && recs * 16 < best) {
        best = recs * 16;
        fmt[b] = G | XL_PHI_SPLIT;
        nrec[b] = recs;
      }
    }
  });
  std::vector<uint64_t> rec0(nb + 1, 0);
  for (int b = 0; b < nb; b++) rec0[b + 1] = rec0[b] + nrec[b];
  if (rec0[nb] >= (1ull << 31)) {
    snprintf(err, errlen, "phi table too large to pack");
    return false;
  }
  out.desc.assign((size_t)nb * 4, 0);
  for (int b = 0; b < nb; b++) {
    const uint32_t G = fmt[b] & 0xffu;
    out.desc[4 * b] = (uint32_t)rec0[b];
    out.desc[4 * b + 1] = fmt[b];
    out.desc[4 * b + 2] = (uint32_t)(((1ull << 32) + G - 1) / G);
  }
  out.rec.assign((size_t)rec0[nb] * 4, 0);
  pool([&](int b) {
    const uint64_t a = (uint64_t)b * B, e = std::min<uint64_t>(n, a + B);
    const uint32_t G = fmt[b] & 0xffu, W = (fmt[b] >> 8) & 0xffu;
    const bool split = (fmt[b] & XL_PHI_SPLIT) != 0;
    uint32_t *rec = out.rec.data() + rec0[b] * 4;
    for (uint64_t g0 = a; g0 < e; g0 += G, rec += 4) {
      rec[0] = bits(g0);
      if (split) {
        // up to three values; s1, s2 = the entries where the second and third start (G: never)
        uint32_t s1 = G, s2 = G, nv = 1;
        rec[1] = rec[2] = rec[0];
        for (uint32_t k = 1; k < G && g0 + k < e; k++) {
          if (bits(g0 + k) == bits(g0 + k - 1)) continue;
          if (nv == 1) {
            s1 = k;
            rec[1] = rec[2] = bits(g0 + k);
          } else {
            s2 = k;
            rec[2] = bits(g0 + k);
          }
          nv++;
        }
        rec[3] = s1 | (s2 << 8);
        continue;
      }
      for (uint32_t k = 1; k < G && g0 + k < e; k++) {
        const uint32_t f = bits(g0) - bits(g0 + k);
        const uint32_t pos = k * W, wi = pos >> 5, sh = pos & 31u;
        rec[1 + wi] |= f << sh;
        if (sh + W > 32) rec[2 + wi] |= f >> (32 - sh);
      }
    }
  });
  // every entry of the packed table against the sweep, through the decode the device uses
  std::atomic<uint64_t> bad{0}, first_bad{~0ull};
  parallel_ranges(0, n - 1, threads, [&](int, uint64_t a, uint64_t e) {
    for (uint64_t i = a; i <= e; i++) {
      const uint32_t *d = out.desc.data() + 4 * (i >> XL_PHI_BINADE_BITS);
      const uint32_t j = (uint32_t)(i & (B - 1)), g = xl_phi_group(j, d[2]);
      const uint32_t *r = out.rec.data() + 4 * ((uint64_t)d[0] + g);
      const uint32_t f = xl_phi_decode_bits(j - g * (d[1] & 0xffu), d[1], r[0], r[1], r[2], r[3]);
      if (f != bits(i)) {
        if (bad.fetch_add(1) == 0) first_bad = i;
      }
    }
  });
  if (bad.load()) {
    snprintf(err, errlen, "packed phi table differs from the sweep at %llu entries (first %llu)",
             (unsigned long long)bad.load(), (unsigned long long)first_bad.load());
    return false;
  }
  return true;
}

extern "C" int dvc_phi_table_check(size_t *packed_bytes, char *msg, int msglen) {
  // y1 = the first float with tanhf(y) == 1 (tanhf is non-decreasing)
  uint32_t lo = XL_TANH_YLO, hi = 0x42000000u;  // tanhf(32) == 1
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (tanhf(xl_bitsf(mid)) == 1.0f) hi = mid;
    else lo = mid + 1;
  }
  const uint32_t y1 = lo;
  std::vector<float> phi((size_t)y1 - XL_TANH_YLO);
  dvc_phi_build(phi.data(), XL_TANH_YLO, y1, 0);
  PhiPacked pk;
  char err[256];
  if (!dvc_phi_pack(phi.data(), XL_TANH_YLO, y1, 0, pk, err, sizeof err)) {
    if (msg && msglen > 0) snprintf(msg, (size_t)msglen, "%s", err);
    return -4;  // DVC_E_DATA
  }
  if (packed_bytes) *packed_bytes = (pk.desc.size() + pk.rec.size()) * 4;
  size_t nsplit = 0;
  for (size_t b = 0; b < pk.desc.size() / 4; b++) nsplit += (pk.desc[4 * b + 1] & XL_PHI_SPLIT) != 0;
  if (msg && msglen > 0)
    snprintf(msg, (size_t)msglen, "%zu entries in %zu binades, %zu records, %zu split binades", phi.size(),
             pk.desc.size() / 4, pk.rec.size() / 4, nsplit);
  return 0;
}
