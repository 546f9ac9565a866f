// Bit-reproducible float elementary functions for the decoder hot path.
//
// The reference decoder's float math calls the host C library: logf and tanhf
// in belief propagation (DvcDec/src/LdpcaDecoder.cpp:513,519,666) and in the
// entropy bound (:135-136), expf in the noise model (noiseModel.cpp:93,126) and
// in motion learning (motionLearning.cpp:111).  Its decisions (accepted ladder
// code, decoded bits) depend on those exact float results, so the device must
// return the same bits as that library for every input the decoder can feed.
//
// Method:
//  1. xl_*_d: double-precision evaluations written here from the table-driven
//     method of P. T. P. Tang ("Table-driven implementation of the exponential
//     function", ACM TOMS 15(2), 1989; "... of the logarithm function", ACM TOMS
//     16(4), 1990), using only IEEE-rounded operations and explicit fused
//     multiply-adds, so host and device produce identical bits:
//       exp:   x = (32k + j) ln2/32 + r, |r| <= ln2/64; e^x = 2^k * T[j] * P(r)
//              with T[j] = 2^(j/32) and P the degree-6 Taylor polynomial;
//       log:   x = 2^e * m, m in [1, 2) split into 128 bins; per bin a
//              reciprocal centre 1/c and log c (bins at and above sqrt 2 fold
//              into [sqrt(1/2), 1) so that values near 1 keep full relative
//              accuracy), log x = (e + f) ln2 + log c + log1p(m/c - 1) with a
//              degree-8 polynomial for log1p.
//     The small tables are computed on the host at table-build time and stored
//     with the correction tables, so host and device always use the same ones.
//     Rounding the double result to float gives the correctly rounded value
//     except in rare near-tie cases.
//  2. Correction tables built on the host by sweeping the C library over the
//     exact input domain (libm_tables.cpp): the inputs where the library's float
//     result differs from part 1, with the library's value, in a hash.  For
//     expf every such input lies within a tiny distance of a float rounding
//     midpoint (the sweep records the largest, exp_tie); the device reads the
//     hash only for results that close to a midpoint (about 1 in 10^5).
//
// The belief-propagation magnitude phi(y) = -logf(tanhf(y)) is not evaluated
// at all: its argument is a float in [2^-31, y1) (y1 = the first float with
// tanhf(y) == 1, above which phi is -0), so the library's value of the whole
// expression is swept once per context for every one of those 2.9e8 floats
// and stored packed (xl_phi_field below, about 170 MB instead of 1.1 GB), so
// that the part the decoder reads stays in the L2 cache.
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define XL_HD __host__ __device__ __forceinline__
#else
#define XL_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define XL_FMA(a, b, c) __fma_rn((a), (b), (c))
#define XL_D2F(a) __double2float_rn(a)
#else
#define XL_FMA(a, b, c) fma((a), (b), (c))
#define XL_D2F(a) ((float)(a))
#endif

// ln 2 = XL_LN2_HI + XL_LN2_LO (44-bit head)
#define XL_LN2_HI 0x1.62e42fefa38p-1
#define XL_LN2_LO 0x1.ef35793c7673p-45
#define XL_INV_LN2 0x1.71547652b82fep+0

// the small tables of part 1 (host copies live in libm_tables.cpp; device copies
// are read through this view, from global or shared memory)
struct XlSmall {
  const double *exp2j;  // [32] 2^(j/32)
  const double *invc;   // [128] reciprocal bin centre
  const double *logc;   // [128] log of the centre, folded bins minus ln 2
  const int *efold;     // [128] 1 for bins folded into [sqrt(1/2), 1)
};

XL_HD uint64_t xl_dbits(double d) {
  union { double d; uint64_t u; } c;
  c.d = d;
  return c.u;
}
XL_HD double xl_bitsd(uint64_t u) {
  union { double d; uint64_t u; } c;
  c.u = u;
  return c.d;
}
XL_HD uint32_t xl_fbits(float f) {
  union { float f; uint32_t u; } c;
  c.f = f;
  return c.u;
}
XL_HD float xl_bitsf(uint32_t u) {
  union { float f; uint32_t u; } c;
  c.u = u;
  return c.f;
}

// e^x for x in [-745, 88]; the decoder uses [-110, 20]
XL_HD double xl_exp_d(double x, const XlSmall &s) {
  const double t = x * (32.0 * XL_INV_LN2);
  const int k = (int)(t >= 0.0 ? t + 0.5 : t - 0.5);
  const double kd = (double)k;
  double r = XL_FMA(-kd, XL_LN2_HI / 32.0, x);
  r = XL_FMA(-kd, XL_LN2_LO / 32.0, r);
  double q = 1.0 / 720.0;
  q = XL_FMA(q, r, 1.0 / 120.0);
  q = XL_FMA(q, r, 1.0 / 24.0);
  q = XL_FMA(q, r, 1.0 / 6.0);
  q = XL_FMA(q, r, 0.5);
  q = XL_FMA(q, r, 1.0);
  const double er = XL_FMA(q, r, 1.0);
  const int j = k & 31, hi = (k - j) / 32;
  // 2^hi in two normal factors
  const int h1 = hi / 2, h2 = hi - h1;
  const double s1 = xl_bitsd((uint64_t)(h1 + 1023) << 52), s2 = xl_bitsd((uint64_t)(h2 + 1023) << 52);
  return ((s.exp2j[j] * er) * s1) * s2;
}

// natural log of a positive double that came from a float (normal as a double)
XL_HD double xl_log_d(double x, const XlSmall &s) {
  const uint64_t u = xl_dbits(x);
  const int e = (int)((u >> 52) & 0x7ff) - 1023;
  const double m = xl_bitsd((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
  const int i = (int)((u >> 45) & 127);
  const double r = XL_FMA(m, s.invc[i], -1.0);
  double q = -1.0 / 8.0;
  q = XL_FMA(q, r, 1.0 / 7.0);
  q = XL_FMA(q, r, -1.0 / 6.0);
  q = XL_FMA(q, r, 1.0 / 5.0);
  q = XL_FMA(q, r, -1.0 / 4.0);
  q = XL_FMA(q, r, 1.0 / 3.0);
  q = XL_FMA(q, r, -0.5);
  const double l1p = XL_FMA(r * r, q, r);
  const double ed = (double)(e + s.efold[i]);
  const double head = XL_FMA(ed, XL_LN2_HI, s.logc[i]);
  return head + XL_FMA(ed, XL_LN2_LO, l1p);
}

// float results of part 1, before corrections
XL_HD float xl_expf_base(float x, const XlSmall &s) { return XL_D2F(xl_exp_d((double)x, s)); }
XL_HD float xl_logf_base(float x, const XlSmall &s) { return XL_D2F(xl_log_d((double)x, s)); }

// Distance of a double from the nearest float rounding boundary (the midpoint
// between two floats of its binade), in units of 2^-52 of the binade: the
// 29 mantissa bits that rounding to float drops, measured from 2^28.  A
// library whose float result differs from the correctly rounded one only for
// doubles this close to a midpoint agrees with XL_D2F(d) everywhere else.
XL_HD uint32_t xl_tie_dist(double d) {
  const uint32_t low = (uint32_t)(xl_dbits(d) & ((1u << 29) - 1));
  return low >= (1u << 28) ? low - (1u << 28) : (1u << 28) - low;
}

// ---- domains (float bit patterns, inclusive) swept by the table builder ----
// logf inputs: LLR from LR in [1e-4/0.9999, 0.9999/1e-4], tanh values in
// [tanh(5e-10), 1], crossover probabilities; every positive float up to 10001
// is swept so that any input the decoder can form is covered.
#define XL_LOG_LO 0x00000001u  // smallest positive subnormal
#define XL_LOG_HI 0x461c4400u  // 10001.0f
// expf inputs: -alpha*d and -0.01*SSE, always <= 0; below -104 the result is 0
#define XL_EXP_LO 0x80000000u  // -0.0f  (negative floats ordered by magnitude)
#define XL_EXP_HI 0xc2d00000u  // -104.0f
// tanh arguments y = (x + 1e-9)/2 with x >= 0, so y >= 5e-10
#define XL_TANH_YLO 0x30000000u  // 2^-31, below the smallest y = 1e-9f/2 (0x3009705f)

// ---- packed table of phi(y) = -logf(tanhf(y)) ----
// Entry i is the library's phi of the float with bits XL_TANH_YLO + i.  The
// entries are split into binades (2^23 consecutive patterns, one exponent of
// y); each binade has a descriptor {first record, format, reciprocal} and is
// cut into groups of G consecutive entries, one 16-byte record per group, in
// one of two formats:
//  * delta format (4 <= G <= 32): word 0 = bits of the group's first value,
//    words 1..3 (96 bits, word 1 lowest) G fields of W = 96 / G bits, field k
//    at bit k*W, field k = bits(v_0) - bits(v_k) (phi falls as y grows; field
//    0 is 0), v_k = word 0 - field k;
//  * split format (format bit 16, 2 <= G <= 255): the group holds at most
//    three distinct values, words 0..2; word 3 holds s1 (bits 0..7) and s2
//    (bits 8..15): v_k = word 0 for k < s1, word 1 for s1 <= k < s2, word 2
//    from s2 on.  Used where y >= 2: there tanhf takes few values and phi
//    jumps by more than a field holds.
// Either way one 16-byte record read gives the value, and the decode is the
// same instructions for both formats (both candidates are formed and one is
// selected), so that lanes reading different binades do not diverge.  The
// group of binade offset j is j / G = umulhi(j, ceil(2^32 / G)) (exact for
// j < 2^23, G < 512).  The builder (libm_tables.cpp) picks the smallest
// feasible layout per binade and checks every entry of the packed table
// against the swept one.
#define XL_PHI_BINADE_BITS 23
#define XL_PHI_SPLIT 0x10000u
#define XL_PHI_MAX_BINADES 64

XL_HD uint32_t xl_umulhi(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// group of binade offset j, recip = ceil(2^32 / G)
XL_HD uint32_t xl_phi_group(uint32_t j, uint32_t recip) { return xl_umulhi(j, recip); }

// field k of a record's words r1..r3; fmt = G | W << 8 (W = 0 in the split format: field 0)
XL_HD uint32_t xl_phi_field(uint32_t k, uint32_t fmt, uint32_t r1, uint32_t r2, uint32_t r3) {
  const uint32_t w = (fmt >> 8) & 0xffu;
  const uint32_t p = k * w;
  const uint32_t wi = p >> 5, sh = p & 31u;
  const uint32_t lo = wi == 0 ? r1 : (wi == 1 ? r2 : r3);
  const uint32_t hi = wi == 0 ? r2 : r3;
#if defined(__CUDA_ARCH__)
  return __funnelshift_r(lo, hi, sh) & ((1u << w) - 1u);
#else
  return (uint32_t)(((((uint64_t)hi) << 32) | lo) >> sh) & ((1u << w) - 1u);
#endif
}

// bits of entry k of a group from its record r0..r3 (both formats; xl_phi reads the record)
XL_HD uint32_t xl_phi_decode_bits(uint32_t k, uint32_t fmt, uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
  const uint32_t delta = r0 - xl_phi_field(k, fmt, r1, r2, r3);
  const uint32_t split = k < (r3 & 0xffu) ? r0 : (k < ((r3 >> 8) & 0xffu) ? r1 : r2);
  return (fmt & XL_PHI_SPLIT) ? split : delta;
}
