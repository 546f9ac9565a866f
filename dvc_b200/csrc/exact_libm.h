// Bit-reproducible float elementary functions for the decoder hot path.
//
// The reference decoder's float math calls the host C library: logf and tanhf
// in belief propagation (DvcDec/src/LdpcaDecoder.cpp:513,519,666) and in the
// entropy bound (:135-136), expf in the noise model (noiseModel.cpp:93,126) and
// in motion learning (motionLearning.cpp:111).  Its decisions (accepted ladder
// code, decoded bits) depend on those exact float results, so the device must
// return the same bits as that library for every input the decoder can feed.
//
// Method (two parts):
//  1. xl_*_d: double-precision evaluations written here from standard
//     mathematics, using only IEEE-rounded +, -, *, / (no fused multiply-add,
//     no library calls), so host and device produce identical bits:
//       exp:   Cody-Waite reduction x = k*ln2 + r (ln2 split into a 44-bit head
//              and a tail), Taylor series of e^r to r^13, scaled by 2^k;
//       log:   x = 2^e * m with m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
//              log m = 2 atanh(s) = 2s(1 + s^2/3 + s^4/5 + ... + s^22/23);
//       expm1: Taylor series to a^18 for |a| < 1/2, else exp(a) - 1.
//     Rounding the double result to float gives the correctly rounded value
//     except in rare near-tie cases.
//  2. Correction tables built on the host by sweeping the C library over the
//     exact input domain (libm_tables.cpp): the inputs where the library's float
//     result differs from part 1, with the library's value.  The library's
//     errors stay below one ulp, so its result is always the float neighbour of
//     part 1's on the side of the double value; for expm1f this lets a plain
//     bitmap mark the exceptions.  The builder verifies this for every input.
//
// tanhf is not swept directly: over the whole decoder domain the library's
// tanhf(y) equals, bit for bit, 1 - 2/(expm1f(2y)+2) for y >= 1 and
// -e/(e+2) with e = expm1f(-2y) for y < 1, evaluated in float; and it is
// exactly 1 from a threshold y1 upward.  The builder checks this identity for
// every y in the domain before writing any table.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define XL_HD __host__ __device__ __forceinline__
#else
#define XL_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define XL_DMUL(a, b) __dmul_rn((a), (b))
#define XL_DADD(a, b) __dadd_rn((a), (b))
#define XL_DSUB(a, b) __dsub_rn((a), (b))
#define XL_DDIV(a, b) __ddiv_rn((a), (b))
#define XL_FADD(a, b) __fadd_rn((a), (b))
#define XL_FSUB(a, b) __fsub_rn((a), (b))
#define XL_FMUL(a, b) __fmul_rn((a), (b))
#define XL_FDIV(a, b) __fdiv_rn((a), (b))
#define XL_D2F(a) __double2float_rn(a)
#else
#define XL_DMUL(a, b) ((a) * (b))
#define XL_DADD(a, b) ((a) + (b))
#define XL_DSUB(a, b) ((a) - (b))
#define XL_DDIV(a, b) ((a) / (b))
#define XL_FADD(a, b) ((a) + (b))
#define XL_FSUB(a, b) ((a) - (b))
#define XL_FMUL(a, b) ((a) * (b))
#define XL_FDIV(a, b) ((a) / (b))
#define XL_D2F(a) ((float)(a))
#endif

// ln 2 = XL_LN2_HI + XL_LN2_LO; the head has 44 significant bits so k*head is
// exact for |k| < 2^9.
#define XL_LN2_HI 0x1.62e42fefa38p-1
#define XL_LN2_LO 0x1.ef35793c7673p-45
#define XL_INV_LN2 0x1.71547652b82fep+0
#define XL_SQRT2 0x1.6a09e667f3bcdp+0

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

// round-half-away of |v| < 2^31 without library calls (the sign of ties does
// not matter for the reduction, only host/device agreement does)
XL_HD int xl_round_int(double v) { return (int)(v >= 0.0 ? XL_DADD(v, 0.5) : XL_DSUB(v, 0.5)); }

// e^x for x in [-745, 709]; used on [-110, 20].
XL_HD double xl_exp_d(double x) {
  const int k = xl_round_int(XL_DMUL(x, XL_INV_LN2));
  const double kd = (double)k;
  const double r = XL_DSUB(XL_DSUB(x, XL_DMUL(kd, XL_LN2_HI)), XL_DMUL(kd, XL_LN2_LO));
  double p = 1.0 / 6227020800.0;          // 1/13!
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 479001600.0);  // 1/12!
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 39916800.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 3628800.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 362880.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 40320.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 5040.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 720.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 120.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 24.0);
  p = XL_DADD(XL_DMUL(p, r), 1.0 / 6.0);
  p = XL_DADD(XL_DMUL(p, r), 0.5);
  // e^r = 1 + r + r^2 p
  const double er = XL_DADD(1.0, XL_DADD(r, XL_DMUL(XL_DMUL(r, r), p)));
  // 2^k as a double (k in [-1022, 1023] here; two steps keep it normal)
  const int k1 = k / 2, k2 = k - k1;
  const double s1 = xl_bitsd((uint64_t)(k1 + 1023) << 52);
  const double s2 = xl_bitsd((uint64_t)(k2 + 1023) << 52);
  return XL_DMUL(XL_DMUL(er, s1), s2);
}

// e^a - 1 for a in [-2, 20]
XL_HD double xl_expm1_d(double a) {
  if (a > -0.5 && a < 0.5) {
    double q = 1.0 / 6402373705728000.0;  // 1/18!
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 355687428096000.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 20922789888000.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 1307674368000.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 87178291200.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 6227020800.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 479001600.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 39916800.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 3628800.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 362880.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 40320.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 5040.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 720.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 120.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 24.0);
    q = XL_DADD(XL_DMUL(q, a), 1.0 / 6.0);
    q = XL_DADD(XL_DMUL(q, a), 0.5);
    // a + a^2 q
    return XL_DADD(a, XL_DMUL(XL_DMUL(a, a), q));
  }
  return XL_DSUB(xl_exp_d(a), 1.0);
}

// natural log of a positive normal double
XL_HD double xl_log_d(double x) {
  const uint64_t u = xl_dbits(x);
  int e = (int)((u >> 52) & 0x7ff) - 1023;
  double m = xl_bitsd((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
  if (m > XL_SQRT2) {
    m = XL_DMUL(m, 0.5);
    e += 1;
  }
  const double s = XL_DDIV(XL_DSUB(m, 1.0), XL_DADD(m, 1.0));
  const double z = XL_DMUL(s, s);
  double q = 1.0 / 23.0;
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 21.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 19.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 17.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 15.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 13.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 11.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 9.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 7.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 5.0);
  q = XL_DADD(XL_DMUL(q, z), 1.0 / 3.0);
  const double s2 = XL_DADD(s, s);
  // log m = 2s + 2s z q
  const double lm = XL_DADD(s2, XL_DMUL(XL_DMUL(s2, z), q));
  const double ed = (double)e;
  return XL_DADD(XL_DMUL(ed, XL_LN2_HI), XL_DADD(lm, XL_DMUL(ed, XL_LN2_LO)));
}

// float results of part 1, before corrections
XL_HD float xl_expf_base(float x) { return XL_D2F(xl_exp_d((double)x)); }
XL_HD float xl_expm1f_base(float a) { return XL_D2F(xl_expm1_d((double)a)); }
XL_HD float xl_logf_base(float x) { return XL_D2F(xl_log_d((double)x)); }

// the float neighbour of r on the side of the double value d (d != r)
XL_HD float xl_step_toward(float r, double d) {
  uint32_t u = xl_fbits(r);
  const bool up = d > (double)r;
  // r is finite and nonzero in every domain used here
  if ((u >> 31) == 0) u = up ? u + 1 : u - 1;
  else u = up ? u - 1 : u + 1;
  return xl_bitsf(u);
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
// tanh arguments y = (x + 1e-9)/2 >= 5e-10; expm1f arguments -2y (y < 1) or 2y
#define XL_TANH_YLO 0x30000000u  // 2^-31, below the smallest y = 1e-9f/2 (0x3009705f)
