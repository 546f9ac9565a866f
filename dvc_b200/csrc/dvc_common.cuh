// Shared device definitions for the Wyner-Ziv decoder kernels (sm_100a).
//
// All float/double arithmetic in these kernels is compiled with -fmad=false so
// that every product and sum is rounded separately, as in the reference's x86
// SSE2 build; divisions and square roots are IEEE (no fast-math).  The only
// fused multiply-adds are the explicit ones of the table-driven exp/log in
// exact_libm.h, which the host table builder evaluates the same way.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "exact_libm.h"
#include "libm_tables.h"

namespace dvc {

// zig-zag band order (DvcDec/src/global.cpp:36-41)
__constant__ int c_zigzag[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};

#define DVC_WZ_B 0
#define DVC_INTRA_B 1
#define DVC_SKIP_B 2

// ------------------------------------------------------------------------
// Library-exact float functions (see exact_libm.h for the method).

// view of the small tables in global memory
__device__ __forceinline__ XlSmall xl_small_global(const XlmDev &t) {
  return XlSmall{t.small->exp2j, t.small->invc, t.small->logc, t.small->efold};
}

// copy the small tables into shared memory (every thread of the block calls
// this; follow with __syncthreads); `buf` holds sizeof(XlmSmallTables) bytes
__device__ __forceinline__ XlSmall xl_small_stage(const XlmDev &t, XlmSmallTables *buf) {
  const uint32_t *src = reinterpret_cast<const uint32_t *>(t.small);
  uint32_t *dst = reinterpret_cast<uint32_t *>(buf);
  for (int i = threadIdx.x; i < (int)(sizeof(XlmSmallTables) / 4); i += blockDim.x) dst[i] = src[i];
  return XlSmall{buf->exp2j, buf->invc, buf->logc, buf->efold};
}

__device__ __forceinline__ float xl_hash_lookup(const uint32_t *tab, uint32_t mask, int shift, uint32_t key,
                                                float fallback) {
  uint32_t s = (key * 0x9E3779B1u) >> shift;
  uint2 kv = __ldg(reinterpret_cast<const uint2 *>(tab + 2 * s));
  if (kv.x == key) return __uint_as_float(kv.y);
  // load factor <= 1/2, so an empty slot ends every probe; the bound is a guard
  for (uint32_t probe = 0; kv.x != 0xFFFFFFFFu && probe < mask; probe++) {
    s = (s + 1) & mask;
    kv = __ldg(reinterpret_cast<const uint2 *>(tab + 2 * s));
    if (kv.x == key) return __uint_as_float(kv.y);
  }
  return fallback;
}

// logf as the C library computes it, for every positive float up to 10001
__device__ __forceinline__ float xl_logf(const XlmDev &t, const XlSmall &s, float x) {
  const uint32_t u = __float_as_uint(x);
  if (!(x > 0.0f) || u >= 0x7f800000u) {
    if (x == 0.0f) return __uint_as_float(0xff800000u);  // -inf
    if (u == 0x7f800000u) return x;                      // +inf
    return __uint_as_float(0x7fc00000u);                 // NaN
  }
  const float m = xl_logf_base(x, s);
  if (u > XL_LOG_HI) return m;
  return xl_hash_lookup(t.log_tab, t.log_mask, t.log_shift, u, m);
}

// expf as the C library computes it, for x <= 0
__device__ __forceinline__ float xl_expf(const XlmDev &t, const XlSmall &s, float x) {
  const uint32_t u = __float_as_uint(x);
  if (x != x) return x;
  if (u >= XL_EXP_HI && (u >> 31)) return 0.0f;  // x <= -104 (and -inf): underflows to +0
  const double d = xl_exp_d((double)x, s);
  const float m = XL_D2F(d);
  if (!(u >> 31)) return m;  // positive arguments do not occur in the decoder
  // every exception with a normal result lies within exp_tie of a midpoint
  if (d >= 0x1p-126 && xl_tie_dist(d) > t.exp_tie) return m;
  return xl_hash_lookup(t.exp_tab, t.exp_mask, t.exp_shift, u, m);
}

// copy the phi descriptors into shared memory (every thread of the block
// calls this; follow with __syncthreads); `buf` holds XL_PHI_MAX_BINADES entries
__device__ __forceinline__ void xl_phi_stage(const XlmDev &t, uint4 *buf) {
  for (int i = threadIdx.x; i < t.phi_nbin; i += blockDim.x) buf[i] = t.phi_desc[i];
}

// -logf(tanhf(y)), the reference's two library calls (LdpcaDecoder.cpp:513,519),
// from the packed table over [tanh_ylo, tanh_y1); -0 where tanhf(y) is 1.
// Every argument the decoder forms is (x + 1e-9f)/2 with x >= 0, so it is at
// least 5e-10 > 2^-31 = tanh_ylo; a smaller one (never formed) clamps to the
// first entry rather than reading outside the table.  `desc` is the binade
// descriptor array (staged in shared memory by xl_phi_stage); one 16-byte
// record read per call, the same instructions in every binade, so that the
// reads of several calls can be in flight together.  Records are cached in
// L1: messages that stay put from one iteration to the next read the same
// records again.
__device__ __forceinline__ float xl_phi(const XlmDev &t, const uint4 *desc, float y) {
  const uint32_t u = __float_as_uint(y);
  const bool one = u >= t.tanh_y1;  // tanhf(y) == 1 (also NaN/negative patterns, never formed)
  const uint32_t i = (!one && u > t.tanh_ylo) ? u - t.tanh_ylo : 0u;
  const uint4 d = desc[i >> XL_PHI_BINADE_BITS];
  const uint32_t j = i & ((1u << XL_PHI_BINADE_BITS) - 1u);
  const uint32_t g = xl_phi_group(j, d.z);
  const uint4 r = tex1Dfetch<uint4>((cudaTextureObject_t)t.phi_tex, (int)(d.x + g));
  const uint32_t v = xl_phi_decode_bits(j - g * (d.y & 0xffu), d.y, r.x, r.y, r.z, r.w);
  return one ? -0.0f : __uint_as_float(v);
}

}  // namespace dvc
