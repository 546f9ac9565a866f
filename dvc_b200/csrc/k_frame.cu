// Wyner-Ziv frame kernels other than LDPCA: side-information creation,
// transforms, correlation-noise model, conditional bit probabilities,
// reconstruction, side-information refinement and motion learning.
//
// Every kernel takes the array of per-frame descriptors of a batch and uses
// blockIdx.y (or blockIdx.x for single-block-per-frame kernels) as the frame
// index, so one launch serves every frame of the batch.  Frames whose
// descriptor is not `active` return at once.
//
// Each kernel restates one reference function (paths in DvcDec/src) with the
// same operation order for every float/double result; the module is compiled
// with -fmad=false so no multiply-add is fused.
#include <cuda_runtime.h>

#include "dvc_common.cuh"
#include "frame_types.h"
#include "kernels.h"

namespace dvc {

#define SEARCH_R 32  // defines.h:8
#define LEARN_R 4    // defines.h:11
#define ML_N 81

__constant__ double c_post_scale[16];
__constant__ double c_pre_scale[16];

// updateSI motion-vector weight 1 + 0.05f * |2v| per integer displacement
// (dx, dy) in [-32, 32]^2 (sideInfoCreation.cpp:667-668), indexed
// (dy + 32) * 65 + dx + 32
__device__ double d_si_weight[65 * 65];

cudaError_t upload_transform_scales(const double *post, const double *pre) {
  cudaError_t e = cudaMemcpyToSymbol(c_post_scale, post, sizeof(double) * 16);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_pre_scale, pre, sizeof(double) * 16)) != cudaSuccess) return e;
  // IEEE square root on the host gives the device's bits (no contraction: -ffp-contract=off)
  static double wt[65 * 65];
  for (int dy = -32; dy <= 32; dy++)
    for (int dx = -32; dx <= 32; dx++) {
      const double vx = (double)(dx << 1), vy = (double)(dy << 1);
      wt[(dy + 32) * 65 + dx + 32] = 1.0 + (double)0.05f * sqrt(vx * vx + vy * vy);
    }
  return cudaMemcpyToSymbol(d_si_weight, wt, sizeof wt);
}

// Does the frame take part in step (band, bit)?  band < 0: frame-level steps.
// Bands are decoded in zig-zag order while Qbits > 0 (DVC_Decoder.cpp:161-165,
// 403-407); bitplanes from Qbits down to 1 (:196).
__device__ __forceinline__ bool in_step(const FrameDev &F, int band, int bit) {
  if (band < 0) return true;
  for (int b = 0; b <= band; b++)
    if (F.qbits[c_zigzag[b]] <= 0) return false;
  return bit <= 0 || bit <= F.qbits[c_zigzag[band]];
}

// ROUND, defines.h:23
__device__ __forceinline__ int dround(double x) { return x >= 0.0 ? (int)(x + 0.5) : -(int)(-x + 0.5); }

// x moved by k units in the last place (x positive and finite)
__device__ __forceinline__ double ulp_shift(double x, int k) {
  return __longlong_as_double(__double_as_longlong(x) + (long long)k);
}

// costFunc, sideInfoCreation.cpp:10-12 (K is the float 0.05f, promoted)
__device__ __forceinline__ double cost_func(double mad, double vx, double vy) {
  return mad * (1.0 + (double)0.05f * sqrt(vx * vx + vy * vy));
}

// computeEndPoint, sideInfoCreation.cpp:14-22
__device__ __forceinline__ int end_point(double st, double v, double scale, int lo, int hi) {
  const int e = (int)((st + v * scale) + 0.5);
  return e < lo ? lo : (e > hi ? hi : e);
}

// forward44, transform.cpp:63-104
__device__ __forceinline__ void forward44(int *blk) {
  int t[16];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    t[c] = blk[c] + blk[4 + c] + blk[8 + c] + blk[12 + c];
    t[4 + c] = (blk[c] << 1) + blk[4 + c] - blk[8 + c] - (blk[12 + c] << 1);
    t[8 + c] = blk[c] - blk[4 + c] - blk[8 + c] + blk[12 + c];
    t[12 + c] = blk[c] - (blk[4 + c] << 1) + (blk[8 + c] << 1) - blk[12 + c];
  }
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int *s = t + 4 * r;
    int *o = blk + 4 * r;
    o[0] = s[0] + s[1] + s[2] + s[3];
    o[1] = (s[0] << 1) + s[1] - s[2] - (s[3] << 1);
    o[2] = s[0] - s[1] - s[2] + s[3];
    o[3] = s[0] - (s[1] << 1) + (s[2] << 1) - s[3];
  }
#pragma unroll
  for (int i = 0; i < 16; i++) blk[i] = dround(((double)blk[i]) * c_post_scale[i]);
}

// inverse44, transform.cpp:106-151
__device__ __forceinline__ void inverse44(int *blk) {
  int t[16];
#pragma unroll
  for (int i = 0; i < 16; i++) blk[i] = dround(((double)blk[i]) * c_pre_scale[i]);
#pragma unroll
  for (int c = 0; c < 4; c++) {
    t[c] = blk[c] + blk[4 + c] + blk[8 + c] + (blk[12 + c] >> 1);
    t[4 + c] = blk[c] + (blk[4 + c] >> 1) - blk[8 + c] - blk[12 + c];
    t[8 + c] = blk[c] - (blk[4 + c] >> 1) - blk[8 + c] + blk[12 + c];
    t[12 + c] = blk[c] - blk[4 + c] + blk[8 + c] - (blk[12 + c] >> 1);
  }
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int *s = t + 4 * r;
    int *o = blk + 4 * r;
    o[0] = s[0] + s[1] + s[2] + (s[3] >> 1);
    o[1] = s[0] + (s[1] >> 1) - s[2] - s[3];
    o[2] = s[0] - (s[1] >> 1) - s[2] + s[3];
    o[3] = s[0] - s[1] + s[2] - (s[3] >> 1);
  }
#pragma unroll
  for (int i = 0; i < 16; i++) blk[i] >>= 6;
}

// argmin with the reference's strict-< row-major scan: lowest cost, then lowest scan index
__device__ __forceinline__ void better(double &c, int &i, double c2, int i2) {
  if (c2 < c || (c2 == c && i2 < i)) {
    c = c2;
    i = i2;
  }
}

template <int NT>
__device__ __forceinline__ void block_argmin(double &c, int &i, double *sc, int *si) {
  for (int o = 16; o > 0; o >>= 1) {
    const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
    better(c, i, c2, i2);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    sc[warp] = c;
    si[warp] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NT / 32; w++) better(c, i, sc[w], si[w]);
    sc[0] = c;
    si[0] = i;
  }
  __syncthreads();
  c = sc[0];
  i = si[0];
}

// lowest (cost, index) over a full warp for costs >= 0 (never NaN): a
// non-negative double orders like its bit pattern, so three 32-bit warp
// reductions give it (high word, low word among the lanes that hold the
// smallest high word, index among the lanes that hold the smallest cost)
__device__ __forceinline__ void warp_argmin_nonneg(double &c, int &i) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(c);
  const unsigned hw = (unsigned)(b >> 32), lw = (unsigned)b;
  const unsigned mh = __reduce_min_sync(0xffffffffu, hw);
  const unsigned ml = __reduce_min_sync(0xffffffffu, hw == mh ? lw : 0xffffffffu);
  const unsigned mi = __reduce_min_sync(0xffffffffu, (hw == mh && lw == ml) ? (unsigned)i : 0xffffffffu);
  c = __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
  i = (int)mi;
}

// block_argmin of two independent (cost, index) pairs with costs >= 0 in one
// reduction; sc and si hold 2 * NT / 32 entries
template <int NT>
__device__ __forceinline__ void block_argmin2(double &c0, int &i0, double &c1, int &i1, double *sc, int *si) {
  warp_argmin_nonneg(c0, i0);
  warp_argmin_nonneg(c1, i1);
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sc[warp] = c0;
    si[warp] = i0;
    sc[NW + warp] = c1;
    si[NW + warp] = i1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NW; w++) {
      better(c0, i0, sc[w], si[w]);
      better(c1, i1, sc[NW + w], si[NW + w]);
    }
    sc[0] = c0;
    si[0] = i0;
    sc[NW] = c1;
    si[NW] = i1;
  }
  __syncthreads();
  c0 = sc[0];
  i0 = si[0];
  c1 = sc[NW];
  i1 = si[NW];
}

// ---------------------------------------------------------------- filters

// lowPassFilter, filter.cpp:214-233
__global__ void lowpass_kernel(const uint8_t *__restrict__ in, int w, int h, uint8_t *__restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w) return;
  double sum = 0;
  for (int m = y - 1; m <= y + 1; m++) {
    if (m < 0 || m >= h) continue;
    for (int n = x - 1; n <= x + 1; n++) {
      if (n < 0 || n >= w) continue;
      sum += (double)in[m * w + n];
    }
  }
  out[y * w + x] = (uint8_t)(sum / 9);
}

// FIR_filter, filter.cpp:55-117, on the output window it keeps.  The taps are
// the separable (1,-5,20,20,-5,1) half-pel filter: /32 horizontally or
// vertically, /1024 at the centre position; zero taps of the reference's 6x6
// tables are skipped (adding +0 to the running sum never changes it).
__global__ void fir_kernel(const uint8_t *__restrict__ in, int w, int h, uint8_t *__restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
  const int w2 = w << 1;
  if (j >= w2) return;
  const double tap[6] = {1.0, -5.0, 20.0, 20.0, -5.0, 1.0};
  const int sub = (j & 1) + ((i & 1) << 1);
  const int cy = i / 2, cx = j / 2;
  auto px = [&](int yy, int xx) {
    yy = yy < 0 ? 0 : (yy > h - 1 ? h - 1 : yy);
    xx = xx < 0 ? 0 : (xx > w - 1 ? w - 1 : xx);
    return (double)in[yy * w + xx];
  };
  uint8_t v;
  if (sub == 0) {
    v = (uint8_t)px(cy, cx);
  } else {
    double sum = 0.0;
    if (sub == 1) {
      for (int jj = 0; jj < 6; jj++) sum += (tap[jj] / 32.0) * px(cy, cx - 2 + jj);
    } else if (sub == 2) {
      for (int ii = 0; ii < 6; ii++) sum += (tap[ii] / 32.0) * px(cy - 2 + ii, cx);
    } else {
      for (int ii = 0; ii < 6; ii++)
        for (int jj = 0; jj < 6; jj++) sum += ((tap[ii] * tap[jj]) / 1024.0) * px(cy - 2 + ii, cx - 2 + jj);
    }
    int r = (int)(sum + 0.5);
    v = (uint8_t)(r < 0 ? 0 : (r > 255 ? 255 : r));
  }
  out[i * w2 + j] = v;
}

cudaError_t launch_ref_planes(const uint8_t *recon, int w, int h, uint8_t *lp, uint8_t *ip, cudaStream_t s) {
  lowpass_kernel<<<dim3((w + 127) / 128, h), 128, 0, s>>>(recon, w, h, lp);
  fir_kernel<<<dim3((2 * w + 127) / 128, 2 * h), 128, 0, s>>>(recon, w, h, ip);
  return cudaGetLastError();
}

// ----------------------------------------------------- side-info creation

// forwardME, sideInfoCreation.cpp:61-118: per 16x16 block of the future
// low-pass frame, full search of +-32 pixels in the past low-pass frame.
template <int NT>
__global__ void __launch_bounds__(NT) forward_me_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, h = F.h, b16w = w / 16;
  const int i = blockIdx.x;
  const int top = (i / b16w) << 4, left = (i % b16w) << 4;
  int st = top - SEARCH_R, sb = top + SEARCH_R, sl = left - SEARCH_R, sr = left + SEARCH_R;
  if (st < 0) st = 0;
  if (sb > h - 16) sb = h - 16;
  if (sl < 0) sl = 0;
  if (sr > w - 16) sr = w - 16;
  const int ww = sr - sl + 16, wh = sb - st + 16;  // staged window (<= 80x80)
  // window rows of 84 bytes in aligned 4-byte words: the window starts at byte
  // `wo` of each row (w is a multiple of 4, so the words of [sl & ~3, sl + ww)
  // stay inside the frame row; ww + 3 <= 84); the block's rows four pixels per
  // word (first pixel lowest)
  constexpr int WS = 84;
  __shared__ __align__(16) uint8_t win[80 * WS];
  __shared__ uint32_t blk4[64];
  __shared__ double sc[NT / 32];
  __shared__ int sidx[NT / 32];
  const int wo = sl & 3, nwd = (wo + ww + 3) >> 2;
  for (int y = threadIdx.x >> 5; y < wh; y += NT / 32) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(F.past_lp + (size_t)(st + y) * w + (sl - wo));
    uint32_t *dst = reinterpret_cast<uint32_t *>(win + y * WS);
    for (int x = threadIdx.x & 31; x < nwd; x += 32) dst[x] = __ldg(src + x);
  }
  for (int k = threadIdx.x; k < 64; k += NT)
    blk4[k] = __ldg(reinterpret_cast<const uint32_t *>(F.future_lp + (size_t)(top + (k >> 2)) * w + left) + (k & 3));
  __syncthreads();
  const int cw = sr - sl + 1, nc = cw * (sb - st + 1);
  double best = 1e300;
  int bi = 0x7fffffff;
  // candidate c = py * cw + pxo, advanced by NT without a division per candidate
  const int dq = NT / cw, dr = NT - dq * cw;
  int py = threadIdx.x / cw, pxo = threadIdx.x - py * cw;
  for (int c = threadIdx.x; c < nc; c += NT) {
    const int X = pxo + wo, sh = (X & 3) * 8;
    const uint32_t *rb = reinterpret_cast<const uint32_t *>(win) + (X >> 2);
    int sad = 0;
#pragma unroll 4
    for (int m = 0; m < 16; m++) {
      const uint32_t *r = rb + (py + m) * (WS / 4);
      const uint32_t w0 = r[0], w1 = r[1], w2 = r[2], w3 = r[3], w4 = r[4];
      sad += (int)__vsadu4(__funnelshift_r(w0, w1, sh), blk4[4 * m]);
      sad += (int)__vsadu4(__funnelshift_r(w1, w2, sh), blk4[4 * m + 1]);
      sad += (int)__vsadu4(__funnelshift_r(w2, w3, sh), blk4[4 * m + 2]);
      sad += (int)__vsadu4(__funnelshift_r(w3, w4, sh), blk4[4 * m + 3]);
    }
    const double vx = (double)(sl + pxo - left), vy = (double)(st + py - top);
    const double cost = cost_func((double)sad, vx, vy);
    if (cost < 10000000.0) better(best, bi, cost, c);
    pxo += dr;
    py += dq;
    if (pxo >= cw) {
      pxo -= cw;
      py++;
    }
  }
  block_argmin<NT>(best, bi, sc, sidx);
  if (threadIdx.x == 0) {
    MVd v{};
    if (bi != 0x7fffffff) {
      const int py = st + bi / cw, px = sl + bi % cw;
      v.px = (double)px;
      v.py = (double)py;
      v.vx = (double)(px - left);
      v.vy = (double)(py - top);
    }
    F.fmv[i] = v;
    F.holes[2 * i] = (double)left * F.ipc + (double)v.px * F.ifc;
    F.holes[2 * i + 1] = (double)top * F.ipc + (double)v.py * F.ifc;
  }
}

// forwardME, sideInfoCreation.cpp:120-142 (nearest projected hole per
// macroblock) and the half-pel scaling of createSideInfo (:511-521)
__global__ void forward_me_post_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, h = F.h, b16w = w / 16, b16n = b16w * (h / 16);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b16n) return;
  const int top = (i / b16w) << 4, left = (i % b16w) << 4;
  const double maxd = w * w + h * h;
  double mind = maxd;
  int bj = -1;
  for (int j = 0; j < b16n; j++) {
    const double hx = F.holes[2 * j], hy = F.holes[2 * j + 1];
    const double d = (left - hx) * (left - hx) + (top - hy) * (top - hy);
    if (d < mind) {
      mind = d;
      bj = j;
    }
  }
  MVd b{};
  if (bj >= 0) b = F.fmv[bj];
  MVd o;
  o.fx = (double)end_point(left, -b.vx, F.ifc, 0, w - 16);
  o.fy = (double)end_point(top, -b.vy, F.ifc, 0, h - 16);
  o.px = (double)end_point(left, b.vx, F.ipc, 0, w - 16);
  o.py = (double)end_point(top, b.vy, F.ipc, 0, h - 16);
  o.vx = o.px - o.fx;
  o.vy = o.py - o.fy;
  // half-pel units
  o.fx *= 2;
  o.fy *= 2;
  o.px *= 2;
  o.py *= 2;
  o.vx = o.px - o.fx;
  o.vy = o.py - o.fy;
  F.mb_mv[i] = o;
}

// bidirectME, sideInfoCreation.cpp:235-310.  The reference visits blocks in
// raster order and updates the vectors in place; a block's search window uses
// its top and left neighbours' updated and its bottom and right neighbours'
// previous vectors.  Blocks on one anti-diagonal are therefore independent:
// this single-block-per-frame kernel walks the anti-diagonals, one warp per
// block, which is equivalent to the raster order.
template <int NT>
__global__ void __launch_bounds__(NT) bidirect_me_kernel(FrameDev *frames, int bl) {
  FrameDev &F = frames[blockIdx.x];
  if (!F.active) return;
  MVd *mv = bl == 16 ? F.mb_mv : F.blk_mv;
  const int w = F.w, h = F.h, bh = h / bl, bw = w / bl, w2 = w << 1, bl2 = bl << 1;
  const int srb = (h << 1) - bl2, srr = w2 - bl2;
  const double scale = F.ipc / F.ifc;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint8_t *fut = F.future_ip, *pas = F.past_ip;
  for (int d = 0; d < bh + bw - 1; d++) {
    const int i0 = d - (bw - 1) > 0 ? d - (bw - 1) : 0;
    const int i1 = d < bh - 1 ? d : bh - 1;
    for (int i = i0 + warp; i <= i1; i += NT / 32) {
      const int j = d - i;
      const int bi = i * bw + j;
      const int y2 = i * bl2, x2 = j * bl2;
      const int st = (i - 1 >= 0) ? (int)mv[bi - bw].fy + bl2 : (int)mv[bi].fy;
      const int sb = (i + 1 < bh) ? (int)mv[bi + bw].fy - bl2 : (int)mv[bi].fy;
      const int sl = (j - 1 >= 0) ? (int)mv[bi - 1].fx + bl2 : (int)mv[bi].fx;
      const int sr = (j + 1 < bw) ? (int)mv[bi + 1].fx - bl2 : (int)mv[bi].fx;
      const int cw = sr - sl + 1, chh = sb - st + 1;
      const int nc = (cw > 0 && chh > 0) ? cw * chh : 0;
      double best = 1e300;
      int bc = 0x7fffffff;
      for (int c = lane; c < nc; c += 32) {
        const int fy = st + c / cw, fx = sl + c % cw;
        const int py = end_point(y2, (double)(y2 - fy), scale, 0, srb);
        const int px = end_point(x2, (double)(x2 - fx), scale, 0, srr);
        int mad = 0;
        for (int m = 0; m < bl2; m += 2) {
          const uint8_t *pr = pas + (py + m) * w2 + px;
          const uint8_t *fr = fut + (fy + m) * w2 + fx;
          for (int n = 0; n < bl2; n += 2) mad += abs((int)fr[n] - (int)pr[n]);
        }
        const double cost = cost_func((double)mad, (double)(px - fx), (double)(py - fy));
        if (cost < 10000000.0) better(best, bc, cost, c);
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double c2 = __shfl_xor_sync(0xffffffffu, best, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, bc, o);
        better(best, bc, c2, i2);
      }
      if (lane == 0 && bc != 0x7fffffff) {
        const int fy = st + bc / cw, fx = sl + bc % cw;
        const int py = end_point(y2, (double)(y2 - fy), scale, 0, srb);
        const int px = end_point(x2, (double)(x2 - fx), scale, 0, srr);
        MVd b;
        b.fx = (double)fx;
        b.fy = (double)fy;
        b.px = (double)px;
        b.py = (double)py;
        b.vx = (double)(px - fx);
        b.vy = (double)(py - fy);
        mv[bi] = b;
      }
    }
    __syncthreads();
  }
}

// createSideInfo, sideInfoCreation.cpp:524-545: 8x8 vectors initialised
// from their macroblock's vector
__global__ void init_blk_mv_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, h = F.h, b8w = w / 8, b8n = b8w * (h / 8), b16w = w / 16;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b8n) return;
  const int i = k / b8w, j = k % b8w;
  const int srb = (h - 8) << 1, srr = (w - 8) << 1;
  const int y2 = i << 4, x2 = j << 4;
  const MVd v = F.mb_mv[(i >> 1) * b16w + (j >> 1)];
  MVd o;
  o.fx = (double)end_point(x2, -v.vx, F.ifc, 0, srr);
  o.fy = (double)end_point(y2, -v.vy, F.ifc, 0, srb);
  o.px = (double)end_point(x2, v.vx, F.ipc, 0, srr);
  o.py = (double)end_point(y2, v.vy, F.ipc, 0, srb);
  o.vx = o.px - o.fx;
  o.vy = o.py - o.fy;
  F.blk_mv[k] = o;
}

// motionFilterAndComp, sideInfoCreation.cpp:325-342: mean squared error per 8x8 block
__global__ void mfc_mse_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, h = F.h, b8n = (w / 8) * (h / 8), w2 = w << 1;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b8n) return;
  const MVd v = F.blk_mv[k];
  const int fy = (int)v.fy, fx = (int)v.fx, py = (int)v.py, px = (int)v.px;
  double s = 0.0;
  for (int m = 0; m < 16; m += 2)
    for (int n = 0; n < 16; n += 2) {
      const double d = (double)F.future_ip[(fy + m) * w2 + fx + n] - (double)F.past_ip[(py + m) * w2 + px + n];
      s += d * d;
    }
  F.mse[k] = s / 64;
}

// motionFilterAndComp, sideInfoCreation.cpp:344-405: weighted vector median
// over the 3x3 neighbourhood, then the new end points
__global__ void mfc_wvmf_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, h = F.h, b8w = w / 8, b8h = h / 8, b8n = b8w * b8h;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b8n) return;
  const int i = k / b8w, j = k % b8w;
  const int srb = (h << 1) - 16, srr = (w << 1) - 16;
  const int y2 = i << 4, x2 = j << 4;
  int nbr[9], cnt = 0;
  for (int m = i - 1; m <= i + 1; m++) {
    if (m < 0 || m >= b8h) continue;
    for (int n = j - 1; n <= j + 1; n++) {
      if (n < 0 || n >= b8w) continue;
      nbr[cnt++] = m * b8w + n;
    }
  }
  const MVd *mv = F.blk_mv;
  const double *mse = F.mse;
  double minw = 0.0;
  int bestb = nbr[0];
  for (int q = 1; q < cnt; q++) {
    const int o = nbr[q];
    const double dx = mv[bestb].vx - mv[o].vx, dy = mv[bestb].vy - mv[o].vy;
    minw += mse[bestb] / mse[o] * sqrt(dx * dx + dy * dy);
  }
  for (int c = 1; c < cnt; c++) {
    const int cb = nbr[c];
    double wv = 0.0;
    for (int q = 0; q < cnt; q++) {
      if (c == q) continue;
      const int o = nbr[q];
      const double dx = mv[cb].vx - mv[o].vx, dy = mv[cb].vy - mv[o].vy;
      wv += mse[cb] / mse[o] * sqrt(dx * dx + dy * dy);
    }
    if (wv < minw) {
      minw = wv;
      bestb = cb;
    }
  }
  const double vx = mv[bestb].vx, vy = mv[bestb].vy;
  MVd o;
  o.fx = (double)end_point(x2, -vx, F.ifc, 0, srr);
  o.fy = (double)end_point(y2, -vy, F.ifc, 0, srb);
  o.px = (double)end_point(x2, vx, F.ipc, 0, srr);
  o.py = (double)end_point(y2, vy, F.ipc, 0, srb);
  o.vx = o.px - o.fx;
  o.vy = o.py - o.fy;
  F.blk_mv2[k] = o;
}

// motionFilterAndComp, sideInfoCreation.cpp:407-434 (bidirectional motion
// compensation -> side information and residue), then copyIntraBlkToSideInfo
// (intra.cpp:271-288)
__global__ void mfc_comp_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, h = F.h, w2 = w << 1;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.z;
  if (x >= w || y >= h) return;
  const int b8 = (y >> 3) * (w >> 3) + (x >> 3);
  const MVd v = F.blk_mv2[b8];
  const int m = (y & 7) << 1, n = (x & 7) << 1;
  const int fi = ((int)v.fy + m) * w2 + (int)v.fx + n, pi = ((int)v.py + m) * w2 + (int)v.px + n;
  const uint8_t fv = F.future_ip[fi], pv = F.past_ip[pi];
  uint8_t s = (uint8_t)(int)((double)fv * F.ifc + (double)pv * F.ipc);
  if (F.mode[b8] == DVC_INTRA_B) s = F.recon[y * w + x];
  F.si[y * w + x] = s;
  F.residue[y * w + x] = ((int)fv - (int)pv) >> 1;
}

// copySkipBlkToRecons, skipBlock.cpp:3-22: skip blocks take the past frame's pixels
__global__ void skip_copy_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || F.skip_mode != 1) return;
  const int w = F.w;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.z;
  if (x >= w) return;
  if (F.mode[(y >> 3) * (w >> 3) + (x >> 3)] == DVC_SKIP_B) F.recon[y * w + x] = F.past[y * w + x];
}

// ------------------------------------------- transforms and noise parameters

// forwardTransform (transform.cpp:153-190) of the residue, every 4x4 block
__global__ void residue_transform_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, b4w = w / 4, b4n = b4w * (F.h / 4);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b4n) return;
  const int i = k / b4w, j = k % b4w;
  int b[16];
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) b[4 * m + n] = F.residue[(4 * i + m) * w + 4 * j + n];
  forward44(b);
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) F.side_trans[(4 * i + m) * w + 4 * j + n] = b[4 * m + n];
}

// noiseParameter, noiseModel.cpp:14-45: band mean and variance of |T| over
// every 4x4 block.  The variance accumulates squares past 2^24, so each band's
// sums run sequentially in raster block order, one thread per band.
// The sums stay sequential in block raster order (one thread per band); the
// block stages 8 block rows of coefficients at a time in shared memory with
// coalesced loads, so those threads read shared memory instead of waiting on
// scattered global loads.
__global__ void __launch_bounds__(256) noise_band_stats_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.x];
  if (!F.active) return;
  constexpr int RB = 8;  // block rows per chunk
  __shared__ int chunk[RB * 4][352];
  const int band = threadIdx.x;
  const int index = c_zigzag[band & 15];
  // bands are coded while Qbits > 0 in zig-zag order; later ones are unused
  bool active = band < 16;
  for (int b = 0; active && b <= band; b++) active = F.qbits[c_zigzag[b]] > 0;
  const int w = F.w, b4w = w / 4, b4h = F.h / 4, b4n = b4w * b4h;
  float mean = 0.0f, var = 0.0f;
  for (int i0 = 0; i0 < b4h; i0 += RB) {
    const int rows = (b4h - i0 < RB ? b4h - i0 : RB) * 4;
    __syncthreads();
    for (int k = threadIdx.x; k < rows * w; k += blockDim.x) {
      const int r = k / w, x = k - r * w;
      chunk[r][x] = F.side_trans[(4 * i0 + r) * w + x];
    }
    __syncthreads();
    if (active)
      for (int i = 0; i < rows / 4; i++)
        for (int j = 0; j < b4w; j++) {
          const float c = fabsf((float)chunk[4 * i + (index >> 2)][4 * j + (index & 3)]);
          mean += c;
          var += c * c;
        }
  }
  if (!active) return;
  mean /= (float)b4n;
  var = var / (float)b4n - mean * mean;
  F.band_mean[band] = mean;
  F.band_var[band] = var;
}

// noiseParameter, noiseModel.cpp:47-73: alpha per WZ coefficient of coded bands
__global__ void noise_alpha_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, b4w = w / 4, b4n = b4w * (F.h / 4);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b4n) return;
  const int i = k / b4w, j = k % b4w;
  if (F.mode[(i >> 1) * (w >> 3) + (j >> 1)] != DVC_WZ_B) return;
  int band = 0, index = c_zigzag[0];
  while (band < 16 && F.qbits[index] > 0) {
    const int ci = (4 * i + (index >> 2)) * w + 4 * j + (index & 3);
    const float t = fabsf((float)F.side_trans[ci]);  // the reference stores |T| back first
    const float d = (float)(int)t - F.band_mean[band];
    const float d2 = d * d;
    F.alpha[ci] = d2 > F.band_var[band] ? sqrtf(2 / d2) : sqrtf(2 / F.band_var[band]);
    band++;
    if (band < 16) index = c_zigzag[band];
  }
}

// overCompleteTransform, transform.cpp:275-298: the 4x4 transform of the side
// information at every pixel offset (values fit 16 bits)
__global__ void over_complete_kernel(FrameDev *frames, int band) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !in_step(F, band, 0)) return;
  const int w = F.w, srw = w - 3;
  const int left = blockIdx.x * blockDim.x + threadIdx.x, top = blockIdx.z;
  if (left >= srw) return;
  int b[16];
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) b[4 * m + n] = F.si[(top + m) * w + left + n];
  forward44(b);
  int16_t *o = F.oct + ((size_t)top * srw + left) * 16;
#pragma unroll
  for (int c = 0; c < 16; c += 2) {
    const uint32_t pk = (uint32_t)(uint16_t)(int16_t)b[c] | ((uint32_t)(uint16_t)(int16_t)b[c + 1] << 16);
    reinterpret_cast<uint32_t *>(o)[c >> 1] = pk;
  }
}

// init_si_ML, motionLearning.cpp:49-68 (every block), and initSMF (:6-47) for WZ blocks
__global__ void init_ml_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active) return;
  const int w = F.w, h = F.h, b4w = w / 4, b4n = b4w * (h / 4), srw = w - 3;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b4n) return;
  const int i = k / b4w, j = k % b4w;
  const int16_t *t = F.oct + ((size_t)(4 * i) * srw + 4 * j) * 16;
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) F.side_trans[(4 * i + m) * w + 4 * j + n] = t[4 * m + n];
  const int s = F.sir_of_blk[k];
  if (s < 0) return;
  const int top = 4 * i, left = 4 * j;
  int st = top - LEARN_R, sb = top + LEARN_R, sl = left - LEARN_R, sr = left + LEARN_R;
  if (st < 0) st = 0;
  if (sb > h - 4) sb = h - 4;
  if (sl < 0) sl = 0;
  if (sr > w - 4) sr = w - 4;
  float *p = F.smf + (size_t)s * ML_N;
  int q = 0;
  for (int m = st; m <= sb; m++)
    for (int n = sl; n <= sr; n++) p[q++] = (m == top && n == left) ? 1.0f : 0.0f;
}

// SMF window of a WZ block (initSMF bounds, motionLearning.cpp:16-27)
struct Win {
  int st, sb, sl, sr;
};
__device__ __forceinline__ Win ml_window(int top, int left, int w, int h) {
  Win r{top - LEARN_R, top + LEARN_R, left - LEARN_R, left + LEARN_R};
  if (r.st < 0) r.st = 0;
  if (r.sb > h - 4) r.sb = h - 4;
  if (r.sl < 0) r.sl = 0;
  if (r.sr > w - 4) r.sr = w - 4;
  return r;
}

// ------------------------------------------------------ correlation noise

// noiseDistribution, noiseModel.cpp:77-132: per WZ block, the (mixture of)
// Laplacian pdf over every coefficient value of the band.  The exponential
// depends only on the integer distance d = |k - range - s_m|, so each block
// first tabulates expf(-alpha*d) (the same float expression) for every d it
// needs, then sums the 81-candidate mixture in the reference's order.
#define NOISE_TAB 2048

// The mixture for up to four values of one lane, k0 + c * 32 * NW (c < NC):
// one table address per candidate serves all of them through immediate
// offsets.  Each value's sum still runs over the candidates in order.
template <int NC, int NW>
__device__ __forceinline__ void noise_mix(const float *e0, const int4 *sc4, const float4 *pr4, int nm4, float *out,
                                          int k0, int rmax) {
  float s[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) s[c] = 0.0f;
  for (int m4 = 0; m4 < nm4; m4++) {
    const int4 v = sc4[m4];
    const float4 p = pr4[m4];
    const float *ax = e0 - v.x, *ay = e0 - v.y, *az = e0 - v.z, *aw = e0 - v.w;
#pragma unroll
    for (int c = 0; c < NC; c++) s[c] += p.x * ax[c * 32 * NW];
#pragma unroll
    for (int c = 0; c < NC; c++) s[c] += p.y * ay[c * 32 * NW];
#pragma unroll
    for (int c = 0; c < NC; c++) s[c] += p.z * az[c * 32 * NW];
#pragma unroll
    for (int c = 0; c < NC; c++) s[c] += p.w * aw[c * 32 * NW];
  }
#pragma unroll
  for (int c = 0; c < NC; c++)
    if (k0 + c * 32 * NW < rmax) out[k0 + c * 32 * NW] = s[c];
}

template <int NT>
__global__ void __launch_bounds__(NT) noise_dist_kernel(FrameDev *frames, XlmDev xt, int band) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !in_step(F, band, 0)) return;
  const int s_idx = blockIdx.x;
  if (s_idx >= F.nsir) return;
  const int w = F.w, h = F.h, b4w = w / 4, srw = w - 3;
  const int index = c_zigzag[band];
  const int range = F.crange[index];
  const int blk = F.sir[s_idx];
  const int top = (blk / b4w) << 2, left = (blk % b4w) << 2;
  constexpr int ML_N4 = (ML_N + 3) & ~3;
  __shared__ float etab[NOISE_TAB];
  __shared__ __align__(16) float prob[ML_N4];
  __shared__ __align__(16) int sc[ML_N4];
  __shared__ int s_n, s_dmax;
  const XlSmall xs = xl_small_global(xt);
  float *out = F.pdf + (size_t)s_idx * F.pdf_stride;
  if (index == 0) {
    const float a = F.alpha[top * w + left];
    const int s = F.oct[((size_t)top * srw + left) * 16];
    for (int k = threadIdx.x; k < range; k += NT) out[k] = xl_expf(xt, xs, -a * (float)abs(k - s));
    return;
  }
  const float a = F.alpha[(top + (index >> 2)) * w + left + (index & 3)];
  // the SMF candidates in row-major window order, gathered in parallel
  const Win wn = ml_window(top, left, w, h);
  const int cw = wn.sr - wn.sl + 1, ncand = cw * (wn.sb - wn.st + 1);
  if (threadIdx.x == 0) s_dmax = 0;
  __syncthreads();
  int mx = 0;
  for (int q = threadIdx.x; q < ncand; q += NT) {
    const int m = wn.st + q / cw, n = wn.sl + q % cw;
    const int v = F.oct[((size_t)m * srw + n) * 16 + index];
    sc[q] = v;
    prob[q] = F.smf[(size_t)s_idx * ML_N + q];
    mx = max(mx, abs(v));
  }
  // pad to a multiple of 4 with zero-probability terms: they add +0 to a
  // non-negative sum, which leaves it unchanged
  for (int q = ncand + threadIdx.x; q < ((ncand + 3) & ~3); q += NT) {
    sc[q] = 0;
    prob[q] = 0.0f;
  }
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&s_dmax, mx);
  if (threadIdx.x == 0) s_n = ncand;
  __syncthreads();
  if (threadIdx.x == 0) s_dmax += range;
  __syncthreads();
  const int nm = s_n, dmax = s_dmax;
  const int rmax = 2 * range + 1;
  if (dmax < NOISE_TAB / 2 - 32) {
    // a symmetric table, etab[ETC + d] = etab[ETC - d] = expf(-a*d), read at
    // pc - v directly: one address per term, no absolute value.  Values are
    // taken in groups of 32 (one per lane); warp w takes groups w, w + NW, ...,
    // up to four per pass.  The last group of a block reads up to 31 entries
    // past dmax for values past rmax, which are not stored: those entries
    // hold 0.
    constexpr int ETC = NOISE_TAB / 2 - 1;
    constexpr int NW = NT / 32;
    for (int d = threadIdx.x; d <= dmax + 31; d += NT) {
      if (d <= dmax) {
        const float e = xl_expf(xt, xs, -a * (float)d);
        etab[ETC + d] = e;
        etab[ETC - d] = e;
      } else {
        etab[ETC + d] = 0.0f;
      }
    }
    __syncthreads();
    const int nm4 = (nm + 3) >> 2;
    const int4 *sc4 = reinterpret_cast<const int4 *>(sc);
    const float4 *pr4 = reinterpret_cast<const float4 *>(prob);
    const int lane = threadIdx.x & 31, groups = (rmax + 31) >> 5;
    for (int g = threadIdx.x >> 5; g < groups; g += 4 * NW) {
      const int k0 = g * 32 + lane, nc = min(4, (groups - g + NW - 1) / NW);
      const float *e0 = etab + ETC + (k0 - range);
      if (nc == 4)
        noise_mix<4, NW>(e0, sc4, pr4, nm4, out, k0, rmax);
      else if (nc == 3)
        noise_mix<3, NW>(e0, sc4, pr4, nm4, out, k0, rmax);
      else if (nc == 2)
        noise_mix<2, NW>(e0, sc4, pr4, nm4, out, k0, rmax);
      else
        noise_mix<1, NW>(e0, sc4, pr4, nm4, out, k0, rmax);
    }
    return;
  }
  const int tab = dmax < NOISE_TAB ? dmax + 1 : NOISE_TAB;
  for (int d = threadIdx.x; d < tab; d += NT) etab[d] = xl_expf(xt, xs, -a * (float)d);
  __syncthreads();
  if (dmax < NOISE_TAB) {
    // every distance is in the table: candidates four at a time, in order
    const int nm4 = (nm + 3) >> 2;
    const int4 *sc4 = reinterpret_cast<const int4 *>(sc);
    const float4 *pr4 = reinterpret_cast<const float4 *>(prob);
    for (int k = threadIdx.x; k < rmax; k += NT) {
      const int pc = k - range;
      float sum = 0.0f;
      for (int m4 = 0; m4 < nm4; m4++) {
        const int4 v = sc4[m4];
        const float4 p = pr4[m4];
        sum += p.x * etab[abs(pc - v.x)];
        sum += p.y * etab[abs(pc - v.y)];
        sum += p.z * etab[abs(pc - v.z)];
        sum += p.w * etab[abs(pc - v.w)];
      }
      out[k] = sum;
    }
    return;
  }
  for (int k = threadIdx.x; k < rmax; k += NT) {
    const int pc = k - range;
    float sum = 0.0f;
    for (int m = 0; m < nm; m++) {
      const int d = abs(pc - sc[m]);
      const float e = d < NOISE_TAB ? etab[d] : xl_expf(xt, xs, -a * (float)d);
      sum += prob[m] * e;
    }
    out[k] = sum;
  }
}

// p[lo0..hi0) and p[lo1..hi1), each summed in ascending order (the float sums
// of condBitProb).  The rows are read 16 bytes at a time once aligned, and
// the two chains advance together, so two additions are in flight.
__device__ __forceinline__ void interval_sums(const float *p, int lo0, int hi0, int lo1, int hi1, float &s0,
                                              float &s1) {
  float a = 0.0f, b = 0.0f;
  int q0 = lo0, q1 = lo1;
  for (; q0 < hi0 && (reinterpret_cast<uintptr_t>(p + q0) & 15); q0++) a += __ldg(p + q0);
  for (; q1 < hi1 && (reinterpret_cast<uintptr_t>(p + q1) & 15); q1++) b += __ldg(p + q1);
  for (; q0 + 4 <= hi0 && q1 + 4 <= hi1; q0 += 4, q1 += 4) {
    const float4 u = __ldg(reinterpret_cast<const float4 *>(p + q0));
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p + q1));
    a += u.x;
    b += v.x;
    a += u.y;
    b += v.y;
    a += u.z;
    b += v.z;
    a += u.w;
    b += v.w;
  }
  for (; q0 + 4 <= hi0; q0 += 4) {
    const float4 u = __ldg(reinterpret_cast<const float4 *>(p + q0));
    a += u.x;
    a += u.y;
    a += u.z;
    a += u.w;
  }
  for (; q1 + 4 <= hi1; q1 += 4) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p + q1));
    b += v.x;
    b += v.y;
    b += v.z;
    b += v.w;
  }
  for (; q0 < hi0; q0++) a += __ldg(p + q0);
  for (; q1 < hi1; q1++) b += __ldg(p + q1);
  s0 = a;
  s1 = b;
}

// condBitProb, noiseModel.cpp:191-310: LR = p0/p1 from sequential interval
// sums of the pdf, one thread per 4x4 block.  Non-WZ blocks get the
// reference's certain-zero ratio when the frame has skip or intra blocks.
__global__ void cond_bit_kernel(FrameDev *frames, int band, int bit) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !in_step(F, band, bit)) return;
  const int w = F.w, b4w = w / 4, b4n = b4w * (F.h / 4);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= b4n) return;
  const int s_idx = F.sir_of_blk[k];
  if (s_idx < 0) {
    if (F.skip_mode == 1 || F.intra_mode == 1) F.lr[k] = 0.9999f / 0.0001f;
    return;
  }
  const int index = c_zigzag[band], step = F.step[index], range = F.crange[index];
  const int i = k / b4w, j = k % b4w;
  const int rc = F.recons_trans[(4 * i + (index >> 2)) * w + 4 * j + (index & 3)];
  const float *p = F.pdf + (size_t)s_idx * F.pdf_stride;
  const int iq = (1 << (bit - 1)) - 1;
  float p0 = 0.0f, p1 = 0.0f;
  // interval ends are clamped to the pdf row; consistent bitstreams never reach the clamp
  if (index == 0) {
    const int b0l = rc << bit, b1l = ((rc << 1) + 1) << (bit - 1);
    const int b0u = b0l + iq, b1u = b1l + iq;
    const int v0l = b0l * step, v1l = b1l * step, v0u = (b0u + 1) * step, v1u = (b1u + 1) * step;
    interval_sums(p, max(v0l, 0), min(v0u, range), max(v1l, 0), min(v1u, range), p0, p1);
  } else {
    const int ls = F.level_shift[index];
    const int b0l = (rc << bit) - ls;
    const int b1l = (((rc << 1) + 1) << (bit - 1)) - ls;
    const int b0u = b0l + iq;
    int b1u = b1l + iq;
    if (b1u > ls) b1u = ls;
    const int v0l = (b0l <= 0) ? (b0l - 1) * step + 1 : b0l * step;
    const int v1l = (b1l <= 0) ? (b1l - 1) * step + 1 : b1l * step;
    const int v0u = ((b0u < 0) ? b0u * step + 1 : (b0u + 1) * step) + range;
    const int v1u = ((b1u < 0) ? b1u * step + 1 : (b1u + 1) * step) + range;
    const int len = 2 * range + 1;
    interval_sums(p, max(v0l + range, 0), min(v0u, len), max(v1l + range, 0), min(v1u, len), p0, p1);
  }
  p0 = p0 / (p0 + p1);
  p1 = 1 - p0;
  float lr;
  if (p0 <= 0.0001)
    lr = (float)(0.0001 / 0.9999);
  else if (p0 >= 0.9999)
    lr = (float)(0.9999 / 0.0001);
  else
    lr = p0 / p1;
  F.lr[k] = lr;
}

// ------------------------------------------------------- reconstruction

// reconstruction (reconstruction.cpp:184-289) of the band's coefficient, then
// inverseTransform (transform.cpp:234-273) of the block; one thread per WZ block
__global__ void recon_kernel(FrameDev *frames, int band) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !in_step(F, band, 0)) return;
  const int s_idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (s_idx >= F.nsir) return;
  const int w = F.w, b4w = w / 4;
  const int blk = F.sir[s_idx];
  const int top = (blk / b4w) << 2, left = (blk % b4w) << 2;
  if (band >= 0) {
    const int index = c_zigzag[band], step = F.step[index];
    const int ci = (top + (index >> 2)) * w + left + (index & 3);
    int lo, hi;
    if (index == 0) {
      const int q = F.recons_trans[ci];
      lo = q * step;
      hi = (q + 1) * step;
    } else {
      const int q = F.recons_trans[ci] - F.level_shift[index];
      if (q == 0) {
        lo = -step + 1;
        hi = step;
      } else if (q > 0) {
        lo = q * step;
        hi = (q + 1) * step;
      } else {
        lo = (q - 1) * step + 1;
        hi = q * step + 1;
      }
    }
    const int sc = F.side_trans[ci];
    const double a = F.alpha[ci];
    int v;
    // The reference rounds with its C library's double exp; this kernel uses
    // the device's.  Both are within an ulp of the true value, and every other
    // operation here is IEEE and identical on both sides, so the rounded result
    // can only differ where moving an exp result by a couple of ulps moves the
    // argument of ROUND across a .5 boundary.  Such steps are counted (every
    // exp result moved by -2 and +2 ulps), so a decode can show that it met none.
    bool tie = false;
    if (a <= 0.0001) {
      v = (lo + hi) / 2;
    } else if (sc < lo || sc >= hi) {
      const double e = exp(a * (double)step);
      const int u = dround(1.0 / a + (double)step / (1.0 - e));
      for (int k = -2; k <= 2 && F.near_ties; k += 4)
        tie |= dround(1.0 / a + (double)step / (1.0 - ulp_shift(e, k))) != u;
      v = sc < lo ? lo + u : hi - u;
    } else {
      const double r = sc - lo, d = hi - sc;
      const double er = exp(-a * r), ed = exp(-a * d);
      const int u = dround(((r + 1.0 / a) * er - (d + 1.0 / a) * ed) / (2.0 - (er + ed)));
      for (int k = 0; k < 4 && F.near_ties; k++) {
        const double er2 = ulp_shift(er, (k & 1) ? 2 : -2), ed2 = ulp_shift(ed, (k & 2) ? 2 : -2);
        tie |= dround(((r + 1.0 / a) * er2 - (d + 1.0 / a) * ed2) / (2.0 - (er2 + ed2))) != u;
      }
      v = sc + u;
    }
    if (tie) atomicAdd(F.near_ties, 1ull);
    F.side_trans[ci] = v;
    F.dbf[ci] = ((v ^ sc) != 0) ? 1 : 0;
  }
  int b[16];
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) b[4 * m + n] = F.side_trans[(top + m) * w + left + n];
  inverse44(b);
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) {
      const int c = b[4 * m + n];
      F.recon[(top + m) * w + left + n] = (uint8_t)(c < 0 ? 0 : (c > 255 ? 255 : c));
    }
}

// -------------------------------------------------- side-info refinement

// sum of the four byte differences |a_i - b_i| plus c
__device__ __forceinline__ uint32_t sad4_acc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// updateSI + subPelRefine, sideInfoCreation.cpp:598-736: per WZ block, +-32
// integer search against the past and future reconstructions (cost = SAD with
// the motion-vector weight; strict-< row-major argmin), a +-1 half-pel
// refinement in the interpolated frames, and the bidirectional average.
template <int NT>
__global__ void __launch_bounds__(NT) update_si_kernel(FrameDev *frames, int band) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !in_step(F, band, 0)) return;
  const int s_idx = blockIdx.x;
  if (s_idx >= F.nsir) return;
  const int w = F.w, h = F.h, b4w = w / 4, w2 = w << 1, h2 = h << 1;
  const int blk = F.sir[s_idx];
  const int top = (blk / b4w) << 2, left = (blk % b4w) << 2;
  int st = top - SEARCH_R, sb = top + SEARCH_R, sl = left - SEARCH_R, sr = left + SEARCH_R;
  if (st < 0) st = 0;
  if (sb > h - 4) sb = h - 4;
  if (sl < 0) sl = 0;
  if (sr > w - 4) sr = w - 4;
  const int ww = sr - sl + 4, wh = sb - st + 4;  // <= 68 x 68
  // windows with a 96-byte row stride: the bytes of [sl & ~15, sl + ww)
  // (at most 6 16-byte chunks), so that the word after any 4-byte group of a
  // row is still inside the row
  constexpr int WS = 96;
  __shared__ __align__(16) uint8_t wp[68 * WS], wf[68 * WS];
  __shared__ uint32_t cur4[4];  // the block's rows, 4 pixels packed per word (first pixel lowest)
  __shared__ int cur[16];
  __shared__ double sca[2 * (NT / 32)];
  __shared__ int sia[2 * (NT / 32)];
  // window rows copied in 16-byte chunks straight to shared memory: lanes are
  // (row of a pair, reference, chunk); w and the planes' bases are multiples
  // of 16, so the chunks of [sl & ~15, sl + ww) are aligned and stay inside
  // the frame row; the window starts at byte `wo` of each shared row
  const int s16 = sl & ~15, wo = sl - s16, nch = (wo + ww + 15) >> 4;
  {
    const int lane = threadIdx.x & 31, ch = lane & 7, ref = (lane >> 3) & 1;
    if (ch < nch) {
      const uint8_t *src = (ref ? F.future : F.past) + (size_t)st * w + s16 + ch * 16;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared((ref ? wf : wp) + ch * 16);
      for (int y = 2 * (threadIdx.x >> 5) + (lane >> 4); y < wh; y += 2 * (NT / 32))
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + y * WS), "l"(src + (size_t)y * w)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  }
  if (threadIdx.x < 16) cur[threadIdx.x] = F.recon[(top + (threadIdx.x >> 2)) * w + left + (threadIdx.x & 3)];
  __syncthreads();
  if (threadIdx.x < 4) {
    const int m = threadIdx.x;
    cur4[m] = (uint32_t)cur[4 * m] | ((uint32_t)cur[4 * m + 1] << 8) | ((uint32_t)cur[4 * m + 2] << 16) |
              ((uint32_t)cur[4 * m + 3] << 24);
  }
  __syncthreads();
  // each thread walks candidate columns of one reference: the SAD of candidate row yo
  // is the sum over m of the 4-pixel SAD of window row yo + m against block
  // row m, accumulated while walking the window rows once.  The weight is at
  // least 1, so cost = sad * weight >= sad (rounding is monotone): a candidate
  // can only match or beat the item's best if sad <= floor(best), and only
  // those are weighed; the rest could neither win nor tie.
  const int cw = sr - sl + 1;
  const uint32_t c0 = cur4[0], c1 = cur4[1], c2 = cur4[2], c3 = cur4[3];
  // 4x4 SAD of the candidate at window offset (yo, xo) of window wb
  auto sad_at = [&](const uint8_t *wb, int yo, int xo) {
    const uint32_t *rw = reinterpret_cast<const uint32_t *>(wb) + ((xo + wo) >> 2) + yo * (WS / 4);
    const int sh = ((xo + wo) & 3) * 8;
    uint32_t sad = sad4_acc(__funnelshift_r(rw[0], rw[1], sh), c0, 0u);
    sad = sad4_acc(__funnelshift_r(rw[WS / 4], rw[WS / 4 + 1], sh), c1, sad);
    sad = sad4_acc(__funnelshift_r(rw[WS / 2], rw[WS / 2 + 1], sh), c2, sad);
    return (int)sad4_acc(__funnelshift_r(rw[3 * WS / 4], rw[3 * WS / 4 + 1], sh), c3, sad);
  };
  // every thread starts from the zero-motion candidate of each reference and
  // from the best candidate of the block's previous refinement (the window is
  // the same in every band); they are candidates like any other, so the lowest
  // (cost, index) is unchanged.  Their cost bounds the item's best from the
  // first row on, so a lane weighs only candidates near the optimum and a
  // warp seldom takes the weighing branch
  // (lanes 0-3 of each warp weigh the four starts; the warp shares them)
  const int y0 = top - st, x0 = left - sl;
  int *last = F.si_mv + 2 * s_idx;
  double bp, bf;
  int ip, jf;
  {
    const int lane = threadIdx.x & 31;
    // lane 0: zero motion in the past window, 1: in the future one, 2 and 3:
    // the previous band's best in each (-1 before the first band)
    const int idx = lane < 2 ? y0 * cw + x0 : (lane < 4 ? last[lane - 2] : -1);
    double c = 1e300;
    if (idx >= 0) {
      const int yo = idx / cw, xo = idx - yo * cw;
      c = (double)sad_at((lane & 1) ? wf : wp, yo, xo) * d_si_weight[(st - top + 32 + yo) * 65 + (sl + xo - left + 32)];
    }
    bp = __shfl_sync(0xffffffffu, c, 0);
    bf = __shfl_sync(0xffffffffu, c, 1);
    ip = jf = y0 * cw + x0;
    const double c2 = __shfl_sync(0xffffffffu, c, 2), c3 = __shfl_sync(0xffffffffu, c, 3);
    const int i2 = __shfl_sync(0xffffffffu, idx, 2), i3 = __shfl_sync(0xffffffffu, idx, 3);
    if (i2 >= 0) better(bp, ip, c2, i2);
    if (i3 >= 0) better(bf, jf, c3, i3);
  }
  // two adjacent candidate columns (xo, xo + 1) of one reference per thread:
  // one row read (two words) serves both, and one vote per four rows covers
  // the eight candidates they complete.  With an odd number of columns the
  // last column of each reference goes candidate by candidate below.
  const int np = cw >> 1;
  for (int pi = threadIdx.x; pi < 2 * np; pi += NT) {
    const bool fut = pi >= np;
    const int xo = 2 * (fut ? pi - np : pi);
    const uint8_t *wb = fut ? wf : wp;
    const uint32_t *row = reinterpret_cast<const uint32_t *>(wb) + ((xo + wo) >> 2);
    const int sh = ((xo + wo) & 3) * 8;
    const double *wt = d_si_weight + (st - top + 32) * 65 + (sl + xo - left + 32);
    // running SADs of candidate rows y-3 .. y (indexed by row & 3) of both columns
    int pa[4] = {0, 0, 0, 0}, pb[4] = {0, 0, 0, 0};
    double best = fut ? bf : bp;
    int bi = fut ? jf : ip, thr = (int)best;
    // window row y is row m of candidate y - m; candidate y - 3 is complete at row y
    auto add_row = [&](int y, int slot) {
      const uint32_t *rw = row + y * (WS / 4);
      const uint32_t lo = rw[0], hi = rw[1];
      const uint32_t va = __funnelshift_r(lo, hi, sh), vb = __funnelshift_rc(lo, hi, sh + 8);
      pa[slot & 3] = (int)sad4_acc(va, c0, 0u);
      pb[slot & 3] = (int)sad4_acc(vb, c0, 0u);
      pa[(slot - 1) & 3] = (int)sad4_acc(va, c1, (uint32_t)pa[(slot - 1) & 3]);
      pb[(slot - 1) & 3] = (int)sad4_acc(vb, c1, (uint32_t)pb[(slot - 1) & 3]);
      pa[(slot - 2) & 3] = (int)sad4_acc(va, c2, (uint32_t)pa[(slot - 2) & 3]);
      pb[(slot - 2) & 3] = (int)sad4_acc(vb, c2, (uint32_t)pb[(slot - 2) & 3]);
      pa[(slot - 3) & 3] = (int)sad4_acc(va, c3, (uint32_t)pa[(slot - 3) & 3]);
      pb[(slot - 3) & 3] = (int)sad4_acc(vb, c3, (uint32_t)pb[(slot - 3) & 3]);
    };
    // column xo + xc, candidate row yo
    auto weigh = [&](int yo, int xc, int sad) {
      if (sad <= thr) {
        const double cst = (double)sad * __ldg(wt + yo * 65 + xc);
        const int idx = yo * cw + xo + xc;
        if (cst < 10000000.0 && (cst < best || (cst == best && idx < bi))) {
          best = cst;
          bi = idx;
          thr = (int)best;
        }
      }
    };
    // rows 0..2 only start candidates (wh >= 4 always: the window holds the block)
    add_row(0, 0);
    add_row(1, 1);
    add_row(2, 2);
    int y = 3;
    // slots of rows y .. y+3 are 3, 0, 1, 2 (y = 3 mod 4); the candidates
    // completed by a group are weighed after it, and only when one lane of the
    // warp has one that can match its best (the lanes run the same rows, so
    // the vote is taken by the whole active warp): a warp branches once per
    // four rows, and rarely.  The (cost, index) order makes the result
    // independent of the order in which candidates are weighed.
    for (; y + 3 < wh; y += 4) {
      int sa[4], sb[4];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        add_row(y + r, 3 + r);
        sa[r] = pa[r & 3];
        sb[r] = pb[r & 3];
      }
      const int mn = min(min(min(sa[0], sa[1]), min(sa[2], sa[3])), min(min(sb[0], sb[1]), min(sb[2], sb[3])));
      if (__any_sync(__activemask(), mn <= thr)) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
          weigh(y + r - 3, 0, sa[r]);
          weigh(y + r - 3, 1, sb[r]);
        }
      }
    }
    for (; y < wh; y++) {  // the last rows; y - 3 mod 4 as above
      const uint32_t *rw = row + y * (WS / 4);
      const uint32_t lo = rw[0], hi = rw[1];
      const int q = y & 3;
      const int done = (q + 1) & 3;  // slot of candidate y - 3
      // the same updates with the slot of row y known only at run time:
      // slot q gets the new candidate, q-1 += row 1, q-2 += row 2, q-3 (= q+1) += row 3
#pragma unroll
      for (int xc = 0; xc < 2; xc++) {
        const uint32_t v = xc ? __funnelshift_rc(lo, hi, sh + 8) : __funnelshift_r(lo, hi, sh);
        int *part = xc ? pb : pa;
        const int s0 = (int)__vsadu4(v, c0), s1 = (int)__vsadu4(v, c1), s2 = (int)__vsadu4(v, c2),
                  s3 = (int)__vsadu4(v, c3);
        int n[4] = {part[0], part[1], part[2], part[3]};
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int d = (q - k) & 3;  // 0: new candidate, 1..3: candidates started 1..3 rows ago
          n[k] = d == 0 ? s0 : d == 1 ? n[k] + s1 : d == 2 ? n[k] + s2 : n[k] + s3;
        }
        part[0] = n[0];
        part[1] = n[1];
        part[2] = n[2];
        part[3] = n[3];
        weigh(y - 3, xc, done == 0 ? n[0] : done == 1 ? n[1] : done == 2 ? n[2] : n[3]);
      }
    }
    if (fut) better(bf, jf, best, bi);
    else better(bp, ip, best, bi);
  }
  if (cw & 1) {
    // the last column (cw - 1) of each reference: candidate k of the past
    // window's column for k < nrow, of the future window's above
    const int nrow = wh - 3, xo = cw - 1;
    for (int k = threadIdx.x; k < 2 * nrow; k += NT) {
      const bool fut = k >= nrow;
      const int yo = k - (fut ? nrow : 0);
      const int sad = sad_at(fut ? wf : wp, yo, xo);
      const double cst = (double)sad * __ldg(d_si_weight + (st - top + 32 + yo) * 65 + (sl + xo - left + 32));
      if (cst < 10000000.0) {
        if (fut) better(bf, jf, cst, yo * cw + xo);
        else better(bp, ip, cst, yo * cw + xo);
      }
    }
  }
  block_argmin2<NT>(bp, ip, bf, jf, sca, sia);
  if (threadIdx.x == 0) {
    last[0] = ip;
    last[1] = jf;
  }
  // subPelRefine in the half-pel planes, no vector weight
  // (sideInfoCreation.cpp:598-640): one thread per (reference, offset) SAD,
  // then the strict-< scan over the offsets in the reference's (di, dj) order
  __shared__ int ssad[18];
  __shared__ int sbest[2][2];
  const int t = threadIdx.x;
  if (t < 18) {
    const int which = t >= 9, k = t - 9 * which;
    const int id = which ? jf : ip;
    const int tt = ((st + id / cw) << 1) + k / 3 - 1, ll = ((sl + id % cw) << 1) + k % 3 - 1;
    int sad = -1;  // offset outside the half-pel plane: not a candidate
    if (tt >= 0 && tt <= h2 - 8 && ll >= 0 && ll <= w2 - 8) {
      const uint8_t *ref = which ? F.future_ip : F.past_ip;
      sad = 0;
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) sad += abs(cur[4 * m + n] - (int)ref[(tt + 2 * m) * w2 + ll + 2 * n]);
    }
    ssad[t] = sad;
  }
  __syncthreads();
  if (t < 2) {
    const int id = t ? jf : ip;
    const int by = st + id / cw, bx = sl + id % cw;
    double minc = 10000000.0;
    int nbx = bx, nby = by;
    for (int k = 0; k < 9; k++) {
      const int sad = ssad[9 * t + k];
      if (sad >= 0 && (double)sad < minc) {
        minc = (double)sad;
        nbx = (bx << 1) + k % 3 - 1;
        nby = (by << 1) + k / 3 - 1;
      }
    }
    sbest[t][0] = nbx;
    sbest[t][1] = nby;
  }
  __syncthreads();
  if (t < 16) {
    const int m = t >> 2, n = t & 3;
    const double pv = (double)F.past_ip[(sbest[0][1] + 2 * m) * w2 + sbest[0][0] + 2 * n];
    const double fv = (double)F.future_ip[(sbest[1][1] + 2 * m) * w2 + sbest[1][0] + 2 * n];
    F.si[(top + m) * w + left + n] = (uint8_t)(int)(pv * F.ipc + fv * F.ifc);
  }
}

// ------------------------------------------------------ motion learning

// bytes a[0..3], the first lowest, from the aligned words that hold them
__device__ __forceinline__ uint32_t load4_u8(const uint8_t *a) {
  const uintptr_t u = reinterpret_cast<uintptr_t>(a);
  const uint32_t *wp = reinterpret_cast<const uint32_t *>(u & ~(uintptr_t)3);
  const uint32_t sh = (uint32_t)(u & 3) * 8;
  const uint32_t lo = wp[0], hi = sh ? wp[1] : 0u;
  return __funnelshift_r(lo, hi, sh);
}

// updateSMF, motionLearning.cpp:70-127: one warp per WZ block.  The block's
// float sum of squared pixel differences only ever holds integers below 2^24
// (16 terms of at most 255^2), so every float step of it is exact and it
// equals the integer sum, taken here four pixels at a time (vabsdiffu4, dp4a).
__global__ void update_smf_kernel(FrameDev *frames, XlmDev xt, int band) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !in_step(F, band, 0)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= F.nsir) return;
  const int w = F.w, h = F.h, b4w = w / 4;
  const int blk = F.sir[warp];
  const int top = (blk / b4w) << 2, left = (blk % b4w) << 2;
  const Win wn = ml_window(top, left, w, h);
  const int cw = wn.sr - wn.sl + 1, nc = cw * (wn.sb - wn.st + 1);
  const XlSmall xs = xl_small_global(xt);
  float *p = F.smf + (size_t)warp * ML_N;
  uint32_t cb[4];
#pragma unroll
  for (int ii = 0; ii < 4; ii++) cb[ii] = load4_u8(F.recon + (size_t)(top + ii) * w + left);
  float pr[3];
  for (int r = 0; r < 3; r++) {
    const int q = lane + 32 * r;
    pr[r] = 0.0f;
    if (q < nc) {
      const int m = wn.st + q / cw, n = wn.sl + q % cw;
      uint32_t sse = 0;
#pragma unroll
      for (int ii = 0; ii < 4; ii++) {
        const uint32_t d = __vabsdiffu4(cb[ii], load4_u8(F.si + (size_t)(m + ii) * w + n));
        sse = __dp4a(d, d, sse);
      }
      pr[r] = xl_expf(xt, xs, (float)-0.01f * (float)sse);
    }
  }
  // sequential sum in candidate order
  float sum = 0.0f;
  for (int q = 0; q < nc; q++) {
    const float v = __shfl_sync(0xffffffffu, pr[q >> 5], q & 31);
    sum += v;
  }
  int center = 0;
  {
    const int cm = top - wn.st, cn = left - wn.sl;
    center = cm * cw + cn;
  }
  for (int r = 0; r < 3; r++) {
    const int q = lane + 32 * r;
    if (q < nc) p[q] = sum > 0.0 ? pr[r] / sum : (q == center ? 1.0f : pr[r]);
  }
}

// update_si_ML, motionLearning.cpp:129-160: ML side coefficients of bands >= first_band
__global__ void update_ml_kernel(FrameDev *frames, int band) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !in_step(F, band, 0)) return;
  const int first_band = band + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s_idx = t >> 4, c = t & 15;
  if (s_idx >= F.nsir || c < first_band) return;
  const int w = F.w, h = F.h, b4w = w / 4, srw = w - 3;
  const int index = c_zigzag[c];
  const int blk = F.sir[s_idx];
  const int top = (blk / b4w) << 2, left = (blk % b4w) << 2;
  const Win wn = ml_window(top, left, w, h);
  const float *p = F.smf + (size_t)s_idx * ML_N;
  float acc = 0.0f;
  int q = 0;
  for (int m = wn.st; m <= wn.sb; m++)
    for (int n = wn.sl; n <= wn.sr; n++) {
      acc += p[q] * (float)(F.oct[((size_t)m * srw + n) * 16 + index]);
      q++;
    }
  F.side_trans[(top + (index >> 2)) * w + left + (index & 3)] = (int)acc;
}

// ------------------------------------------------------------- launchers

// ------------------------------------------------------------ deblocking
//
// The reference's deblocking filter (DvcDec/src/deblock.cpp:346-386): every
// vertical 4x4 block edge in raster order, then every horizontal one, each
// filtered from a decision taken on the frame before filtering
// (deblock_44_decision, :228-344) with the strength and thresholds of the
// H.264 in-loop filter.  Decisions are independent, so one thread takes each
// edge; the filter of an edge touches up to three pixels on each side and
// only its own pixel lines, so one thread walks each pixel row (vertical
// edges) and then each pixel column (horizontal edges) in the reference's
// order.

// alpha, beta and tc0 by QP (H.264 tables 8-16 and 8-17; deblock.cpp:16-37)
__constant__ uint8_t c_db_alpha[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,   0,   0,   0,   0,   0,   0,   0,   4,   4,
                                       5,  6,  7,  8,  9,  10, 12, 13, 15,  17,  20,  22,  25,  28,  32,  36,  40,  45,
                                       50, 56, 63, 71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
__constant__ uint8_t c_db_beta[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  0,  2,  2,
                                      2, 3, 3, 3, 3, 4, 4, 4, 6,  6,  7,  7,  8,  8,  9,  9,  10, 10,
                                      11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
__constant__ uint8_t c_db_tc0[52][3] = {
    {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},
    {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},    {0, 0, 0},
    {0, 0, 0},   {0, 0, 1},   {0, 0, 1},   {0, 0, 1},    {0, 0, 1},    {0, 1, 1},    {0, 1, 1},    {1, 1, 1},
    {1, 1, 1},   {1, 1, 1},   {1, 1, 1},   {1, 1, 2},    {1, 1, 2},    {1, 1, 2},    {1, 1, 2},    {1, 2, 3},
    {1, 2, 3},   {2, 2, 3},   {2, 2, 4},   {2, 3, 4},    {2, 3, 4},    {3, 3, 5},    {3, 4, 6},    {3, 4, 6},
    {4, 5, 7},   {4, 5, 8},   {4, 6, 9},   {5, 7, 10},   {6, 8, 11},   {6, 8, 13},   {7, 10, 14},  {8, 11, 16},
    {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};
// quantiser table (reconstruction.cpp:9-43): the WZ-edge weights are Qtable[i] / sum
__constant__ int c_db_qtable[9][16] = {
    {0},
    {16, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0, 4, 4, 0, 0},
    {64, 16, 8, 8, 16, 8, 8, 4, 8, 8, 4, 4, 8, 4, 4, 0},
    {64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0},
    {128, 64, 32, 16, 64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 0}};

#define DB_NONE 0
#define DB_WZ 1    // both sides WZ blocks: strength from the reconstruction flags and variances
#define DB_ISWZ 2  // an intra or skip side: H.264-style strength 1..4
#define DB_BSMAX 0.14

// weighted count of the coefficients reconstruction changed, and the
// "flat block" indicator, of the 4x4 block at (bx, by) (deblock.cpp:286-327)
__device__ void db_block_stats(const FrameDev &F, int bx, int by, double &phi, double &chi) {
  const int *qt = c_db_qtable[F.qindex];
  int qsum = 0;
  for (int i = 0; i < 16; i++) qsum += qt[i];
  phi = 0.0;
  int sum = 0, sq = 0;
  for (int m = 0; m < 4; m++) {
    const int idx = ((by << 2) + m) * F.w + (bx << 2);
    for (int n = 0; n < 4; n++) {
      if (F.dbf[idx + n]) phi += (double)qt[(m << 2) + n] / (double)qsum;
      const int v = F.recon[idx + n];
      sum += v;
      sq += v * v;
    }
  }
  const double var = (double)sq / 16.0 - ((double)sum / 16.0) * ((double)sum / 16.0);
  chi = var < 50.0 ? 1.0 : 0.0;
}

// deblock_44_decision (deblock.cpp:228-344) for the edge between 4x4 blocks 1 and 2
__device__ int db_decide(const FrameDev &F, int x1, int y1, int x2, int y2, double &bs) {
  const int b8w = F.w >> 3;
  const int p1 = (y1 >> 1) * b8w + (x1 >> 1), p2 = (y2 >> 1) * b8w + (x2 >> 1);
  const int t1 = F.mode[p1], t2 = F.mode[p2];
  if (t1 == DVC_INTRA_B && t2 == DVC_INTRA_B) {
    bs = 3.0;
    return DB_ISWZ;
  }
  if (t1 == DVC_INTRA_B || t2 == DVC_INTRA_B) {
    bs = (t1 == DVC_WZ_B || t2 == DVC_WZ_B) ? 4.0 : 3.0;
    return DB_ISWZ;
  }
  if (t1 == DVC_SKIP_B && t2 == DVC_SKIP_B) {
    bs = 0.0;
    return DB_NONE;
  }
  if (t1 == DVC_SKIP_B || t2 == DVC_SKIP_B) {
    if (F.past_is_wz) {
      const int ps = t1 == DVC_SKIP_B ? p1 : p2;
      bs = F.past_mode[ps] == DVC_INTRA_B ? 2.0 : 1.0;
    } else {
      bs = 2.0;
    }
    return DB_ISWZ;
  }
  double phi1, chi1, phi2, chi2;
  db_block_stats(F, x1, y1, phi1, chi1);
  db_block_stats(F, x2, y2, phi2, chi2);
  const double P = 0.9;
  bs = DB_BSMAX * (P * ((phi1 + phi2) / 2.0) + (1.0 - P) * ((chi1 + chi2) / 2.0));
  return bs > 0.0 ? DB_WZ : DB_NONE;
}

// vertical edges at i*W4 + j (j < W4-1), horizontal edges at n + i*W4 + j (i < H4-1)
__global__ void deblock_decide_kernel(FrameDev *frames) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !F.deblock) return;
  const int w4 = F.w >> 2, h4 = F.h >> 2, n = w4 * h4;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2 * n) return;
  const int dir = e >= n, k = dir ? e - n : e, i = k / w4, j = k - i * w4;
  double bs = 0.0;
  int mode = DB_NONE;
  if (dir == 0 ? j < w4 - 1 : i < h4 - 1) mode = dir == 0 ? db_decide(F, j, i, j + 1, i, bs) : db_decide(F, j, i, j, i + 1, bs);
  F.db_mode[e] = (uint8_t)mode;
  F.db_bs[e] = bs;
}

__device__ __forceinline__ int db_clip3(int lo, int hi, int x) { return x < lo ? lo : x > hi ? hi : x; }

// deblock_filter (deblock.cpp:40-206) on one pixel line across one edge: p[0..7*st]
// holds L3 L2 L1 L0 | R0 R1 R2 R3
__device__ void db_line(uint8_t *p, int st, int mode, double bs, const FrameDev &F) {
  const int alpha = c_db_alpha[F.db_qp], beta = c_db_beta[F.db_qp];
  const int L3 = p[0], L2 = p[st], L1 = p[2 * st], L0 = p[3 * st];
  const int R0 = p[4 * st], R1 = p[5 * st], R2 = p[6 * st], R3 = p[7 * st];
  if (!(abs(R0 - L0) < alpha && abs(R0 - R1) < beta && abs(L0 - L1) < beta)) return;
  const double mu = DB_BSMAX * 0.5;
  const bool strong = mode == DB_ISWZ ? (int)bs == 4 : bs > mu;
  if (strong) {
    const int RL0 = L0 + R0;
    const int small_gap = abs(R0 - L0) < ((alpha >> 2) + 2);
    const int aq = (abs(R0 - R2) < beta) & small_gap, ap = (abs(L0 - L2) < beta) & small_gap;
    if (ap) {
      p[3 * st] = (uint8_t)((R1 + ((L1 + RL0) << 1) + L2 + 4) >> 3);
      p[2 * st] = (uint8_t)((L2 + L1 + RL0 + 2) >> 2);
      p[st] = (uint8_t)((((L3 + L2) << 1) + L2 + L1 + RL0 + 4) >> 3);
    } else {
      p[3 * st] = (uint8_t)(((L1 << 1) + L0 + R1 + 2) >> 2);
    }
    if (aq) {
      p[4 * st] = (uint8_t)((L1 + ((R1 + RL0) << 1) + R2 + 4) >> 3);
      p[5 * st] = (uint8_t)((R2 + R0 + L0 + R1 + 2) >> 2);
      p[6 * st] = (uint8_t)((((R3 + R2) << 1) + R2 + R1 + RL0 + 4) >> 3);
    } else {
      p[4 * st] = (uint8_t)(((R1 << 1) + R0 + L1 + 2) >> 2);
    }
    return;
  }
  if (mode == DB_WZ && !(bs > 0.0)) return;
  const int RL0 = (L0 + R0 + 1) >> 1;
  const int aq = abs(R0 - R2) < beta, ap = abs(L0 - L2) < beta;
  const int C0 = mode == DB_ISWZ ? (int)c_db_tc0[F.db_qp][(int)bs - 1] : (int)(bs * (F.db_pow - 1));
  const int tc0 = C0 + ap + aq;
  const int dif = db_clip3(-tc0, tc0, (((R0 - L0) << 2) + (L1 - R1) + 4) >> 3);
  if (ap) p[2 * st] = (uint8_t)(p[2 * st] + db_clip3(-C0, C0, (L2 + RL0 - (L1 << 1)) >> 1));
  p[3 * st] = (uint8_t)db_clip3(0, 255, L0 + dif);
  p[4 * st] = (uint8_t)db_clip3(0, 255, R0 - dif);
  if (aq) p[5 * st] = (uint8_t)(p[5 * st] + db_clip3(-C0, C0, (R2 + RL0 - (R1 << 1)) >> 1));
}

// pass 0: copy the frame; pass 1: vertical edges along each pixel row; pass 2:
// horizontal edges down each pixel column; pass 3: copy the result back
__global__ void deblock_pass_kernel(FrameDev *frames, int pass) {
  FrameDev &F = frames[blockIdx.y];
  if (!F.active || !F.deblock) return;
  const int w = F.w, h = F.h, w4 = w >> 2, h4 = h >> 2, n = w4 * h4;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (pass == 0) {
    if (t < w * h) F.db_img[t] = F.recon[t];
  } else if (pass == 1) {
    if (t >= h) return;
    const int i = t >> 2;
    for (int j = 0; j < w4 - 1; j++) {
      const int e = i * w4 + j;
      if (F.db_mode[e] != DB_NONE) db_line(F.db_img + (size_t)t * w + (j << 2), 1, F.db_mode[e], F.db_bs[e], F);
    }
  } else if (pass == 2) {
    if (t >= w) return;
    const int j = t >> 2;
    for (int i = 0; i < h4 - 1; i++) {
      const int e = n + i * w4 + j;
      if (F.db_mode[e] != DB_NONE) db_line(F.db_img + (size_t)(i << 2) * w + t, w, F.db_mode[e], F.db_bs[e], F);
    }
  } else {
    if (t < w * h) F.recon[t] = F.db_img[t];
  }
}

cudaError_t launch_deblock(FrameDev *fr, int nf, int w, int h, cudaStream_t s) {
  const int n = (w / 4) * (h / 4);
  deblock_decide_kernel<<<dim3((2 * n + 127) / 128, nf), 128, 0, s>>>(fr);
  deblock_pass_kernel<<<dim3((w * h + 127) / 128, nf), 128, 0, s>>>(fr, 0);
  deblock_pass_kernel<<<dim3((h + 127) / 128, nf), 128, 0, s>>>(fr, 1);
  deblock_pass_kernel<<<dim3((w + 127) / 128, nf), 128, 0, s>>>(fr, 2);
  deblock_pass_kernel<<<dim3((w * h + 127) / 128, nf), 128, 0, s>>>(fr, 3);
  return cudaGetLastError();
}

static inline dim3 g2(int n, int tpb, int frames) { return dim3((n + tpb - 1) / tpb, frames); }

// threads per search block of the two motion searches (the candidate columns
// or positions each thread walks follow from it); process-wide, set when a
// context is created (dvc_b200.autotune picks them; the output never depends on them)
static int g_si_threads = 64, g_fme_threads = 256;

void set_me_shapes(int si_threads, int fme_threads) {
  g_si_threads = (si_threads == 128 || si_threads == 256) ? si_threads : 64;
  g_fme_threads = (fme_threads == 128 || fme_threads == 512) ? fme_threads : 256;
}

cudaError_t launch_side_info(FrameDev *fr, int nf, int w, int h, cudaStream_t s) {
  const int b16n = (w / 16) * (h / 16), b8n = (w / 8) * (h / 8);
  if (g_fme_threads == 128)
    forward_me_kernel<128><<<dim3(b16n, nf), 128, 0, s>>>(fr);
  else if (g_fme_threads == 512)
    forward_me_kernel<512><<<dim3(b16n, nf), 512, 0, s>>>(fr);
  else
    forward_me_kernel<256><<<dim3(b16n, nf), 256, 0, s>>>(fr);
  forward_me_post_kernel<<<g2(b16n, 128, nf), 128, 0, s>>>(fr);
  bidirect_me_kernel<1024><<<nf, 1024, 0, s>>>(fr, 16);
  init_blk_mv_kernel<<<g2(b8n, 128, nf), 128, 0, s>>>(fr);
  bidirect_me_kernel<1024><<<nf, 1024, 0, s>>>(fr, 8);
  mfc_mse_kernel<<<g2(b8n, 128, nf), 128, 0, s>>>(fr);
  mfc_wvmf_kernel<<<g2(b8n, 128, nf), 128, 0, s>>>(fr);
  mfc_comp_kernel<<<dim3((w + 127) / 128, nf, h), 128, 0, s>>>(fr);
  return cudaGetLastError();
}

cudaError_t launch_frame_prep(FrameDev *fr, int nf, int w, int h, cudaStream_t s) {
  const int b4n = (w / 4) * (h / 4);
  residue_transform_kernel<<<g2(b4n, 128, nf), 128, 0, s>>>(fr);
  noise_band_stats_kernel<<<nf, 256, 0, s>>>(fr);
  noise_alpha_kernel<<<g2(b4n, 128, nf), 128, 0, s>>>(fr);
  over_complete_kernel<<<dim3((w - 3 + 127) / 128, nf, h - 3), 128, 0, s>>>(fr, -1);
  init_ml_kernel<<<g2(b4n, 128, nf), 128, 0, s>>>(fr);
  skip_copy_kernel<<<dim3((w + 127) / 128, nf, h), 128, 0, s>>>(fr);
  return cudaGetLastError();
}

// A batch whose frames have no WZ block (every block intra or skipped) has
// max_nsir == 0: the per-WZ-block kernels have nothing to do and are not launched.
// The block has about one warp per 128 values of the widest pdf of the band
// (2 * max_range + 1 values), so that each lane sums up to four of them.
cudaError_t launch_noise_dist(FrameDev *fr, int nf, int max_nsir, const XlmDev &xt, int band, int max_range,
                              cudaStream_t s) {
  if (max_nsir <= 0) return cudaSuccess;
  const dim3 grid(max_nsir, nf);
  const int warps = (2 * max_range + 1 + 127) / 128;
  if (warps <= 2)
    noise_dist_kernel<64><<<grid, 64, 0, s>>>(fr, xt, band);
  else if (warps <= 4)
    noise_dist_kernel<128><<<grid, 128, 0, s>>>(fr, xt, band);
  else
    noise_dist_kernel<256><<<grid, 256, 0, s>>>(fr, xt, band);
  return cudaGetLastError();
}

cudaError_t launch_cond_bit(FrameDev *fr, int nf, int w, int h, int band, int bit, cudaStream_t s) {
  cond_bit_kernel<<<g2((w / 4) * (h / 4), 128, nf), 128, 0, s>>>(fr, band, bit);
  return cudaGetLastError();
}

cudaError_t launch_band_end(FrameDev *fr, int nf, int w, int h, int max_nsir, int band, const XlmDev &xt,
                            cudaStream_t s) {
  if (max_nsir <= 0) return cudaSuccess;
  recon_kernel<<<g2(max_nsir, 128, nf), 128, 0, s>>>(fr, band);
  if (g_si_threads == 64)
    update_si_kernel<64><<<dim3(max_nsir, nf), 64, 0, s>>>(fr, band);
  else if (g_si_threads == 256)
    update_si_kernel<256><<<dim3(max_nsir, nf), 256, 0, s>>>(fr, band);
  else
    update_si_kernel<128><<<dim3(max_nsir, nf), 128, 0, s>>>(fr, band);
  over_complete_kernel<<<dim3((w - 3 + 127) / 128, nf, h - 3), 128, 0, s>>>(fr, band);
  update_smf_kernel<<<g2(max_nsir * 32, 128, nf), 128, 0, s>>>(fr, xt, band);
  update_ml_kernel<<<g2(max_nsir * 16, 128, nf), 128, 0, s>>>(fr, band);
  return cudaGetLastError();
}

cudaError_t launch_final_inverse(FrameDev *fr, int nf, int max_nsir, cudaStream_t s) {
  if (max_nsir <= 0) return cudaSuccess;
  recon_kernel<<<g2(max_nsir, 128, nf), 128, 0, s>>>(fr, -1);
  return cudaGetLastError();
}

}  // namespace dvc
