/* Test infrastructure: CPU restatement of the reference DvcDec WZ-frame decoder
 * hot path in ParallelMode 0.  See dvc_oracle.h.  This file is the checker for
 * the CUDA path; nothing in the product links it.
 *
 * Arithmetic notes that make the restatement bit-identical to the reference
 * (a C++ program): where the reference calls log/exp/tanh/sqrt/abs on a float
 * argument, C++ overload resolution selects the float functions, so this C
 * code calls logf/expf/tanhf/sqrtf/fabsf explicitly; on double arguments the
 * double functions; on int arguments the int abs.  Compile with
 * -ffp-contract=off on x86-64 (SSE2), as oracle/Makefile does. */
#include "dvc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ROUND(x) ((x) >= 0.0 ? (int)((x) + 0.5) : -(int)(-(x) + 0.5)) /* defines.h:23 */
#define SEARCHRANGE 32                                                  /* defines.h:8 */
#define LEARNSEARCHRANGE 4                                              /* defines.h:11 */
#define ML_RANGE 81
#define KCOST 0.05f                                                     /* defines.h:10 */
#define MU 0.01f                                                        /* defines.h:13 */
#define WZ_B 0
#define INTRA_B 1
#define SKIP_B 2
#define MAX_ITERATIONS 50                                               /* LdpcaDecoder.h:4 */
#define LOG2 (0.693147181f)                                             /* LdpcaDecoder.cpp:18 */

/* global.cpp:36-41 */
static const int zigzag[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
/* reconstruction.cpp:9-78 */
static const int qtable[9][16] = {
    {0},
    {16, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0, 4, 4, 0, 0},
    {64, 16, 8, 8, 16, 8, 8, 4, 8, 8, 4, 4, 8, 4, 4, 0},
    {64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0},
    {128, 64, 32, 16, 64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 0}};
static const int qbits_table[9][16] = {
    {0},
    {4, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0},
    {5, 4, 3, 2, 4, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0},
    {5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0, 2, 2, 0, 0},
    {6, 4, 3, 3, 4, 3, 3, 2, 3, 3, 2, 2, 3, 2, 2, 0},
    {6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0},
    {7, 6, 5, 4, 6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 0}};

/* CRC-8, polynomial x^8+x^2+x+1, init 0, no final xor (crc8.h:20-67); the
 * byte table is generated here from the polynomial. */
static uint8_t crc_table[256];
static int crc_ready;
static void crc_init(void) {
  for (int b = 0; b < 256; b++) {
    uint8_t c = (uint8_t)b;
    for (int k = 0; k < 8; k++) c = (uint8_t)((c & 0x80) ? ((c << 1) ^ 0x07) : (c << 1));
    crc_table[b] = c;
  }
  crc_ready = 1;
}

/* transform.cpp:12-61 */
static double post_scale[16], pre_scale[16];
static int transform_ready;
static void transform_init(void) {
  double a = 0.5, b = sqrt(0.4);
  double a2 = 0.25, b2 = 0.4, ab = a * b;
  const double ps[16] = {a2, ab / 2, a2, ab / 2, ab / 2, b2 / 4, ab / 2, b2 / 4,
                         a2, ab / 2, a2, ab / 2, ab / 2, b2 / 4, ab / 2, b2 / 4};
  const double pr[16] = {a2, ab, a2, ab, ab, b2, ab, b2, a2, ab, a2, ab, ab, b2, ab, b2};
  for (int i = 0; i < 16; i++) {
    post_scale[i] = ps[i];
    pre_scale[i] = pr[i] * 64.0;
  }
  transform_ready = 1;
}

int dvco_qbits_per_block(int q) {
  int s = 0;
  for (int j = 0; j < 16; j++) s += qbits_table[q][j];
  return s;
}

/* ------------------------------------------------------------------ LDPCA */

/* BitToByte (LdpcaDecoder.cpp:41-70) followed by CRC8 (crc8.h:57-67). */
uint8_t dvco_crc8_bits(const uint8_t *bits, int n) {
  if (!crc_ready) crc_init();
  uint8_t crc = 0, tmp = 0;
  int i;
  for (i = 0; i < n; i++) {
    tmp |= bits[i];
    if (((i + 1) & 7) == 0) {
      crc = crc_table[crc ^ tmp];
      tmp = 0;
    } else {
      tmp <<= 1;
    }
  }
  if (n & 7) crc = crc_table[crc ^ (uint8_t)(tmp << (7 - (n & 7)))];
  return crc;
}

/* Encoder side, DvcEnc/src/LdpcaEncoder.cpp:76-85: syndrome = H*x over the
 * full-rate rows (the last ladder code), then prefix XOR. */
void dvco_accumulated_syndrome(const dvco_ladder *L, const uint8_t *src, uint8_t *acc) {
  const int *ir = L->ir + (size_t)(L->num_codes - 1) * L->e;
  memset(acc, 0, (size_t)L->n);
  for (int k = 0; k < L->n; k++)
    for (int l = L->jc[k]; l < L->jc[k + 1]; l++) acc[ir[l]] ^= src[k];
  for (int k = 1; k < L->n; k++) acc[k] ^= acc[k - 1];
}

/* ComputeCE, LdpcaDecoder.cpp:127-143 */
float dvco_compute_ce(const float *prob, int n) {
  float bound = 0.0f;
  for (int k = 0; k < n; k++) {
    float pco = prob[k] / (1.0f + prob[k]);
    float tmp = logf(1 - pco);
    bound += (pco * (-logf(pco) + tmp) - tmp) / LOG2;
  }
  bound /= (float)n;
  return bound;
}

static inline int32_t fbits(float f) {
  int32_t i;
  memcpy(&i, &f, 4);
  return i;
}

/* beliefPropagation, LdpcaDecoder.cpp:462-580 */
int dvco_belief_propagation(const dvco_ladder *L, const float *llr_in, const uint8_t *syndrome,
                            uint8_t *decoded, int m, int code, int max_iter, int *iters) {
  const int n = L->n, ne = L->e;
  const int *ir = L->ir + (size_t)code * ne;
  const int *jc = L->jc;
  float *ext = (float *)malloc(sizeof(float) * ne);
  float *mag = (float *)malloc(sizeof(float) * ne);
  signed char *sgn = (signed char *)malloc((size_t)ne);
  signed char *buf = (signed char *)malloc((size_t)(m > ne ? m : ne));
  float *row = (float *)malloc(sizeof(float) * m);
  float *overall = (float *)malloc(sizeof(float) * n);
  int ok = 0, it;
  for (int k = 0; k < n; k++)
    for (int l = jc[k]; l < jc[k + 1]; l++) ext[l] = llr_in[k];
  for (it = 0; it < max_iter; it++) {
    for (int k = 0; k < ne; k++) {
      sgn[k] = (signed char)((fbits(ext[k]) >> 31) | 1);
      mag[k] = (float)sgn[k] * ext[k];
    }
    for (int k = 0; k < m; k++) buf[k] = (signed char)(1 - (signed char)(syndrome[k] << 1));
    for (int k = 0; k < ne; k++) buf[ir[k]] = (signed char)((buf[ir[k]] ^ sgn[k]) | 1);
    for (int k = 0; k < ne; k++) sgn[k] = (signed char)((sgn[k] ^ buf[ir[k]]) | 1);
    for (int k = 0; k < m; k++) row[k] = 0;
    for (int k = 0; k < ne; k++) mag[k] = -logf(tanhf((mag[k] + (float)0.000000001) / 2));
    for (int k = 0; k < ne; k++) row[ir[k]] += mag[k];
    for (int k = 0; k < ne; k++)
      mag[k] = -logf(tanhf((row[ir[k]] - mag[k] + (float)0.000000001) / 2)) * (float)sgn[k];
    for (int k = 0; k < n; k++) {
      float tmp = llr_in[k];
      for (int l = jc[k]; l < jc[k + 1]; l++) tmp += mag[l];
      for (int l = jc[k]; l < jc[k + 1]; l++) ext[l] = tmp - mag[l];
      overall[k] = tmp;
    }
    for (int k = 0; k < n; k++) decoded[k] = (uint8_t)((fbits(overall[k]) >> 31) & 1);
    for (int k = 0; k < m; k++) row[k] = syndrome[k];
    for (int k = 0; k < n; k++)
      for (int l = jc[k]; l < jc[k + 1]; l++) row[ir[l]] += (float)decoded[k];
    int wrong = 0;
    for (int k = 0; k < m; k++)
      if ((((int)row[k]) & 1) != 0) {
        wrong++;
        break;
      }
    if (wrong == 0) {
      ok = 1;
      it++;
      break;
    }
  }
  if (iters) *iters = it;
  free(ext);
  free(mag);
  free(sgn);
  free(buf);
  free(row);
  free(overall);
  return ok;
}

/* invH_mul, LdpcaDecoder.cpp:584-643: decoded = inv(H) * syndrome over GF(2),
 * with the syndrome packed MSB-first into bytes as BitToWord does. */
static void invh_mul(const dvco_ladder *L, uint8_t *decoded, const uint8_t *syndrome) {
  const int n = L->n, words = (n + 31) >> 5;
  uint32_t *sw = (uint32_t *)calloc((size_t)words, 4);
  uint8_t *bytes = (uint8_t *)sw;
  for (int i = 0; i < n; i++)
    if (syndrome[i]) bytes[i >> 3] |= (uint8_t)(0x80 >> (i & 7));
  for (int j = 0; j < n; j++) {
    uint32_t t = 0;
    for (int k = 0; k < words; k++) t ^= L->invh[(size_t)j * words + k] & sw[k];
    decoded[j] = (uint8_t)(__builtin_popcount(t) & 1);
  }
  free(sw);
}

/* LdpcaDecoder, LdpcaDecoder.cpp:646-771 (ParallelMode 0 branch). */
int dvco_ldpca_decode(const dvco_ladder *L, float *lr, const uint8_t *acc, uint8_t *decoded, int *rate,
                      uint8_t crc, float entropy, int *start_code) {
  return dvco_ldpca_decode_iter(L, lr, acc, decoded, rate, crc, entropy, start_code, MAX_ITERATIONS);
}

/* The same with another cap on BP iterations per ladder code (the reference's
 * is the compile-time MAX_ITERATIONS, 50). */
int dvco_ldpca_decode_iter(const dvco_ladder *L, float *lr, const uint8_t *acc, uint8_t *decoded, int *rate,
                           uint8_t crc, float entropy, int *start_code, int max_iter) {
  const int n = L->n;
  int start = 0;
  while (start < L->num_codes - 1 &&
         (float)((L->n / L->period) * L->bpp[start]) / (float)n < entropy)
    start++;
  if (start_code) *start_code = start;
  for (int k = 0; k < n; k++) lr[k] = logf(lr[k]);
  uint8_t *synd = (uint8_t *)malloc((size_t)n);
  int code;
  for (code = start; code < L->num_codes; code++) {
    const int m = (n / L->period) * L->bpp[code];
    const int nb = L->bpp[code];
    const int *idx = L->idx + (size_t)code * L->period;
    *rate = m + 8;
    int cur = idx[0], prev;
    synd[0] = acc[cur];
    for (int k = 1; k < m; k++) {
      prev = cur;
      cur = idx[k % nb] + (k / nb) * L->period;
      synd[k] = acc[cur] ^ acc[prev];
    }
    if (m == n) {
      invh_mul(L, decoded, synd);
      break;
    }
    if (dvco_belief_propagation(L, lr, synd, decoded, m, code, max_iter, NULL)) {
      if (dvco_crc8_bits(decoded, n) == crc) break;
    }
  }
  free(synd);
  return code;
}

/* ------------------------------------------------------------- transforms */

/* forward44, transform.cpp:63-104 */
static void forward44(int *blk) {
  int t[16];
  for (int c = 0; c < 4; c++) {
    t[c] = blk[c] + blk[4 + c] + blk[8 + c] + blk[12 + c];
    t[4 + c] = (blk[c] << 1) + blk[4 + c] - blk[8 + c] - (blk[12 + c] << 1);
    t[8 + c] = blk[c] - blk[4 + c] - blk[8 + c] + blk[12 + c];
    t[12 + c] = blk[c] - (blk[4 + c] << 1) + (blk[8 + c] << 1) - blk[12 + c];
  }
  for (int r = 0; r < 4; r++) {
    int *o = blk + 4 * r;
    const int *s = t + 4 * r;
    o[0] = s[0] + s[1] + s[2] + s[3];
    o[1] = (s[0] << 1) + s[1] - s[2] - (s[3] << 1);
    o[2] = s[0] - s[1] - s[2] + s[3];
    o[3] = s[0] - (s[1] << 1) + (s[2] << 1) - s[3];
  }
  for (int i = 0; i < 16; i++) blk[i] = ROUND(((double)blk[i]) * post_scale[i]);
}

/* inverse44, transform.cpp:106-151 */
static void inverse44(int *blk) {
  int t[16];
  for (int i = 0; i < 16; i++) blk[i] = ROUND(((double)blk[i]) * pre_scale[i]);
  for (int c = 0; c < 4; c++) {
    t[c] = blk[c] + blk[4 + c] + blk[8 + c] + (blk[12 + c] >> 1);
    t[4 + c] = blk[c] + (blk[4 + c] >> 1) - blk[8 + c] - blk[12 + c];
    t[8 + c] = blk[c] - (blk[4 + c] >> 1) - blk[8 + c] + blk[12 + c];
    t[12 + c] = blk[c] - blk[4 + c] + blk[8 + c] - (blk[12 + c] >> 1);
  }
  for (int r = 0; r < 4; r++) {
    int *o = blk + 4 * r;
    const int *s = t + 4 * r;
    o[0] = s[0] + s[1] + s[2] + (s[3] >> 1);
    o[1] = s[0] + (s[1] >> 1) - s[2] - s[3];
    o[2] = s[0] - (s[1] >> 1) - s[2] + s[3];
    o[3] = s[0] - s[1] + s[2] - (s[3] >> 1);
  }
  for (int i = 0; i < 16; i++) blk[i] >>= 6;
}

/* forwardTransform, transform.cpp:153-190 (every 4x4 block) */
void dvco_forward_transform(int w, int h, const int *in, int *out) {
  if (!transform_ready) transform_init();
  for (int i = 0; i < h / 4; i++)
    for (int j = 0; j < w / 4; j++) {
      int b[16];
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) b[4 * m + n] = in[(4 * i + m) * w + 4 * j + n];
      forward44(b);
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) out[(4 * i + m) * w + 4 * j + n] = b[4 * m + n];
    }
}

/* overCompleteTransform, transform.cpp:275-298: trans16[((top*(w-3))+left)*16 + c] */
void dvco_over_complete_transform(int w, int h, const uint8_t *pix, int *trans) {
  if (!transform_ready) transform_init();
  int idx = 0;
  for (int top = 0; top <= h - 4; top++)
    for (int left = 0; left <= w - 4; left++) {
      int *b = trans + (size_t)idx * 16;
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) b[4 * m + n] = pix[(top + m) * w + left + n];
      forward44(b);
      idx++;
    }
}

/* ---------------------------------------------------------------- filters */

/* lowPassFilter, filter.cpp:214-233 */
void dvco_low_pass(const uint8_t *in, int w, int h, uint8_t *out) {
  for (int i = 0; i < h; i++)
    for (int j = 0; j < w; j++) {
      double sum = 0;
      for (int m = i - 1; m <= i + 1; m++) {
        if (m < 0 || m >= h) continue;
        for (int n = j - 1; n <= j + 1; n++) {
          if (n < 0 || n >= w) continue;
          sum += (double)in[m * w + n];
        }
      }
      out[i * w + j] = (uint8_t)(sum / 9);
    }
}

/* FilterCoef, filter.cpp:30-52: separable 6-tap (1,-5,20,20,-5,1) half-pel taps. */
static double fir_coef[3][36];
static int fir_ready;
static void fir_init(void) {
  static const double tap[6] = {1.0, -5.0, 20.0, 20.0, -5.0, 1.0};
  memset(fir_coef, 0, sizeof fir_coef);
  for (int j = 0; j < 6; j++) fir_coef[0][2 * 6 + j] = tap[j] / 32.0; /* horizontal half */
  for (int i = 0; i < 6; i++) fir_coef[1][i * 6 + 2] = tap[i] / 32.0; /* vertical half */
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) fir_coef[2][i * 6 + j] = (tap[i] * tap[j]) / 1024.0; /* centre */
  fir_ready = 1;
}

static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }

/* FIR_filter, filter.cpp:55-117, restricted to the output window it keeps
 * (rows/cols 0..2h-1, 0..2w-1 of the half-pel plane). */
void dvco_fir_half_pel(const uint8_t *in, int w, int h, uint8_t *out) {
  if (!fir_ready) fir_init();
  const int w2 = w << 1, h2 = h << 1;
  for (int i = 0; i < h2; i++) {
    const int ysub2 = ((i + 8) & 1) << 1;
    for (int j = 0; j < w2; j++) {
      const int sub = ((j + 8) & 1) + ysub2;
      if (sub) {
        double sum = 0.0;
        for (int ii = 0; ii < 6; ii++) {
          int py = imax(0, imin(h - 1, i / 2 - 2 + ii));
          for (int jj = 0; jj < 6; jj++) {
            int px = imax(0, imin(w - 1, j / 2 - 2 + jj));
            sum += (fir_coef[sub - 1][ii * 6 + jj] * in[py * w + px]);
          }
        }
        out[i * w2 + j] = (uint8_t)imax(0, imin(255, (int)(sum + 0.5)));
      } else {
        out[i * w2 + j] = in[imax(0, imin(h - 1, i / 2)) * w + imax(0, imin(w - 1, j / 2))];
      }
    }
  }
}

/* ----------------------------------------------------------- side info */

typedef struct { double x, y; } pt;
typedef struct { pt past, future, vec; } mvec;

/* costFunc, sideInfoCreation.cpp:10-12 */
static inline double cost_func(double mad, double vx, double vy) {
  return mad * (1.0 + KCOST * sqrt(vx * vx + vy * vy));
}

/* computeEndPoint, sideInfoCreation.cpp:14-22 */
static inline int end_point(double st, double v, double scale, int lo, int hi) {
  int e = (int)((st + v * scale) + 0.5);
  return e < lo ? lo : (e > hi ? hi : e);
}

/* bidirectME, sideInfoCreation.cpp:235-310 (mv updated in place, raster order) */
static void bidirect_me(int w, int h, const uint8_t *fut2, const uint8_t *pas2, double ifc, double ipc,
                        mvec *mv, int bl) {
  const int bh = h / bl, bw = w / bl, w2 = w << 1, h2 = h << 1, bl2 = bl << 1;
  const int srb = h2 - bl2, srr = w2 - bl2;
  int bi = 0;
  for (int i = 0; i < bh; i++) {
    const int y2 = i * bl2;
    for (int j = 0; j < bw; j++) {
      const int x2 = j * bl2;
      int st = (i - 1 >= 0) ? (int)mv[bi - bw].future.y + bl2 : (int)mv[bi].future.y;
      int sb = (i + 1 < bh) ? (int)mv[bi + bw].future.y - bl2 : (int)mv[bi].future.y;
      int sl = (j - 1 >= 0) ? (int)mv[bi - 1].future.x + bl2 : (int)mv[bi].future.x;
      int sr = (j + 1 < bw) ? (int)mv[bi + 1].future.x - bl2 : (int)mv[bi].future.x;
      double minc = 10000000.0;
      mvec best = mv[bi];
      const double scale = ipc / ifc;
      for (int fy = st; fy <= sb; fy++) {
        const int py = end_point(y2, (double)(y2 - fy), scale, 0, srb);
        for (int fx = sl; fx <= sr; fx++) {
          const int px = end_point(x2, (double)(x2 - fx), scale, 0, srr);
          int mad = 0;
          for (int m = 0; m < bl2; m += 2) {
            const int pi = (py + m) * w2 + px, fi = (fy + m) * w2 + fx;
            for (int n = 0; n < bl2; n += 2) mad += abs((int)fut2[fi + n] - (int)pas2[pi + n]);
          }
          const double vx = (double)(px - fx), vy = (double)(py - fy);
          const double c = cost_func((double)mad, vx, vy);
          if (c < minc) {
            minc = c;
            best.future.x = (double)fx;
            best.future.y = (double)fy;
            best.past.x = (double)px;
            best.past.y = (double)py;
            best.vec.x = vx;
            best.vec.y = vy;
          }
        }
      }
      mv[bi++] = best;
    }
  }
}

/* createSideInfo with forwardME and motionFilterAndComp,
 * sideInfoCreation.cpp:24-145, 312-551. */
void dvco_create_side_info(int w, int h, const uint8_t *past, const uint8_t *future, int past_idx,
                           int future_idx, int cur_idx, uint8_t *si, int *residue) {
  const int fs = w * h;
  const int b16w = w / 16, b16h = h / 16, b16n = b16w * b16h;
  const int b8w = w / 8, b8h = h / 8, b8n = b8w * b8h;
  uint8_t *lp_p = (uint8_t *)malloc((size_t)fs), *lp_f = (uint8_t *)malloc((size_t)fs);
  uint8_t *ip_p = (uint8_t *)malloc((size_t)fs * 4), *ip_f = (uint8_t *)malloc((size_t)fs * 4);
  dvco_low_pass(past, w, h, lp_p);
  dvco_fir_half_pel(past, w, h, ip_p);
  dvco_low_pass(future, w, h, lp_f);
  dvco_fir_half_pel(future, w, h, ip_f);
  const double ifc = (double)(future_idx - cur_idx) / (double)(future_idx - past_idx);
  const double ipc = (double)(cur_idx - past_idx) / (double)(future_idx - past_idx);

  /* forwardME (sideInfoCreation.cpp:61-145) on the low-pass frames */
  mvec *mbmv = (mvec *)calloc((size_t)b16n, sizeof(mvec));
  mvec *fmv = (mvec *)calloc((size_t)b16n, sizeof(mvec));
  pt *holes = (pt *)calloc((size_t)b16n, sizeof(pt));
  {
    const int srb = h - 16, srr = w - 16;
    for (int i = 0; i < b16n; i++) {
      const int top = (i / b16w) << 4, left = (i % b16w) << 4;
      int s_top = top - SEARCHRANGE, s_bot = top + SEARCHRANGE, s_l = left - SEARCHRANGE, s_r = left + SEARCHRANGE;
      if (s_top < 0) s_top = 0;
      if (s_bot > srb) s_bot = srb;
      if (s_l < 0) s_l = 0;
      if (s_r > srr) s_r = srr;
      double minc = 10000000.0;
      mvec best;
      memset(&best, 0, sizeof best);
      for (int py = s_top; py <= s_bot; py++)
        for (int px = s_l; px <= s_r; px++) {
          int sad = 0;
          for (int m = 0; m < 16; m++)
            for (int n = 0; n < 16; n++)
              sad += abs((int)lp_f[(top + m) * w + left + n] - (int)lp_p[(py + m) * w + px + n]);
          const double vx = (double)(px - left), vy = (double)(py - top);
          const double c = cost_func((double)sad, vx, vy);
          if (c < minc) {
            minc = c;
            best.past.x = (double)px;
            best.past.y = (double)py;
            best.vec.x = vx;
            best.vec.y = vy;
          }
        }
      fmv[i] = best;
      holes[i].x = (double)left * ipc + (double)best.past.x * ifc;
      holes[i].y = (double)top * ipc + (double)best.past.y * ifc;
    }
    const double maxd = w * w + h * h;
    for (int i = 0; i < b16n; i++) {
      const int top = (i / b16w) << 4, left = (i % b16w) << 4;
      double mind = maxd;
      mvec best;
      memset(&best, 0, sizeof best);
      for (int j = 0; j < b16n; j++) {
        double d = (left - holes[j].x) * (left - holes[j].x) + (top - holes[j].y) * (top - holes[j].y);
        if (d < mind) {
          mind = d;
          best = fmv[j];
        }
      }
      mvec *o = &mbmv[i];
      o->future.x = (double)end_point(left, -best.vec.x, ifc, 0, srr);
      o->future.y = (double)end_point(top, -best.vec.y, ifc, 0, srb);
      o->past.x = (double)end_point(left, best.vec.x, ipc, 0, srr);
      o->past.y = (double)end_point(top, best.vec.y, ipc, 0, srb);
      o->vec.x = o->past.x - o->future.x;
      o->vec.y = o->past.y - o->future.y;
    }
  }
  /* half-pel scaling then 16x16 bidirectional ME (sideInfoCreation.cpp:511-522) */
  for (int i = 0; i < b16n; i++) {
    mvec v = mbmv[i];
    v.future.x *= 2;
    v.future.y *= 2;
    v.past.x *= 2;
    v.past.y *= 2;
    v.vec.x = v.past.x - v.future.x;
    v.vec.y = v.past.y - v.future.y;
    mbmv[i] = v;
  }
  bidirect_me(w, h, ip_f, ip_p, ifc, ipc, mbmv, 16);
  /* 8x8 initialisation from the macroblock vectors (sideInfoCreation.cpp:524-545) */
  mvec *bmv = (mvec *)calloc((size_t)b8n, sizeof(mvec));
  {
    const int srb = (h - 8) << 1, srr = (w - 8) << 1;
    int bi = 0;
    for (int i = 0; i < b8h; i++) {
      const int mbrow = (i >> 1) * b16w, y2 = i << 4;
      for (int j = 0; j < b8w; j++) {
        const int x2 = j << 4;
        pt v = mbmv[mbrow + (j >> 1)].vec;
        mvec o;
        o.future.x = (double)end_point(x2, -v.x, ifc, 0, srr);
        o.future.y = (double)end_point(y2, -v.y, ifc, 0, srb);
        o.past.x = (double)end_point(x2, v.x, ipc, 0, srr);
        o.past.y = (double)end_point(y2, v.y, ipc, 0, srb);
        o.vec.x = o.past.x - o.future.x;
        o.vec.y = o.past.y - o.future.y;
        bmv[bi++] = o;
      }
    }
  }
  bidirect_me(w, h, ip_f, ip_p, ifc, ipc, bmv, 8);

  /* motionFilterAndComp, sideInfoCreation.cpp:312-436 */
  {
    const int w2 = w << 1, h2 = h << 1;
    const int srb = h2 - 16, srr = w2 - 16;
    double *mse = (double *)malloc(sizeof(double) * b8n);
    for (int i = 0; i < b8n; i++) {
      const int fy = (int)bmv[i].future.y, fx = (int)bmv[i].future.x;
      const int py = (int)bmv[i].past.y, px = (int)bmv[i].past.x;
      double s = 0.0;
      for (int m = 0; m < 16; m += 2)
        for (int n = 0; n < 16; n += 2) {
          double d = (double)ip_f[(fy + m) * w2 + fx + n] - (double)ip_p[(py + m) * w2 + px + n];
          s += d * d;
        }
      mse[i] = s / 64;
    }
    mvec *nb = (mvec *)malloc(sizeof(mvec) * b8n);
    int bi = 0;
    for (int i = 0; i < b8h; i++) {
      const int y2 = i << 4;
      for (int j = 0; j < b8w; j++) {
        const int x2 = j << 4;
        int nbr[9], cnt = 0;
        for (int m = i - 1; m <= i + 1; m++) {
          if (m < 0 || m >= b8h) continue;
          for (int n = j - 1; n <= j + 1; n++) {
            if (n < 0 || n >= b8w) continue;
            nbr[cnt++] = m * b8w + n;
          }
        }
        double minw = 0.0;
        int bestb = nbr[0];
        for (int k = 1; k < cnt; k++) {
          const int o = nbr[k];
          double dx = bmv[bestb].vec.x - bmv[o].vec.x, dy = bmv[bestb].vec.y - bmv[o].vec.y;
          minw += mse[bestb] / mse[o] * sqrt(dx * dx + dy * dy);
        }
        for (int c = 1; c < cnt; c++) {
          const int cb = nbr[c];
          double wv = 0.0;
          for (int k = 0; k < cnt; k++) {
            if (c == k) continue;
            const int o = nbr[k];
            double dx = bmv[cb].vec.x - bmv[o].vec.x, dy = bmv[cb].vec.y - bmv[o].vec.y;
            wv += mse[cb] / mse[o] * sqrt(dx * dx + dy * dy);
          }
          if (wv < minw) {
            minw = wv;
            bestb = cb;
          }
        }
        pt v = bmv[bestb].vec;
        mvec o;
        o.future.x = (double)end_point(x2, -v.x, ifc, 0, srr);
        o.future.y = (double)end_point(y2, -v.y, ifc, 0, srb);
        o.past.x = (double)end_point(x2, v.x, ipc, 0, srr);
        o.past.y = (double)end_point(y2, v.y, ipc, 0, srb);
        o.vec.x = o.past.x - o.future.x;
        o.vec.y = o.past.y - o.future.y;
        nb[bi++] = o;
      }
    }
    memcpy(bmv, nb, sizeof(mvec) * b8n);
    free(nb);
    free(mse);
    bi = 0;
    for (int i = 0; i < b8h; i++) {
      const int y = i << 3;
      for (int j = 0; j < b8w; j++) {
        const int x = j << 3;
        const mvec v = bmv[bi++];
        const int fy = (int)v.future.y, fx = (int)v.future.x, py = (int)v.past.y, px = (int)v.past.x;
        for (int m = 0; m < 16; m += 2) {
          const int pi = (py + m) * w2 + px, fi = (fy + m) * w2 + fx, ci = (y + (m >> 1)) * w + x;
          for (int n = 0; n < 16; n += 2) {
            si[ci + (n >> 1)] = (uint8_t)(int)((double)ip_f[fi + n] * ifc + (double)ip_p[pi + n] * ipc);
            residue[ci + (n >> 1)] = ((int)ip_f[fi + n] - (int)ip_p[pi + n]) >> 1;
          }
        }
      }
    }
  }
  free(bmv);
  free(mbmv);
  free(fmv);
  free(holes);
  free(lp_p);
  free(lp_f);
  free(ip_p);
  free(ip_f);
}

/* --------------------------------------------------------- frame decode */

typedef struct {
  int top, left, s_top, s_bot, s_left, s_right, blk;
} sinfo;

typedef struct {
  float prob[ML_RANGE];
  int s_top, s_left, s_right, s_bot, blk, len;
} smf_t;

/* updateSI + subPelRefine, sideInfoCreation.cpp:598-736 */
static void sub_pel_refine(const double *block, const uint8_t *ref, int *bx, int *by, int w2, int h2) {
  const int srb = h2 - 8, srr = w2 - 8;
  const int ix = (*bx) << 1, iy = (*by) << 1;
  double minc = 10000000.0;
  for (int i = -1; i <= 1; i++) {
    const int top = iy + i;
    if (top < 0 || top > srb) continue;
    for (int j = -1; j <= 1; j++) {
      const int left = ix + j;
      if (left < 0 || left > srr) continue;
      double c = 0.0;
      int k = 0, row = top * w2 + left;
      for (int m = 0; m < 8; m += 2) {
        c += fabs(block[k++] - (double)ref[row]);
        c += fabs(block[k++] - (double)ref[row + 2]);
        c += fabs(block[k++] - (double)ref[row + 4]);
        c += fabs(block[k++] - (double)ref[row + 6]);
        row += w2 << 1;
      }
      if (c < minc) {
        minc = c;
        *bx = left;
        *by = top;
      }
    }
  }
}

static void update_si(int w, int h, uint8_t *si, const uint8_t *rec, const uint8_t *past, const uint8_t *fut,
                      const uint8_t *past2, const uint8_t *fut2, double ifc, double ipc, const sinfo *sir, int nsir) {
  const int w2 = w << 1, h2 = h << 1;
  for (int i = 0; i < nsir; i++) {
    const sinfo s = sir[i];
    double block[16];
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++) block[4 * m + n] = (double)rec[(s.top + m) * w + s.left + n];
    int pbx = 0, pby = 0, fbx = 0, fby = 0;
    double pmin = 10000000.0, fmin = 10000000.0;
    for (int y = s.s_top; y <= s.s_bot; y++)
      for (int x = s.s_left; x <= s.s_right; x++) {
        double pc = 0.0, fc = 0.0;
        int k = 0;
        for (int m = 0; m < 4; m++) {
          const int r = (y + m) * w + x;
          for (int n = 0; n < 4; n++) {
            pc += fabs(block[k] - (double)past[r + n]);
            fc += fabs(block[k] - (double)fut[r + n]);
            k++;
          }
        }
        const double vx = (double)((x - s.left) << 1), vy = (double)((y - s.top) << 1);
        pc = cost_func(pc, vx, vy);
        fc = cost_func(fc, vx, vy);
        if (pc < pmin) {
          pbx = x;
          pby = y;
          pmin = pc;
        }
        if (fc < fmin) {
          fbx = x;
          fby = y;
          fmin = fc;
        }
      }
    sub_pel_refine(block, past2, &pbx, &pby, w2, h2);
    sub_pel_refine(block, fut2, &fbx, &fby, w2, h2);
    for (int m = 0; m < 8; m += 2) {
      const int r = (s.top + (m >> 1)) * w + s.left, pr = (pby + m) * w2 + pbx, fr = (fby + m) * w2 + fbx;
      for (int n = 0; n < 8; n += 2)
        si[r + (n >> 1)] = (uint8_t)(int)((double)past2[pr + n] * ipc + (double)fut2[fr + n] * ifc);
    }
  }
}

/* noiseParameter, noiseModel.cpp:9-75 (writes |T| back into trans like the reference) */
static void noise_parameter(int w, int h, int q, int *trans, float *alpha, const uint8_t *mode) {
  float mean[16] = {0}, var[16] = {0};
  const int b4w = w / 4, b4h = h / 4, b8w = w / 8, b4n = b4w * b4h;
  for (int i = 0; i < b4h; i++)
    for (int j = 0; j < b4w; j++) {
      int band = 0, index = zigzag[0];
      while (qbits_table[q][index] > 0) {
        const int ci = (4 * i + (index >> 2)) * w + 4 * j + (index & 3);
        float c = fabsf((float)trans[ci]);
        mean[band] += c;
        var[band] += c * c;
        trans[ci] = (int)c;
        band++;
        index = zigzag[band];
      }
    }
  {
    int band = 0, index = zigzag[0];
    while (qbits_table[q][index] > 0) {
      mean[band] /= (float)b4n;
      var[band] = var[band] / (float)b4n - mean[band] * mean[band];
      band++;
      index = zigzag[band];
    }
  }
  for (int i = 0; i < b4h; i++)
    for (int j = 0; j < b4w; j++) {
      if (mode[(i >> 1) * b8w + (j >> 1)] != WZ_B) continue;
      int band = 0, index = zigzag[0];
      while (qbits_table[q][index] > 0) {
        const int ci = (4 * i + (index >> 2)) * w + 4 * j + (index & 3);
        float d = (float)trans[ci] - mean[band];
        float d2 = d * d;
        if (d2 > var[band])
          alpha[ci] = sqrtf(2 / d2);
        else
          alpha[ci] = sqrtf(2 / var[band]);
        band++;
        index = zigzag[band];
      }
    }
}

/* noiseDistribution, noiseModel.cpp:77-132 */
static float *noise_distribution(int w, int range, int index, const float *alpha, const smf_t *smf,
                                 const int *trans, const sinfo *sir, int nsir) {
  const int srw = w - 3;
  float *dist;
  if (index == 0) {
    dist = (float *)malloc(sizeof(float) * (size_t)nsir * range);
    for (int i = 0; i < nsir; i++) {
      float *p = dist + (size_t)i * range;
      const float a = alpha[sir[i].top * w + sir[i].left];
      const int s = trans[((size_t)sir[i].top * srw + sir[i].left) * 16 + 0];
      for (int k = 0; k < range; k++) p[k] = expf(-a * (float)abs(k - s));
    }
  } else {
    const int rmax = (range << 1) + 1, row = index >> 2, col = index & 3;
    dist = (float *)malloc(sizeof(float) * (size_t)nsir * rmax);
    for (int i = 0; i < nsir; i++) {
      const float a = alpha[(sir[i].top + row) * w + sir[i].left + col];
      const smf_t *b = &smf[i];
      int sc[ML_RANGE], n = 0;
      for (int m = b->s_top; m <= b->s_bot; m++)
        for (int x = b->s_left; x <= b->s_right; x++) sc[n++] = trans[((size_t)m * srw + x) * 16 + index];
      float *p = dist + (size_t)i * rmax;
      for (int k = 0; k < rmax; k++) {
        float sum = 0.0f;
        const int pc = k - range;
        for (int m = 0; m < n; m++) sum += b->prob[m] * expf(-a * (float)abs(pc - sc[m]));
        p[k] = sum;
      }
    }
  }
  return dist;
}

/* condBitProb, noiseModel.cpp:191-310 */
static void cond_bit_prob(int w, float *lr, int index, int bit, int step, const int *rt, int range,
                          const float *dist, const sinfo *sir, int nsir, int level_shift) {
  const int iq = (1 << (bit - 1)) - 1;
  if (index == 0) {
    for (int i = 0; i < nsir; i++) {
      const int rc = rt[sir[i].top * w + sir[i].left];
      const float *p = dist + (size_t)i * range;
      const int b0l = rc << bit, b1l = ((rc << 1) + 1) << (bit - 1);
      const int b0u = b0l + iq, b1u = b1l + iq;
      const int v0l = b0l * step, v1l = b1l * step, v0u = (b0u + 1) * step, v1u = (b1u + 1) * step;
      float p0 = 0.0f, p1 = 0.0f;
      for (int k = v0l; k < v0u; k++) p0 += p[k];
      for (int k = v1l; k < v1u; k++) p1 += p[k];
      p0 = p0 / (p0 + p1);
      p1 = 1 - p0;
      if (p0 <= 0.0001)
        lr[sir[i].blk] = (float)(0.0001 / 0.9999);
      else if (p0 >= 0.9999)
        lr[sir[i].blk] = (float)(0.9999 / 0.0001);
      else
        lr[sir[i].blk] = p0 / p1;
    }
  } else {
    const int row = index >> 2, col = index & 3, rmax = (range << 1) + 1;
    for (int i = 0; i < nsir; i++) {
      const int rc = rt[(sir[i].top + row) * w + sir[i].left + col];
      const float *p = dist + (size_t)i * rmax;
      const int b0l = (rc << bit) - level_shift;
      const int b1l = (((rc << 1) + 1) << (bit - 1)) - level_shift;
      const int b0u = b0l + iq;
      int b1u = b1l + iq;
      if (b1u > level_shift) b1u = level_shift;
      int v0l, v1l, v0u, v1u;
      v0l = (b0l <= 0) ? (b0l - 1) * step + 1 : b0l * step;
      v1l = (b1l <= 0) ? (b1l - 1) * step + 1 : b1l * step;
      v0u = (b0u < 0) ? b0u * step + 1 : (b0u + 1) * step;
      v1u = (b1u < 0) ? b1u * step + 1 : (b1u + 1) * step;
      float p0 = 0.0f, p1 = 0.0f;
      v0u += range;
      for (int k = v0l + range; k < v0u; k++) p0 += p[k];
      v1u += range;
      for (int k = v1l + range; k < v1u; k++) p1 += p[k];
      p0 = p0 / (p0 + p1);
      p1 = 1 - p0;
      if (p0 <= 0.0001)
        lr[sir[i].blk] = (float)(0.0001 / 0.9999);
      else if (p0 >= 0.9999)
        lr[sir[i].blk] = (float)(0.9999 / 0.0001);
      else
        lr[sir[i].blk] = p0 / p1;
    }
  }
}

/* updateSMF, motionLearning.cpp:70-127 */
static void update_smf(int w, smf_t *smf, const uint8_t *rec, const uint8_t *si, const sinfo *sir, int nsir) {
  for (int i = 0; i < nsir; i++) {
    float block[16];
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++) block[4 * m + n] = (float)rec[(sir[i].top + m) * w + sir[i].left + n];
    smf_t b = smf[i];
    int k = 0;
    float sum = 0.0f;
    for (int m = b.s_top; m <= b.s_bot; m++)
      for (int x = b.s_left; x <= b.s_right; x++) {
        float sse = 0.0f;
        int bi = 0;
        for (int ii = 0; ii < 4; ii++)
          for (int jj = 0; jj < 4; jj++) {
            float d = block[bi++] - (float)si[(m + ii) * w + x + jj];
            sse += d * d;
          }
        b.prob[k] = expf((float)-MU * sse);
        sum += b.prob[k];
        k++;
      }
    if (sum > 0.0) {
      for (int m = 0; m < k; m++) b.prob[m] = b.prob[m] / sum;
    } else {
      b.prob[b.blk] = 1.0f;
    }
    smf[i] = b;
  }
}

/* update_si_ML, motionLearning.cpp:129-160 */
static void update_si_ml(int w, int *side_trans, const int *trans, int band, const smf_t *smf, const sinfo *sir,
                         int nsir) {
  const int srw = w - 3;
  for (int i = 0; i < nsir; i++) {
    float block[16] = {0};
    const smf_t *b = &smf[i];
    int k = 0;
    for (int m = b->s_top; m <= b->s_bot; m++)
      for (int x = b->s_left; x <= b->s_right; x++) {
        const float p = b->prob[k];
        const int *t = trans + ((size_t)m * srw + x) * 16;
        for (int c = band; c < 16; c++) {
          const int index = zigzag[c];
          block[index] += p * (float)(t[index]);
        }
        k++;
      }
    for (int c = band; c < 16; c++) {
      const int index = zigzag[c];
      side_trans[(sir[i].top + (index >> 2)) * w + sir[i].left + (index & 3)] = (int)block[index];
    }
  }
}

/* reconstruction, reconstruction.cpp:184-289 */
static void reconstruct_band(int w, int h, const int *rt, int *st, int index, const float *alpha, int step,
                             const uint8_t *mode, uint8_t *dbf, int level_shift) {
  const int b4w = w / 4, b4h = h / 4, b8w = w / 8, row = index >> 2, col = index & 3;
  for (int i = 0; i < b4h; i++)
    for (int j = 0; j < b4w; j++) {
      if (mode[(i >> 1) * b8w + (j >> 1)] != WZ_B) continue;
      const int ci = ((i << 2) + row) * w + (j << 2) + col;
      int lo, hi;
      if (index == 0) {
        const int q = rt[ci];
        lo = q * step;
        hi = (q + 1) * step;
      } else {
        const int q = rt[ci] - level_shift;
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
      const int sc = st[ci];
      const double a = alpha[ci];
      if (a <= 0.0001) {
        st[ci] = (lo + hi) / 2;
      } else if (sc < lo) {
        st[ci] = lo + ROUND(1.0 / a + (double)step / (1.0 - exp(a * (double)step)));
      } else if (sc >= hi) {
        st[ci] = hi - ROUND(1.0 / a + (double)step / (1.0 - exp(a * (double)step)));
      } else {
        double r = sc - lo, d = hi - sc;
        double er = exp(-a * r), ed = exp(-a * d);
        st[ci] = sc + ROUND(((r + 1.0 / a) * er - (d + 1.0 / a) * ed) / (2.0 - (er + ed)));
      }
      dbf[ci] = ((st[ci] ^ sc) != 0) ? 1 : 0;
    }
}

/* inverseTransform, transform.cpp:234-273 (WZ blocks only) */
static void inverse_transform_wz(int w, const int *st, uint8_t *rec, const sinfo *sir, int nsir) {
  for (int i = 0; i < nsir; i++) {
    int b[16];
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++) b[4 * m + n] = st[(sir[i].top + m) * w + sir[i].left + n];
    inverse44(b);
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++) {
        int c = b[4 * m + n];
        rec[(sir[i].top + m) * w + sir[i].left + n] = (uint8_t)(c < 0 ? 0 : (c > 255 ? 255 : c));
      }
  }
}

/* decodeGOP body for one WZ frame, DVC_Decoder.cpp:39-435 (intraRecon and the
 * deblocking filter excluded: the caller supplies intra pixels in f->recon and
 * filters afterwards using f->deblock_flag). */
int dvco_decode_wz_frame(const dvco_ladder *L, dvco_frame *f) {
  if (!transform_ready) transform_init();
  const int w = f->w, h = f->h, fs = w * h, q = f->qindex;
  const int b4w = w / 4, b4h = h / 4, b4n = b4w * b4h, b8w = w / 8, b8h = h / 8;
  const int *qt = qtable[q], *qb = qbits_table[q];
  int level_shift[16] = {0};
  for (int j = 1; j < 16; j++)
    if (qt[j] > 0) level_shift[j] = (qt[j] - 2) / 2; /* wzbitstream.cpp:172-175 */
  if (L->n != b4n) return -1;

  uint8_t *si = (uint8_t *)malloc((size_t)fs);
  int *residue = (int *)malloc(sizeof(int) * fs);
  dvco_create_side_info(w, h, f->past, f->future, f->past_idx, f->future_idx, f->cur_idx, si, residue);
  /* copyIntraBlkToSideInfo, intra.cpp:271-288 */
  for (int i = 0; i < b8h; i++)
    for (int j = 0; j < b8w; j++)
      if (f->mode[i * b8w + j] == INTRA_B)
        for (int m = 0; m < 8; m++) memcpy(si + (8 * i + m) * w + 8 * j, f->recon + (8 * i + m) * w + 8 * j, 8);
  if (f->si_initial) memcpy(f->si_initial, si, (size_t)fs);

  int *side_trans = (int *)malloc(sizeof(int) * fs);
  dvco_forward_transform(w, h, residue, side_trans);
  float *alpha = (float *)calloc((size_t)fs, sizeof(float));
  noise_parameter(w, h, q, side_trans, alpha, f->mode);
  if (f->alpha) memcpy(f->alpha, alpha, sizeof(float) * fs);

  /* initSIR, sideInfoCreation.cpp:554-596 */
  sinfo *sir = (sinfo *)malloc(sizeof(sinfo) * b4n);
  int nsir = 0;
  for (int i = 0; i < b4h; i++) {
    const int top = i << 2;
    int st = top - SEARCHRANGE, sb = top + SEARCHRANGE;
    if (st < 0) st = 0;
    if (sb > h - 4) sb = h - 4;
    for (int j = 0; j < b4w; j++) {
      if (f->mode[(i >> 1) * b8w + (j >> 1)] != WZ_B) continue;
      const int left = j << 2;
      int sl = left - SEARCHRANGE, sr = left + SEARCHRANGE;
      if (sl < 0) sl = 0;
      if (sr > w - 4) sr = w - 4;
      sinfo s = {top, left, st, sb, sl, sr, i * b4w + j};
      sir[nsir++] = s;
    }
  }
  /* initSMF, motionLearning.cpp:6-47 */
  smf_t *smf = (smf_t *)malloc(sizeof(smf_t) * (nsir > 0 ? nsir : 1));
  for (int i = 0; i < nsir; i++) {
    const int top = sir[i].top, left = sir[i].left;
    int st = top - LEARNSEARCHRANGE, sb = top + LEARNSEARCHRANGE;
    int sl = left - LEARNSEARCHRANGE, sr = left + LEARNSEARCHRANGE;
    if (st < 0) st = 0;
    if (sb > h - 4) sb = h - 4;
    if (sl < 0) sl = 0;
    if (sr > w - 4) sr = w - 4;
    int k = 0;
    for (int m = st; m <= sb; m++)
      for (int n = sl; n <= sr; n++) {
        if (m == top && n == left) {
          smf[i].blk = k;
          smf[i].prob[k++] = 1.0f;
        } else {
          smf[i].prob[k++] = 0.0f;
        }
      }
    smf[i].s_top = st;
    smf[i].s_bot = sb;
    smf[i].s_left = sl;
    smf[i].s_right = sr;
    smf[i].len = k;
  }
  const int srw = w - 3, srh = h - 3;
  int *oct = (int *)malloc(sizeof(int) * 16 * (size_t)srw * srh);
  dvco_over_complete_transform(w, h, si, oct);
  /* init_si_ML, motionLearning.cpp:49-68 */
  for (int i = 0; i < b4h; i++)
    for (int j = 0; j < b4w; j++) {
      const int *t = oct + ((size_t)(4 * i) * srw + 4 * j) * 16;
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) side_trans[(4 * i + m) * w + 4 * j + n] = t[4 * m + n];
    }

  /* step sizes and coefficient ranges, DVC_Decoder.cpp:139-152 */
  int step[16], crange[16], wz_bits = 0;
  step[0] = 1024 / qt[0];
  crange[0] = 1024;
  for (int i = 1; i < 16; i++) {
    if (qt[i] > 0) {
      step[i] = (int)ceil((double)((f->ac_range[i] + 1) << 1) / (double)qt[i]);
      wz_bits += 10;
      crange[i] = (level_shift[i] + 1) * step[i] - 1;
    } else {
      step[i] = 0;
    }
  }
  /* copySkipBlkToRecons, skipBlock.cpp:3-22 */
  if (f->skip_mode == 1)
    for (int i = 0; i < b8h; i++)
      for (int j = 0; j < b8w; j++)
        if (f->mode[i * b8w + j] == SKIP_B)
          for (int m = 0; m < 8; m++) memcpy(f->recon + (8 * i + m) * w + 8 * j, f->past + (8 * i + m) * w + 8 * j, 8);

  const double ifc = (double)(f->future_idx - f->cur_idx) / (double)(f->future_idx - f->past_idx);
  const double ipc = (double)(f->cur_idx - f->past_idx) / (double)(f->future_idx - f->past_idx);
  uint8_t *past2 = (uint8_t *)malloc((size_t)fs * 4), *fut2 = (uint8_t *)malloc((size_t)fs * 4);
  dvco_fir_half_pel(f->past, w, h, past2);
  dvco_fir_half_pel(f->future, w, h, fut2);

  int *rt = (int *)calloc((size_t)fs, sizeof(int));
  float *lr = (float *)malloc(sizeof(float) * b4n);
  uint8_t *dec = (uint8_t *)malloc((size_t)b4n);
  uint8_t *acc = (uint8_t *)malloc((size_t)b4n);
  uint8_t *dbf = f->deblock_flag ? f->deblock_flag : (uint8_t *)malloc((size_t)fs);
  memset(dbf, 0, (size_t)fs);
  int plane = 0;
  const int synd_bytes = b4n >> 3;
  for (int band = 0; band < 16; band++) {
    const int index = zigzag[band];
    const int qbits = qb[index];
    if (qbits <= 0) break;
    const int range = crange[index];
    float *dist = noise_distribution(w, range, index, alpha, smf, oct, sir, nsir);
    for (int bit = qbits; bit > 0; bit--) {
      if (f->skip_mode == 1 || f->intra_mode == 1)
        for (int i = 0; i < b4n; i++) lr[i] = 0.9999f / 0.0001f;
      cond_bit_prob(w, lr, index, bit, step[index], rt, range, dist, sir, nsir, level_shift[index]);
      const float ent = dvco_compute_ce(lr, b4n);
      if (f->entropy) f->entropy[plane] = ent;
      /* ByteToBit, LdpcaDecoder.cpp:81-107 */
      const uint8_t *bytes = f->acc_synd + (size_t)plane * synd_bytes;
      for (int i = 0; i < b4n; i++) acc[i] = (uint8_t)((bytes[i >> 3] >> (7 - (i & 7))) & 1);
      int rate = 0, start = 0;
      const int accepted = dvco_ldpca_decode(L, lr, acc, dec, &rate, f->crc[plane], ent, &start);
      if (f->start_code) f->start_code[plane] = start;
      if (f->accepted_code) f->accepted_code[plane] = accepted;
      wz_bits += rate;
      /* putBitplaneToCoeff, bitplane.cpp:4-22 */
      {
        const int row = index >> 2, col = index & 3;
        int bi = 0;
        for (int i = 0; i < b4h; i++)
          for (int j = 0; j < b4w; j++, bi++)
            if (f->mode[(i >> 1) * b8w + (j >> 1)] == WZ_B) {
              const int ci = ((i << 2) + row) * w + (j << 2) + col;
              rt[ci] = (rt[ci] << 1) + (int)dec[bi];
            }
      }
      plane++;
    }
    reconstruct_band(w, h, rt, side_trans, index, alpha, step[index], f->mode, dbf, level_shift[index]);
    inverse_transform_wz(w, side_trans, f->recon, sir, nsir);
    update_si(w, h, si, f->recon, f->past, f->future, past2, fut2, ifc, ipc, sir, nsir);
    free(dist);
    dvco_over_complete_transform(w, h, si, oct);
    update_smf(w, smf, f->recon, si, sir, nsir);
    update_si_ml(w, side_trans, oct, band + 1, smf, sir, nsir);
  }
  inverse_transform_wz(w, side_trans, f->recon, sir, nsir);
  if (f->si_final) memcpy(f->si_final, si, (size_t)fs);
  f->wz_bits = wz_bits;

  if (!f->deblock_flag) free(dbf);
  free(rt);
  free(lr);
  free(dec);
  free(acc);
  free(past2);
  free(fut2);
  free(oct);
  free(smf);
  free(sir);
  free(alpha);
  free(side_trans);
  free(residue);
  free(si);
  return 0;
}

/* ---------------------------------------------------------------- deblocking
 * deblock, DvcDec/src/deblock.cpp:346-386: edge decisions on the unfiltered
 * frame (deblock_44_decision, :228-344), edges filtered in place in raster
 * order, vertical edges (between horizontal neighbours) first
 * (deblock_filter, :40-226).  type_map: per 8x8 block 0 WZ, 1 intra, 2 skip;
 * past_mode: the past reference's block modes when it is a WZ frame (NULL
 * for a key frame, :270-287). */
static const unsigned char db_alpha[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,   0,   0,   0,   0,   0,   0,   0,   4,   4,
                                           5,  6,  7,  8,  9,  10, 12, 13, 15,  17,  20,  22,  25,  28,  32,  36,  40,  45,
                                           50, 56, 63, 71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
static const unsigned char db_beta[52] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4,
                                          6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
/* the H.264 tc0 table by strength 1..3 (strength 0 and 4 columns unused or equal) */
static const unsigned char db_tc0[52][5] = {
    {0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},
    {0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},{0,0,0,0,0},
    {0,0,0,0,0},{0,0,0,1,1},{0,0,0,1,1},{0,0,0,1,1},{0,0,0,1,1},{0,0,1,1,1},{0,0,1,1,1},{0,1,1,1,1},
    {0,1,1,1,1},{0,1,1,1,1},{0,1,1,1,1},{0,1,1,2,2},{0,1,1,2,2},{0,1,1,2,2},{0,1,1,2,2},{0,1,2,3,3},
    {0,1,2,3,3},{0,2,2,3,3},{0,2,2,4,4},{0,2,3,4,4},{0,2,3,4,4},{0,3,3,5,5},{0,3,4,6,6},{0,3,4,6,6},
    {0,4,5,7,7},{0,4,5,8,8},{0,4,6,9,9},{0,5,7,10,10},{0,6,8,11,11},{0,6,8,13,13},{0,7,10,14,14},{0,8,11,16,16},
    {0,9,12,18,18},{0,10,13,20,20},{0,11,15,23,23},{0,13,17,25,25}};

enum { DB_NONE = 0, DB_WZ = 1, DB_ISWZ = 2 };

static int db_iabs(int v) { return v < 0 ? -v : v; }
static int db_clip3(int lo, int hi, int v) { return v < lo ? lo : (v > hi ? hi : v); }

/* one 4x4 block: did any coefficient change its side-information value
 * (weighted), and is the pixel variance below 50 */
static void db_block(const uint8_t *rec, const uint8_t *flag, int w, int bx, int by, const double *weight, double *phi,
                     double *chi) {
  int sum = 0, sq = 0;
  *phi = 0.0;
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) {
      const int idx = (by * 4 + m) * w + bx * 4 + n;
      if (flag[idx]) *phi += weight[m * 4 + n];
      sum += rec[idx];
      sq += rec[idx] * rec[idx];
    }
  const double var = (double)sq / 16.0 - ((double)sum / 16.0) * ((double)sum / 16.0);
  *chi = var < 50.0 ? 1.0 : 0.0;
}

/* deblock_44_decision: filter mode and strength of the edge between blocks 1 and 2 */
static int db_decide(const uint8_t *rec, const uint8_t *flag, const uint8_t *type_map, const uint8_t *past_mode, int w,
                     int x1, int y1, int x2, int y2, const double *weight, double *bs) {
  const int b8w = w / 8;
  const int t1 = type_map[(y1 >> 1) * b8w + (x1 >> 1)], t2 = type_map[(y2 >> 1) * b8w + (x2 >> 1)];
  if (t1 == 1 || t2 == 1) {
    *bs = (t1 == 1 && t2 == 1) ? 3.0 : ((t1 == 0 || t2 == 0) ? 4.0 : 3.0);
    return DB_ISWZ;
  }
  if (t1 == 2 && t2 == 2) {
    *bs = 0.0;
    return DB_NONE;
  }
  if (t1 == 2 || t2 == 2) {
    const int sp = t1 == 2 ? (y1 >> 1) * b8w + (x1 >> 1) : (y2 >> 1) * b8w + (x2 >> 1);
    *bs = past_mode ? (past_mode[sp] == 1 ? 2.0 : 1.0) : 2.0;
    return DB_ISWZ;
  }
  if (t1 == 0 && t2 == 0) {
    double phi1, chi1, phi2, chi2;
    db_block(rec, flag, w, x1, y1, weight, &phi1, &chi1);
    db_block(rec, flag, w, x2, y2, weight, &phi2, &chi2);
    const double P = 0.9;
    *bs = 0.14 * (P * ((phi1 + phi2) / 2.0) + (1.0 - P) * ((chi1 + chi2) / 2.0));
    return *bs > 0.0 ? DB_WZ : DB_NONE;
  }
  return DB_NONE;
}

/* the four pixel lines across one edge; p[k] is the k-th pixel of a line
 * counted from block 1's far side (p[0..3] block 1, p[4..7] block 2) */
static void db_filter(int dir, int mode, double bs, uint8_t *img, int w, int x1, int y1, int x2, int y2, int qp,
                      double pow_qp) {
  const int step = dir ? w : 1;
  const int alpha = db_alpha[qp], beta = db_beta[qp];
  for (int line = 0; line < 4; line++) {
    uint8_t *P = img + (y1 * 4 + (dir ? 0 : line)) * w + x1 * 4 + (dir ? line : 0);
    uint8_t *Q = img + (y2 * 4 + (dir ? 0 : line)) * w + x2 * 4 + (dir ? line : 0);
    const int L3 = P[0], L2 = P[step], L1 = P[2 * step], L0 = P[3 * step];
    const int R0 = Q[0], R1 = Q[step], R2 = Q[2 * step], R3 = Q[3 * step];
    if (!(db_iabs(R0 - L0) < alpha && db_iabs(R0 - R1) < beta && db_iabs(L0 - L1) < beta)) continue;
    const int strong = (mode == DB_ISWZ) ? ((int)bs == 4) : (bs > 0.14 * 0.5);
    if (mode == DB_WZ && !(bs > 0.0)) continue;
    if (strong) {
      const int rl0 = L0 + R0, small_gap = db_iabs(R0 - L0) < ((alpha >> 2) + 2);
      const int aq = (db_iabs(R0 - R2) < beta) & small_gap, ap = (db_iabs(L0 - L2) < beta) & small_gap;
      if (ap) {
        P[3 * step] = (uint8_t)((R1 + ((L1 + rl0) << 1) + L2 + 4) >> 3);
        P[2 * step] = (uint8_t)((L2 + L1 + rl0 + 2) >> 2);
        P[step] = (uint8_t)((((L3 + L2) << 1) + L2 + L1 + rl0 + 4) >> 3);
      } else {
        P[3 * step] = (uint8_t)(((L1 << 1) + L0 + R1 + 2) >> 2);
      }
      if (aq) {
        Q[0] = (uint8_t)((L1 + ((R1 + rl0) << 1) + R2 + 4) >> 3);
        Q[step] = (uint8_t)((R2 + R0 + L0 + R1 + 2) >> 2);
        Q[2 * step] = (uint8_t)((((R3 + R2) << 1) + R2 + R1 + rl0 + 4) >> 3);
      } else {
        Q[0] = (uint8_t)(((R1 << 1) + R0 + L1 + 2) >> 2);
      }
    } else {
      const int rl0 = (L0 + R0 + 1) >> 1;
      const int aq = db_iabs(R0 - R2) < beta, ap = db_iabs(L0 - L2) < beta;
      const int c0 = mode == DB_ISWZ ? db_tc0[qp][(int)bs] : (int)(bs * (pow_qp - 1));
      const int tc = c0 + ap + aq;
      const int dif = db_clip3(-tc, tc, (((R0 - L0) << 2) + (L1 - R1) + 4) >> 3);
      /* the p1 / q1 updates add to the byte without clipping (it wraps), :186-197 */
      if (ap) P[2 * step] = (uint8_t)(P[2 * step] + db_clip3(-c0, c0, (L2 + rl0 - (L1 << 1)) >> 1));
      P[3 * step] = (uint8_t)db_clip3(0, 255, L0 + dif);
      Q[0] = (uint8_t)db_clip3(0, 255, R0 - dif);
      if (aq) Q[step] = (uint8_t)(Q[step] + db_clip3(-c0, c0, (R2 + rl0 - (R1 << 1)) >> 1));
    }
  }
}

void dvco_deblock(const uint8_t *recon, const uint8_t *flag, const uint8_t *type_map, const uint8_t *past_mode, int w,
                  int h, int qindex, int intra_qp, uint8_t *out) {
  const int b4w = w / 4, b4h = h / 4;
  double weight[16];
  int sum = 0;
  for (int i = 0; i < 16; i++) sum += qtable[qindex][i];
  for (int i = 0; i < 16; i++) weight[i] = (double)qtable[qindex][i] / (double)sum;
  const double pow_qp = pow(2, (double)intra_qp / 6.0);
  memcpy(out, recon, (size_t)w * h);
  for (int dir = 0; dir < 2; dir++) {
    const int xd = dir ? 0 : 1, yd = dir ? 1 : 0;
    for (int i = 0; i < b4h - yd; i++)
      for (int j = 0; j < b4w - xd; j++) {
        double bs = 0.0;
        const int mode = db_decide(recon, flag, type_map, past_mode, w, j, i, j + xd, i + yd, weight, &bs);
        if (mode == DB_WZ || mode == DB_ISWZ) db_filter(dir, mode, bs, out, w, j, i, j + xd, i + yd, intra_qp, pow_qp);
      }
  }
}

/* ---- intra blocks (IntraMode 1): intraRecon, DvcDec/src/intra.cpp:252-268 ----
 *
 * CAVLC entropy decoding of the 4x4 luma blocks (vlc.cpp:423-761), restated
 * from the H.264 syntax (ITU-T H.264 9.2): coeff_token, trailing-one signs,
 * levels (level_prefix / level_suffix with the adaptive suffix length),
 * total_zeros and run_before.  The code tables are the standard's tables 9-5
 * (0 <= nC < 8), 9-9a and 9-10, written as {length, value} pairs; the reference
 * holds the same tables (vlc.cpp:89-198, 423-470).  Codes are matched bit by
 * bit: after each bit, every entry of that length is compared. */
typedef struct {
  uint8_t len;
  uint16_t code;
} vlc_code;

/* coeff_token by nC class (nC < 2, < 4, < 8), [TotalCoeff][TrailingOnes] */
static const vlc_code ct_tab[3][17][4] = {
    {{{1, 1}, {0, 0}, {0, 0}, {0, 0}},
     {{6, 5}, {2, 1}, {0, 0}, {0, 0}},
     {{8, 7}, {6, 4}, {3, 1}, {0, 0}},
     {{9, 7}, {8, 6}, {7, 5}, {5, 3}},
     {{10, 7}, {9, 6}, {8, 5}, {6, 3}},
     {{11, 7}, {10, 6}, {9, 5}, {7, 4}},
     {{13, 15}, {11, 6}, {10, 5}, {8, 4}},
     {{13, 11}, {13, 14}, {11, 5}, {9, 4}},
     {{13, 8}, {13, 10}, {13, 13}, {10, 4}},
     {{14, 15}, {14, 14}, {13, 9}, {11, 4}},
     {{14, 11}, {14, 10}, {14, 13}, {13, 12}},
     {{15, 15}, {15, 14}, {14, 9}, {14, 12}},
     {{15, 11}, {15, 10}, {15, 13}, {14, 8}},
     {{16, 15}, {15, 1}, {15, 9}, {15, 12}},
     {{16, 11}, {16, 14}, {16, 13}, {15, 8}},
     {{16, 7}, {16, 10}, {16, 9}, {16, 12}},
     {{16, 4}, {16, 6}, {16, 5}, {16, 8}}},
    {{{2, 3}, {0, 0}, {0, 0}, {0, 0}},
     {{6, 11}, {2, 2}, {0, 0}, {0, 0}},
     {{6, 7}, {5, 7}, {3, 3}, {0, 0}},
     {{7, 7}, {6, 10}, {6, 9}, {4, 5}},
     {{8, 7}, {6, 6}, {6, 5}, {4, 4}},
     {{8, 4}, {7, 6}, {7, 5}, {5, 6}},
     {{9, 7}, {8, 6}, {8, 5}, {6, 8}},
     {{11, 15}, {9, 6}, {9, 5}, {6, 4}},
     {{11, 11}, {11, 14}, {11, 13}, {7, 4}},
     {{12, 15}, {11, 10}, {11, 9}, {9, 4}},
     {{12, 11}, {12, 14}, {12, 13}, {11, 12}},
     {{12, 8}, {12, 10}, {12, 9}, {11, 8}},
     {{13, 15}, {13, 14}, {13, 13}, {12, 12}},
     {{13, 11}, {13, 10}, {13, 9}, {13, 12}},
     {{13, 7}, {14, 11}, {13, 6}, {13, 8}},
     {{14, 9}, {14, 8}, {14, 10}, {13, 1}},
     {{14, 7}, {14, 6}, {14, 5}, {14, 4}}},
    {{{4, 15}, {0, 0}, {0, 0}, {0, 0}},
     {{6, 15}, {4, 14}, {0, 0}, {0, 0}},
     {{6, 11}, {5, 15}, {4, 13}, {0, 0}},
     {{6, 8}, {5, 12}, {5, 14}, {4, 12}},
     {{7, 15}, {5, 10}, {5, 11}, {4, 11}},
     {{7, 11}, {5, 8}, {5, 9}, {4, 10}},
     {{7, 9}, {6, 14}, {6, 13}, {4, 9}},
     {{7, 8}, {6, 10}, {6, 9}, {4, 8}},
     {{8, 15}, {7, 14}, {7, 13}, {5, 13}},
     {{8, 11}, {8, 14}, {7, 10}, {6, 12}},
     {{9, 15}, {8, 10}, {8, 13}, {7, 12}},
     {{9, 11}, {9, 14}, {8, 9}, {8, 12}},
     {{9, 8}, {9, 10}, {9, 13}, {8, 8}},
     {{10, 13}, {9, 7}, {9, 9}, {9, 12}},
     {{10, 9}, {10, 12}, {10, 11}, {10, 10}},
     {{10, 5}, {10, 8}, {10, 7}, {10, 6}},
     {{10, 1}, {10, 4}, {10, 3}, {10, 2}}},
};

/* total_zeros for TotalCoeff 1..15 (row TotalCoeff - 1), [total_zeros] */
static const vlc_code tz_tab[15][16] = {
    {{1, 1}, {3, 3}, {3, 2}, {4, 3}, {4, 2}, {5, 3}, {5, 2}, {6, 3}, {6, 2}, {7, 3}, {7, 2}, {8, 3}, {8, 2}, {9, 3}, {9, 2}, {9, 1}},
    {{3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {4, 5}, {4, 4}, {4, 3}, {4, 2}, {5, 3}, {5, 2}, {6, 3}, {6, 2}, {6, 1}, {6, 0}},
    {{4, 5}, {3, 7}, {3, 6}, {3, 5}, {4, 4}, {4, 3}, {3, 4}, {3, 3}, {4, 2}, {5, 3}, {5, 2}, {6, 1}, {5, 1}, {6, 0}},
    {{5, 3}, {3, 7}, {4, 5}, {4, 4}, {3, 6}, {3, 5}, {3, 4}, {4, 3}, {3, 3}, {4, 2}, {5, 2}, {5, 1}, {5, 0}},
    {{4, 5}, {4, 4}, {4, 3}, {3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {4, 2}, {5, 1}, {4, 1}, {5, 0}},
    {{6, 1}, {5, 1}, {3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {3, 2}, {4, 1}, {3, 1}, {6, 0}},
    {{6, 1}, {5, 1}, {3, 5}, {3, 4}, {3, 3}, {2, 3}, {3, 2}, {4, 1}, {3, 1}, {6, 0}},
    {{6, 1}, {4, 1}, {5, 1}, {3, 3}, {2, 3}, {2, 2}, {3, 2}, {3, 1}, {6, 0}},
    {{6, 1}, {6, 0}, {4, 1}, {2, 3}, {2, 2}, {3, 1}, {2, 1}, {5, 1}},
    {{5, 1}, {5, 0}, {3, 1}, {2, 3}, {2, 2}, {2, 1}, {4, 1}},
    {{4, 0}, {4, 1}, {3, 1}, {3, 2}, {1, 1}, {3, 3}},
    {{4, 0}, {4, 1}, {2, 1}, {1, 1}, {3, 1}},
    {{3, 0}, {3, 1}, {1, 1}, {2, 1}},
    {{2, 0}, {2, 1}, {1, 1}},
    {{1, 0}, {1, 1}},
};

/* run_before for zerosLeft 1..6 and > 6 (row min(zerosLeft, 7) - 1), [run_before] */
static const vlc_code rb_tab[7][15] = {
    {{1, 1}, {1, 0}},
    {{1, 1}, {2, 1}, {2, 0}},
    {{2, 3}, {2, 2}, {2, 1}, {2, 0}},
    {{2, 3}, {2, 2}, {2, 1}, {3, 1}, {3, 0}},
    {{2, 3}, {2, 2}, {3, 3}, {3, 2}, {3, 1}, {3, 0}},
    {{2, 3}, {3, 0}, {3, 1}, {3, 3}, {3, 2}, {3, 5}, {3, 4}},
    {{3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {3, 2}, {3, 1}, {4, 1}, {5, 1}, {6, 1}, {7, 1}, {8, 1}, {9, 1}, {10, 1}, {11, 1}},
};

typedef struct {
  const uint8_t *buf;
  size_t nbits, pos;
  int bad; /* set when a read runs past the end or a code is not in its table */
} ib_reader;

static int ib_bit(ib_reader *r) {
  if (r->pos >= r->nbits) {
    r->bad = 1;
    return 0;
  }
  const int b = (r->buf[r->pos >> 3] >> (7 - (int)(r->pos & 7))) & 1; /* MSB first, GetBits vlc.cpp:366-401 */
  r->pos++;
  return b;
}

static int ib_bits(ib_reader *r, int n) {
  int v = 0;
  for (int i = 0; i < n; i++) v = (v << 1) | ib_bit(r);
  return v;
}

/* Index of the entry of tab[0..count) the next bits spell, or -1. */
static int ib_vlc(ib_reader *r, const vlc_code *tab, int count) {
  int v = 0;
  for (int len = 1; len <= 16 && !r->bad; len++) {
    v = (v << 1) | ib_bit(r);
    for (int i = 0; i < count; i++)
      if (tab[i].len == len && tab[i].code == v) return i;
  }
  r->bad = 1;
  return -1;
}

/* One level (H.264 9.2.2.1; Level_VLC0 / Level_VLCN, vlc.cpp:231-364):
 * level_prefix zeros, a suffix of levelSuffixSize bits, levelCode, and the
 * signed level (levelCode + 2) >> 1 for even codes, (-levelCode - 1) >> 1 for
 * odd ones. */
static int ib_level(ib_reader *r, int suffix_length, int first_adjust) {
  int prefix = 0;
  while (!r->bad && !ib_bit(r)) prefix++;
  int size = suffix_length;
  if (prefix == 14 && suffix_length == 0) size = 4;
  if (prefix >= 15) size = prefix - 3;
  int code = ((prefix < 15 ? prefix : 15) << suffix_length) + (size ? ib_bits(r, size) : 0);
  if (prefix >= 15 && suffix_length == 0) code += 15;
  if (prefix >= 16) code += (1 << (prefix - 3)) - 4096;
  if (first_adjust) code += 2; /* first non-trailing-one level when TrailingOnes < 3 */
  return (code & 1) ? (-code - 1) >> 1 : (code + 2) >> 1;
}

/* residual_block_cavlc of one 4x4 luma block (vlc.cpp:613-761): coefficients
 * in zig-zag order into scan[16]; returns TotalCoeff. */
static int ib_block(ib_reader *r, int nc, int scan[16]) {
  int total, t1;
  memset(scan, 0, 16 * sizeof(int));
  if (nc >= 8) { /* 6-bit fixed-length coeff_token: TotalCoeff - 1 and TrailingOnes, 000011 = none */
    const int v = ib_bits(r, 6);
    total = (v >> 2) + 1;
    t1 = v & 3;
    if (v == 3) total = t1 = 0;
  } else {
    const int i = ib_vlc(r, &ct_tab[nc < 2 ? 0 : nc < 4 ? 1 : 2][0][0], 17 * 4);
    if (i < 0) return 0;
    total = i / 4;
    t1 = i % 4;
  }
  if (total == 0 || r->bad) return 0;
  int level[16], run[16];
  for (int i = 0; i < t1; i++) level[i] = ib_bit(r) ? -1 : 1; /* trailing ones, highest frequency first */
  int suffix_length = (total > 10 && t1 < 3) ? 1 : 0;
  for (int i = t1; i < total; i++) {
    level[i] = ib_level(r, suffix_length, i == t1 && t1 < 3);
    const int a = level[i] < 0 ? -level[i] : level[i];
    if (suffix_length == 0) suffix_length = 1;
    if (a > (3 << (suffix_length - 1)) && suffix_length < 6) suffix_length++;
  }
  int zeros_left = 0;
  if (total < 16) {
    zeros_left = ib_vlc(r, tz_tab[total - 1], 16);
    if (zeros_left < 0) return 0;
  }
  for (int i = 0; i < total - 1; i++) {
    run[i] = 0;
    if (zeros_left > 0) {
      run[i] = ib_vlc(r, rb_tab[(zeros_left < 7 ? zeros_left : 7) - 1], 15);
      if (run[i] < 0) return 0;
    }
    zeros_left -= run[i];
  }
  run[total - 1] = zeros_left;
  if (zeros_left < 0) {
    r->bad = 1;
    return 0;
  }
  int pos = -1; /* lowest frequency last: walk back from level[total-1] */
  for (int i = total - 1; i >= 0; i--) {
    pos += run[i] + 1;
    if (pos > 15) {
      r->bad = 1;
      return 0;
    }
    scan[pos] = level[i];
  }
  return total;
}

/* 4x4 inverse core transform of intra blocks (intra.cpp:35-80): columns
 * first, then rows, then >> 6 without rounding. */
static void intra_inverse44(int *b) {
  int t[16];
  for (int c = 0; c < 4; c++) {
    const int x0 = b[c], x1 = b[4 + c], x2 = b[8 + c], x3 = b[12 + c];
    t[c] = x0 + x1 + x2 + (x3 >> 1);
    t[4 + c] = x0 + (x1 >> 1) - x2 - x3;
    t[8 + c] = x0 - (x1 >> 1) - x2 + x3;
    t[12 + c] = x0 - x1 + x2 - (x3 >> 1);
  }
  for (int r = 0; r < 4; r++) {
    const int *x = t + 4 * r;
    b[4 * r] = x[0] + x[1] + x[2] + (x[3] >> 1);
    b[4 * r + 1] = x[0] + (x[1] >> 1) - x[2] - x[3];
    b[4 * r + 2] = x[0] - (x[1] >> 1) - x[2] + x[3];
    b[4 * r + 3] = x[0] - x[1] + x[2] - (x[3] >> 1);
  }
  for (int i = 0; i < 16; i++) b[i] >>= 6;
}

int dvco_intra_decode_frame(const uint8_t *buf, size_t nbytes, size_t *bit_offset, int w, int h, int intra_qp,
                            const uint8_t *mode, uint8_t *recon) {
  if (!transform_ready) transform_init();
  const int b4w = w / 4, b4h = h / 4, b8w = w / 8;
  ib_reader r = {buf, nbytes * 8, *bit_offset, 0};
  int *nnz = (int *)calloc((size_t)b4w * b4h, sizeof(int));
  if (!nnz) return -1;
  const double qstep = pow(2.0, ((double)intra_qp - 4.0) / 6.0); /* intra.cpp:253 */
#define IS_INTRA(bx, by) (mode[((by) >> 1) * b8w + ((bx) >> 1)] == INTRA_B)
  for (int by = 0; by < b4h && !r.bad; by++)
    for (int bx = 0; bx < b4w && !r.bad; bx++) {
      if (!IS_INTRA(bx, by)) continue;
      /* neighbours count when they lie in an intra 8x8 block (getNeighbour intra.cpp:83-121) */
      const int left = bx > 0 && IS_INTRA(bx - 1, by), up = by > 0 && IS_INTRA(bx, by - 1);
      /* nC (predict_nnz vlc.cpp:564-611) */
      int nc = 0;
      if (left) nc += nnz[by * b4w + bx - 1];
      if (up) nc += nnz[(by - 1) * b4w + bx];
      if (left && up) nc = (nc + 1) >> 1;
      int scan[16], blk[16];
      nnz[by * b4w + bx] = ib_block(&r, nc, scan);
      /* de-quantisation in double (read_one_block intra.cpp:187-215) */
      for (int i = 0; i < 16; i++) blk[i] = 0;
      for (int k = 0; k < 16; k++) blk[zigzag[k]] = scan[k];
      for (int i = 0; i < 16; i++) blk[i] = ROUND((double)blk[i] * qstep * pre_scale[i]);
      intra_inverse44(blk);
      /* DC prediction from the intra neighbours' decoded pixels (intra4x4_dc_pred intra.cpp:124-185) */
      const int x0 = 4 * bx, y0 = 4 * by;
      int s = 0;
      if (up)
        for (int i = 0; i < 4; i++) s += recon[(y0 - 1) * w + x0 + i];
      if (left)
        for (int i = 0; i < 4; i++) s += recon[(y0 + i) * w + x0 - 1];
      const int dc = (up && left) ? (s + 4) >> 3 : (up || left) ? (s + 2) >> 2 : 128;
      /* SampleRecon intra.cpp:218-238 */
      for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) {
          const int v = blk[4 * y + x] + dc;
          recon[(y0 + y) * w + x0 + x] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
#undef IS_INTRA
  free(nnz);
  if (r.bad) return -1;
  *bit_offset = r.pos;
  return 0;
}
