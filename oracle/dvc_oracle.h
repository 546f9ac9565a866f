/* Test infrastructure: CPU restatement of the reference DvcDec Wyner-Ziv frame
 * decoder hot path (ParallelMode 0 arithmetic), used only as the checker for
 * the CUDA path in tests/, smoke() and the CPU-baseline leg of bench.py.
 *
 * Everything is restated from the reference sources (paths relative to the
 * reference tree, DvcDec/src unless noted); each function cites the file:line
 * it follows.  Float and double operations are written in the reference's order
 * and compiled without FMA contraction, and the same libm entry points are
 * called (logf, tanhf, expf, sqrtf, exp, sqrt), so results are bit-identical to
 * the reference decoder built with g++ on this machine.  Parity is pinned by
 * tests against oracle/_ref (the reference compiled from its own sources).
 */
#ifndef DVC_ORACLE_H
#define DVC_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* LDPCA ladder tables (ReadLdpcaLadderFile_LdpcaDecoder.cpp:150-201). */
typedef struct {
  int num_codes, n, e, period;
  const int *jc;        /* [n+1] */
  const int *bpp;       /* [num_codes] bitsPerPeriod */
  const int *idx;       /* [num_codes*period] idxPerPeriod, row-padded */
  const int *ir;        /* [num_codes*e] row of every edge */
  const uint32_t *invh; /* [n*ceil(n/32)] inverse of the full-rate H, reference file layout */
} dvco_ladder;

/* One LDPCA decode of one bitplane (LdpcaDecoder.cpp:646-771, mode 0).
 * lr[n] holds p0/p1 on entry and log(p0/p1) on exit, as in the reference.
 * acc_bits[n]: accumulated syndrome, one bit per byte.  Returns the accepted
 * code index; *start_code receives the first code tried. */
int dvco_ldpca_decode(const dvco_ladder *L, float *lr, const uint8_t *acc_bits, uint8_t *decoded,
                      int *rate, uint8_t crc, float entropy, int *start_code);

/* dvco_ldpca_decode with max_iter BP iterations per ladder code instead of 50. */
int dvco_ldpca_decode_iter(const dvco_ladder *L, float *lr, const uint8_t *acc_bits, uint8_t *decoded,
                           int *rate, uint8_t crc, float entropy, int *start_code, int max_iter);

/* Sum-product BP on one code (LdpcaDecoder.cpp:462-580); returns 1 if all
 * parity checks hold within max_iter iterations. *iters gets the iteration count. */
int dvco_belief_propagation(const dvco_ladder *L, const float *llr, const uint8_t *syndrome,
                            uint8_t *decoded, int m, int code, int max_iter, int *iters);

float dvco_compute_ce(const float *lr, int n);                   /* LdpcaDecoder.cpp:127-143 */
uint8_t dvco_crc8_bits(const uint8_t *bits, int n);              /* crc8.h + BitToByte */
void dvco_accumulated_syndrome(const dvco_ladder *L, const uint8_t *source_bits,
                               uint8_t *acc_bits);               /* DvcEnc LdpcaEncoder.cpp:64-95 */

/* Whole WZ frame (DVC_Decoder.cpp:26-445 for one frameIdx). */
typedef struct {
  int w, h, qindex;
  const uint8_t *past, *future; /* reconstructed reference frames [w*h] */
  int past_idx, future_idx, cur_idx;
  const uint8_t *mode;          /* [w*h/64] 0 WZ, 1 intra, 2 skip */
  int skip_mode, intra_mode;
  const int *ac_range;          /* [16] */
  const uint8_t *crc;           /* [qbits] */
  const uint8_t *acc_synd;      /* [qbits][n/8] bytes as in the bitstream */
  uint8_t *recon;               /* [w*h] in: intra blocks decoded; out: decoded frame (pre-deblocking) */
  /* outputs (optional ones may be NULL) */
  int wz_bits;                  /* 10 per coded AC band + sum of (m+8) */
  int *start_code, *accepted_code; /* [qbits] */
  uint8_t *deblock_flag;        /* [w*h] */
  float *alpha;                 /* [w*h] */
  uint8_t *si_initial;          /* [w*h] side info after createSideInfo + intra copy */
  uint8_t *si_final;            /* [w*h] side info after the last updateSI */
  float *entropy;               /* [qbits] */
} dvco_frame;

int dvco_decode_wz_frame(const dvco_ladder *L, dvco_frame *f);

/* Stage-level entry points used by unit tests. */
void dvco_low_pass(const uint8_t *in, int w, int h, uint8_t *out);            /* filter.cpp:214-233 */
void dvco_fir_half_pel(const uint8_t *in, int w, int h, uint8_t *out);        /* filter.cpp:55-117 */
void dvco_create_side_info(int w, int h, const uint8_t *past, const uint8_t *future,
                           int past_idx, int future_idx, int cur_idx,
                           uint8_t *si, int *residue);                          /* sideInfoCreation.cpp:438-551 */
void dvco_forward_transform(int w, int h, const int *in, int *out);            /* transform.cpp:153-190 */
void dvco_over_complete_transform(int w, int h, const uint8_t *pix, int *trans16); /* transform.cpp:275-298 */
int dvco_qbits_per_block(int qindex);
/* deblock, DvcDec/src/deblock.cpp:346-386 (type_map per 8x8 block: 0 WZ, 1 intra, 2 skip;
 * past_mode NULL when the past reference is a key frame) */
void dvco_deblock(const uint8_t *recon, const uint8_t *flag, const uint8_t *type_map, const uint8_t *past_mode, int w,
                  int h, int qindex, int intra_qp, uint8_t *out);
/* intra blocks of one frame, intraRecon DvcDec/src/intra.cpp:252-268: decodes every
 * 4x4 block of the 8x8 blocks with mode 1 (raster order over the frame's 4x4
 * blocks) from the sequence's intra bit string buf[nbytes], starting at
 * *bit_offset, and writes their pixels into recon[w*h]; other pixels are left
 * alone.  Returns 0 and advances *bit_offset, or -1 when the string ends inside
 * a block or holds a code that is not in its table. */
int dvco_intra_decode_frame(const uint8_t *buf, size_t nbytes, size_t *bit_offset, int w, int h, int intra_qp,
                            const uint8_t *mode, uint8_t *recon);

#ifdef __cplusplus
}
#endif
#endif
