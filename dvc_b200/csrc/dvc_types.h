// Plain-data structures shared by the host driver and the kernels.
#pragma once
#include <stdint.h>

#include "libm_tables.h"

namespace dvc {

// LDPCA ladder for one codeword length, resident in device memory.
// Derived from the reference's ladder tables (ReadLdpcaLadderFile_LdpcaDecoder.cpp:150-201):
// per code c the syndrome length m_c = (n/period)*bpp[c], its rate m_c/n, the
// row of every edge, plus layouts this decoder adds for parallel BP: per code
// the row-order positions of the edges (each row's edges contiguous, in
// increasing edge order, so that row sums keep the reference's summation
// order), the CRC-8 contribution of each single source bit, and the GF(2)
// inverse of the full-rate matrix with bit i of row j at word i/32, bit i%32.
struct LadderDev {
  int n, e, period, num_codes, invh_words;
  const int *jc;          // [n+1]
  const int *bpp;         // [num_codes]
  const int *idx;         // [num_codes*period]
  const int *synd_len;    // [num_codes]
  const float *code_rate; // [num_codes]
  const int *row_ptr;     // [num_codes*(n+1)] first row-order position of each row
  // Edges are numbered column-major (edge e = 3k + i is the i-th edge of column
  // k, every column has degree 3); row-order position p lists each row's edges
  // in increasing e, rows in order.
  const uint16_t *pos;       // [num_codes*e] row-order position of edge e
  const uint16_t *rid;       // [num_codes*e] row of row-order position p
  const uint16_t *ir_full;   // [e] row of edge e in the full-rate code (the encoder's matrix)
  const uint8_t *crc_tab;    // [n]
  const uint32_t *invh;      // [n*invh_words]
};

// One LDPCA decode request: a bitplane of one WZ frame.
struct LdpcaJob {
  int active;            // 0: the block returns at once (frame not in this step)
  const float *lr;       // [n] p0/p1 per 4x4 block (condBitProb output)
  const uint8_t *acc;    // [n/8] accumulated syndrome bytes, MSB first
  int crc;               // CRC-8 of the source bitplane
  uint8_t *decoded;      // [n] decoded bits (may be null)
  int *result;           // [4] rate (m+8), first code tried, accepted code, BP iterations run
  float *entropy;        // conditional entropy bound (may be null)
  int use_given_entropy; // 1: take the bound from given_entropy instead of computing it
  float given_entropy;
  float *llr_out;        // [n] log(p0/p1) written back (may alias lr), or null
  // optional fused putBitplaneToCoeff (bitplane.cpp:4-22)
  int *recons_trans;     // [w*h] quantisation indices, or null
  const uint8_t *mode;   // [w*h/64] block modes
  int w, index_in_blk;
};

// Scratch of the speculative ladder form (k_ldpca.cu): per codeword the lowest
// successful code, summed BP iterations and first code; per (codeword, block)
// the code it succeeded with and its decoded bits.
struct LdpcaSpec {
  int *best = nullptr, *iters = nullptr, *start = nullptr, *done = nullptr, *slot_code = nullptr;
  uint8_t *slot_dec = nullptr;
};

// Batched form (k_ldpca_batch.cu): one codeword of a mixed-length batch.
struct LdpcaBatchCw {
  int cif;          // 1: n = 6336 (CIF ladder), 0: n = 1584 (QCIF ladder)
  int crc;          // CRC-8 of the source bits
  int given_start;  // first ladder code to try, or -1: the conditional-entropy bound picks it
  long long lr_off, acc_off, dec_off;  // offsets of its LRs (floats), accumulated syndrome and decoded bits (bytes)
};

// Ladder state of one codeword of a batch.
struct LdpcaBatchState {
  int start;                 // first code
  int best;                  // lowest code that succeeded so far (LDPCA_NONE: none)
  int fin;                   // 1 once a group has been elected to finalise the codeword
  int nsucc;                 // successes so far (each takes the next slot)
  unsigned long long mask;   // bit c - start: code c has finished
  int succ_code[4];          // code that filled each slot
  int iters[64];             // BP iterations of code start + k
};

// Arguments of the batched launch (all device pointers).
struct LdpcaBatch {
  LadderDev L_cif, L_qcif;
  XlmDev xt;
  const LdpcaBatchCw *cw;
  LdpcaBatchState *state;
  uint32_t *slot_bits;       // [count * 4 * 198] packed decoded bits of successes
  const float *lr;
  const uint8_t *acc;
  uint8_t *decoded;          // may be null
  int *results;              // [count * 4] rate, first code, accepted code, BP iterations of the ladder
  float *entropy;            // [count] conditional-entropy bound, may be null
  const int *cif, *qcif;     // indices of the CIF and of the QCIF codewords
  int n_cif, n_qcif;
  int last_cif, last_qcif;   // full-rate code index of each ladder
  int *ctr;                  // [2] queue heads (CIF, QCIF), zeroed before the launch
  unsigned long long *work;  // BP iterations run, abandoned and skipped-over codes included
  int max_iter;
};

}  // namespace dvc
