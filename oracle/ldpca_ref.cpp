// Test infrastructure (oracle side): the reference's own LdpcaDecoder, callable
// per codeword through ctypes, for LDPCA known-answer fixtures that no decoded
// sequence reaches (full-rate codewords, the batched codeword microbenchmark).
//
// Built only by oracle/Makefile into oracle/_ref/libldpcaref.so from the
// reference's unmodified decoder objects.  The reference keeps its ladder in
// process globals (ReadLdpcaLadderFile_LdpcaDecoder.cpp:12-20) read by
// ReadLadder_decoder (:131-220), and its BP scratch in buffers allocated by
// initLdpcaBuffer (LdpcaDecoder.cpp:145-153); ldpcaref_load sets both up for
// one codeword length, in ParallelMode 0 (the sequential decoder,
// LdpcaDecoder.cpp:718-720).  Loading another length replaces the first.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "global.h"
#include "LdpcaDecoder.h"

extern int codeLength;
extern float *codeRate;
extern int numCodes;

void ReadLadder_decoder(char *LadderFileName, char *InverseHmatrixFileName);

extern "C" {

// Read the ladder (.lad) and inverse-H (.bin) files of one codeword length.
// Returns the code length read, or -1.
int ldpcaref_load(const char *lad, const char *inv) {
  FILE *a = fopen(lad, "r"), *b = fopen(inv, "rb");
  if (!a || !b) {
    if (a) fclose(a);
    if (b) fclose(b);
    return -1;
  }
  fclose(a);
  fclose(b);
  codingOption.ParallelMode = 0;
  ReadLadder_decoder(const_cast<char *>(lad), const_cast<char *>(inv));
  initLdpcaBuffer();
  return codeLength;
}

// The ladder's rate of code c (codeRate[c] = syndLength/N as float).
float ldpcaref_code_rate(int c) { return (c >= 0 && c < numCodes) ? codeRate[c] : -1.0f; }

int ldpcaref_num_codes(void) { return numCodes; }

// ComputeCE (LdpcaDecoder.cpp:127-143): the conditional-entropy rate bound of
// the likelihood ratios lr[N].
float ldpcaref_compute_ce(const float *lr) { return ComputeCE(const_cast<float *>(lr)); }

// One LdpcaDecoder call (LdpcaDecoder.cpp:646-771).  lr[N] is the intrinsic
// likelihood ratio p0/p1 (copied: the reference takes its log in place),
// acc_bits[N] the accumulated syndrome one bit per byte (ByteToBit layout),
// bound the rate lower bound that selects the first code.  Writes the decoded
// bits and returns the rate (syndrome length + 8).
int ldpcaref_decode(const float *lr, const unsigned char *acc_bits, unsigned char crc, float bound,
                    unsigned char *decoded) {
  float *l = (float *)malloc(sizeof(float) * codeLength);
  unsigned char *acc = (unsigned char *)malloc(codeLength);
  memcpy(l, lr, sizeof(float) * codeLength);
  memcpy(acc, acc_bits, codeLength);
  int rate = 0;
  LdpcaDecoder(l, acc, decoded, &rate, crc, bound);
  free(l);
  free(acc);
  return rate;
}
}
