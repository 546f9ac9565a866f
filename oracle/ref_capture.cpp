// Test infrastructure (oracle side): link-time hooks that record the reference
// decoder's per-stage inputs and outputs while it runs in ParallelMode 0.
//
// Built only by oracle/Makefile into oracle/_ref/DvcDec_capture, by linking the
// reference's own unmodified objects with `-Wl,--wrap=<symbol>` so that every
// call from DVC_Decoder.o into a hot-path function goes through the hooks below
// first.  The hooks write a flat record stream (tag, length, payload) to the
// file named by $DVC_CAPTURE; tests/golden/capture.py parses it.
//
// Hooked reference functions (all in DvcDec/src):
//   createSideInfo      sideInfoCreation.cpp:438   -> SI + residue after the call
//   noiseParameter      noiseModel.cpp:9           -> alpha[] after the call
//   noiseDistribution   noiseModel.cpp:77          -> pdf checksum per band
//   condBitProb         noiseModel.cpp:191         -> LR[] per bitplane
//   ComputeCE           LdpcaDecoder.cpp:127       -> entropy per bitplane
//   LdpcaDecoder        LdpcaDecoder.cpp:646       -> inputs/outputs per bitplane
//   reconstruction      reconstruction.cpp:184     -> sideTrans and deblockFlag after the call
//   deblock             deblock.cpp:346            -> frame, flags, modes, past index in; filtered frame out
//   updateSI            sideInfoCreation.cpp:642   -> SI after the call
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>

#include "global.h"

extern int *syndLength;
extern int numCodes;
extern int codeLength;

static FILE *g_out = nullptr;

static FILE *out() {
  if (!g_out) {
    const char *p = getenv("DVC_CAPTURE");
    if (!p) return nullptr;
    g_out = fopen(p, "wb");
  }
  return g_out;
}

static void rec(const char tag[4], const void *a, uint32_t na, const void *b = nullptr, uint32_t nb = 0) {
  FILE *f = out();
  if (!f) return;
  uint32_t n = na + nb;
  fwrite(tag, 1, 4, f);
  fwrite(&n, 4, 1, f);
  if (na) fwrite(a, 1, na, f);
  if (nb) fwrite(b, 1, nb, f);
  fflush(f);
}

static uint64_t fnv_bytes(const void *p, size_t n) {
  const unsigned char *c = (const unsigned char *)p;
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; i++) { h ^= c[i]; h *= 1099511628211ull; }
  return h;
}

extern "C" {

// ---- createSideInfo(int past, int future, int current, SideInfo *si)
void __real__Z14createSideInfoiiiP8SideInfo(int, int, int, SideInfo *);
void __wrap__Z14createSideInfoiiiP8SideInfo(int past, int future, int current, SideInfo *si) {
  __real__Z14createSideInfoiiiP8SideInfo(past, future, current, si);
  int32_t hdr[4] = {past, future, current, FrameSize};
  rec("FRAM", hdr, sizeof hdr);
  rec("SIC0", si->sideInfoFrame, FrameSize);
  rec("RES0", si->residueFrame, FrameSize * 4);
}

// ---- noiseParameter(int *transFrame, float *alpha, unsigned char *BlockModeFlag)
void __real__Z14noiseParameterPiPfPh(int *, float *, unsigned char *);
void __wrap__Z14noiseParameterPiPfPh(int *trans, float *alpha, unsigned char *flags) {
  rec("RTRN", trans, FrameSize * 4);
  rec("MODE", flags, Block88Num);
  __real__Z14noiseParameterPiPfPh(trans, alpha, flags);
  rec("ALPH", alpha, FrameSize * 4);
}

// ---- float *noiseDistribution(int range, int indexInBlk, float *alpha, SMF*, Trans*, SIR*)
float *__real__Z17noiseDistributioniiPfP3SMFP5TransP3SIR(int, int, float *, SMF *, Trans *, SIR *);
float *__wrap__Z17noiseDistributioniiPfP3SMFP5TransP3SIR(int range, int index, float *alpha, SMF *smf, Trans *tr, SIR *sir) {
  float *d = __real__Z17noiseDistributioniiPfP3SMFP5TransP3SIR(range, index, alpha, smf, tr, sir);
  size_t per = (index == 0) ? (size_t)range : (size_t)(2 * range + 1);
  size_t n = per * (size_t)sir->searchCandidate;
  uint64_t h = fnv_bytes(d, n * 4);
  int32_t hdr[4] = {range, index, sir->searchCandidate, (int32_t)per};
  rec("PDFH", hdr, sizeof hdr, &h, 8);
  const char *full = getenv("DVC_CAPTURE_PDF");
  if (full && atoi(full)) rec("PDF_", d, (uint32_t)(n * 4));
  return d;
}

// ---- condBitProb(float *LR, int indexInBlk, int bit, int stepSize, int *reconsTrans, int range, float *dist, SIR*)
void __real__Z11condBitProbPfiiiPiiS_P3SIR(float *, int, int, int, int *, int, float *, SIR *);
void __wrap__Z11condBitProbPfiiiPiiS_P3SIR(float *LR, int index, int bit, int step, int *rt, int range, float *dist, SIR *sir) {
  __real__Z11condBitProbPfiiiPiiS_P3SIR(LR, index, bit, step, rt, range, dist, sir);
  int32_t hdr[4] = {index, bit, step, range};
  rec("CBPH", hdr, sizeof hdr);
}

// ---- float ComputeCE(float *prob)
float __real__Z9ComputeCEPf(float *);
float __wrap__Z9ComputeCEPf(float *prob) {
  float e = __real__Z9ComputeCEPf(prob);
  rec("CENT", &e, 4);
  return e;
}

// ---- LdpcaDecoder(float *LR, unsigned char *accSynd, unsigned char *decoded, int *rate, unsigned char crc, float entropy)
void __real__Z12LdpcaDecoderPfPhS0_Pihf(float *, unsigned char *, unsigned char *, int *, unsigned char, float);
void __wrap__Z12LdpcaDecoderPfPhS0_Pihf(float *LR, unsigned char *acc, unsigned char *dec, int *rate, unsigned char crc, float entropy) {
  // LdpcaDecoder turns LR into log(LR) in place, so record the inputs first.
  int32_t hdr[3] = {codeLength, (int32_t)crc, 0};
  memcpy(&hdr[2], &entropy, 4);
  rec("LDIN", hdr, sizeof hdr);
  rec("LDLR", LR, codeLength * 4);
  rec("LDAS", acc, codeLength);
  __real__Z12LdpcaDecoderPfPhS0_Pihf(LR, acc, dec, rate, crc, entropy);
  rec("LDLL", LR, codeLength * 4);
  rec("LDDE", dec, codeLength);
  int32_t r = *rate;
  rec("LDRT", &r, 4);
}

// ---- reconstruction(int *reconsTrans, int *sideTrans, int indexInBlk, float *alpha, int *stepSize, unsigned char *modes, unsigned char *deblockFlag)
void __real__Z14reconstructionPiS_iPfS_PhS1_(int *, int *, int, float *, int *, unsigned char *, unsigned char *);
void __wrap__Z14reconstructionPiS_iPfS_PhS1_(int *rt, int *st, int index, float *alpha, int *step, unsigned char *modes, unsigned char *dbf) {
  rec("QIDX", rt, FrameSize * 4);
  rec("STIN", st, FrameSize * 4);
  __real__Z14reconstructionPiS_iPfS_PhS1_(rt, st, index, alpha, step, modes, dbf);
  int32_t hdr[2] = {index, step[index]};
  rec("RECH", hdr, sizeof hdr);
  rec("STOU", st, FrameSize * 4);
  rec("DBFL", dbf, FrameSize);
}

// ---- deblock(unsigned char *deblockimg, unsigned char *recon, unsigned char *deblockFlag, unsigned char *type_map, int begin)
void __real__Z7deblockPhS_S_S_i(unsigned char *, unsigned char *, unsigned char *, unsigned char *, int);
void __wrap__Z7deblockPhS_S_S_i(unsigned char *out, unsigned char *recon, unsigned char *flag, unsigned char *modes,
                                int begin) {
  rec("DBIN", recon, FrameSize);
  rec("DBFG", flag, FrameSize);
  rec("DBMD", modes, FrameSize / 64);
  int32_t b = begin;
  rec("DBBG", &b, 4);
  __real__Z7deblockPhS_S_S_i(out, recon, flag, modes, begin);
  rec("DBOU", out, FrameSize);
}

// ---- updateSI(SideInfo *si, unsigned char *recons, int current, int past, int future, SIR*)
void __real__Z8updateSIP8SideInfoPhiiiP3SIR(SideInfo *, unsigned char *, int, int, int, SIR *);
void __wrap__Z8updateSIP8SideInfoPhiiiP3SIR(SideInfo *si, unsigned char *recons, int cur, int past, int fut, SIR *sir) {
  rec("RCIN", recons, FrameSize);
  __real__Z8updateSIP8SideInfoPhiiiP3SIR(si, recons, cur, past, fut, sir);
  rec("SIUP", si->sideInfoFrame, FrameSize);
}

}  // extern "C"
