// The reference-side binding of libdvc_b200, compiled: the reference's own
// DvcDec (its main, configuration, bitstream, intra, frame I/O and RD report
// objects, unmodified) with the WZ-frame decode of ParallelMode 2/3 routed to
// this repository's GPU library.
//
// Built by oracle/Makefile into oracle/_ref/DvcDec_b200: the reference's
// objects (its configuration parser compiled with -DCUDA, as in its GPU build,
// so that ParallelMode 2 and 3 are accepted: configfile.cpp:278-284) are linked
// with -Wl,--wrap=decodeGOP, so main's calls of decodeGOP
// (DvcDec/src/main.cpp:132-142) come here.  With ParallelMode 0 or 1 the call
// goes on to the reference's own decodeGOP (DVC_Decoder.cpp:26-474).  With
// ParallelMode 2 or 3 this function does what decodeGOP does around the
// decode (DVC_Decoder.cpp:38-46 and 454-473: the intra blocks by the
// reference's intraRecon, the rate, the timing, the PSNR, the recursion over
// the GOP) and hands the frame itself to dvc_decode_wz_frames: side
// information, noise model, LDPCA ladder, reconstruction, refinement, motion
// learning and the deblocking filter on the GPU.  skipGOP (the intra replay of
// -startFrame) is the reference's own.
//
// The library's context is created on the first call, on the GPU of -GPUid,
// with the ladder data from $DVC_B200_DATA and the table cache in
// $DVC_B200_TABLES (both required: the library's dvc_b200/ladders and
// dvc_b200/_tables directories).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "global.h"
#include "frame.h"
#include "intra.h"
#include "reconstruction.h"

#include "../include/dvc_b200.h"

extern "C" void __real__Z9decodeGOPii(int begin, int end);

static dvc_ctx *g_ctx = nullptr;

static dvc_ctx *context() {
  if (g_ctx) return g_ctx;
  const char *data = getenv("DVC_B200_DATA");
  const char *tables = getenv("DVC_B200_TABLES");
  if (!data || !tables) {
    fprintf(stderr, "DvcDec_b200: set DVC_B200_DATA and DVC_B200_TABLES\n");
    exit(2);
  }
  if (dvc_create(data, tables, codingOption.GPUid < 0 ? 0 : codingOption.GPUid, &g_ctx) != DVC_OK) {
    fprintf(stderr, "DvcDec_b200: GPU set-up failed: %s\n", dvc_last_error(g_ctx));
    exit(2);
  }
  return g_ctx;
}

extern "C" void __wrap__Z9decodeGOPii(int begin, int end) {
  if (codingOption.ParallelMode < 2) {
    __real__Z9decodeGOPii(begin, end);
    return;
  }
  const int m = (begin + end) / 2;
  if (m <= begin) return;
  TimeStamp st_time, end_time;
  timeStart(&st_time);
  decodedFrames[m].isWZFrame = 1;
  EncodedFrame &E = encodedFrames[m];
  // 1. intra blocks (DVC_Decoder.cpp:41-46)
  if (E.intraMode) {
    intraRecon(decodedFrames[m].reconsFrame, &E);
    E.intraBlockBits += IntraBS.frame_bitoffset - IntraBS.prev_frame_bitoffset;
    IntraBS.prev_frame_bitoffset = IntraBS.frame_bitoffset;
  }
  // 2-7. the WZ decode on the GPU
  const int nb = Block44Num / 8;
  std::vector<uint8_t> acc((size_t)QbitsNumPerBlk * nb);
  for (int j = 0; j < QbitsNumPerBlk; j++) memcpy(&acc[(size_t)j * nb], E.AccumulatedSyndrome[j], nb);
  dvc_wz_frame f;
  memset(&f, 0, sizeof f);
  f.width = codingOption.FrameWidth;
  f.height = codingOption.FrameHeight;
  f.qindex = codingOption.Qindex;
  f.past_idx = begin;
  f.future_idx = end;
  f.cur_idx = m;
  f.past = decodedFrames[begin].reconsFrame;
  f.future = decodedFrames[end].reconsFrame;
  f.mode = E.BlockModeFlag;
  f.skip_mode = E.skipMode;
  f.intra_mode = E.intraMode;
  f.ac_range = E.ACRange;
  f.crc = E.CRC;
  f.acc_synd = acc.data();
  f.recon = decodedFrames[m].reconsFrame;
  f.deblock = codingOption.DeblockingMode;
  f.intra_qp = codingOption.IntraQP;
  f.past_mode = decodedFrames[begin].isWZFrame ? encodedFrames[begin].BlockModeFlag : nullptr;
  if (dvc_decode_wz_frames(context(), 1, &f) != DVC_OK) {
    fprintf(stderr, "DvcDec_b200: decoding frame %d failed: %s\n", m, dvc_last_error(g_ctx));
    exit(2);
  }
  // 8. rate, time, PSNR (DVC_Decoder.cpp:131, 147, 269, 454-456)
  decodedFrames[m].bitRate = E.skipBlockBits + E.intraBlockBits + f.wz_bits;
  decodedFrames[m].decodeTime = timeElapse(st_time, &end_time);
  decodedFrames[m].PSNR = psnr(decodedFrames[m].reconsFrame, oriFrames[m]);
  __wrap__Z9decodeGOPii(begin, m);
  __wrap__Z9decodeGOPii(m, end);
}
