// Per-frame device descriptor shared by the frame kernels and the host driver.
#pragma once
#include <stdint.h>

namespace dvc {

// motion vector as the reference keeps it (global.h:118-126): past/future
// block positions and their difference, all doubles
struct MVd {
  double px, py, fx, fy, vx, vy;
};

struct FrameDev {
  int w, h, qindex, nsir, skip_mode, intra_mode;
  double ifc, ipc;  // (future-cur)/(future-past), (cur-past)/(future-past)
  // reference frames: reconstruction, 3x3 low-pass, 2x half-pel interpolation
  const uint8_t *past, *future, *past_lp, *future_lp, *past_ip, *future_ip;
  const uint8_t *mode;        // [w*h/64] 0 WZ, 1 intra, 2 skip
  const int *sir;             // [nsir] raster index of each WZ 4x4 block (initSIR order)
  const int *sir_of_blk;      // [w*h/16] WZ list position or -1
  int step[16], crange[16], level_shift[16], qbits[16];
  // state and outputs
  uint8_t *recon, *si, *dbf;
  int *residue, *side_trans, *recons_trans;
  float *alpha, *smf, *pdf, *lr;
  int *si_mv;                 // [2*nsir] last refinement's best candidate index, past then future (-1: none)
  int16_t *oct;               // [(h-3)*(w-3)*16] over-complete transform of the side information
  MVd *mb_mv, *fmv, *blk_mv, *blk_mv2;
  double *holes, *mse;        // [b16n*2], [b88n]
  float *band_mean, *band_var;  // [16]
  int pdf_stride;             // floats per WZ block row of pdf
  // deblocking (deblock.cpp:346-386): on/off, IntraQP, 2^(IntraQP/6) from the
  // host's pow, the past reference's modes when it is a WZ frame
  int deblock, db_qp, past_is_wz;
  double db_pow;
  const uint8_t *past_mode;   // [w*h/64]
  uint8_t *db_img, *db_mode;  // [w*h] filtered copy; [2*w*h/16] edge mode (vertical edges, then horizontal)
  double *db_bs;              // [2*w*h/16] edge strength
  // reconstruction steps whose rounding could depend on the last bits of exp
  // (counted by recon_kernel; null: not counted)
  unsigned long long *near_ties;
  int active;                 // 0: the descriptor is a placeholder, every kernel skips it
};

}  // namespace dvc
