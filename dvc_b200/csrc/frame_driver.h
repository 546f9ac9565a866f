// Host driver of batched WZ-frame decoding on the device.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "context.h"
#include "frame_types.h"

namespace dvc {

// quantiser tables and derived per-frame constants (reconstruction.cpp:9-78,
// wzbitstream.cpp:165-175, DVC_Decoder.cpp:139-152)
extern const int kQTable[9][16];
extern const int kQBits[9][16];
extern const int kZigzag[16];
int qbits_per_block(int q);

// One WZ frame of a batch.  Reference frames and the output live on the device.
struct FrameSpec {
  int w = 0, h = 0, qindex = 0;
  const uint8_t *past = nullptr, *future = nullptr;        // device [w*h]
  const uint8_t *past_lp = nullptr, *future_lp = nullptr;  // device [w*h]
  const uint8_t *past_ip = nullptr, *future_ip = nullptr;  // device [4*w*h]
  int past_idx = 0, future_idx = 0, cur_idx = 0;
  const uint8_t *mode = nullptr;  // host [w*h/64], null = every block WZ
  int skip_mode = 0, intra_mode = 0;
  int ac_range[16] = {0};
  const uint8_t *crc = nullptr;   // host [qbits]
  const uint8_t *acc = nullptr;   // host [qbits*w*h/128]
  uint8_t *recon = nullptr;       // device [w*h]; intra blocks filled in by the caller
  uint8_t *deblock_flag = nullptr;  // device [w*h] out, or null
  int deblock = 0, intra_qp = 0;    // deblocking filter after decoding, with IntraQP thresholds
  const uint8_t *past_mode = nullptr;  // host [w*h/64] modes of a WZ past reference, null for a key frame
  // optional device copies of intermediate stages (stage-level parity checks)
  uint8_t *dbg_si_initial = nullptr;  // side information after createSideInfo + intra copy
  float *dbg_alpha = nullptr;         // noise parameters
  uint8_t *dbg_si_final = nullptr;    // side information after the last refinement
  float *dbg_lr = nullptr;            // [qbits * w*h/16] condBitProb likelihood ratios of every bitplane
};

struct FrameResult {
  int wz_bits = 0;                // 10 per coded AC band + sum over bitplanes of (m+8)
  std::vector<int> planes;        // per bitplane: rate, first code, accepted code, BP iterations
  std::vector<float> entropy;     // per bitplane conditional-entropy bound
};

struct Slot {
  int w = 0, h = 0;
  DevBuf si, dbf, residue, side_trans, recons_trans, alpha, lr, oct, smf, pdf;
  DevBuf mb_mv, fmv, blk_mv, blk_mv2, holes, mse, stats, in, out;
  DevBuf db_img, db_mode, db_bs;  // deblocking: filtered copy, per-edge mode and strength
  DevBuf si_mv;                   // side-info refinement: last best candidate per WZ block and reference
  bool ensure(int w, int h, size_t pdf_floats, size_t in_bytes, size_t out_bytes, cudaStream_t alloc = nullptr);
  void release();
};

// Kernel-level measurements, filled while Context-level profiling is on.
struct ProfileStats {
  double ldpca_ms = 0;      // summed CUDA-event time of LDPCA ladder launches
  long long ldpca_launches = 0, ldpca_codewords = 0, bp_iterations = 0;
  long long kernel_launches = 0;  // every kernel this library launched
};

class FrameBatcher {
 public:
  // prepare: per-frame constants, block lists, packed inputs, descriptors and
  // LDPCA jobs, uploaded once; execute: the kernels only (no host transfer, no
  // synchronisation); collect: per-bitplane results to the host.
  // concurrent_frames: frames expected to decode on the device at the same time
  // (this batch included; 0 = this batch alone), which sets the speculation width
  bool prepare(Context &ctx, const std::vector<FrameSpec> &frames, cudaStream_t stream, int concurrent_frames = 0);
  bool execute(Context &ctx, cudaStream_t stream, int max_iter = 50, ProfileStats *prof = nullptr);
  bool collect(Context &ctx, std::vector<FrameResult> &results, cudaStream_t stream);
  // asynchronous form of collect: enqueue the result copies on the stream, and
  // after the stream has passed them (event or sync) parse them on the host
  bool enqueue_results(Context &ctx, cudaStream_t stream);
  void read_results(std::vector<FrameResult> &results);
  // device bytes held by the batcher's slots
  size_t device_bytes() const;
  // after the stream has been synchronised: add the recorded LDPCA event times to prof
  void harvest(ProfileStats *prof);
  bool decode(Context &ctx, const std::vector<FrameSpec> &frames, std::vector<FrameResult> &results,
              cudaStream_t stream, int max_iter = 50, ProfileStats *prof = nullptr);
  void release();
  size_t slots() const { return slots_.size(); }
  // grow device buffers in the order of this stream (the batcher is only used
  // on it), so that a growth does not wait for other streams' work
  void set_alloc_stream(cudaStream_t s) { alloc_stream_ = s; }
  int frames() const { return nf_; }
  // launches execute() issues (for the launch counter)
  long long launches_per_execute() const;

 private:
  std::vector<Slot> slots_;
  DevBuf frames_dev_, jobs_dev_, spec_;
  cudaStream_t alloc_stream_ = nullptr;
  int spec_k_ = 1;
  void *pinned_ = nullptr;
  size_t pinned_bytes_ = 0;
  std::vector<void *> retired_pinned_;  // outgrown pinned buffers, freed by release()
  bool ensure_pinned(size_t b);
  // prepared state
  struct Step {
    int band, bit;
  };
  std::vector<Step> steps_;
  std::vector<FrameDev> fd_;
  std::vector<int> qb_, wz_bits0_;
  std::vector<int> plane_of_;  // [step * frames + frame]: the frame's bitplane decoded at that step, or -1
  std::vector<const FrameSpec *> specs_;
  std::vector<FrameSpec> spec_copy_;
  int nf_ = 0, w_ = 0, h_ = 0, max_nsir_ = 0;
  size_t res_off_ = 0;
  const LadderDev *L_ = nullptr;
  std::vector<cudaEvent_t> ev_;  // start/stop pairs of the LDPCA launches of one execute()
  int ev_used_ = 0;
};

}  // namespace dvc
