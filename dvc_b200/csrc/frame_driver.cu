// Batched WZ-frame decoding on the device.  See frame_driver.h.
//
// Order of work for a batch (DVC_Decoder.cpp:26-435 for each frame):
//   side information (createSideInfo) -> residue transform, noise parameters,
//   over-complete transform, ML initialisation, skip copy -> for every band:
//   noise distribution; for every bitplane: conditional bit probabilities, LDPCA
//   ladder (with the bitplane appended to the quantisation indices); then
//   reconstruction + inverse transform, side-information refinement,
//   over-complete transform, motion learning -> final inverse transform.
// Frames run in lockstep over (band, bitplane) steps; a frame whose quantiser
// has no such step is skipped by the kernels, so mixed Q can share a batch.
#include "frame_driver.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "kernels.h"

namespace dvc {

const int kZigzag[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
const int kQTable[9][16] = {
    {0},
    {16, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0, 4, 4, 0, 0},
    {64, 16, 8, 8, 16, 8, 8, 4, 8, 8, 4, 4, 8, 4, 4, 0},
    {64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0},
    {128, 64, 32, 16, 64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 0}};
const int kQBits[9][16] = {
    {0},
    {4, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0},
    {5, 4, 3, 2, 4, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0},
    {5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0, 2, 2, 0, 0},
    {6, 4, 3, 3, 4, 3, 3, 2, 3, 3, 2, 2, 3, 2, 2, 0},
    {6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0},
    {7, 6, 5, 4, 6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 0}};

int qbits_per_block(int q) {
  int s = 0;
  for (int j = 0; j < 16; j++) s += kQBits[q][j];
  return s;
}

// kernels in k_frame.cu
cudaError_t upload_transform_scales(const double *post, const double *pre);
cudaError_t launch_side_info(FrameDev *fr, int nf, int w, int h, cudaStream_t s);
cudaError_t launch_frame_prep(FrameDev *fr, int nf, int w, int h, cudaStream_t s);
cudaError_t launch_noise_dist(FrameDev *fr, int nf, int max_nsir, const XlmDev &xt, int band, int max_range,
                              cudaStream_t s);
cudaError_t launch_cond_bit(FrameDev *fr, int nf, int w, int h, int band, int bit, cudaStream_t s);
cudaError_t launch_band_end(FrameDev *fr, int nf, int w, int h, int max_nsir, int band, const XlmDev &xt,
                            cudaStream_t s);
cudaError_t launch_final_inverse(FrameDev *fr, int nf, int max_nsir, cudaStream_t s);
cudaError_t launch_deblock(FrameDev *fr, int nf, int w, int h, cudaStream_t s);

static bool g_scales_done = false;

// initTransform, transform.cpp:12-61
static cudaError_t ensure_scales() {
  if (g_scales_done) return cudaSuccess;
  const double a = 0.5, b = sqrt(0.4);
  const double a2 = 0.25, b2 = 0.4, ab = a * b;
  const double post[16] = {a2, ab / 2, a2, ab / 2, ab / 2, b2 / 4, ab / 2, b2 / 4,
                           a2, ab / 2, a2, ab / 2, ab / 2, b2 / 4, ab / 2, b2 / 4};
  const double pr[16] = {a2, ab, a2, ab, ab, b2, ab, b2, a2, ab, a2, ab, ab, b2, ab, b2};
  double pre[16];
  for (int i = 0; i < 16; i++) pre[i] = pr[i] * 64.0;
  cudaError_t e = upload_transform_scales(post, pre);
  if (e == cudaSuccess) g_scales_done = true;
  return e;
}

bool Slot::ensure(int w_, int h_, size_t pdf_floats, size_t in_bytes, size_t out_bytes, cudaStream_t a) {
  const size_t fs = (size_t)w_ * h_, n = fs / 16;
  const size_t b16n = fs / 256, b8n = fs / 64, octn = (size_t)(w_ - 3) * (h_ - 3) * 16;
  bool ok = si.ensure(fs, a) && dbf.ensure(fs, a) && residue.ensure(fs * 4, a) && side_trans.ensure(fs * 4, a) &&
            recons_trans.ensure(fs * 4, a) && alpha.ensure(fs * 4, a) && lr.ensure(n * 4, a) &&
            oct.ensure(octn * 2, a) && smf.ensure(n * 81 * 4, a) && pdf.ensure(pdf_floats * 4, a) &&
            mb_mv.ensure(b16n * sizeof(MVd), a) && fmv.ensure(b16n * sizeof(MVd), a) &&
            blk_mv.ensure(b8n * sizeof(MVd), a) && blk_mv2.ensure(b8n * sizeof(MVd), a) && holes.ensure(b16n * 16, a) &&
            mse.ensure(b8n * 8, a) && stats.ensure(32 * 4, a) && in.ensure(in_bytes, a) && out.ensure(out_bytes, a) &&
            db_img.ensure(fs, a) && db_mode.ensure(2 * n, a) && db_bs.ensure(2 * n * 8, a) && si_mv.ensure(2 * n * 4, a);
  w = w_;
  h = h_;
  return ok;
}

void Slot::release() {
  DevBuf *all[] = {&si, &dbf, &residue, &side_trans, &recons_trans, &alpha, &lr, &oct, &smf, &pdf,
                   &mb_mv, &fmv, &blk_mv, &blk_mv2, &holes, &mse, &stats, &in, &out, &db_img, &db_mode, &db_bs,
                   &si_mv};
  for (DevBuf *b : all) b->release();
}

bool FrameBatcher::ensure_pinned(size_t b) {
  if (b <= pinned_bytes_) return true;
  // grow by at least half (and to 4 MB at first), so that a stream of batches
  // of changing sizes rarely frees and pins host memory again
  b = std::max(b, std::max(pinned_bytes_ + pinned_bytes_ / 2, (size_t)4 << 20));
  // freeing pinned memory waits for the whole device: keep the outgrown
  // buffer until release() (growth is geometric, so at most about twice the
  // final size is held)
  if (pinned_) retired_pinned_.push_back(pinned_);
  pinned_ = nullptr;
  pinned_bytes_ = 0;
  if (cudaMallocHost(&pinned_, b) != cudaSuccess) return false;
  pinned_bytes_ = b;
  return true;
}

void FrameBatcher::release() {
  for (cudaEvent_t e : ev_) cudaEventDestroy(e);
  ev_.clear();
  for (auto &s : slots_) s.release();
  slots_.clear();
  frames_dev_.release();
  jobs_dev_.release();
  spec_.release();
  if (pinned_) cudaFreeHost(pinned_);
  for (void *p : retired_pinned_) cudaFreeHost(p);
  retired_pinned_.clear();
  pinned_ = nullptr;
  pinned_bytes_ = 0;
}

static size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

bool FrameBatcher::prepare(Context &ctx, const std::vector<FrameSpec> &frames, cudaStream_t s, int concurrent) {
  const int nf = (int)frames.size();
  nf_ = 0;
  if (nf == 0) return true;
  const int w = frames[0].w, h = frames[0].h;
  const int n = w * h / 16, nb = n / 8, b8n = w * h / 64;
  for (const FrameSpec &f : frames) {
    if (f.w != w || f.h != h) return ctx.fail("a batch must share one frame size");
    if (f.qindex < 1 || f.qindex > 8) return ctx.fail("Qindex out of range 1..8");
    if (!f.past || !f.future || !f.past_ip || !f.future_ip || !f.past_lp || !f.future_lp || !f.recon)
      return ctx.fail("missing device frame pointer");
    // update_si copies the references in 16-byte chunks, the forward motion
    // search reads the low-pass planes in 4-byte words
    if ((((uintptr_t)f.past | (uintptr_t)f.future) & 15u) || (((uintptr_t)f.past_lp | (uintptr_t)f.future_lp) & 3u))
      return ctx.fail("reference frames must be 16-byte aligned (low-pass planes 4-byte)");
    if (!f.crc || !f.acc) return ctx.fail("missing bitplane data");
    if (f.future_idx == f.past_idx) return ctx.fail("past and future reference are the same frame");
  }
  const LadderDev *L = ctx.ladder(n);
  if (!L) return ctx.fail("no LDPCA ladder for " + std::to_string(n) + "-bit codewords");
  if (!ctx.cuda_ok(ensure_scales(), "transform scales")) return false;

  // ---- host-side per-frame constants, WZ block lists and upload packing
  std::vector<FrameDev> fd(nf);
  std::vector<std::vector<int>> plane_base(nf);
  int max_nsir = 0;
  struct Packed {
    size_t mode, sir, sob, crc, acc, pmode, total;
  };
  std::vector<Packed> pk(nf);
  std::vector<int> qb(nf);
  size_t pinned_need = 0;
  for (int f = 0; f < nf; f++) {
    const FrameSpec &F = frames[f];
    qb[f] = qbits_per_block(F.qindex);
    Packed &p = pk[f];
    p.mode = 0;
    p.sir = align16(p.mode + b8n);
    p.sob = align16(p.sir + (size_t)n * 4);
    p.crc = align16(p.sob + (size_t)n * 4);
    p.acc = align16(p.crc + (size_t)qb[f]);
    p.pmode = align16(p.acc + (size_t)qb[f] * nb);
    p.total = align16(p.pmode + b8n);
    pinned_need += p.total;
  }
  const size_t fd_off = pinned_need;
  pinned_need += align16(sizeof(FrameDev) * nf);
  // LDPCA steps: (band, bit) while any frame codes the band
  std::vector<Step> steps;
  for (int band = 0; band < 16; band++) {
    int maxbits = 0;
    for (int f = 0; f < nf; f++) {
      bool coded = true;
      for (int b = 0; b <= band; b++) coded = coded && kQBits[frames[f].qindex][kZigzag[b]] > 0;
      if (coded) maxbits = std::max(maxbits, kQBits[frames[f].qindex][kZigzag[band]]);
    }
    if (maxbits == 0) break;
    for (int bit = maxbits; bit >= 1; bit--) steps.push_back({band, bit});
  }
  const size_t jobs_off = pinned_need;
  pinned_need += align16(sizeof(LdpcaJob) * steps.size() * nf);
  const size_t res_off = pinned_need;
  size_t res_bytes = 0;
  for (int f = 0; f < nf; f++) res_bytes += (size_t)qb[f] * 20;
  pinned_need += align16(res_bytes);
  if (!ensure_pinned(pinned_need)) return ctx.fail("pinned host allocation failed");
  uint8_t *pin = (uint8_t *)pinned_;

  if ((int)slots_.size() < nf) slots_.resize(nf);
  wz_bits0_.assign(nf, 0);
  size_t off = 0;
  for (int f = 0; f < nf; f++) {
    const FrameSpec &F = frames[f];
    const int q = F.qindex;
    FrameDev &D = fd[f];
    memset(&D, 0, sizeof D);
    D.w = w;
    D.h = h;
    D.qindex = q;
    D.skip_mode = F.skip_mode;
    D.intra_mode = F.intra_mode;
    D.ifc = (double)(F.future_idx - F.cur_idx) / (double)(F.future_idx - F.past_idx);
    D.ipc = (double)(F.cur_idx - F.past_idx) / (double)(F.future_idx - F.past_idx);
    D.active = 1;
    D.near_ties = ctx.near_ties.as<unsigned long long>();
    int level_shift[16] = {0};
    for (int j = 1; j < 16; j++)
      if (kQTable[q][j] > 0) level_shift[j] = (kQTable[q][j] - 2) / 2;
    int wz_bits = 0;
    D.step[0] = 1024 / kQTable[q][0];
    D.crange[0] = 1024;
    for (int i = 1; i < 16; i++) {
      if (kQTable[q][i] > 0) {
        D.step[i] = (int)ceil((double)((F.ac_range[i] + 1) << 1) / (double)kQTable[q][i]);
        wz_bits += 10;
        D.crange[i] = (level_shift[i] + 1) * D.step[i] - 1;
      } else {
        D.step[i] = 0;
        D.crange[i] = 0;
      }
    }
    wz_bits0_[f] = wz_bits;
    for (int i = 0; i < 16; i++) {
      D.level_shift[i] = level_shift[i];
      D.qbits[i] = kQBits[q][i];
    }
    size_t pdf_stride = 1024;
    for (int band = 0; band < 16 && kQBits[q][kZigzag[band]] > 0; band++) {
      const int idx = kZigzag[band];
      if (idx == 0) continue;
      if (D.crange[idx] < 0 || D.crange[idx] > (1 << 20)) return ctx.fail("AC range out of bounds");
      pdf_stride = std::max(pdf_stride, (size_t)(2 * D.crange[idx] + 1));
    }
    D.pdf_stride = (int)pdf_stride;
    // packed inputs: mode map, WZ block list (initSIR order), block -> list position, CRCs, syndromes
    uint8_t *P = pin + off;
    const Packed &p = pk[f];
    if (F.mode)
      memcpy(P + p.mode, F.mode, b8n);
    else
      memset(P + p.mode, 0, b8n);
    int *sir = (int *)(P + p.sir), *sob = (int *)(P + p.sob);
    int nsir = 0;
    for (int k = 0; k < n; k++) {
      const int i = k / (w / 4), j = k % (w / 4);
      const uint8_t md = P[p.mode + (i >> 1) * (w / 8) + (j >> 1)];
      if (md == 0) {
        sob[k] = nsir;
        sir[nsir++] = k;
      } else {
        sob[k] = -1;
      }
    }
    D.nsir = nsir;
    max_nsir = std::max(max_nsir, nsir);
    memcpy(P + p.crc, F.crc, qb[f]);
    if (F.past_mode)
      memcpy(P + p.pmode, F.past_mode, b8n);
    else
      memset(P + p.pmode, 0, b8n);
    memcpy(P + p.acc, F.acc, (size_t)qb[f] * nb);
    Slot &S = slots_[f];
    if (!S.ensure(w, h, (size_t)std::max(nsir, 1) * pdf_stride, p.total, (size_t)qb[f] * 20 + 64, alloc_stream_))
      return ctx.fail("device allocation for frame slot failed");
    uint8_t *in = S.in.as<uint8_t>();
    D.mode = in + p.mode;
    D.sir = (const int *)(in + p.sir);
    D.sir_of_blk = (const int *)(in + p.sob);
    D.past = F.past;
    D.future = F.future;
    D.past_lp = F.past_lp;
    D.future_lp = F.future_lp;
    D.past_ip = F.past_ip;
    D.future_ip = F.future_ip;
    D.recon = F.recon;
    D.si = S.si.as<uint8_t>();
    D.dbf = F.deblock_flag ? F.deblock_flag : S.dbf.as<uint8_t>();
    D.residue = S.residue.as<int>();
    D.side_trans = S.side_trans.as<int>();
    D.recons_trans = S.recons_trans.as<int>();
    D.alpha = S.alpha.as<float>();
    D.smf = S.smf.as<float>();
    D.si_mv = S.si_mv.as<int>();
    D.pdf = S.pdf.as<float>();
    D.lr = S.lr.as<float>();
    D.oct = S.oct.as<int16_t>();
    D.mb_mv = S.mb_mv.as<MVd>();
    D.fmv = S.fmv.as<MVd>();
    D.blk_mv = S.blk_mv.as<MVd>();
    D.blk_mv2 = S.blk_mv2.as<MVd>();
    D.holes = S.holes.as<double>();
    D.mse = S.mse.as<double>();
    D.band_mean = S.stats.as<float>();
    D.band_var = S.stats.as<float>() + 16;
    D.deblock = F.deblock ? 1 : 0;
    D.db_qp = std::min(51, std::max(0, F.intra_qp));
    D.db_pow = pow(2, (double)D.db_qp / 6.0);  // deblock.cpp:174, with the host's C library
    D.past_is_wz = F.past_mode != nullptr;
    D.past_mode = in + p.pmode;
    D.db_img = S.db_img.as<uint8_t>();
    D.db_mode = S.db_mode.as<uint8_t>();
    D.db_bs = S.db_bs.as<double>();
    // bitplane index of each (band, bit) in this frame's bitstream order
    plane_base[f].assign(16, 0);
    int acc_planes = 0;
    for (int band = 0; band < 16; band++) {
      plane_base[f][band] = acc_planes;
      acc_planes += kQBits[q][kZigzag[band]];
    }
    if (!ctx.cuda_ok(cudaMemcpyAsync(S.in.p, P, p.total, cudaMemcpyHostToDevice, s), "H2D frame inputs")) return false;
    off += p.total;
  }
  FrameDev *fd_pin = (FrameDev *)(pin + fd_off);
  memcpy(fd_pin, fd.data(), sizeof(FrameDev) * nf);
  if (!frames_dev_.ensure(sizeof(FrameDev) * nf, alloc_stream_)) return ctx.fail("device allocation failed");
  if (!ctx.cuda_ok(cudaMemcpyAsync(frames_dev_.p, fd_pin, sizeof(FrameDev) * nf, cudaMemcpyHostToDevice, s),
                   "H2D frame descriptors"))
    return false;
  FrameDev *fdev = frames_dev_.as<FrameDev>();

  // LDPCA jobs for every step
  LdpcaJob *jobs = (LdpcaJob *)(pin + jobs_off);
  plane_of_.assign(steps.size() * nf, -1);
  for (size_t si = 0; si < steps.size(); si++) {
    const int band = steps[si].band, bit = steps[si].bit, index = kZigzag[band];
    for (int f = 0; f < nf; f++) {
      LdpcaJob &J = jobs[si * nf + f];
      memset(&J, 0, sizeof J);
      const int q = frames[f].qindex;
      bool coded = true;
      for (int b = 0; b <= band; b++) coded = coded && kQBits[q][kZigzag[b]] > 0;
      if (!coded || bit > kQBits[q][index]) continue;
      const int plane = plane_base[f][band] + (kQBits[q][index] - bit);
      plane_of_[si * nf + f] = plane;
      Slot &S = slots_[f];
      J.active = 1;
      J.lr = fd[f].lr;
      J.acc = S.in.as<uint8_t>() + pk[f].acc + (size_t)plane * nb;
      J.crc = frames[f].crc[plane];
      J.result = S.out.as<int>() + plane * 4;
      J.entropy = (float *)(S.out.as<uint8_t>() + (size_t)qb[f] * 16) + plane;
      J.recons_trans = fd[f].recons_trans;
      J.mode = fd[f].mode;
      J.w = w;
      J.index_in_blk = index;
    }
  }
  if (!jobs_dev_.ensure(sizeof(LdpcaJob) * std::max<size_t>(1, steps.size() * nf), alloc_stream_))
    return ctx.fail("device allocation failed");
  if (!steps.empty() &&
      !ctx.cuda_ok(cudaMemcpyAsync(jobs_dev_.p, jobs, sizeof(LdpcaJob) * steps.size() * nf, cudaMemcpyHostToDevice, s),
                   "H2D jobs"))
    return false;

  // speculative ladder width: spread each codeword over idle SMs when the batch is small
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device);
    // speculation pays even on a full GPU (it shortens the slowest codeword of
    // every lockstep bitplane step); on the bench's 640 CIF frames the
    // autotuner measured 4 blocks per codeword fastest (911 ms a step, against
    // 956 at 8, 966 at 2 and 1168 at 1); at least 4 blocks per codeword, more
    // when SMs are idle.  DVC_LDPCA_SPEC_FLOOR replaces the floor of 4 (the
    // autotuner's setting), DVC_LDPCA_SPEC fixes the width outright
    int floor_k = 4;
    if (const char *e = getenv("DVC_LDPCA_SPEC_FLOOR")) floor_k = std::max(1, std::min(32, atoi(e)));
    int k = std::max(floor_k, sms / std::max(1, std::max(nf, concurrent)));
    if (const char *e = getenv("DVC_LDPCA_SPEC")) k = atoi(e);
    spec_k_ = std::max(1, std::min(32, k));
    if (!spec_.ensure(ldpca_spec_scratch_bytes(n, nf, spec_k_), alloc_stream_))
      return ctx.fail("device allocation failed");
    if (!ctx.cuda_ok(ldpca_spec_reset(ldpca_spec_carve(spec_.p, nf, spec_k_), nf, spec_k_, s), "LDPCA scratch"))
      return false;
  }
  steps_ = steps;
  fd_ = fd;
  qb_ = qb;
  spec_copy_ = frames;
  nf_ = nf;
  w_ = w;
  h_ = h;
  max_nsir_ = max_nsir;
  res_off_ = res_off;
  L_ = L;
  return true;
}

long long FrameBatcher::launches_per_execute() const {
  if (nf_ == 0) return 0;
  long long bands = 0;
  for (size_t i = 0; i < steps_.size(); i++)
    if (i == 0 || steps_[i].band != steps_[i - 1].band) bands++;
  bool deblock = false;
  for (const FrameDev &f : fd_) deblock = deblock || f.deblock;
  // side info 8, prep 6, per band 1 + 5, per step condBitProb + ladder, final 1, deblocking 5
  return 8 + 6 + bands * 6 + (long long)steps_.size() * 2 + 1 + (deblock ? 5 : 0);
}

bool FrameBatcher::execute(Context &ctx, cudaStream_t s, int max_iter, ProfileStats *prof) {
  if (nf_ == 0) return true;
  const int nf = nf_, w = w_, h = h_, max_nsir = max_nsir_;
  const std::vector<FrameDev> &fd = fd_;
  const std::vector<FrameSpec> &frames = spec_copy_;
  const std::vector<Step> &steps = steps_;
  const LadderDev *L = L_;
  FrameDev *fdev = frames_dev_.as<FrameDev>();
  for (int f = 0; f < nf; f++) {
    if (!ctx.cuda_ok(cudaMemsetAsync(fd[f].recons_trans, 0, (size_t)w * h * 4, s), "memset")) return false;
    if (!ctx.cuda_ok(cudaMemsetAsync(fd[f].si_mv, 0xff, (size_t)w * h / 16 * 8, s), "memset")) return false;
    if (!ctx.cuda_ok(cudaMemsetAsync(fd[f].dbf, 0, (size_t)w * h, s), "memset")) return false;
    if (!ctx.cuda_ok(cudaMemsetAsync(fd[f].alpha, 0, (size_t)w * h * 4, s), "memset")) return false;
  }
  ev_used_ = 0;
  if (prof)
    while (ev_.size() < 2 * steps.size()) {
      cudaEvent_t e;
      if (!ctx.cuda_ok(cudaEventCreate(&e), "event")) return false;
      ev_.push_back(e);
    }
  // ---- the decode
  if (!ctx.cuda_ok(launch_side_info(fdev, nf, w, h, s), "side information")) return false;
  if (!ctx.cuda_ok(launch_frame_prep(fdev, nf, w, h, s), "frame preparation")) return false;
  for (int f = 0; f < nf; f++) {
    if (frames[f].dbg_si_initial &&
        !ctx.cuda_ok(cudaMemcpyAsync(frames[f].dbg_si_initial, fd[f].si, (size_t)w * h, cudaMemcpyDeviceToDevice, s),
                     "debug copy"))
      return false;
    if (frames[f].dbg_alpha &&
        !ctx.cuda_ok(cudaMemcpyAsync(frames[f].dbg_alpha, fd[f].alpha, (size_t)w * h * 4, cudaMemcpyDeviceToDevice, s),
                     "debug copy"))
      return false;
  }
  size_t si = 0;
  while (si < steps.size()) {
    const int band = steps[si].band;
    int max_range = 0;
    for (int f = 0; f < nf; f++) max_range = std::max(max_range, fd[f].crange[kZigzag[band]]);
    if (!ctx.cuda_ok(launch_noise_dist(fdev, nf, max_nsir, ctx.xlm, band, max_range, s), "noise distribution"))
      return false;
    for (; si < steps.size() && steps[si].band == band; si++) {
      if (!ctx.cuda_ok(launch_cond_bit(fdev, nf, w, h, band, steps[si].bit, s), "conditional bit probability"))
        return false;
      for (int f = 0; f < nf; f++)
        if (frames[f].dbg_lr && plane_of_[si * nf + f] >= 0) {
          const size_t n = (size_t)w * h / 16;
          if (!ctx.cuda_ok(cudaMemcpyAsync(frames[f].dbg_lr + (size_t)plane_of_[si * nf + f] * n, fd[f].lr, n * 4,
                                           cudaMemcpyDeviceToDevice, s),
                           "debug copy"))
            return false;
        }
      if (prof) cudaEventRecord(ev_[ev_used_], s);
      if (!ctx.cuda_ok(launch_ldpca_spec(*L, jobs_dev_.as<LdpcaJob>() + si * nf, nf, ctx.xlm, max_iter, spec_k_,
                                         ldpca_spec_carve(spec_.p, nf, spec_k_), s),
                       "LDPCA"))
        return false;
      if (prof) {
        cudaEventRecord(ev_[ev_used_ + 1], s);
        ev_used_ += 2;
        prof->ldpca_launches++;
        prof->ldpca_codewords += nf;
      }
    }
    if (!ctx.cuda_ok(launch_band_end(fdev, nf, w, h, max_nsir, band, ctx.xlm, s), "band reconstruction")) return false;
  }
  if (!ctx.cuda_ok(launch_final_inverse(fdev, nf, max_nsir, s), "inverse transform")) return false;
  bool any_deblock = false;
  for (int f = 0; f < nf; f++) any_deblock = any_deblock || fd[f].deblock;
  if (any_deblock && !ctx.cuda_ok(launch_deblock(fdev, nf, w, h, s), "deblocking")) return false;
  for (int f = 0; f < nf; f++)
    if (frames[f].dbg_si_final &&
        !ctx.cuda_ok(cudaMemcpyAsync(frames[f].dbg_si_final, fd[f].si, (size_t)w * h, cudaMemcpyDeviceToDevice, s),
                     "debug copy"))
      return false;

  if (prof) prof->kernel_launches += launches_per_execute();
  return true;
}

void FrameBatcher::harvest(ProfileStats *prof) {
  for (int i = 0; i + 1 < ev_used_; i += 2) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ev_[i], ev_[i + 1]) == cudaSuccess && prof) prof->ldpca_ms += ms;
  }
  ev_used_ = 0;
}

bool FrameBatcher::enqueue_results(Context &ctx, cudaStream_t s) {
  uint8_t *rp = (uint8_t *)pinned_ + res_off_;
  size_t ro = 0;
  for (int f = 0; f < nf_; f++) {
    if (!ctx.cuda_ok(cudaMemcpyAsync(rp + ro, slots_[f].out.p, (size_t)qb_[f] * 20, cudaMemcpyDeviceToHost, s), "D2H"))
      return false;
    ro += (size_t)qb_[f] * 20;
  }
  return true;
}

void FrameBatcher::read_results(std::vector<FrameResult> &results) {
  results.assign(nf_, FrameResult());
  const uint8_t *rp = (const uint8_t *)pinned_ + res_off_;
  size_t ro = 0;
  for (int f = 0; f < nf_; f++) {
    results[f].wz_bits = wz_bits0_[f];
    const int *r = (const int *)(rp + ro);
    const float *e = (const float *)(rp + ro + (size_t)qb_[f] * 16);
    results[f].planes.assign(r, r + qb_[f] * 4);
    results[f].entropy.assign(e, e + qb_[f]);
    for (int p = 0; p < qb_[f]; p++) results[f].wz_bits += r[4 * p];
    ro += (size_t)qb_[f] * 20;
  }
}

size_t FrameBatcher::device_bytes() const {
  size_t b = frames_dev_.bytes + jobs_dev_.bytes + spec_.bytes;
  for (const Slot &S : slots_) {
    const DevBuf *all[] = {&S.si, &S.dbf, &S.residue, &S.side_trans, &S.recons_trans, &S.alpha, &S.lr, &S.oct,
                           &S.smf, &S.pdf, &S.mb_mv, &S.fmv, &S.blk_mv, &S.blk_mv2, &S.holes, &S.mse, &S.stats,
                           &S.in, &S.out};
    for (const DevBuf *d : all) b += d->bytes;
  }
  return b;
}

bool FrameBatcher::collect(Context &ctx, std::vector<FrameResult> &results, cudaStream_t s) {
  if (!enqueue_results(ctx, s)) return false;
  if (!ctx.cuda_ok(cudaStreamSynchronize(s), "decode")) return false;
  read_results(results);
  return true;
}

bool FrameBatcher::decode(Context &ctx, const std::vector<FrameSpec> &frames, std::vector<FrameResult> &results,
                          cudaStream_t s, int max_iter, ProfileStats *prof) {
  results.clear();
  if (frames.empty()) return true;
  if (!(prepare(ctx, frames, s) && execute(ctx, s, max_iter, prof) && collect(ctx, results, s))) return false;
  harvest(prof);
  return true;
}

}  // namespace dvc
