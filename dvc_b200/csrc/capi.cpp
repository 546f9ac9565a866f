// C ABI of libdvc_b200.so (declared in include/dvc_b200.h).
#include "../../include/dvc_b200.h"

#include <string.h>

#include <new>
#include <vector>

#include <algorithm>
#include <array>
#include <map>

#include "context.h"
#include "frame_driver.h"
#include "kernels.h"

struct dvc_ctx {
  dvc::Context c;
  dvc::FrameBatcher batcher;
  // device copies of host frames handed to dvc_decode_wz_frames
  std::vector<dvc::DevBuf> ref, lp, ip, out, dbf;
  dvc::DevBuf dbg;
};

namespace dvc {
cudaError_t launch_ref_planes(const uint8_t *recon, int w, int h, uint8_t *lp, uint8_t *ip, cudaStream_t s);
Context *context_of(dvc_ctx *ctx) { return &ctx->c; }
}

using dvc::Context;

static int cuda_status(Context &c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return DVC_OK;
  c.err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? DVC_E_NOMEM : DVC_E_CUDA;
}

extern "C" int dvc_create(const char *data_dir, const char *table_dir, int device, dvc_ctx **out) {
  if (!out || !data_dir) return DVC_E_ARG;
  *out = nullptr;
  dvc_ctx *h = new (std::nothrow) dvc_ctx();
  if (!h) return DVC_E_NOMEM;
  if (!h->c.init(data_dir, table_dir, device)) {
    // keep the handle so the caller can read the message
    *out = h;
    return h->c.err.find("CUDA") != std::string::npos || h->c.err.find("cuda") != std::string::npos ? DVC_E_CUDA
                                                                                                      : DVC_E_DATA;
  }
  *out = h;
  return DVC_OK;
}

extern "C" void dvc_destroy(dvc_ctx *ctx) {
  if (!ctx) return;
  ctx->batcher.release();
  for (auto *v : {&ctx->ref, &ctx->lp, &ctx->ip, &ctx->out, &ctx->dbf})
    for (auto &b : *v) b.release();
  ctx->dbg.release();
  ctx->c.release();
  delete ctx;
}

extern "C" const char *dvc_last_error(dvc_ctx *ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

static int ldpca_run(Context &c, int n, int count, const float *lr, const uint8_t *acc, const uint8_t *crc,
                     uint8_t *decoded, int *results, float *entropy, int max_iter, const float *given_entropy,
                     float *llr_back) {
  const dvc::LadderDev *L = c.ladder(n);
  if (!L) {
    c.err = "no ladder for codeword length " + std::to_string(n);
    return DVC_E_ARG;
  }
  if (count <= 0 || !lr || !acc || !crc || !results || max_iter <= 0) {
    c.err = "dvc_ldpca_decode: bad arguments";
    return DVC_E_ARG;
  }
  const size_t nb = (size_t)n / 8;
  if (!c.ld_lr.ensure((size_t)count * n * 4) || !c.ld_acc.ensure((size_t)count * nb) ||
      !c.ld_dec.ensure((size_t)count * n) || !c.ld_res.ensure((size_t)count * 16) ||
      !c.ld_ent.ensure((size_t)count * 4) || !c.ld_jobs.ensure((size_t)count * sizeof(dvc::LdpcaJob))) {
    c.err = "device allocation failed";
    return DVC_E_NOMEM;
  }
  std::vector<dvc::LdpcaJob> jobs(count);
  for (int i = 0; i < count; i++) {
    dvc::LdpcaJob &j = jobs[i];
    memset(&j, 0, sizeof j);
    j.active = 1;
    j.lr = c.ld_lr.as<float>() + (size_t)i * n;
    j.acc = c.ld_acc.as<uint8_t>() + (size_t)i * nb;
    j.crc = crc[i];
    j.decoded = c.ld_dec.as<uint8_t>() + (size_t)i * n;
    j.result = c.ld_res.as<int>() + (size_t)i * 4;
    j.entropy = c.ld_ent.as<float>() + i;
    if (given_entropy) {
      j.use_given_entropy = 1;
      j.given_entropy = given_entropy[i];
    }
    if (llr_back) j.llr_out = c.ld_lr.as<float>() + (size_t)i * n;
  }
  cudaStream_t s = c.stream;
  int st;
  if ((st = cuda_status(c, cudaMemcpyAsync(c.ld_lr.p, lr, (size_t)count * n * 4, cudaMemcpyHostToDevice, s), "H2D lr")))
    return st;
  if ((st = cuda_status(c, cudaMemcpyAsync(c.ld_acc.p, acc, (size_t)count * nb, cudaMemcpyHostToDevice, s), "H2D acc")))
    return st;
  if ((st = cuda_status(c, cudaMemcpyAsync(c.ld_jobs.p, jobs.data(), jobs.size() * sizeof(dvc::LdpcaJob),
                                           cudaMemcpyHostToDevice, s),
                        "H2D jobs")))
    return st;
  if ((st = cuda_status(c, dvc::launch_ldpca(*L, c.ld_jobs.as<dvc::LdpcaJob>(), count, c.xlm, max_iter, s), "ldpca launch")))
    return st;
  if (decoded &&
      (st = cuda_status(c, cudaMemcpyAsync(decoded, c.ld_dec.p, (size_t)count * n, cudaMemcpyDeviceToHost, s), "D2H dec")))
    return st;
  if ((st = cuda_status(c, cudaMemcpyAsync(results, c.ld_res.p, (size_t)count * 16, cudaMemcpyDeviceToHost, s), "D2H res")))
    return st;
  if (entropy &&
      (st = cuda_status(c, cudaMemcpyAsync(entropy, c.ld_ent.p, (size_t)count * 4, cudaMemcpyDeviceToHost, s), "D2H ent")))
    return st;
  if (llr_back &&
      (st = cuda_status(c, cudaMemcpyAsync(llr_back, c.ld_lr.p, (size_t)count * n * 4, cudaMemcpyDeviceToHost, s),
                        "D2H llr")))
    return st;
  if ((st = cuda_status(c, cudaStreamSynchronize(s), "ldpca sync"))) return st;
  return DVC_OK;
}

extern "C" int dvc_ldpca_decode(dvc_ctx *ctx, int n, int count, const float *lr, const uint8_t *acc, const uint8_t *crc,
                                uint8_t *decoded, int *results, float *entropy, int max_iter) {
  if (!ctx) return DVC_E_ARG;
  return ldpca_run(ctx->c, n, count, lr, acc, crc, decoded, results, entropy, max_iter, nullptr, nullptr);
}

extern "C" int dvc_ldpca_decode_batch(dvc_ctx *ctx, int count, const int *n, const float *lr, const uint8_t *acc,
                                      const uint8_t *crc, const int *start, uint8_t *decoded, int *results,
                                      float *entropy, int max_iter, long long *bp_iterations, double *kernel_ms) {
  if (!ctx) return DVC_E_ARG;
  Context &c = ctx->c;
  if (count <= 0 || count > (1 << 22) || !n || !lr || !acc || !crc || !results || max_iter <= 0) {
    c.err = "dvc_ldpca_decode_batch: bad arguments";
    return DVC_E_ARG;
  }
  const dvc::LadderDev *Lc = c.ladder(6336), *Lq = c.ladder(1584);
  if (!Lc || !Lq) {
    c.err = "dvc_ldpca_decode_batch: ladders missing";
    return DVC_E_DATA;
  }
  std::vector<dvc::LdpcaBatchCw> cw(count);
  std::vector<int> lists;
  lists.reserve(count);
  long long lr_off = 0, byte_off = 0;
  for (int i = 0; i < count; i++) {
    if (n[i] != 1584 && n[i] != 6336) {
      c.err = "dvc_ldpca_decode_batch: codeword " + std::to_string(i) + " has length " + std::to_string(n[i]) +
              " (1584 or 6336)";
      return DVC_E_ARG;
    }
    cw[i].cif = n[i] == 6336;
    cw[i].crc = crc[i];
    cw[i].given_start = start ? start[i] : -1;
    if (start && (start[i] < 0 || start[i] > 64)) {
      c.err = "dvc_ldpca_decode_batch: start level out of range";
      return DVC_E_ARG;
    }
    cw[i].lr_off = lr_off;
    cw[i].acc_off = byte_off / 8;
    cw[i].dec_off = byte_off;
    lr_off += n[i];
    byte_off += n[i];
  }
  for (int i = 0; i < count; i++)
    if (cw[i].cif) lists.push_back(i);
  const int n_cif = (int)lists.size();
  for (int i = 0; i < count; i++)
    if (!cw[i].cif) lists.push_back(i);
  // layout of bt_cw: the codeword descriptors, the two index lists, then (16-byte
  // aligned, for the 64-bit counter's atomics) the queue heads and the work counter
  const size_t list_off = sizeof(dvc::LdpcaBatchCw) * count;
  const size_t ctr_off = (list_off + sizeof(int) * count + 15) & ~(size_t)15;
  if (!c.bt_lr.ensure((size_t)lr_off * 4) || !c.bt_acc.ensure((size_t)byte_off / 8) ||
      !c.bt_dec.ensure((size_t)byte_off) || !c.bt_res.ensure((size_t)count * 16) || !c.bt_ent.ensure((size_t)count * 4) ||
      !c.bt_cw.ensure(ctr_off + 32) ||
      !c.bt_state.ensure(dvc::ldpca_batch_state_bytes(count))) {
    c.err = "device allocation failed";
    return DVC_E_NOMEM;
  }
  dvc::LdpcaBatch A{};
  A.L_cif = *Lc;
  A.L_qcif = *Lq;
  A.xt = c.xlm;
  uint8_t *cwb = c.bt_cw.as<uint8_t>();
  A.cw = (const dvc::LdpcaBatchCw *)cwb;
  int *list_dev = (int *)(cwb + list_off);
  A.cif = list_dev;
  A.qcif = list_dev + n_cif;
  A.n_cif = n_cif;
  A.n_qcif = count - n_cif;
  A.last_cif = Lc->num_codes - 1;
  A.last_qcif = Lq->num_codes - 1;
  A.ctr = (int *)(cwb + ctr_off);
  A.work = (unsigned long long *)(cwb + ctr_off + 16);
  A.state = c.bt_state.as<dvc::LdpcaBatchState>();
  A.slot_bits = (uint32_t *)(c.bt_state.as<uint8_t>() + sizeof(dvc::LdpcaBatchState) * count);
  A.lr = c.bt_lr.as<float>();
  A.acc = c.bt_acc.as<uint8_t>();
  A.decoded = decoded ? c.bt_dec.as<uint8_t>() : nullptr;
  A.results = c.bt_res.as<int>();
  A.entropy = c.bt_ent.as<float>();
  A.max_iter = max_iter;
  cudaStream_t s = c.stream;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  int st;
  if ((st = cuda_status(c, cudaMemcpyAsync(c.bt_lr.p, lr, (size_t)lr_off * 4, cudaMemcpyHostToDevice, s), "H2D lr")) ||
      (st = cuda_status(c, cudaMemcpyAsync(c.bt_acc.p, acc, (size_t)byte_off / 8, cudaMemcpyHostToDevice, s), "H2D acc")) ||
      (st = cuda_status(c, cudaMemcpyAsync(cwb, cw.data(), sizeof(dvc::LdpcaBatchCw) * count, cudaMemcpyHostToDevice, s),
                        "H2D codewords")) ||
      (st = cuda_status(c, cudaMemcpyAsync(list_dev, lists.data(), sizeof(int) * count, cudaMemcpyHostToDevice, s),
                        "H2D lists")))
    return st;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (kernel_ms && ((st = cuda_status(c, cudaEventCreate(&e0), "event")) ||
                    (st = cuda_status(c, cudaEventCreate(&e1), "event"))))
    return st;
  if (e0) cudaEventRecord(e0, s);
  st = cuda_status(c, dvc::launch_ldpca_batch(A, count, sms, s), "ldpca batch launch");
  if (e1) cudaEventRecord(e1, s);
  unsigned long long work = 0;
  if (!st && decoded)
    st = cuda_status(c, cudaMemcpyAsync(decoded, c.bt_dec.p, (size_t)byte_off, cudaMemcpyDeviceToHost, s), "D2H dec");
  if (!st)
    st = cuda_status(c, cudaMemcpyAsync(results, c.bt_res.p, (size_t)count * 16, cudaMemcpyDeviceToHost, s), "D2H res");
  if (!st && entropy)
    st = cuda_status(c, cudaMemcpyAsync(entropy, c.bt_ent.p, (size_t)count * 4, cudaMemcpyDeviceToHost, s), "D2H ent");
  if (!st) st = cuda_status(c, cudaMemcpyAsync(&work, A.work, 8, cudaMemcpyDeviceToHost, s), "D2H work");
  if (!st) st = cuda_status(c, cudaStreamSynchronize(s), "ldpca batch sync");
  if (!st && kernel_ms) {
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    *kernel_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!st && bp_iterations) *bp_iterations = (long long)work;
  return st;
}

extern "C" int dvc_ldpca_encode(dvc_ctx *ctx, int n, int count, const uint8_t *bits, uint8_t *acc, uint8_t *crc) {
  if (!ctx) return DVC_E_ARG;
  Context &c = ctx->c;
  const dvc::LadderDev *L = c.ladder(n);
  if (!L) {
    c.err = "no ladder for codeword length " + std::to_string(n);
    return DVC_E_ARG;
  }
  if (count <= 0 || !bits || !acc || !crc) {
    c.err = "dvc_ldpca_encode: bad arguments";
    return DVC_E_ARG;
  }
  const size_t nb = (size_t)n / 8;
  if (!c.ld_dec.ensure((size_t)count * n) || !c.ld_acc.ensure((size_t)count * nb) || !c.ld_res.ensure((size_t)count)) {
    c.err = "device allocation failed";
    return DVC_E_NOMEM;
  }
  cudaStream_t s = c.stream;
  int st;
  if ((st = cuda_status(c, cudaMemcpyAsync(c.ld_dec.p, bits, (size_t)count * n, cudaMemcpyHostToDevice, s), "H2D bits")) ||
      (st = cuda_status(c, dvc::launch_ldpca_encode(*L, c.ld_dec.as<uint8_t>(), count, c.ld_acc.as<uint8_t>(),
                                                    c.ld_res.as<uint8_t>(), s),
                        "ldpca encode")) ||
      (st = cuda_status(c, cudaMemcpyAsync(acc, c.ld_acc.p, (size_t)count * nb, cudaMemcpyDeviceToHost, s), "D2H acc")) ||
      (st = cuda_status(c, cudaMemcpyAsync(crc, c.ld_res.p, (size_t)count, cudaMemcpyDeviceToHost, s), "D2H crc")) ||
      (st = cuda_status(c, cudaStreamSynchronize(s), "ldpca encode sync")))
    return st;
  return DVC_OK;
}

extern "C" int dvc_LdpcaDecoder(dvc_ctx *ctx, int n, float *LR_intrinsic, const unsigned char *accumulatedSyndrome,
                                unsigned char *decoded, int *rate, unsigned char crc_encoder, float RateLowerBound) {
  if (!ctx || !LR_intrinsic || !accumulatedSyndrome || !decoded || !rate || (n & 7)) return DVC_E_ARG;
  std::vector<uint8_t> bytes((size_t)n / 8, 0);
  for (int i = 0; i < n; i++)
    if (accumulatedSyndrome[i] & 1) bytes[i >> 3] |= (uint8_t)(0x80 >> (i & 7));
  int res[4];
  uint8_t crc = crc_encoder;
  // like the reference, LR_intrinsic comes back as log(LR) (LdpcaDecoder.cpp:663-667)
  int st = ldpca_run(ctx->c, n, 1, LR_intrinsic, bytes.data(), &crc, decoded, res, nullptr, 50, &RateLowerBound,
                     LR_intrinsic);
  if (st != DVC_OK) return st;
  *rate = res[0];
  return DVC_OK;
}

static int decode_frames(dvc_ctx *ctx, int count, dvc_wz_frame *frames, uint8_t *dbg_si0, float *dbg_alpha,
                         uint8_t *dbg_si1, float *dbg_lr = nullptr);

extern "C" int dvc_decode_wz_frames(dvc_ctx *ctx, int count, dvc_wz_frame *frames) {
  return decode_frames(ctx, count, frames, nullptr, nullptr, nullptr);
}

extern "C" int dvc_debug_wz_frame(dvc_ctx *ctx, dvc_wz_frame *frame, uint8_t *si_initial, float *alpha,
                                  uint8_t *si_final) {
  return decode_frames(ctx, 1, frame, si_initial, alpha, si_final);
}

extern "C" int dvc_debug_wz_frame_lr(dvc_ctx *ctx, dvc_wz_frame *frame, float *lr_planes) {
  if (!ctx || !frame || !lr_planes) return DVC_E_ARG;
  return decode_frames(ctx, 1, frame, nullptr, nullptr, nullptr, lr_planes);
}

extern "C" int dvc_recon_near_ties(dvc_ctx *ctx, long long *count) {
  if (!ctx || !count) return DVC_E_ARG;
  dvc::Context &c = ctx->c;
  unsigned long long v = 0;
  int st;
  if ((st = cuda_status(c, cudaMemcpy(&v, c.near_ties.p, 8, cudaMemcpyDeviceToHost), "near-tie counter"))) return st;
  *count = (long long)v;
  return DVC_OK;
}

static int decode_frames(dvc_ctx *ctx, int count, dvc_wz_frame *frames, uint8_t *dbg_si0, float *dbg_alpha,
                         uint8_t *dbg_si1, float *dbg_lr) {
  if (!ctx) return DVC_E_ARG;
  Context &c = ctx->c;
  if (count <= 0 || !frames) {
    c.err = "dvc_decode_wz_frames: no frames";
    return DVC_E_ARG;
  }
  const int w = frames[0].width, h = frames[0].height;
  for (int i = 0; i < count; i++) {
    const dvc_wz_frame &f = frames[i];
    if (f.width != w || f.height != h || !((w == 176 && h == 144) || (w == 352 && h == 288))) {
      c.err = "frames must all be QCIF (176x144) or all CIF (352x288)";
      return DVC_E_ARG;
    }
    if (f.qindex < 1 || f.qindex > 8 || !f.past || !f.future || !f.ac_range || !f.crc || !f.acc_synd || !f.recon) {
      c.err = "dvc_decode_wz_frames: bad frame " + std::to_string(i);
      return DVC_E_ARG;
    }
  }
  const size_t fs = (size_t)w * h;
  cudaStream_t s = c.stream;
  // distinct reference frames (by host pointer), each uploaded once with its planes
  std::map<const uint8_t *, int> refs;
  for (int i = 0; i < count; i++)
    for (const uint8_t *p : {frames[i].past, frames[i].future})
      if (!refs.count(p)) {
        const int k = (int)refs.size();
        refs[p] = k;
      }
  const size_t nr = refs.size();
  if (ctx->ref.size() < nr) {
    ctx->ref.resize(nr);
    ctx->lp.resize(nr);
    ctx->ip.resize(nr);
  }
  if (ctx->out.size() < (size_t)count) {
    ctx->out.resize(count);
    ctx->dbf.resize(count);
  }
  int st;
  for (auto &kv : refs) {
    const int k = kv.second;
    if (!ctx->ref[k].ensure(fs) || !ctx->lp[k].ensure(fs) || !ctx->ip[k].ensure(fs * 4)) {
      c.err = "device allocation failed";
      return DVC_E_NOMEM;
    }
    if ((st = cuda_status(c, cudaMemcpyAsync(ctx->ref[k].p, kv.first, fs, cudaMemcpyHostToDevice, s), "H2D ref")))
      return st;
    if ((st = cuda_status(c, dvc::launch_ref_planes(ctx->ref[k].as<uint8_t>(), w, h, ctx->lp[k].as<uint8_t>(),
                                                    ctx->ip[k].as<uint8_t>(), s),
                          "reference planes")))
      return st;
  }
  std::vector<dvc::FrameSpec> specs(count);
  for (int i = 0; i < count; i++) {
    const dvc_wz_frame &f = frames[i];
    if (!ctx->out[i].ensure(fs) || !ctx->dbf[i].ensure(fs)) {
      c.err = "device allocation failed";
      return DVC_E_NOMEM;
    }
    if ((st = cuda_status(c, cudaMemcpyAsync(ctx->out[i].p, f.recon, fs, cudaMemcpyHostToDevice, s), "H2D recon")))
      return st;
    dvc::FrameSpec &S = specs[i];
    S.w = w;
    S.h = h;
    S.qindex = f.qindex;
    const int pr = refs[f.past], fr = refs[f.future];
    S.past = ctx->ref[pr].as<uint8_t>();
    S.future = ctx->ref[fr].as<uint8_t>();
    S.past_lp = ctx->lp[pr].as<uint8_t>();
    S.future_lp = ctx->lp[fr].as<uint8_t>();
    S.past_ip = ctx->ip[pr].as<uint8_t>();
    S.future_ip = ctx->ip[fr].as<uint8_t>();
    S.past_idx = f.past_idx;
    S.future_idx = f.future_idx;
    S.cur_idx = f.cur_idx;
    S.mode = f.mode;
    S.skip_mode = f.skip_mode;
    S.intra_mode = f.intra_mode;
    S.deblock = f.deblock;
    S.intra_qp = f.intra_qp;
    S.past_mode = f.past_mode;
    for (int j = 0; j < 16; j++) S.ac_range[j] = f.ac_range[j];
    S.crc = f.crc;
    S.acc = f.acc_synd;
    S.recon = ctx->out[i].as<uint8_t>();
    S.deblock_flag = ctx->dbf[i].as<uint8_t>();
  }
  dvc::DevBuf &dbg = ctx->dbg;
  const size_t lr_bytes = dbg_lr ? (size_t)dvc::qbits_per_block(frames[0].qindex) * (fs / 16) * 4 : 0;
  if (dbg_si0 || dbg_alpha || dbg_si1 || dbg_lr) {
    if (!dbg.ensure(fs * 6 + lr_bytes)) {
      c.err = "device allocation failed";
      return DVC_E_NOMEM;
    }
    specs[0].dbg_si_initial = dbg.as<uint8_t>();
    specs[0].dbg_si_final = dbg.as<uint8_t>() + fs;
    specs[0].dbg_alpha = (float *)(dbg.as<uint8_t>() + 2 * fs);
    if (dbg_lr) specs[0].dbg_lr = (float *)(dbg.as<uint8_t>() + 6 * fs);
  }
  std::vector<dvc::FrameResult> res;
  if (!ctx->batcher.decode(c, specs, res, s)) return c.err.find("alloc") != std::string::npos ? DVC_E_NOMEM : DVC_E_CUDA;
  for (int i = 0; i < count; i++) {
    dvc_wz_frame &f = frames[i];
    if ((st = cuda_status(c, cudaMemcpyAsync(f.recon, ctx->out[i].p, fs, cudaMemcpyDeviceToHost, s), "D2H recon")))
      return st;
    if (f.deblock_flag &&
        (st = cuda_status(c, cudaMemcpyAsync(f.deblock_flag, ctx->dbf[i].p, fs, cudaMemcpyDeviceToHost, s), "D2H dbf")))
      return st;
  }
  if (dbg_si0 && (st = cuda_status(c, cudaMemcpyAsync(dbg_si0, dbg.p, fs, cudaMemcpyDeviceToHost, s), "D2H dbg")))
    return st;
  if (dbg_si1 &&
      (st = cuda_status(c, cudaMemcpyAsync(dbg_si1, dbg.as<uint8_t>() + fs, fs, cudaMemcpyDeviceToHost, s), "D2H dbg")))
    return st;
  if (dbg_alpha &&
      (st = cuda_status(c, cudaMemcpyAsync(dbg_alpha, dbg.as<uint8_t>() + 2 * fs, fs * 4, cudaMemcpyDeviceToHost, s),
                        "D2H dbg")))
    return st;
  if (dbg_lr && (st = cuda_status(c, cudaMemcpyAsync(dbg_lr, dbg.as<uint8_t>() + 6 * fs, lr_bytes,
                                                      cudaMemcpyDeviceToHost, s), "D2H dbg")))
    return st;
  if ((st = cuda_status(c, cudaStreamSynchronize(s), "decode sync"))) return st;
  for (int i = 0; i < count; i++) {
    dvc_wz_frame &f = frames[i];
    f.wz_bits = res[i].wz_bits;
    if (f.plane_results) memcpy(f.plane_results, res[i].planes.data(), res[i].planes.size() * sizeof(int));
    if (f.plane_entropy) memcpy(f.plane_entropy, res[i].entropy.data(), res[i].entropy.size() * sizeof(float));
  }
  return DVC_OK;
}

// ---------------------------------------------------------------- sessions

struct dvc_session {
  dvc_ctx *ctx = nullptr;
  int w = 0, h = 0, count = 0;
  std::vector<dvc::DevBuf> ref, lp, ip;   // reference frames given by the caller (+ derived planes)
  std::vector<dvc::DevBuf> out, olp, oip; // decoded frames (+ derived planes of those used as references)
  std::vector<dvc::DevBuf> init;          // initial recon (intra pixels) of frames with intra blocks
  std::vector<char> is_ref;               // frame i's output is a reference of a later level
  std::vector<dvc::FrameBatcher> batches;
  std::vector<std::vector<int>> batch_frames;  // frame indices of each batch
  std::vector<std::vector<int>> batch_deps;    // batches whose outputs each batch reads
  std::vector<int> batch_stream;
  std::vector<cudaEvent_t> batch_done;
  std::vector<cudaStream_t> streams;
  std::vector<std::vector<dvc::FrameResult>> results;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  std::vector<cudaEvent_t> done;
  dvc::ProfileStats prof;
  long long runs = 0, replays = 0;
  // the whole run as one CUDA graph, captured on the second unprofiled run and
  // replayed after that; graph_failed: capture did not work, stay eager
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  bool graph_failed = false;
};

static void session_release(dvc_session *S) {
  for (auto &b : S->batches) b.release();
  for (auto *v : {&S->ref, &S->lp, &S->ip, &S->out, &S->olp, &S->oip, &S->init})
    for (auto &b : *v) b.release();
  for (cudaStream_t st : S->streams) cudaStreamDestroy(st);
  for (cudaEvent_t e : S->done) cudaEventDestroy(e);
  for (cudaEvent_t e : S->batch_done) cudaEventDestroy(e);
  if (S->t0) cudaEventDestroy(S->t0);
  if (S->t1) cudaEventDestroy(S->t1);
  if (S->graph_exec) cudaGraphExecDestroy(S->graph_exec);
  if (S->graph) cudaGraphDestroy(S->graph);
  S->graph_exec = nullptr;
  S->graph = nullptr;
}

extern "C" int dvc_session_create(dvc_ctx *ctx, int count, const dvc_wz_frame *frames, int max_batch, int nstreams,
                                  dvc_session **out) {
  if (!ctx || !out || count <= 0 || !frames) return DVC_E_ARG;
  Context &c = ctx->c;
  *out = nullptr;
  if (max_batch <= 0) max_batch = count;
  if (nstreams <= 0) nstreams = 1;
  const int w = frames[0].width, h = frames[0].height;
  for (int i = 0; i < count; i++) {
    const dvc_wz_frame &f = frames[i];
    if (f.width != w || f.height != h || !((w == 176 && h == 144) || (w == 352 && h == 288)) || f.qindex < 1 ||
        f.qindex > 8 || !f.past || !f.future || !f.ac_range || !f.crc || !f.acc_synd || !f.recon) {
      c.err = "dvc_session_create: bad frame " + std::to_string(i);
      return DVC_E_ARG;
    }
  }
  // A reference pointer equal to another frame's recon pointer names that
  // frame's decoded output: the frame then decodes in a later level.
  std::map<const uint8_t *, int> recon_of;
  for (int i = 0; i < count; i++) recon_of[frames[i].recon] = i;
  std::vector<std::array<int, 2>> dep(count, {-1, -1});
  std::map<const uint8_t *, int> refs;
  for (int i = 0; i < count; i++)
    for (int k = 0; k < 2; k++) {
      const uint8_t *p = k == 0 ? frames[i].past : frames[i].future;
      auto it = recon_of.find(p);
      if (it != recon_of.end()) {
        if (it->second == i) {
          c.err = "dvc_session_create: frame " + std::to_string(i) + " references its own output";
          return DVC_E_ARG;
        }
        dep[i][k] = it->second;
      } else if (!refs.count(p)) {
        const int n = (int)refs.size();
        refs[p] = n;
      }
    }
  std::vector<int> level(count, -1);
  for (int pass = 0, left = count; left > 0; pass++) {
    int placed = 0;
    for (int i = 0; i < count; i++) {
      if (level[i] >= 0) continue;
      bool ready = true;  // every reference decoded in an earlier level
      for (int k = 0; k < 2; k++)
        if (dep[i][k] >= 0 && (level[dep[i][k]] < 0 || level[dep[i][k]] >= pass)) ready = false;
      if (ready) {
        level[i] = pass;
        placed++;
      }
    }
    if (!placed) {
      c.err = "dvc_session_create: circular references between frames";
      return DVC_E_ARG;
    }
    left -= placed;
  }
  dvc_session *S = new (std::nothrow) dvc_session();
  if (!S) return DVC_E_NOMEM;
  S->ctx = ctx;
  S->w = w;
  S->h = h;
  S->count = count;
  const size_t fs = (size_t)w * h;
  int st = DVC_OK;
  auto bail = [&](int code) {
    session_release(S);
    delete S;
    return code;
  };
  S->ref.resize(refs.size());
  S->lp.resize(refs.size());
  S->ip.resize(refs.size());
  S->out.resize(count);
  S->olp.resize(count);
  S->oip.resize(count);
  S->init.resize(count);
  S->is_ref.assign(count, 0);
  for (int i = 0; i < count; i++)
    for (int k = 0; k < 2; k++)
      if (dep[i][k] >= 0) S->is_ref[dep[i][k]] = 1;
  cudaStream_t s0 = c.stream;
  for (auto &kv : refs) {
    const int k = kv.second;
    if (!S->ref[k].ensure(fs) || !S->lp[k].ensure(fs) || !S->ip[k].ensure(fs * 4)) {
      c.err = "device allocation failed";
      return bail(DVC_E_NOMEM);
    }
    if ((st = cuda_status(c, cudaMemcpyAsync(S->ref[k].p, kv.first, fs, cudaMemcpyHostToDevice, s0), "H2D ref")) ||
        (st = cuda_status(c, dvc::launch_ref_planes(S->ref[k].as<uint8_t>(), w, h, S->lp[k].as<uint8_t>(),
                                                    S->ip[k].as<uint8_t>(), s0),
                          "reference planes")))
      return bail(st);
  }
  for (int i = 0; i < count; i++) {
    if (!S->out[i].ensure(fs) || (S->is_ref[i] && (!S->olp[i].ensure(fs) || !S->oip[i].ensure(fs * 4))) ||
        (frames[i].intra_mode && !S->init[i].ensure(fs))) {
      c.err = "device allocation failed";
      return bail(DVC_E_NOMEM);
    }
    if ((st = cuda_status(c, cudaMemcpyAsync(S->out[i].p, frames[i].recon, fs, cudaMemcpyHostToDevice, s0), "H2D")))
      return bail(st);
    if (frames[i].intra_mode &&
        (st = cuda_status(c, cudaMemcpyAsync(S->init[i].p, frames[i].recon, fs, cudaMemcpyHostToDevice, s0), "H2D")))
      return bail(st);
  }
  if ((st = cuda_status(c, cudaStreamSynchronize(s0), "session upload"))) return bail(st);
  for (int k = 0; k < nstreams; k++) {
    cudaStream_t sk;
    if ((st = cuda_status(c, cudaStreamCreateWithFlags(&sk, cudaStreamNonBlocking), "stream"))) return bail(st);
    S->streams.push_back(sk);
    cudaEvent_t e;
    if ((st = cuda_status(c, cudaEventCreate(&e), "event"))) return bail(st);
    S->done.push_back(e);
  }
  if ((st = cuda_status(c, cudaEventCreate(&S->t0), "event")) || (st = cuda_status(c, cudaEventCreate(&S->t1), "event")))
    return bail(st);
  // batches: level by level, frames of a level in the caller's order, at most
  // max_batch per batch, streams assigned round-robin
  const int nlev = *std::max_element(level.begin(), level.end()) + 1;
  std::vector<int> batch_of(count, -1);
  for (int lv = 0; lv < nlev; lv++) {
    std::vector<int> fl;
    for (int i = 0; i < count; i++)
      if (level[i] == lv) fl.push_back(i);
    for (size_t a = 0; a < fl.size(); a += max_batch) {
      const int b = (int)S->batch_frames.size();
      S->batch_frames.emplace_back(fl.begin() + a, fl.begin() + std::min(fl.size(), a + (size_t)max_batch));
      S->batch_stream.push_back(b % nstreams);
      std::vector<int> deps;
      for (int i : S->batch_frames[b]) {
        batch_of[i] = b;
        for (int k = 0; k < 2; k++)
          if (dep[i][k] >= 0 && std::find(deps.begin(), deps.end(), batch_of[dep[i][k]]) == deps.end())
            deps.push_back(batch_of[dep[i][k]]);
      }
      S->batch_deps.push_back(deps);
    }
  }
  const int nb = (int)S->batch_frames.size();
  S->batches.resize(nb);
  S->results.resize(nb);
  for (int b = 0; b < nb; b++) {
    cudaEvent_t e;
    if ((st = cuda_status(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event"))) return bail(st);
    S->batch_done.push_back(e);
    std::vector<dvc::FrameSpec> specs;
    for (int i : S->batch_frames[b]) {
      const dvc_wz_frame &f = frames[i];
      dvc::FrameSpec sp;
      sp.w = w;
      sp.h = h;
      sp.qindex = f.qindex;
      for (int k = 0; k < 2; k++) {
        const uint8_t *pl, *pp, *pi;
        if (dep[i][k] >= 0) {
          const int d = dep[i][k];
          pl = S->out[d].as<uint8_t>();
          pp = S->olp[d].as<uint8_t>();
          pi = S->oip[d].as<uint8_t>();
        } else {
          const int r = refs[k == 0 ? f.past : f.future];
          pl = S->ref[r].as<uint8_t>();
          pp = S->lp[r].as<uint8_t>();
          pi = S->ip[r].as<uint8_t>();
        }
        (k == 0 ? sp.past : sp.future) = pl;
        (k == 0 ? sp.past_lp : sp.future_lp) = pp;
        (k == 0 ? sp.past_ip : sp.future_ip) = pi;
      }
      sp.past_idx = f.past_idx;
      sp.future_idx = f.future_idx;
      sp.cur_idx = f.cur_idx;
      sp.mode = f.mode;
      sp.skip_mode = f.skip_mode;
      sp.intra_mode = f.intra_mode;
      sp.deblock = f.deblock;
      sp.intra_qp = f.intra_qp;
      sp.past_mode = f.past_mode;
      for (int j = 0; j < 16; j++) sp.ac_range[j] = f.ac_range[j];
      sp.crc = f.crc;
      sp.acc = f.acc_synd;
      sp.recon = S->out[i].as<uint8_t>();
      specs.push_back(sp);
    }
    cudaStream_t sb = S->streams[S->batch_stream[b]];
    // frames decoding at once: one batch per stream
    const int concurrent = std::min(count, nstreams * max_batch);
    if (!S->batches[b].prepare(c, specs, sb, concurrent)) return bail(DVC_E_CUDA);
    if ((st = cuda_status(c, cudaStreamSynchronize(sb), "session prepare"))) return bail(st);
  }
  *out = S;
  return DVC_OK;
}

// every operation of one run, forked from streams[0] at `fork` and joined back
// to it: the batches in level order (a batch waits for the batches it reads),
// the planes of decoded frames that later levels use as references, and, when
// `results` is set, the per-bitplane result copies
static int session_enqueue(dvc_session *S, bool profile, bool results, cudaEvent_t fork) {
  Context &c = S->ctx->c;
  const int ns = (int)S->streams.size();
  const size_t fs = (size_t)S->w * S->h;
  int st;
  cudaStream_t s0 = S->streams[0];
  if ((st = cuda_status(c, cudaEventRecord(fork, s0), "event"))) return st;
  for (int k = 1; k < ns; k++)
    if ((st = cuda_status(c, cudaStreamWaitEvent(S->streams[k], fork, 0), "wait"))) return st;
  for (size_t b = 0; b < S->batches.size(); b++) {
    cudaStream_t sb = S->streams[S->batch_stream[b]];
    for (int d : S->batch_deps[b])
      if ((st = cuda_status(c, cudaStreamWaitEvent(sb, S->batch_done[d], 0), "wait"))) return st;
    for (int i : S->batch_frames[b])
      if (S->init[i].p &&
          (st = cuda_status(c, cudaMemcpyAsync(S->out[i].p, S->init[i].p, fs, cudaMemcpyDeviceToDevice, sb), "D2D")))
        return st;
    if (!S->batches[b].execute(c, sb, 50, profile ? &S->prof : nullptr)) return DVC_E_CUDA;
    for (int i : S->batch_frames[b]) {
      if (!S->is_ref[i]) continue;
      if ((st = cuda_status(c, dvc::launch_ref_planes(S->out[i].as<uint8_t>(), S->w, S->h, S->olp[i].as<uint8_t>(),
                                                      S->oip[i].as<uint8_t>(), sb),
                            "reference planes")))
        return st;
      if (profile) S->prof.kernel_launches += 2;  // low-pass and half-pel kernels
    }
    if (results && !S->batches[b].enqueue_results(c, sb)) return DVC_E_CUDA;
    if ((st = cuda_status(c, cudaEventRecord(S->batch_done[b], sb), "event"))) return st;
  }
  for (int k = 1; k < ns; k++) {
    if ((st = cuda_status(c, cudaEventRecord(S->done[k], S->streams[k]), "event"))) return st;
    if ((st = cuda_status(c, cudaStreamWaitEvent(s0, S->done[k], 0), "wait"))) return st;
  }
  return DVC_OK;
}

// capture one run into S->graph_exec; false (and eager runs from then on) if
// the capture or the instantiation fails
static bool session_capture(dvc_session *S) {
  cudaStream_t s0 = S->streams[0];
  if (cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
  const int st = session_enqueue(S, false, true, S->t0);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s0, &g);
  if (st != DVC_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return false;
  }
  cudaGraphExec_t x = nullptr;
  if (cudaGraphInstantiate(&x, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    cudaGetLastError();
    return false;
  }
  S->graph = g;
  S->graph_exec = x;
  return true;
}

extern "C" int dvc_session_run(dvc_session *S, int profile, double *elapsed_ms) {
  if (!S) return DVC_E_ARG;
  Context &c = S->ctx->c;
  const int ns = (int)S->streams.size();
  int st;
  cudaStream_t s0 = S->streams[0];
  // from the second unprofiled run on, replay the captured graph (the first
  // run is eager: it sets the kernels' attributes and fills the buffers)
  if (!profile && S->runs >= 1 && !S->graph_failed && !S->graph_exec && !session_capture(S)) S->graph_failed = true;
  if (!profile && S->graph_exec) {
    if ((st = cuda_status(c, cudaEventRecord(S->t0, s0), "event"))) return st;
    if ((st = cuda_status(c, cudaGraphLaunch(S->graph_exec, s0), "graph launch"))) return st;
    if ((st = cuda_status(c, cudaEventRecord(S->t1, s0), "event"))) return st;
    if ((st = cuda_status(c, cudaEventSynchronize(S->t1), "session run"))) return st;
    for (size_t b = 0; b < S->batches.size(); b++) S->batches[b].read_results(S->results[b]);
    S->replays++;
  } else {
    if ((st = session_enqueue(S, profile != 0, false, S->t0))) return st;
    if ((st = cuda_status(c, cudaEventRecord(S->t1, s0), "event"))) return st;
    for (size_t b = 0; b < S->batches.size(); b++)
      if (!S->batches[b].collect(c, S->results[b], S->streams[S->batch_stream[b]])) return DVC_E_CUDA;
    if ((st = cuda_status(c, cudaEventSynchronize(S->t1), "session run"))) return st;
    for (int k = 0; k < ns; k++)
      if ((st = cuda_status(c, cudaStreamSynchronize(S->streams[k]), "session collect"))) return st;
    if (profile)
      for (auto &b : S->batches) b.harvest(&S->prof);
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, S->t0, S->t1);
  if (elapsed_ms) *elapsed_ms = ms;
  S->runs++;
  return DVC_OK;
}

extern "C" int dvc_session_replays(dvc_session *S, long long *replays) {
  if (!S || !replays) return DVC_E_ARG;
  *replays = S->replays;
  return DVC_OK;
}

extern "C" int dvc_session_frame(dvc_session *S, int index, uint8_t *recon, int *wz_bits, int *plane_results) {
  if (!S || index < 0 || index >= S->count) return DVC_E_ARG;
  Context &c = S->ctx->c;
  for (size_t b = 0; b < S->batch_frames.size(); b++)
    for (size_t j = 0; j < S->batch_frames[b].size(); j++)
      if (S->batch_frames[b][j] == index) {
        if (S->results[b].size() <= j) {
          c.err = "dvc_session_frame: no completed run";
          return DVC_E_ARG;
        }
        const dvc::FrameResult &r = S->results[b][j];
        if (wz_bits) *wz_bits = r.wz_bits;
        if (plane_results) memcpy(plane_results, r.planes.data(), r.planes.size() * sizeof(int));
        if (recon) {
          int st = cuda_status(c, cudaMemcpy(recon, S->out[index].p, (size_t)S->w * S->h, cudaMemcpyDeviceToHost),
                               "D2H recon");
          if (st) return st;
        }
        return DVC_OK;
      }
  return DVC_E_ARG;
}

extern "C" int dvc_session_profile(dvc_session *S, double *out5) {
  if (!S || !out5) return DVC_E_ARG;
  out5[0] = S->prof.ldpca_ms;
  out5[1] = (double)S->prof.ldpca_launches;
  out5[2] = (double)S->prof.ldpca_codewords;
  out5[3] = (double)S->prof.kernel_launches;
  out5[4] = (double)S->runs;
  return DVC_OK;
}

extern "C" void dvc_session_destroy(dvc_session *S) {
  if (!S) return;
  session_release(S);
  delete S;
}
