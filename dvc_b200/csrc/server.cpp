// Continuous-batching WZ decode server (dvc_server_* in include/dvc_b200.h).
//
// Requests (one WZ frame each, with their reference frames) are queued by
// submit().  poll() does the scheduling: it retires finished cohorts (an event
// per stream tells when the device is done with one) and forms new cohorts for
// idle streams from the queue: frames of one size (any quantisers), up to
// max_cohort of them, admitted while the estimated device memory of the frames
// in flight stays within the budget.  While other cohorts are decoding, a
// cohort that would start short of max_cohort waits up to the batch window for
// company; the speculation width of its ladders is set from all frames then in
// flight, so that many small cohorts do not oversubscribe the SMs.  Each cohort runs the whole frame pipeline
// on its own stream (side information, noise model, every bitplane's ladder with
// the syndrome-request feedback on the device, reconstruction, refinement), so
// cohorts on different streams overlap on the GPU and a request that arrives
// while others are decoding starts as soon as a stream and memory are free.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/dvc_b200.h"
#include "context.h"
#include "frame_driver.h"

namespace dvc {
Context *context_of(dvc_ctx *ctx);
cudaError_t launch_ref_planes(const uint8_t *recon, int w, int h, uint8_t *lp, uint8_t *ip, cudaStream_t s);
}  // namespace dvc

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  long long ticket = 0;
  int w = 0, h = 0, q = 0, past_idx = 0, future_idx = 0, cur_idx = 0, skip_mode = 0, intra_mode = 0;
  int deblock = 0, intra_qp = 0;
  std::vector<uint8_t> past_mode;  // empty: the past reference is a key frame
  int ac_range[16] = {0};
  std::vector<uint8_t> past, future, mode, crc, acc, recon;
  bool has_mode = false;
  size_t est_bytes = 0;
  Clock::time_point t_submit, t_done;
  int status = DVC_OK;
  int wz_bits = 0;
  std::vector<int> planes;
};

struct Cohort {
  dvc::FrameBatcher batcher;
  std::vector<std::shared_ptr<Request>> reqs;
  std::vector<dvc::DevBuf> ref, lp, ip, out;
  uint8_t *pinned_out = nullptr;
  size_t pinned_bytes = 0;
  cudaEvent_t done = nullptr;
  bool active = false;
  size_t charged = 0;
};

// estimated device bytes of one frame in flight (frame slot + its references);
// the noise pdf is bounded by the largest coefficient range of the frame's bands
size_t frame_bytes(int w, int h, int q, const int *ac_range) {
  const size_t fs = (size_t)w * h, n = fs / 16;
  size_t stride = 1024;
  for (int band = 0; band < 16 && dvc::kQBits[q][dvc::kZigzag[band]] > 0; band++) {
    const int i = dvc::kZigzag[band];
    if (i == 0 || dvc::kQTable[q][i] <= 0) continue;
    const int step = (int)((2 * (ac_range[i] + 1) + dvc::kQTable[q][i] - 1) / dvc::kQTable[q][i]);
    const int ls = (dvc::kQTable[q][i] - 2) / 2;
    stride = std::max(stride, (size_t)(2 * ((ls + 1) * step - 1) + 1));
  }
  const size_t slot = fs * 18 + n * 4 + (size_t)(w - 3) * (h - 3) * 32 + n * 81 * 4 + n * stride * 4 +
                      fs / 256 * 48 * 2 + fs / 64 * 56 * 2 + (size_t)dvc::qbits_per_block(q) * (n / 8 + 24);
  const size_t refs = 2 * fs * 6 + fs;  // two references with low-pass and half-pel planes, output
  const size_t spec = (size_t)32 * n;   // speculative ladder slots
  return slot + refs + spec + (1 << 16);
}

}  // namespace

struct dvc_server {
  dvc_ctx *ctx = nullptr;
  dvc::Context *c = nullptr;
  size_t budget = 0, used = 0;
  int max_cohort = 8;
  std::vector<cudaStream_t> streams;
  std::vector<Cohort> cohorts;
  std::mutex mu;
  std::deque<std::shared_ptr<Request>> pending;
  std::map<long long, std::shared_ptr<Request>> finished;
  long long next_ticket = 1;
  long long completed = 0;
  // a partial cohort waits this long for company while another cohort is decoding
  int batch_window_us = 2000;
};

static int srv_fail(dvc_server *S, int code, const std::string &m) {
  S->c->err = m;
  return code;
}

extern "C" int dvc_server_create(dvc_ctx *ctx, size_t mem_budget_bytes, int nstreams, int max_cohort,
                                 dvc_server **out) {
  if (!ctx || !out || nstreams <= 0 || max_cohort <= 0 || mem_budget_bytes == 0) return DVC_E_ARG;
  *out = nullptr;
  dvc_server *S = new (std::nothrow) dvc_server();
  if (!S) return DVC_E_NOMEM;
  S->ctx = ctx;
  S->c = dvc::context_of(ctx);
  S->budget = mem_budget_bytes;
  S->max_cohort = max_cohort;
  S->cohorts.resize(nstreams);
  // cohort buffers grow with cudaMallocAsync / cudaFreeAsync: keep freed memory
  // in this process's pool rather than handing it back to the driver at every
  // synchronisation (a process-local attribute of the current device's pool)
  {
    cudaMemPool_t pool;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  for (int i = 0; i < nstreams; i++) {
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->cohorts[i].done, cudaEventDisableTiming) != cudaSuccess) {
      S->c->err = "dvc_server_create: stream/event creation failed";
      for (cudaStream_t x : S->streams) cudaStreamDestroy(x);
      delete S;
      return DVC_E_CUDA;
    }
    S->streams.push_back(st);
  }
  *out = S;
  return DVC_OK;
}

extern "C" int dvc_server_submit(dvc_server *S, const dvc_wz_frame *f, long long *ticket) {
  if (!S || !f || !ticket) return DVC_E_ARG;
  const int w = f->width, h = f->height;
  if (!((w == 176 && h == 144) || (w == 352 && h == 288)) || f->qindex < 1 || f->qindex > 8 || !f->past ||
      !f->future || !f->ac_range || !f->crc || !f->acc_synd || f->future_idx == f->past_idx)
    return srv_fail(S, DVC_E_ARG, "dvc_server_submit: bad frame");
  auto r = std::make_shared<Request>();
  const size_t fs = (size_t)w * h;
  const int qb = dvc::qbits_per_block(f->qindex);
  r->w = w;
  r->h = h;
  r->q = f->qindex;
  r->past_idx = f->past_idx;
  r->future_idx = f->future_idx;
  r->cur_idx = f->cur_idx;
  r->skip_mode = f->skip_mode;
  r->intra_mode = f->intra_mode;
  r->deblock = f->deblock;
  r->intra_qp = f->intra_qp;
  if (f->past_mode) r->past_mode.assign(f->past_mode, f->past_mode + fs / 64);
  memcpy(r->ac_range, f->ac_range, sizeof r->ac_range);
  r->past.assign(f->past, f->past + fs);
  r->future.assign(f->future, f->future + fs);
  if (f->mode) {
    r->mode.assign(f->mode, f->mode + fs / 64);
    r->has_mode = true;
  }
  r->crc.assign(f->crc, f->crc + qb);
  r->acc.assign(f->acc_synd, f->acc_synd + (size_t)qb * (fs / 128));
  r->recon.assign(fs, 0);
  if (f->recon) memcpy(r->recon.data(), f->recon, fs);
  r->est_bytes = frame_bytes(w, h, f->qindex, f->ac_range);
  if (r->est_bytes > S->budget)
    return srv_fail(S, DVC_E_NOMEM,
                    "dvc_server_submit: one frame needs ~" + std::to_string(r->est_bytes >> 20) +
                        " MB of device memory, above the server budget of " + std::to_string(S->budget >> 20) + " MB");
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(S->mu);
  r->ticket = S->next_ticket++;
  *ticket = r->ticket;
  S->pending.push_back(r);
  return DVC_OK;
}

// start a cohort on stream i from the queue; returns false (with err) on a CUDA failure
static bool start_cohort(dvc_server *S, int i) {
  dvc::Context &c = *S->c;
  Cohort &C = S->cohorts[i];
  C.reqs.clear();
  // frames of one size, oldest first, within the memory budget (quantisers may
  // differ: each frame takes part only in the band/bitplane steps it codes)
  std::shared_ptr<Request> head;
  {
    // dynamic batching: while other cohorts keep the GPU busy, a partial cohort
    // waits up to the batch window for more frames of its kind
    bool busy = false;
    for (auto &o : S->cohorts) busy = busy || o.active;
    if (busy && !S->pending.empty()) {
      const Request &h0 = *S->pending.front();
      int same = 0;
      for (auto &p : S->pending)
        if (p->w == h0.w && p->h == h0.h) same++;
      const double waited = std::chrono::duration<double, std::micro>(Clock::now() - h0.t_submit).count();
      if (same < S->max_cohort && waited < S->batch_window_us) return true;
    }
  }
  for (auto it = S->pending.begin(); it != S->pending.end();) {
    Request &r = **it;
    if (!head) {
      if (S->used + r.est_bytes > S->budget) break;  // the oldest waits for memory
      head = *it;
    } else if (r.w != head->w || r.h != head->h || S->used + r.est_bytes > S->budget) {
      ++it;
      continue;
    }
    S->used += r.est_bytes;
    C.charged += r.est_bytes;
    C.reqs.push_back(*it);
    it = S->pending.erase(it);
    if ((int)C.reqs.size() >= S->max_cohort) break;
  }
  if (C.reqs.empty()) return true;
  const int nf = (int)C.reqs.size(), w = head->w, h = head->h;
  const size_t fs = (size_t)w * h;
  cudaStream_t s = S->streams[i];
  if ((int)C.ref.size() < 2 * nf) {
    C.ref.resize(2 * nf);
    C.lp.resize(2 * nf);
    C.ip.resize(2 * nf);
  }
  if ((int)C.out.size() < nf) C.out.resize(nf);
  if (C.pinned_bytes < fs * nf) {
    // once, for the largest cohort (CIF frames, max_cohort of them): freeing
    // pinned memory waits for the whole device
    const size_t most = std::max(fs * nf, (size_t)352 * 288 * S->max_cohort);
    if (C.pinned_out) cudaFreeHost(C.pinned_out);
    C.pinned_out = nullptr;
    if (cudaMallocHost((void **)&C.pinned_out, most) != cudaSuccess) return c.fail("pinned allocation failed");
    C.pinned_bytes = most;
  }
  std::vector<dvc::FrameSpec> specs(nf);
  for (int f = 0; f < nf; f++) {
    Request &r = *C.reqs[f];
    for (int k = 0; k < 2; k++) {
      dvc::DevBuf &rb = C.ref[2 * f + k], &lb = C.lp[2 * f + k], &ib = C.ip[2 * f + k];
      if (!rb.ensure(fs, s) || !lb.ensure(fs, s) || !ib.ensure(4 * fs, s)) return c.fail("device allocation failed");
      const std::vector<uint8_t> &src = k == 0 ? r.past : r.future;
      if (!c.cuda_ok(cudaMemcpyAsync(rb.p, src.data(), fs, cudaMemcpyHostToDevice, s), "H2D reference") ||
          !c.cuda_ok(dvc::launch_ref_planes(rb.as<uint8_t>(), w, h, lb.as<uint8_t>(), ib.as<uint8_t>(), s),
                     "reference planes"))
        return false;
    }
    if (!C.out[f].ensure(fs, s)) return c.fail("device allocation failed");
    if (!c.cuda_ok(cudaMemcpyAsync(C.out[f].p, r.recon.data(), fs, cudaMemcpyHostToDevice, s), "H2D recon"))
      return false;
    dvc::FrameSpec &sp = specs[f];
    sp.w = w;
    sp.h = h;
    sp.qindex = r.q;
    sp.past = C.ref[2 * f].as<uint8_t>();
    sp.future = C.ref[2 * f + 1].as<uint8_t>();
    sp.past_lp = C.lp[2 * f].as<uint8_t>();
    sp.future_lp = C.lp[2 * f + 1].as<uint8_t>();
    sp.past_ip = C.ip[2 * f].as<uint8_t>();
    sp.future_ip = C.ip[2 * f + 1].as<uint8_t>();
    sp.past_idx = r.past_idx;
    sp.future_idx = r.future_idx;
    sp.cur_idx = r.cur_idx;
    sp.mode = r.has_mode ? r.mode.data() : nullptr;
    sp.skip_mode = r.skip_mode;
    sp.intra_mode = r.intra_mode;
    sp.deblock = r.deblock;
    sp.intra_qp = r.intra_qp;
    sp.past_mode = r.past_mode.empty() ? nullptr : r.past_mode.data();
    memcpy(sp.ac_range, r.ac_range, sizeof sp.ac_range);
    sp.crc = r.crc.data();
    sp.acc = r.acc.data();
    sp.recon = C.out[f].as<uint8_t>();
  }
  int in_flight = 0;
  for (auto &o : S->cohorts) in_flight += (int)o.reqs.size();
  C.batcher.set_alloc_stream(s);
  if (!C.batcher.prepare(c, specs, s, in_flight) || !C.batcher.execute(c, s, 50, nullptr)) return false;
  for (int f = 0; f < nf; f++)
    if (!c.cuda_ok(cudaMemcpyAsync(C.pinned_out + f * fs, C.out[f].p, fs, cudaMemcpyDeviceToHost, s), "D2H recon"))
      return false;
  if (!C.batcher.enqueue_results(c, s) || !c.cuda_ok(cudaEventRecord(C.done, s), "event")) return false;
  C.active = true;
  return true;
}

extern "C" int dvc_server_poll(dvc_server *S, int *completed) {
  if (!S) return DVC_E_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  int got = 0;
  for (size_t i = 0; i < S->cohorts.size(); i++) {
    Cohort &C = S->cohorts[i];
    if (!C.active) continue;
    const cudaError_t q = cudaEventQuery(C.done);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return srv_fail(S, DVC_E_CUDA, std::string("cohort failed: ") + cudaGetErrorString(q));
    std::vector<dvc::FrameResult> res;
    C.batcher.read_results(res);
    const auto now = Clock::now();
    const size_t fs = (size_t)C.reqs[0]->w * C.reqs[0]->h;
    for (size_t f = 0; f < C.reqs.size(); f++) {
      Request &r = *C.reqs[f];
      memcpy(r.recon.data(), C.pinned_out + f * fs, fs);
      r.wz_bits = res[f].wz_bits;
      r.planes = res[f].planes;
      r.t_done = now;
      S->finished[r.ticket] = C.reqs[f];
      got++;
    }
    S->used -= C.charged;
    C.charged = 0;
    C.reqs.clear();
    C.active = false;
  }
  for (size_t i = 0; i < S->cohorts.size() && !S->pending.empty(); i++)
    if (!S->cohorts[i].active && !start_cohort(S, (int)i)) return DVC_E_CUDA;
  S->completed += got;
  if (completed) *completed = got;
  return DVC_OK;
}

extern "C" int dvc_server_result(dvc_server *S, long long ticket, uint8_t *recon, int *wz_bits, int *plane_results,
                                 double *latency_ms) {
  if (!S) return DVC_E_ARG;
  std::shared_ptr<Request> r;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->finished.find(ticket);
    if (it == S->finished.end()) return srv_fail(S, DVC_E_ARG, "dvc_server_result: ticket not finished");
    r = it->second;
    S->finished.erase(it);
  }
  if (recon) memcpy(recon, r->recon.data(), r->recon.size());
  if (wz_bits) *wz_bits = r->wz_bits;
  if (plane_results) memcpy(plane_results, r->planes.data(), r->planes.size() * sizeof(int));
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  return DVC_OK;
}

extern "C" int dvc_server_finished(dvc_server *S, long long *tickets, int cap, int *count) {
  if (!S || !count || cap < 0 || (cap > 0 && !tickets)) return DVC_E_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  int n = 0;
  for (auto it = S->finished.begin(); it != S->finished.end() && n < cap; ++it) tickets[n++] = it->first;
  *count = n;
  return DVC_OK;
}

extern "C" int dvc_server_stats(dvc_server *S, long long *pending, long long *in_flight, size_t *bytes_in_flight) {
  if (!S) return DVC_E_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  long long inflight = 0;
  for (auto &C : S->cohorts) inflight += (long long)C.reqs.size();
  if (pending) *pending = (long long)S->pending.size();
  if (in_flight) *in_flight = inflight;
  if (bytes_in_flight) *bytes_in_flight = S->used;
  return DVC_OK;
}

extern "C" int dvc_server_config(dvc_server *S, int batch_window_us) {
  if (!S || batch_window_us < 0) return DVC_E_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  S->batch_window_us = batch_window_us;
  return DVC_OK;
}

extern "C" void dvc_server_destroy(dvc_server *S) {
  if (!S) return;
  for (size_t i = 0; i < S->cohorts.size(); i++) {
    Cohort &C = S->cohorts[i];
    if (C.active) cudaEventSynchronize(C.done);
    C.batcher.release();
    for (auto *v : {&C.ref, &C.lp, &C.ip, &C.out})
      for (auto &b : *v) b.release();
    if (C.pinned_out) cudaFreeHost(C.pinned_out);
    if (C.done) cudaEventDestroy(C.done);
    cudaStreamDestroy(S->streams[i]);
  }
  delete S;
}
