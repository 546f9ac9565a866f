// C ABI of libdvc_b200.so (declared in include/dvc_b200.h).
#include "../../include/dvc_b200.h"

#include <string.h>

#include <new>
#include <vector>

#include "context.h"
#include "kernels.h"

struct dvc_ctx {
  dvc::Context c;
};

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
