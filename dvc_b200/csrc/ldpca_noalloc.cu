// LDPCA ladder decode that performs no device allocation at call time.
//
// Who needs it: callers that must not call cudaMalloc once they are running.
// cudaMalloc can synchronise the whole device (stalling every other stream of
// a serving pipeline), is not allowed inside CUDA stream capture, and fails in
// processes where another framework's memory pool has already reserved the
// device memory.  Such callers keep their own device buffers for inputs and
// outputs and need an entry point that brings no scratch of its own.
//
// The only scratch this decode needs beyond its inputs and outputs is the
// array of per-codeword job descriptors the LDPCA kernel reads.  Here it lives
// in a file-scope __device__ array of fixed size (kMaxCodewords descriptors,
// about 100 KB), which every GPU that loads this library holds until the
// process exits.  Host code cannot use the array's name as a device address,
// so the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and keeps it; make that first
// call before any stream capture.  A small kernel writes every descriptor field
// of the codewords of a call on the device, so nothing carries over between
// calls.  All calls share the one array: calls that overlap on the GPU (for
// example on two streams) overwrite each other's descriptors and race.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/dvc_b200.h"
#include "context.h"
#include "kernels.h"

namespace {

constexpr int kMaxCodewords = DVC_NOALLOC_MAX_CODEWORDS;  // sizeof(LdpcaJob) is 96 bytes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) dvc::LdpcaJob g_jobs[kMaxCodewords];

std::mutex g_mu;
dvc::LdpcaJob *g_jobs_addr[kMaxDevices] = {nullptr};

// every field of each descriptor is written, so no state survives a call
__global__ void fill_jobs_kernel(dvc::LdpcaJob *jobs, int count, int n, const float *lr, const uint8_t *acc,
                                 const uint8_t *crc, uint8_t *decoded, int *results, float *entropy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  dvc::LdpcaJob j;
  memset(&j, 0, sizeof j);
  j.active = 1;
  j.lr = lr + (size_t)i * n;
  j.acc = acc + (size_t)i * (n / 8);
  j.crc = crc[i];
  j.decoded = decoded ? decoded + (size_t)i * n : nullptr;
  j.result = results + (size_t)i * 4;
  j.entropy = entropy ? entropy + i : nullptr;
  jobs[i] = j;
}

}  // namespace

struct dvc_ctx;
namespace dvc {
Context *context_of(dvc_ctx *ctx);
}

extern "C" int dvc_ldpca_decode_noalloc(dvc_ctx *ctx, int n, int count, const float *d_lr, const uint8_t *d_acc,
                                        const uint8_t *d_crc, uint8_t *d_decoded, int *d_results, float *d_entropy,
                                        int max_iter, void *stream) {
  if (!ctx) return DVC_E_ARG;
  dvc::Context &c = *dvc::context_of(ctx);
  if (count <= 0 || !d_lr || !d_acc || !d_crc || !d_results || max_iter <= 0) {
    c.err = "dvc_ldpca_decode_noalloc: bad arguments";
    return DVC_E_ARG;
  }
  if (count > kMaxCodewords) {
    c.err = "dvc_ldpca_decode_noalloc: " + std::to_string(count) + " codewords exceed the limit of " +
            std::to_string(kMaxCodewords) + " per call";
    return DVC_E_ARG;
  }
  const dvc::LadderDev *L = c.ladder(n);
  if (!L) {
    c.err = "dvc_ldpca_decode_noalloc: no ladder for codeword length " + std::to_string(n);
    return DVC_E_ARG;
  }
  if (c.device < 0 || c.device >= kMaxDevices) {
    c.err = "dvc_ldpca_decode_noalloc: device ordinal out of range";
    return DVC_E_ARG;
  }
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) {
    c.err = "dvc_ldpca_decode_noalloc: cudaGetDevice failed";
    return DVC_E_CUDA;
  }
  if (cur != c.device && cudaSetDevice(c.device) != cudaSuccess) {
    c.err = "dvc_ldpca_decode_noalloc: cudaSetDevice failed";
    return DVC_E_CUDA;
  }
  dvc::LdpcaJob *jobs = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_jobs_addr[c.device]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_jobs);
      if (e != cudaSuccess) {
        c.err = std::string("dvc_ldpca_decode_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
        if (cur != c.device) cudaSetDevice(cur);
        return DVC_E_CUDA;
      }
      g_jobs_addr[c.device] = (dvc::LdpcaJob *)p;
    }
    jobs = g_jobs_addr[c.device];
  }
  cudaStream_t s = (cudaStream_t)stream;
  fill_jobs_kernel<<<(count + 127) / 128, 128, 0, s>>>(jobs, count, n, d_lr, d_acc, d_crc, d_decoded, d_results,
                                                       d_entropy);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = dvc::launch_ldpca(*L, jobs, count, c.xlm, max_iter, s);
  if (cur != c.device) cudaSetDevice(cur);
  if (e != cudaSuccess) {
    c.err = std::string("dvc_ldpca_decode_noalloc: ") + cudaGetErrorString(e);
    return DVC_E_CUDA;
  }
  return DVC_OK;
}
