// Per-device decoder context: library-exact math tables, LDPCA ladders,
// streams and reusable device buffers.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dvc_types.h"
#include "ladder.h"
#include "libm_tables.h"

namespace dvc {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  bool ensure(size_t b);
  // the same, but a growth frees and allocates in the order of `stream`
  // (cudaFreeAsync / cudaMallocAsync), without waiting for work on other streams;
  // for buffers used on that stream only (stream nullptr: as ensure)
  bool ensure(size_t b, cudaStream_t stream);
  void release();
  template <class T>
  T *as() const { return (T *)p; }
};

struct Context {
  int device = 0;
  std::string data_dir, table_dir;
  std::string err;
  XlmHost xlm_host;
  XlmDev xlm{};
  std::vector<void *> xlm_allocs;
  size_t phi_bytes = 0;  // device bytes of the packed phi table
  std::vector<LadderHost> ladders_host;
  std::vector<LadderGpu> ladders_gpu;
  cudaStream_t stream = nullptr;
  // scratch for the batched LDPCA entry point
  DevBuf ld_lr, ld_acc, ld_dec, ld_res, ld_ent, ld_jobs;
  // buffers of the batched LDPCA entry point (dvc_ldpca_decode_batch)
  DevBuf bt_lr, bt_acc, bt_dec, bt_res, bt_ent, bt_cw, bt_state;
  // count of reconstruction steps near a rounding tie (recon_kernel), one
  // unsigned 64-bit word, zeroed at set-up
  DevBuf near_ties;

  bool init(const char *data_dir, const char *table_dir, int device);
  void release();
  const LadderDev *ladder(int n) const;
  const LadderHost *ladder_host(int n) const;
  bool fail(const std::string &m) {
    err = m;
    return false;
  }
  bool cuda_ok(cudaError_t e, const char *what);
};

}  // namespace dvc
