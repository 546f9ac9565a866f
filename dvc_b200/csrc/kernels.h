// Launch entry points of the decoder kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "dvc_types.h"
#include "libm_tables.h"

namespace dvc {

size_t ldpca_smem_size(int n, int e);
cudaError_t launch_ldpca(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt,
                         int max_iter, cudaStream_t stream);

}  // namespace dvc
