// Launch entry points of the decoder kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "dvc_types.h"
#include "libm_tables.h"

namespace dvc {

size_t ldpca_smem_size(int n, int e);
// direct form: one block per codeword, no scratch
cudaError_t launch_ldpca(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt,
                         int max_iter, cudaStream_t stream);
// speculative form: K blocks per codeword, the last of them writes the result;
// scratch from ldpca_spec_carve, put in its initial state once by
// ldpca_spec_reset (each launch leaves it so for the next)
size_t ldpca_spec_scratch_bytes(int n, int num_jobs, int K);
LdpcaSpec ldpca_spec_carve(void *base, int num_jobs, int K);
cudaError_t ldpca_spec_reset(const LdpcaSpec &sp, int num_jobs, int K, cudaStream_t stream);
cudaError_t launch_ldpca_spec(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt,
                              int max_iter, int K, const LdpcaSpec &sp, cudaStream_t stream);
void set_ldpca_threads(int nt);
// encoder: accumulated syndromes (n/8 bytes, MSB first) and CRC-8 of `count` source bitplanes
cudaError_t launch_ldpca_encode(const LadderDev &L, const uint8_t *bits_dev, int count, uint8_t *acc_dev,
                                uint8_t *crc_dev, cudaStream_t stream);

}  // namespace dvc
