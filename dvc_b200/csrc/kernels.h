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
// threads per codeword block of the ladder kernel: CIF 1024 or 512, QCIF 1024,
// 512 or 256 (other values select the defaults, 1024 for both)
void set_ldpca_threads(int nt, int nt_qcif);
// threads per search block of updateSI (64, 128 or 256) and of the forward
// motion search (128, 256 or 512); other values select 128 and 256
void set_me_shapes(int si_threads, int fme_threads);
// L2 persisting access window of the LDPCA kernels' table reads (num_bytes 0: none)
void set_phi_window(const void *base, size_t num_bytes, float hit_ratio);
// batched form: one persistent launch over codewords of both lengths
// (k_ldpca_batch.cu); state + slot bytes per codeword from ldpca_batch_state_bytes
size_t ldpca_batch_state_bytes(int count);
cudaError_t launch_ldpca_batch(LdpcaBatch A, int count, int grid, cudaStream_t stream);
// encoder: accumulated syndromes (n/8 bytes, MSB first) and CRC-8 of `count` source bitplanes
cudaError_t launch_ldpca_encode(const LadderDev &L, const uint8_t *bits_dev, int count, uint8_t *acc_dev,
                                uint8_t *crc_dev, cudaStream_t stream);

}  // namespace dvc
