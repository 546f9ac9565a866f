// LDPCA encoder on the device: accumulated syndromes and CRC-8 of many source
// bitplanes at once (LdpcaEncoder.cpp:64-95, crc8.h:57-67), for generating
// decoder inputs on the GPU and for encode/decode round trips.
//
// One block per codeword: the full-rate syndrome s = H x (every column has
// degree 3, edge e = 3k + i in row ir_full[e]) is built with shared-memory
// xors, the accumulated syndrome is its inclusive prefix xor over rows, packed
// MSB first as the bitstream stores it, and the CRC is the xor of the
// single-bit CRCs of the set source bits (the CRC is linear for a fixed length
// with zero initial value and no final xor).
#include <cuda_runtime.h>

#include "dvc_types.h"
#include "kernels.h"

namespace dvc {

template <int NT>
__global__ void __launch_bounds__(NT) ldpca_encode_kernel(LadderDev L, const uint8_t *__restrict__ bits,
                                                          uint8_t *__restrict__ acc_bytes, uint8_t *__restrict__ crc) {
  extern __shared__ uint32_t s_synd[];  // [n] one word per row (0/1)
  __shared__ uint32_t s_part[NT / 32];
  __shared__ uint32_t s_carry;
  const int n = L.n, cw = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint8_t *x = bits + (size_t)cw * n;
  for (int r = tid; r < n; r += NT) s_synd[r] = 0;
  __syncthreads();
  uint32_t c = 0;
  for (int k = tid; k < n; k += NT)
    if (x[k] & 1) {
      c ^= __ldg(L.crc_tab + k);
#pragma unroll
      for (int i = 0; i < 3; i++) atomicXor(&s_synd[__ldg(L.ir_full + 3 * k + i)], 1u);
    }
  // CRC: xor over the block
  for (int o = 16; o > 0; o >>= 1) c ^= __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) s_part[warp] = c;
  __syncthreads();
  if (tid == 0) {
    uint32_t t = 0;
    for (int w = 0; w < NT / 32; w++) t ^= s_part[w];
    crc[cw] = (uint8_t)t;
    s_carry = 0;
  }
  __syncthreads();
  // inclusive prefix xor over rows, NT rows at a time; pack 8 rows per byte
  uint8_t *out = acc_bytes + (size_t)cw * (n / 8);
  for (int base = 0; base < n; base += NT) {
    const int r = base + tid;
    uint32_t v = r < n ? s_synd[r] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v ^= u;
    }
    if (lane == 31) s_part[warp] = v;
    __syncthreads();
    uint32_t pre = s_carry;
    for (int w = 0; w < warp; w++) pre ^= s_part[w];
    v ^= pre;
    if (r < n) s_synd[r] = v;
    __syncthreads();
    if (tid == NT - 1) s_carry = v;
    __syncthreads();
  }
  for (int b = tid; b < n / 8; b += NT) {
    uint32_t byte = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) byte |= (s_synd[8 * b + i] & 1u) << (7 - i);
    out[b] = (uint8_t)byte;
  }
}

cudaError_t launch_ldpca_encode(const LadderDev &L, const uint8_t *bits_dev, int count, uint8_t *acc_dev,
                                uint8_t *crc_dev, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  ldpca_encode_kernel<256><<<count, 256, (size_t)L.n * 4, stream>>>(L, bits_dev, acc_dev, crc_dev);
  return cudaGetLastError();
}

}  // namespace dvc
