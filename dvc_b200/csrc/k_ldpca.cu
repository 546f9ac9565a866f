// LDPCA rate-adaptive decoding on the device: one thread block per codeword
// runs the whole request ladder (start code from the conditional-entropy bound,
// syndrome of each ladder code from the accumulated syndrome, sum-product belief
// propagation with the parity early stop, CRC-8 acceptance, and the GF(2)
// inverse at full rate) with no host round trip between requests.
//
// Reference: DvcDec/src/LdpcaDecoder.cpp LdpcaDecoder (:646-771),
// beliefPropagation (:462-580), ComputeCE (:127-143), invH_mul (:624-643).
// The per-edge arithmetic, the order of every float sum (row sums in edge
// order, column sums in edge order, the entropy sum in block order) and the
// library functions (logf, tanhf via exact_libm) follow the reference exactly,
// so decoded bits, accepted codes and rates are identical to it.
//
// Shared-memory layout per codeword (n bits, e edges; CIF n=6336, e=19008):
//   msg[e] f32   the single edge-message array, updated in place:
//                v->c message -> phi(|v->c|) -> c->v message -> next v->c
//   llr[n] f32   log(p0/p1)
//   rowt[n] f32  row sums of phi (m <= n rows)
//   sgn[e/32]    sign bits of the v->c messages
//   dec[n], synd[n], acc[n] u8  (synd bit 1 holds the row sign parity during BP)
// CIF: 148 KB, one block per SM; QCIF: 37 KB.
#include <cuda_runtime.h>

#include "dvc_common.cuh"
#include "dvc_types.h"
#include "kernels.h"

namespace dvc {

#define LDPCA_LOG2 (0.693147181f)  // LdpcaDecoder.cpp:18

static __host__ __device__ size_t ldpca_smem_bytes(int n, int e) {
  size_t b = 0;
  b += (size_t)e * 4;                  // msg
  b += (size_t)n * 4;                  // llr
  b += (size_t)n * 4;                  // rowt
  b += (size_t)((e + 31) / 32) * 4;    // sgn
  b += (size_t)n * 3;                  // dec, synd, acc
  return (b + 15) & ~(size_t)15;
}

size_t ldpca_smem_size(int n, int e) { return ldpca_smem_bytes(n, e); }

template <int NT>
__global__ void __launch_bounds__(NT, 1)
    ldpca_ladder_kernel(LadderDev L, const LdpcaJob *__restrict__ jobs, XlmDev xt, int max_iter) {
  extern __shared__ __align__(16) uint8_t smem[];
  const LdpcaJob J = jobs[blockIdx.x];
  if (!J.active) return;
  const int n = L.n, E = L.e, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float *msg = reinterpret_cast<float *>(smem);
  float *llr = msg + E;
  float *rowt = llr + n;
  uint32_t *sgn = reinterpret_cast<uint32_t *>(rowt + n);
  uint8_t *dec = reinterpret_cast<uint8_t *>(sgn + (E + 31) / 32);
  uint8_t *synd = dec + n;
  uint8_t *acc = synd + n;
  __shared__ uint32_t s_ured[NT / 32];
  __shared__ int s_start, s_accepted;
  __shared__ float s_entropy;

  // accumulated syndrome bits (ByteToBit, LdpcaDecoder.cpp:81-107) and the
  // entropy terms (ComputeCE): H = sum_k (P(-log P + log(1-P)) - log(1-P)) / LOG2, P = LR/(1+LR)
  for (int k = tid; k < n; k += NT) {
    acc[k] = (uint8_t)((J.acc[k >> 3] >> (7 - (k & 7))) & 1);
    const float lr = J.lr[k];
    const float pco = lr / (1.0f + lr);
    const float tmp = xl_logf(xt, 1.0f - pco);
    msg[k] = (pco * (-xl_logf(xt, pco) + tmp) - tmp) / LDPCA_LOG2;
    llr[k] = xl_logf(xt, lr);  // LdpcaDecoder.cpp:665-666
    if (J.llr_out) J.llr_out[k] = llr[k];
  }
  __syncthreads();
  if (tid == 0) {
    // the bound is a sequential float sum in block order
    float h = 0.0f;
    for (int k = 0; k < n; k++) h += msg[k];
    h /= (float)n;
    if (J.use_given_entropy) h = J.given_entropy;
    int start = 0;
    while (start < L.num_codes - 1 && L.code_rate[start] < h) start++;
    s_entropy = h;
    s_start = start;
    s_accepted = L.num_codes - 1;
  }
  __syncthreads();
  const int start = s_start;
  int total_iters = 0;

  for (int code = start; code < L.num_codes; code++) {
    const int m = L.synd_len[code];
    const int nb = L.bpp[code];
    const int *idx = L.idx + (size_t)code * L.period;
    // syndrome of this code: differences of the accumulated syndrome at the
    // kept positions (LdpcaDecoder.cpp:684-693)
    for (int k = tid; k < m; k += NT) {
      const int cur = idx[k % nb] + (k / nb) * L.period;
      uint8_t s = acc[cur];
      if (k > 0) s ^= acc[idx[(k - 1) % nb] + ((k - 1) / nb) * L.period];
      synd[k] = s;
    }
    __syncthreads();

    if (m == n) {
      // full rate: decoded = inv(H) * syndrome over GF(2) (LdpcaDecoder.cpp:695-716)
      uint32_t *sw = sgn;  // reuse: n/32 syndrome words
      for (int base = warp * 32; base < n; base += NT) {
        const int k = base + lane;
        const uint32_t b = __ballot_sync(0xffffffffu, k < n && synd[k]);
        if (lane == 0) sw[base >> 5] = b;
      }
      __syncthreads();
      for (int j = tid; j < n; j += NT) {
        const uint32_t *row = L.invh + (size_t)j * L.invh_words;
        uint32_t x = 0;
        for (int w = 0; w < L.invh_words; w++) x ^= row[w] & sw[w];
        dec[j] = (uint8_t)(__popc(x) & 1);
      }
      __syncthreads();
      if (tid == 0) s_accepted = code;
      break;
    }

    // ---- belief propagation (beliefPropagation, LdpcaDecoder.cpp:462-580)
    const int *rp = L.row_ptr + (size_t)code * (n + 1);
    const uint16_t *re = L.row_edge + (size_t)code * E;
    const uint16_t *ir = L.ir + (size_t)code * E;
    for (int e = tid; e < E; e += NT) msg[e] = llr[L.edge_col[e]];
    __syncthreads();
    bool converged = false;
    int it = 0;
    for (; it < max_iter && !converged; it++) {
      // (1) sign and magnitude of every v->c message; phi of the magnitude
      for (int base = warp * 32; base < E; base += NT) {
        const int e = base + lane;
        bool neg = false;
        if (e < E) {
          const float v = msg[e];
          neg = (__float_as_uint(v) >> 31) != 0;
          const float mag = neg ? -v : v;
          msg[e] = xl_phi(xt, (mag + 1e-9f) / 2.0f);
        }
        const uint32_t b = __ballot_sync(0xffffffffu, neg);
        if (lane == 0) sgn[base >> 5] = b;
      }
      __syncthreads();
      // (2) per row: sum of phi in edge order, sign parity incl. the syndrome
      for (int r = tid; r < m; r += NT) {
        float s = 0.0f;
        uint32_t par = synd[r] & 1u;
        for (int p = rp[r]; p < rp[r + 1]; p++) {
          const int e = re[p];
          s += msg[e];
          par ^= (sgn[e >> 5] >> (e & 31)) & 1u;
        }
        rowt[r] = s;
        synd[r] = (uint8_t)((synd[r] & 1u) | (par << 1));  // bit 1: sign parity of the row
      }
      __syncthreads();
      // (3) c->v messages: phi(row sum - own phi) with the product of the other signs
      for (int e = tid; e < E; e += NT) {
        const int r = ir[e];
        const float c = xl_phi(xt, (rowt[r] - msg[e] + 1e-9f) / 2.0f);
        const uint32_t neg = ((uint32_t)synd[r] >> 1) ^ ((sgn[e >> 5] >> (e & 31)) & 1u);
        msg[e] = c * (neg ? -1.0f : 1.0f);
      }
      __syncthreads();
      // (4) per column: total in edge order, extrinsic messages, hard decision
      for (int k = tid; k < n; k += NT) {
        const int e0 = L.jc[k], e1 = L.jc[k + 1];
        float tmp = llr[k];
        for (int e = e0; e < e1; e++) tmp += msg[e];
        for (int e = e0; e < e1; e++) msg[e] = tmp - msg[e];
        dec[k] = (uint8_t)(__float_as_uint(tmp) >> 31);
      }
      __syncthreads();
      // (5) parity check of every row
      int wrong = 0;
      for (int r = tid; r < m; r += NT) {
        uint32_t par = synd[r] & 1u;
        for (int p = rp[r]; p < rp[r + 1]; p++) par ^= dec[L.edge_col[re[p]]];
        wrong |= (int)par;
      }
      converged = __syncthreads_or(wrong) == 0;
    }
    total_iters += it;
    // restore the plain syndrome bits (bit 1 held the row sign parity)
    for (int k = tid; k < m; k += NT) synd[k] &= 1u;
    __syncthreads();
    if (converged) {
      // CRC-8 of the decoded bitplane as the xor of single-bit CRCs
      uint32_t c = 0;
      for (int k = tid; k < n; k += NT)
        if (dec[k]) c ^= L.crc_tab[k];
      for (int o = 16; o > 0; o >>= 1) c ^= __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) s_ured[warp] = c;
      __syncthreads();
      if (tid == 0) {
        uint32_t t = 0;
        for (int w = 0; w < NT / 32; w++) t ^= s_ured[w];
        s_ured[0] = t;
      }
      __syncthreads();
      const bool ok = (int)(s_ured[0] & 0xffu) == J.crc;
      __syncthreads();
      if (ok) {
        if (tid == 0) s_accepted = code;
        break;
      }
    }
  }
  __syncthreads();
  const int accepted = s_accepted;
  if (tid == 0) {
    J.result[0] = L.synd_len[accepted] + 8;
    J.result[1] = start;
    J.result[2] = accepted;
    J.result[3] = total_iters;
    if (J.entropy) *J.entropy = s_entropy;
  }
  if (J.decoded)
    for (int k = tid; k < n; k += NT) J.decoded[k] = dec[k];
  if (J.recons_trans) {
    // putBitplaneToCoeff (bitplane.cpp:4-22): append the bit to WZ blocks' indices
    const int b4w = J.w >> 2, b8w = J.w >> 3;
    const int row = J.index_in_blk >> 2, col = J.index_in_blk & 3;
    for (int k = tid; k < n; k += NT) {
      const int i = k / b4w, j = k - i * b4w;
      if (J.mode[(i >> 1) * b8w + (j >> 1)] == DVC_WZ_B) {
        int *p = J.recons_trans + ((i << 2) + row) * J.w + (j << 2) + col;
        *p = (*p << 1) + (int)dec[k];
      }
    }
  }
}

cudaError_t launch_ldpca(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt,
                         int max_iter, cudaStream_t stream) {
  if (num_jobs <= 0) return cudaSuccess;
  constexpr int NT = 1024;
  const size_t smem = ldpca_smem_bytes(L.n, L.e);
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(ldpca_ladder_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  ldpca_ladder_kernel<NT><<<num_jobs, NT, smem, stream>>>(L, jobs_dev, xt, max_iter);
  return cudaGetLastError();
}

}  // namespace dvc
