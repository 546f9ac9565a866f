// LDPCA rate-adaptive decoding on the device: the whole request ladder (start
// code from the conditional-entropy bound, syndrome of each ladder code from the
// accumulated syndrome, sum-product belief propagation with the parity early
// stop, CRC-8 acceptance, and the GF(2) inverse at full rate) with no host round
// trip between requests.
//
// Reference: DvcDec/src/LdpcaDecoder.cpp LdpcaDecoder (:646-771),
// beliefPropagation (:462-580), ComputeCE (:127-143), invH_mul (:624-643).
// The per-edge arithmetic, the order of every float sum (row sums in edge
// order, column sums in edge order, the entropy sum in block order) and the
// library functions (logf, tanhf via exact_libm) follow the reference exactly,
// so decoded bits, accepted codes and rates are identical to it.
//
// Two launch forms share one kernel:
//  * direct (K = 1, no scratch): one thread block per codeword walks the ladder
//    code by code, exactly as the reference does;
//  * speculative (K >= 1, scratch): K blocks per codeword try the ladder codes
//    start+k, start+k+K, ... concurrently.  A code is accepted by the reference
//    iff BP converges and the CRC matches and no lower code was accepted, i.e.
//    the accepted code is the lowest code that succeeds; blocks publish
//    successes with atomicMin, stop at (or abandon) codes above the best success
//    so far, and the last of the K blocks to finish (a counter with fences)
//    picks the lowest success (or the full-rate inverse when none), writes the
//    outputs and resets the codeword's scratch for the next launch, so results
//    are identical to the sequential ladder while idle SMs shorten it, with one
//    launch per bitplane step.
//
// Edge messages are kept in row order (each row's edges contiguous, in
// increasing edge index), so a row sum is a sequential pass over contiguous
// shared memory in the reference's summation order; columns (every column has
// degree 3) reach their edges through the per-code position array.  The
// parity check of an iteration's hard decision is folded into the next row
// pass.  The magnitude phi(y) = -logf(tanhf(y)) is one record read of the
// packed table (dvc_common.cuh; its hot part stays in L2), and the reads of a
// pass are issued in batches so that several are in flight per thread.  Shared
// memory is kept under 132 KB so that the rest of the SM's 256 KB stays L1
// cache for the per-code position arrays and the table records that
// successive iterations read again.
//
// Shared memory per codeword (n bits, e edges; CIF n=6336, e=19008: 124 KB):
//   msg[e]  f32  edge messages by row-order position, in place:
//                phi(|v->c|) -> c->v -> next phi(|v->c|)
//   rowt[n] f32  row sums (after decoding: the decoded bits, one byte each)
//   sgd[e]  u8   bit 0: sign of the v->c message, bit 1: hard decision of its column
//   rpar[n] u8   bit 0: syndrome bit of the row, bit 1: sign parity of the row
// The log-LRs of a thread's columns stay in registers.
#include <cuda_runtime.h>

#include <atomic>

#include "dvc_common.cuh"
#include "dvc_types.h"
#include "kernels.h"

namespace dvc {

#define LDPCA_LOG2 (0.693147181f)  // LdpcaDecoder.cpp:18
#define LDPCA_NONE 0x7f7f7f7f      // "no success yet" (memset pattern 0x7f)

// largest codeword length; each thread keeps the log-LRs of up to
// LDPCA_MAX_N / NT columns in registers
#define LDPCA_MAX_N 6336

static __host__ __device__ size_t ldpca_smem_bytes(int n, int e) {
  size_t b = (size_t)e * 4;  // msg
  b += (size_t)n * 4;        // rowt
  b += (size_t)e;            // sgd
  b += (size_t)n;            // rpar
  return (b + 15) & ~(size_t)15;
}

size_t ldpca_smem_size(int n, int e) { return ldpca_smem_bytes(n, e); }

// fused bitplane insertion (putBitplaneToCoeff, bitplane.cpp:4-22)
__device__ __forceinline__ void put_bitplane(const LdpcaJob &J, const uint8_t *dec, int n) {
  const int b4w = J.w >> 2, b8w = J.w >> 3;
  const int row = J.index_in_blk >> 2, col = J.index_in_blk & 3;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int i = k / b4w, j = k - i * b4w;
    if (J.mode[(i >> 1) * b8w + (j >> 1)] == DVC_WZ_B) {
      int *p = J.recons_trans + ((i << 2) + row) * J.w + (j << 2) + col;
      *p = (*p << 1) + (int)dec[k];
    }
  }
}

// decoded = inv(H) * syndrome of the full-rate code (LdpcaDecoder.cpp:695-716);
// syndrome words are built in `sw` (n/32 words of shared memory)
__device__ void invh_decode(const LadderDev &L, const uint8_t *synd, uint8_t *dec, uint32_t *sw) {
  const int n = L.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nt = blockDim.x;
  for (int base = warp * 32; base < n; base += nt) {
    const int k = base + lane;
    const uint32_t b = __ballot_sync(0xffffffffu, k < n && (synd[k] & 1));
    if (lane == 0) sw[base >> 5] = b;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += nt) {
    const uint32_t *row = L.invh + (size_t)j * L.invh_words;
    uint32_t x = 0;
    for (int w = 0; w < L.invh_words; w++) x ^= __ldg(row + w) & sw[w];
    dec[j] = (uint8_t)(__popc(x) & 1);
  }
  __syncthreads();
}

// syndrome of ladder code `code` from the accumulated syndrome bits (LdpcaDecoder.cpp:684-693)
__device__ __forceinline__ void build_syndrome(const LadderDev &L, int code, const uint8_t *acc, uint8_t *synd) {
  const int m = L.synd_len[code], nb = L.bpp[code];
  const int *idx = L.idx + (size_t)code * L.period;
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    uint8_t s = acc[idx[k % nb] + (k / nb) * L.period];
    if (k > 0) s ^= acc[idx[(k - 1) % nb] + ((k - 1) / nb) * L.period];
    synd[k] = s;
  }
}

// the same from the packed accumulated-syndrome bytes (MSB first, ByteToBit)
__device__ __forceinline__ uint8_t acc_bit(const uint8_t *packed, int i) {
  return (uint8_t)((__ldg(packed + (i >> 3)) >> (7 - (i & 7))) & 1);
}
__device__ __forceinline__ void build_syndrome_packed(const LadderDev &L, int code, const uint8_t *packed,
                                                      uint8_t *synd) {
  const int m = L.synd_len[code], nb = L.bpp[code];
  const int *idx = L.idx + (size_t)code * L.period;
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    uint8_t s = acc_bit(packed, idx[k % nb] + (k / nb) * L.period);
    if (k > 0) s ^= acc_bit(packed, idx[(k - 1) % nb] + ((k - 1) / nb) * L.period);
    synd[k] = s;
  }
}

template <int NT>
__global__ void __launch_bounds__(NT, 1)
    ldpca_ladder_kernel(LadderDev L, const LdpcaJob *__restrict__ jobs, XlmDev xt, int max_iter, int K,
                        LdpcaSpec sp) {
  constexpr int MAXC = (LDPCA_MAX_N + NT - 1) / NT;  // columns per thread
  constexpr int UNR = 8;                             // edge-pass table reads in flight per thread
  constexpr int CB = NT >= 1024 ? 1 : 4;             // column-pass columns per batch (3 reads each)
  extern __shared__ __align__(16) uint8_t smem[];
  const int j = blockIdx.x / K, kk = blockIdx.x - j * K;
  const LdpcaJob J = jobs[j];
  if (!J.active) return;
  const bool spec = sp.best != nullptr;
  const int n = L.n, E = L.e, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float *msg = reinterpret_cast<float *>(smem);
  float *rowt = msg + E;
  uint8_t *sgd = reinterpret_cast<uint8_t *>(rowt + n);
  uint8_t *rpar = sgd + E;
  uint8_t *dec = reinterpret_cast<uint8_t *>(rowt);  // decoded bits, once BP is over
  __shared__ uint32_t s_ured[NT / 32];
  __shared__ int s_start, s_accepted, s_stop;
  __shared__ uint4 s_pdesc[XL_PHI_MAX_BINADES];
  const XlSmall xs = xl_small_global(xt);
  xl_phi_stage(xt, s_pdesc);

  // accumulated syndrome bits (ByteToBit, LdpcaDecoder.cpp:81-107), entropy
  // terms H_k = (P(-log P + log(1-P)) - log(1-P)) / LOG2 with P = LR/(1+LR)
  // (ComputeCE), and log LR (LdpcaDecoder.cpp:665-666)
  float llr[MAXC];
#pragma unroll
  for (int c = 0; c < MAXC; c++) {
    const int k = tid + c * NT;
    llr[c] = 0.0f;
    if (k < n) {
      const float lr = J.lr[k];
      const float pco = lr / (1.0f + lr);
      const float tmp = xl_logf(xt, xs, 1.0f - pco);
      msg[k] = (pco * (-xl_logf(xt, xs, pco) + tmp) - tmp) / LDPCA_LOG2;
      llr[c] = xl_logf(xt, xs, lr);
      if (J.llr_out && kk == 0) J.llr_out[k] = llr[c];
    }
  }
  __syncthreads();
  if (tid == 0) {
    // the bound is a sequential float sum in block order
    float h = 0.0f;
    int k = 0;
    for (; k + 8 <= n; k += 8) {
      const float v0 = msg[k], v1 = msg[k + 1], v2 = msg[k + 2], v3 = msg[k + 3];
      const float v4 = msg[k + 4], v5 = msg[k + 5], v6 = msg[k + 6], v7 = msg[k + 7];
      h += v0;
      h += v1;
      h += v2;
      h += v3;
      h += v4;
      h += v5;
      h += v6;
      h += v7;
    }
    for (; k < n; k++) h += msg[k];
    h /= (float)n;
    if (J.use_given_entropy) h = J.given_entropy;
    int start = 0;
    while (start < L.num_codes - 1 && L.code_rate[start] < h) start++;
    s_start = start;
    s_accepted = L.num_codes - 1;
    if (kk == 0) {
      if (J.entropy) *J.entropy = h;
      if (spec) sp.start[j] = start;
    }
  }
  __syncthreads();
  const int start = s_start;
  const int last = L.num_codes - 1;
  int total_iters = 0;
  volatile int *bestp = spec ? sp.best + j : nullptr;

  for (int code = start + kk; code < last; code += K) {
    if (spec) {
      if (tid == 0) s_stop = *bestp < code;
      __syncthreads();
      if (s_stop) break;
    }
    const int m = L.synd_len[code];
    const uint16_t *__restrict__ pos = L.pos + (size_t)code * E;
    const uint16_t *__restrict__ rid = L.rid + (size_t)code * E;
    build_syndrome_packed(L, code, J.acc, rpar);
    __syncthreads();
    const int *rp = L.row_ptr + (size_t)code * (n + 1);
    // first magnitudes: phi(|LLR|) on the three edges of each column
    {
      float ph[MAXC];
#pragma unroll
      for (int c = 0; c < MAXC; c++)
        ph[c] = tid + c * NT < n ? xl_phi(xt, s_pdesc, (fabsf(llr[c]) + 1e-9f) / 2.0f) : 0.0f;
#pragma unroll
      for (int c = 0; c < MAXC; c++) {
        const int k = tid + c * NT;
        if (k < n) {
          const uint8_t ng = (uint8_t)(__float_as_uint(llr[c]) >> 31);
#pragma unroll
          for (int i = 0; i < 3; i++) {
            const int p = __ldg(pos + 3 * k + i);
            msg[p] = ph[c];
            sgd[p] = ng;
          }
        }
      }
    }
    __syncthreads();
    bool converged = false;
    int it = 0;
    for (;;) {
      // (R) rows: sum of the magnitudes in edge order and the sign parity with
      //     the syndrome bit, for the next edge pass; from the second pass on
      //     also the parity check of the previous hard decision
      int wrong = 0;
      for (int r = tid; r < m; r += NT) {
        const int p0 = rp[r], p1 = rp[r + 1];
        float s = 0.0f;
        uint32_t x = 0;  // bit 0: xor of signs, bit 1: xor of decisions
        for (int p = p0; p < p1; p++) {
          s += msg[p];
          x ^= sgd[p];
        }
        const uint32_t syn = rpar[r] & 1u;
        rowt[r] = s;
        rpar[r] = (uint8_t)(syn | (((x & 1u) ^ syn) << 1));
        wrong |= (int)(((x >> 1) ^ syn) & 1u);
      }
      if (spec && tid == 0) s_stop = *bestp < code;
      const int any_wrong = __syncthreads_or(wrong);
      if (it > 0 && !any_wrong) {
        converged = true;
        break;
      }
      // abandon a code above a known success
      if (it == max_iter || (spec && s_stop)) break;
      it++;
      // (E) edges: c->v = phi(row sum - own magnitude) with the product of
      //     the other signs
      for (int p0 = tid; p0 < E; p0 += UNR * NT) {
        float c[UNR];
        int rr[UNR];
#pragma unroll
        for (int q = 0; q < UNR; q++) {
          // lanes past the last edge repeat it (no branch, so that the UNR
          // table reads are in flight together) and store nothing
          const int p = min(p0 + q * NT, E - 1);
          rr[q] = __ldg(rid + p);
          c[q] = xl_phi(xt, s_pdesc, (rowt[rr[q]] - msg[p] + 1e-9f) / 2.0f);
        }
#pragma unroll
        for (int q = 0; q < UNR; q++) {
          const int p = p0 + q * NT;
          if (p < E) msg[p] = c[q] * ((((uint32_t)rpar[rr[q]] >> 1) ^ (sgd[p] & 1u)) ? -1.0f : 1.0f);
        }
      }
      __syncthreads();
      // (C) columns: total in edge order, hard decision, extrinsic messages
      //     and their magnitudes for the next iteration
#pragma unroll
      for (int c0 = 0; c0 < MAXC; c0 += CB) {
        float ph[CB][3];
        uint32_t sb[CB][3];
        int pp[CB][3];
#pragma unroll
        for (int b = 0; b < CB; b++) {
          const int c = c0 + b, k = tid + c * NT;
          if (c < MAXC && k < n) {
            float mv[3];
#pragma unroll
            for (int i = 0; i < 3; i++) {
              pp[b][i] = __ldg(pos + 3 * k + i);
              mv[i] = msg[pp[b][i]];
            }
            float tmp = llr[c];
            tmp += mv[0];
            tmp += mv[1];
            tmp += mv[2];
            const uint32_t d = __float_as_uint(tmp) >> 31;
#pragma unroll
            for (int i = 0; i < 3; i++) {
              const float v = tmp - mv[i];
              sb[b][i] = (__float_as_uint(v) >> 31) | (d << 1);
              ph[b][i] = xl_phi(xt, s_pdesc, (fabsf(v) + 1e-9f) / 2.0f);
            }
          }
        }
#pragma unroll
        for (int b = 0; b < CB; b++) {
          const int c = c0 + b, k = tid + c * NT;
          if (c < MAXC && k < n)
#pragma unroll
            for (int i = 0; i < 3; i++) {
              msg[pp[b][i]] = ph[b][i];
              sgd[pp[b][i]] = (uint8_t)sb[b][i];
            }
        }
      }
      __syncthreads();
    }
    total_iters += it;
    if (!converged) continue;
    // hard decision of each column (bit 1 of its edges' sgd) into dec, and the
    // CRC-8 of the decoded bitplane as the xor of single-bit CRCs (the CRC is
    // linear for a fixed length with zero initial value and no final xor)
    uint32_t c = 0;
    for (int k = tid; k < n; k += NT) {
      const uint8_t d = (uint8_t)((sgd[__ldg(pos + 3 * k)] >> 1) & 1u);
      dec[k] = d;
      if (d) c ^= __ldg(L.crc_tab + k);
    }
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
      if (spec) {
        uint8_t *slot = sp.slot_dec + (size_t)blockIdx.x * n;
        for (int k = tid; k < n; k += NT) slot[k] = dec[k];
        __syncthreads();
        if (tid == 0) {
          sp.slot_code[blockIdx.x] = code;
          __threadfence();
          atomicMin(sp.best + j, code);
        }
      }
      break;
    }
  }
  if (spec) {
    // the last of the codeword's K blocks to finish writes its result: the
    // lowest successful code (or the full-rate inverse when no code below it
    // succeeded), then puts the codeword's scratch back to its initial state
    // for the next launch (no memset between the steps of a batch)
    __shared__ int s_slot, s_iters;
    __syncthreads();
    if (tid == 0) {
      atomicAdd(sp.iters + j, total_iters);
      __threadfence();
      s_stop = atomicAdd(sp.done + j, 1) == K - 1;
    }
    __syncthreads();
    if (!s_stop) return;
    __threadfence();
    if (tid == 0) {
      const int best = __ldcg(sp.best + j);
      int acc = last, slot = -1;
      if (best != LDPCA_NONE && best < last)
        for (int k = 0; k < K; k++)
          if (__ldcg(sp.slot_code + j * K + k) == best) {
            slot = k;
            acc = best;
          }
      s_accepted = acc;
      s_slot = slot;
      s_iters = __ldcg(sp.iters + j);
    }
    __syncthreads();
    if (s_slot >= 0) {
      const uint8_t *src = sp.slot_dec + (size_t)(j * K + s_slot) * n;
      for (int k = tid; k < n; k += NT) dec[k] = __ldcg(src + k);
    }
    total_iters = s_iters;
    for (int k = tid; k < K; k += NT) sp.slot_code[j * K + k] = -1;
    if (tid == 0) {
      sp.best[j] = LDPCA_NONE;
      sp.iters[j] = 0;
      sp.done[j] = 0;
    }
  }
  __syncthreads();
  const int accepted = s_accepted;
  if (accepted == last) {
    build_syndrome_packed(L, last, J.acc, rpar);
    __syncthreads();
    invh_decode(L, rpar, dec, reinterpret_cast<uint32_t *>(msg));
  }
  if (tid == 0) {
    J.result[0] = L.synd_len[accepted] + 8;
    J.result[1] = start;
    J.result[2] = accepted;
    J.result[3] = total_iters;
  }
  if (J.decoded)
    for (int k = tid; k < n; k += NT) J.decoded[k] = dec[k];
  if (J.recons_trans) put_bitplane(J, dec, n);
}

template <int NT>
static cudaError_t launch_nt(const LadderDev &L, const LdpcaJob *jobs, int num_jobs, const XlmDev &xt, int max_iter,
                             int K, const LdpcaSpec &sp, cudaStream_t stream) {
  if (L.n > LDPCA_MAX_N) return cudaErrorInvalidValue;
  const size_t smem = ldpca_smem_bytes(L.n, L.e);
  // the attribute is per device: set it once for each device
  static std::atomic<uint64_t> attr_set{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    const size_t most = ldpca_smem_bytes(LDPCA_MAX_N, 3 * LDPCA_MAX_N);
    e = cudaFuncSetAttribute(ldpca_ladder_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most);
    if (e != cudaSuccess) return e;
    // the smallest shared-memory split that holds one block, so that the rest
    // of the SM's 256 KB is L1 for the phi records, which BP iterations re-read
    // (percent of the 228 KB maximum; the driver rounds up to a supported split)
    const int pct = (int)(((most + 4096) * 100 + 228 * 1024 - 1) / (228 * 1024));
    e = cudaFuncSetAttribute(ldpca_ladder_kernel<NT>, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e != cudaSuccess) return e;
    attr_set.fetch_or(bit);
  }
  ldpca_ladder_kernel<NT><<<num_jobs * K, NT, smem, stream>>>(L, jobs, xt, max_iter, K, sp);
  return cudaGetLastError();
}

static int g_ldpca_threads = 1024;

void set_ldpca_threads(int nt) { g_ldpca_threads = (nt == 512) ? 512 : 1024; }

cudaError_t launch_ldpca(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt, int max_iter,
                         cudaStream_t stream) {
  if (num_jobs <= 0) return cudaSuccess;
  LdpcaSpec none{};
  return g_ldpca_threads == 512 ? launch_nt<512>(L, jobs_dev, num_jobs, xt, max_iter, 1, none, stream)
                                : launch_nt<1024>(L, jobs_dev, num_jobs, xt, max_iter, 1, none, stream);
}

size_t ldpca_spec_scratch_bytes(int n, int num_jobs, int K) {
  return (size_t)num_jobs * 16 + (size_t)num_jobs * K * 4 + (size_t)num_jobs * K * n + 64;
}

LdpcaSpec ldpca_spec_carve(void *base, int num_jobs, int K) {
  LdpcaSpec sp;
  uint8_t *p = (uint8_t *)base;
  sp.best = (int *)p;
  p += (size_t)num_jobs * 4;
  sp.iters = (int *)p;
  p += (size_t)num_jobs * 4;
  sp.start = (int *)p;
  p += (size_t)num_jobs * 4;
  sp.done = (int *)p;
  p += (size_t)num_jobs * 4;
  sp.slot_code = (int *)p;
  p += (size_t)num_jobs * K * 4;
  sp.slot_dec = p;
  return sp;
}

cudaError_t ldpca_spec_reset(const LdpcaSpec &sp, int num_jobs, int K, cudaStream_t stream) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(sp.best, 0x7f, (size_t)num_jobs * 4, stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(sp.iters, 0, (size_t)num_jobs * 4, stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(sp.done, 0, (size_t)num_jobs * 4, stream)) != cudaSuccess) return e;
  return cudaMemsetAsync(sp.slot_code, 0xff, (size_t)num_jobs * K * 4, stream);
}

cudaError_t launch_ldpca_spec(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt,
                              int max_iter, int K, const LdpcaSpec &sp, cudaStream_t stream) {
  if (num_jobs <= 0) return cudaSuccess;
  return g_ldpca_threads == 512 ? launch_nt<512>(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream)
                                : launch_nt<1024>(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream);
}

}  // namespace dvc
