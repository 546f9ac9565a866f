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
// The per-code BP, the syndrome, the inverse and the shared-memory layout are
// in ldpca_bp.cuh.
#include <cuda_runtime.h>

#include <atomic>

#include "dvc_common.cuh"
#include "dvc_types.h"
#include "kernels.h"
#include "ldpca_bp.cuh"

namespace dvc {

size_t ldpca_smem_size(int n, int e) { return ldpca_smem_bytes(n, e); }

// One thread block of NT threads per (codeword, speculative slot), each thread
// holding MAXC = ceil(n / NT) columns, MINB blocks per SM.  By default NT = 1024 for both lengths
// (CIF: one block per SM, 124 KB of shared memory; QCIF: 31 KB, 5 edges per
// thread); QCIF codewords can also run with 256 or 512 threads, four or two
// blocks per SM (the autotuner measures which is faster).
// the QCIF shape that owns its SM stages the code's index tables in shared
// memory (ld_try_code); the others read them from global memory
template <int NT, int MAXC>
__host__ __device__ constexpr bool ldpca_stage() {
  return NT == 1024 && MAXC <= 2;
}

template <int NT, int MAXC, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    ldpca_ladder_kernel(LadderDev L, const LdpcaJob *__restrict__ jobs, XlmDev xt, int max_iter, int K,
                        LdpcaSpec sp) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int j = blockIdx.x / K, kk = blockIdx.x - j * K;
  const LdpcaJob J = jobs[j];
  if (!J.active) return;
  const bool spec = sp.best != nullptr;
  const LdGroup<NT, true> g{(int)threadIdx.x, 0};
  const int n = L.n, tid = threadIdx.x;
  const LdSmem S = ld_carve(smem, n, L.e, ldpca_stage<NT, MAXC>());
  __shared__ uint32_t s_ured[NT / 32];
  __shared__ int s_start, s_accepted, s_stop;
  __shared__ uint4 s_pdesc[XL_PHI_MAX_BINADES];
  const XlSmall xs = xl_small_global(xt);
  xl_phi_stage(xt, s_pdesc);

  // accumulated syndrome bits (ByteToBit, LdpcaDecoder.cpp:81-107), log LR and
  // the entropy terms (ComputeCE), the bound as a sequential sum in block order
  float llr[MAXC];
  ld_llr(g, n, J.lr, xt, xs, llr, S.msg, (J.llr_out && kk == 0) ? J.llr_out : nullptr);
  ld_stage_acc(g, J.acc, n, S.accs);
  g.sync();
  if (tid == 0) {
    float h = ld_entropy_sum(S.msg, n);
    if (J.use_given_entropy) h = J.given_entropy;
    const int start = ld_start_code(L, h);
    s_start = start;
    s_accepted = L.num_codes - 1;
    if (kk == 0) {
      if (J.entropy) *J.entropy = h;
      if (spec) sp.start[j] = start;
    }
  }
  g.sync();
  const int start = s_start;
  const int last = L.num_codes - 1;
  int total_iters = 0;
  volatile int *bestp = spec ? sp.best + j : nullptr;

  for (int code = start + kk; code < last; code += K) {
    if (spec) {
      if (tid == 0) s_stop = *bestp < code;
      g.sync();
      if (s_stop) break;
    }
    int it = 0;
    const int ok = ld_try_code<LdGroup<NT, true>, MAXC, ldpca_stage<NT, MAXC>()>(g, L, code, llr, J.crc, xt, s_pdesc,
                                                                                  max_iter, bestp, S, s_ured, &s_stop, it);
    total_iters += it;
    if (ok) {
      if (tid == 0) s_accepted = code;
      if (spec) {
        uint8_t *slot = sp.slot_dec + (size_t)blockIdx.x * n;
        for (int k = tid; k < n; k += NT) slot[k] = S.dec[k];
        g.sync();
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
    g.sync();
    if (tid == 0) {
      atomicAdd(sp.iters + j, total_iters);
      __threadfence();
      s_stop = atomicAdd(sp.done + j, 1) == K - 1;
    }
    g.sync();
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
    g.sync();
    if (s_slot >= 0) {
      const uint8_t *src = sp.slot_dec + (size_t)(j * K + s_slot) * n;
      for (int k = tid; k < n; k += NT) S.dec[k] = __ldcg(src + k);
    }
    total_iters = s_iters;
    for (int k = tid; k < K; k += NT) sp.slot_code[j * K + k] = -1;
    if (tid == 0) {
      sp.best[j] = LDPCA_NONE;
      sp.iters[j] = 0;
      sp.done[j] = 0;
    }
  }
  g.sync();
  const int accepted = s_accepted;
  if (accepted == last) {
    ld_build_syndrome(g, L, last, S.accs, S.rpar);
    g.sync();
    ld_invh_decode(g, L, S.rpar, S.dec, reinterpret_cast<uint32_t *>(S.msg));
  }
  if (tid == 0) {
    J.result[0] = L.synd_len[accepted] + 8;
    J.result[1] = start;
    J.result[2] = accepted;
    J.result[3] = total_iters;
  }
  if (J.decoded)
    for (int k = tid; k < n; k += NT) J.decoded[k] = S.dec[k];
  if (J.recons_trans) ld_put_bitplane(g, J, S.dec, n);
}

// the L2 persisting window of the table reads (set when a context is created;
// process-wide like the launch shapes)
static cudaAccessPolicyWindow g_phi_window = {};

void set_phi_window(const void *base, size_t num_bytes, float hit_ratio) {
  g_phi_window = cudaAccessPolicyWindow{};
  if (!base || num_bytes == 0) return;
  g_phi_window.base_ptr = const_cast<void *>(base);
  g_phi_window.num_bytes = num_bytes;
  g_phi_window.hitRatio = hit_ratio;
  g_phi_window.hitProp = cudaAccessPropertyPersisting;
  g_phi_window.missProp = cudaAccessPropertyStreaming;
}

// the window as a launch attribute; returns the number of attributes (0 or 1)
unsigned phi_window_attr(cudaLaunchAttribute &a) {
  if (g_phi_window.num_bytes == 0) return 0;
  a.id = cudaLaunchAttributeAccessPolicyWindow;
  a.val.accessPolicyWindow = g_phi_window;
  return 1;
}

template <int NT, int MAXC, int MINB>
static cudaError_t launch_nt(const LadderDev &L, const LdpcaJob *jobs, int num_jobs, const XlmDev &xt, int max_iter,
                             int K, const LdpcaSpec &sp, cudaStream_t stream) {
  if (L.n > LDPCA_MAX_N || LDPCA_COLS(L.n, NT) > MAXC) return cudaErrorInvalidValue;
  const size_t smem = ldpca_smem_bytes(L.n, L.e, ldpca_stage<NT, MAXC>());
  // the attributes are per device: set them once for each device
  static std::atomic<uint64_t> attr_set{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    e = cudaFuncSetAttribute(ldpca_ladder_kernel<NT, MAXC, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // the smallest shared-memory split that holds the blocks an SM runs (MINB
    // of them), so that the rest of the SM's 256 KB is L1 for the
    // phi records, which BP iterations re-read (percent of the 228 KB maximum;
    // the driver rounds up to a supported split)
    const size_t need = (size_t)MINB * (smem + 4096);
    const int pct = (int)((need * 100 + 228 * 1024 - 1) / (228 * 1024));
    e = cudaFuncSetAttribute(ldpca_ladder_kernel<NT, MAXC, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             pct > 100 ? 100 : pct);
    if (e != cudaSuccess) return e;
    attr_set.fetch_or(bit);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(num_jobs * K);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  cfg.attrs = attr;
  cfg.numAttrs = phi_window_attr(attr[0]);
  return cudaLaunchKernelEx(&cfg, ldpca_ladder_kernel<NT, MAXC, MINB>, L, jobs, xt, max_iter, K, sp);
}

// threads per codeword block: CIF 1024 (or 512), QCIF 1024 (or 256, 512)
static int g_ldpca_threads = 1024, g_ldpca_threads_qcif = 1024;

void set_ldpca_threads(int nt, int nt_qcif) {
  g_ldpca_threads = (nt == 512) ? 512 : 1024;
  g_ldpca_threads_qcif = (nt_qcif == 256 || nt_qcif == 512) ? nt_qcif : 1024;
}

static cudaError_t launch_shape(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt,
                                int max_iter, int K, const LdpcaSpec &sp, cudaStream_t stream) {
  if (L.n == 1584) {
    if (g_ldpca_threads_qcif == 1024) return launch_nt<1024, 2, 1>(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream);
    if (g_ldpca_threads_qcif == 512) return launch_nt<512, 4, 2>(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream);
    return launch_nt<256, 7, 4>(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream);
  }
  if (g_ldpca_threads == 512) return launch_nt<512, 13, 1>(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream);
  return launch_nt<1024, 7, 1>(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream);
}

cudaError_t launch_ldpca(const LadderDev &L, const LdpcaJob *jobs_dev, int num_jobs, const XlmDev &xt, int max_iter,
                         cudaStream_t stream) {
  if (num_jobs <= 0) return cudaSuccess;
  LdpcaSpec none{};
  return launch_shape(L, jobs_dev, num_jobs, xt, max_iter, 1, none, stream);
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
  return launch_shape(L, jobs_dev, num_jobs, xt, max_iter, K, sp, stream);
}

}  // namespace dvc
