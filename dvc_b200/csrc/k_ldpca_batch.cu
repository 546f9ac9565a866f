// Batched LDPCA decoding in one persistent launch: thousands of codewords of
// both lengths (QCIF n = 1584, CIF n = 6336), each from its own start level,
// each walking the rate-adaptive ladder (LdpcaDecoder.cpp:646-771) to the
// lowest code whose BP converges with a matching CRC, or to the full-rate
// inverse.
//
// Work items are (codeword, ladder code) pairs on two device queues, CIF first,
// each ordered breadth-first by the code's offset above the codeword's start:
// first the start code of every codeword, then the next code of every
// codeword, and so on.  A persistent grid of one 1024-thread block per SM pops
// CIF items with the whole block, then splits each block into four 256-thread
// groups (named barriers 1-4, a quarter of the shared memory each) that pop
// QCIF items independently.  An item whose code lies above a success already
// published for its codeword is skipped, and a running one is abandoned as soon
// as such a success appears.
//
// The result equals the sequential ladder's: the reference accepts the lowest
// code at or above the start that converges with a matching CRC.  Successes are
// published with atomicMin; each finished item sets its code's bit in the
// codeword's 64-bit mask; once every code from the start up to the lowest
// success (or, with none, up to the last code below full rate) has finished,
// the group that completes the set is elected (atomicExch) to finalise the
// codeword: the winner's decoded bits from its slot (or the GF(2) inverse at
// full rate), the rate, start, accepted code and the BP iterations the
// sequential ladder would have run (the per-code counts from the start to the
// accepted code).  A success stores its bits in one of four slots per
// codeword; a fifth concurrent success finds none, and the finaliser then
// decodes the accepted code again (BP is deterministic).
#include <cuda_runtime.h>

#include <atomic>

#include "dvc_common.cuh"
#include "dvc_types.h"
#include "kernels.h"
#include "ldpca_bp.cuh"

namespace dvc {

unsigned phi_window_attr(cudaLaunchAttribute &a);

namespace {

constexpr int kSlots = 4;
constexpr int kWords = (LDPCA_MAX_N + 31) / 32;  // packed decoded bits per slot

// the decoded bits of a group's codeword, packed 32 to a word (bit b of word w = bit 32w+b)
template <class G>
__device__ void pack_bits(const G &g, const uint8_t *dec, int n, uint32_t *out) {
  for (int w = g.t; w < (n + 31) / 32; w += G::NT) {
    uint32_t x = 0;
    for (int b = 0; b < 32 && w * 32 + b < n; b++) x |= (uint32_t)dec[w * 32 + b] << b;
    out[w] = x;
  }
}

// the codeword's result once every code up to `acc`, the accepted code (the
// lowest success, or the full-rate code), has finished; `acc` is the same for
// every thread of the group
template <class G, int MAXC>
__device__ void finalise(const G &g, const LdpcaBatch &A, const LadderDev &L, int j, int acc, const LdSmem &S,
                         uint32_t *s_ured, int *s_flag, const uint4 *pdesc) {
  const LdpcaBatchCw &C = A.cw[j];
  LdpcaBatchState &st = A.state[j];
  const int n = L.n, last = L.num_codes - 1, start = st.start;
  if (acc == last) {
    ld_build_syndrome(g, L, last, S.accs, S.rpar);
    g.sync();
    ld_invh_decode(g, L, S.rpar, S.dec, reinterpret_cast<uint32_t *>(S.msg));
  } else {
    if (g.t == 0) {
      int slot = -1;
      const int ns = min(__ldcg(&st.nsucc), kSlots);
      for (int s = 0; s < ns; s++)
        if (__ldcg(&st.succ_code[s]) == acc) slot = s;
      *s_flag = slot;
    }
    g.sync();
    const int slot = *s_flag;
    g.sync();
    if (slot >= 0) {
      const uint32_t *src = A.slot_bits + ((size_t)j * kSlots + slot) * kWords;
      for (int k = g.t; k < n; k += G::NT) S.dec[k] = (uint8_t)((__ldcg(src + (k >> 5)) >> (k & 31)) & 1u);
    } else {
      // every slot was taken by other successes: decode the accepted code again
      const XlSmall xs = xl_small_global(A.xt);
      float llr[MAXC];
      ld_llr(g, n, A.lr + C.lr_off, A.xt, xs, llr, nullptr, nullptr);
      int it = 0;
      ld_try_code(g, L, acc, llr, C.crc, A.xt, pdesc, A.max_iter, nullptr, S, s_ured, s_flag, it);
    }
    g.sync();
  }
  if (g.t == 0) {
    int iters = 0;
    for (int c = start; c <= min(acc, last - 1); c++) iters += __ldcg(&st.iters[c - start]);
    int *r = A.results + (size_t)j * 4;
    r[0] = L.synd_len[acc] + 8;
    r[1] = start;
    r[2] = acc;
    r[3] = iters;
  }
  if (A.decoded)
    for (int k = g.t; k < n; k += G::NT) A.decoded[C.dec_off + k] = S.dec[k];
  g.sync();
}

// one (codeword, code) item
template <class G, int MAXC>
__device__ void run_item(const G &g, const LdpcaBatch &A, const LadderDev &L, int j, int code,
                         const LdSmem &S, uint32_t *s_ured, int *s_flag, const uint4 *pdesc) {
  const LdpcaBatchCw &C = A.cw[j];
  LdpcaBatchState &st = A.state[j];
  const int n = L.n, last = L.num_codes - 1;
  const int start = st.start;
  const XlSmall xs = xl_small_global(A.xt);
  float llr[MAXC];
  ld_llr(g, n, A.lr + C.lr_off, A.xt, xs, llr, nullptr, nullptr);
  ld_stage_acc(g, A.acc + C.acc_off, n, S.accs);
  g.sync();
  int it = 0;
  const int ok = ld_try_code(g, L, code, llr, C.crc, A.xt, pdesc, A.max_iter, &st.best, S, s_ured, s_flag, it);
  if (g.t == 0) {
    st.iters[code - start] = it;
    atomicAdd(A.work, (unsigned long long)it);
  }
  if (ok) {
    if (g.t == 0) *s_flag = atomicAdd(&st.nsucc, 1);
    g.sync();
    const int slot = *s_flag;
    if (slot < kSlots) pack_bits(g, S.dec, n, A.slot_bits + ((size_t)j * kSlots + slot) * kWords);
    __threadfence();
    g.sync();
    if (g.t == 0) {
      if (slot < kSlots) st.succ_code[slot] = code;
      __threadfence();
      atomicMin(&st.best, code);
    }
  }
  // completion: this code's bit, then whether every code up to the lowest
  // success (or every code below full rate, with none) has finished
  g.sync();
  if (g.t == 0) {
    __threadfence();
    const unsigned long long bit = 1ull << (code - start);
    const unsigned long long m = atomicOr(&st.mask, bit) | bit;
    __threadfence();
    const int best = __ldcg(&st.best);
    const int top = (best == LDPCA_NONE || best >= last) ? last - 1 : best;
    const int need = top - start + 1;
    const unsigned long long want = need >= 64 ? ~0ull : ((1ull << need) - 1ull);
    // elected: the accepted code (every code at or below it has finished, so
    // no lower success can still appear); otherwise -1
    const bool elected = ((m & want) == want) && atomicExch(&st.fin, 1) == 0;
    *s_flag = elected ? ((best == LDPCA_NONE || best >= last) ? last : best) : -1;
  }
  g.sync();
  const int acc = *s_flag;
  g.sync();
  if (acc >= 0) finalise<G, MAXC>(g, A, L, j, acc, S, s_ured, s_flag, pdesc);
}

// next valid item of a queue (one thread): codeword index in the high bits, code in the low 8; -1 when empty
__device__ int pop_item(const LdpcaBatch &A, int which) {
  const int count = which ? A.n_qcif : A.n_cif;
  const int *list = which ? A.qcif : A.cif;
  const int last = which ? A.last_qcif : A.last_cif;
  int *ctr = A.ctr + which;
  for (;;) {
    const long long q = atomicAdd(ctr, 1);
    if (q >= (long long)count * 64) return -1;
    const int k = (int)(q / count), j = list[q % count];
    const LdpcaBatchState &st = A.state[j];
    const int code = st.start + k;
    if (code >= last) continue;
    if (__ldcg(&st.best) < code || __ldcg(&st.fin)) continue;
    return (j << 8) | code;
  }
}

}  // namespace

// per codeword: the entropy bound and the start code (or the given start), and
// the ladder state reset; one block of 256 threads per codeword
__global__ void __launch_bounds__(256) ldpca_batch_prep_kernel(LdpcaBatch A) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int j = blockIdx.x;
  const LdpcaBatchCw &C = A.cw[j];
  const LadderDev &L = C.cif ? A.L_cif : A.L_qcif;
  const int n = L.n;
  float *terms = reinterpret_cast<float *>(smem);
  const XlSmall xs = xl_small_global(A.xt);
  const float *lr = A.lr + C.lr_off;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const float v = lr[k];
    const float pco = v / (1.0f + v);
    const float tmp = xl_logf(A.xt, xs, 1.0f - pco);
    terms[k] = (pco * (-xl_logf(A.xt, xs, pco) + tmp) - tmp) / LDPCA_LOG2;
  }
  __syncthreads();
  LdpcaBatchState &st = A.state[j];
  if (threadIdx.x == 0) {
    const float h = ld_entropy_sum(terms, n);
    if (A.entropy) A.entropy[j] = h;
    st.start = C.given_start >= 0 ? min(C.given_start, L.num_codes - 1) : ld_start_code(L, h);
    st.best = LDPCA_NONE;
    st.fin = 0;
    st.nsucc = 0;
    st.mask = 0ull;
  }
  // a start at full rate has no BP item: finalise it here with the inverse
  __syncthreads();
  if (st.start == L.num_codes - 1) {
    uint8_t *synd = smem;
    uint32_t *sw = reinterpret_cast<uint32_t *>(smem + ((n + 15) & ~15));
    uint8_t *dec = smem + ((n + 15) & ~15) + 4 * ((n + 31) / 32) + 16;
    const LdGroup<256, true> g{(int)threadIdx.x, 0};
    ld_build_syndrome(g, L, L.num_codes - 1, A.acc + C.acc_off, synd);
    g.sync();
    ld_invh_decode(g, L, synd, dec, sw);
    if (threadIdx.x == 0) {
      st.fin = 1;
      int *r = A.results + (size_t)j * 4;
      r[0] = L.synd_len[L.num_codes - 1] + 8;
      r[1] = st.start;
      r[2] = st.start;
      r[3] = 0;
    }
    if (A.decoded)
      for (int k = threadIdx.x; k < n; k += blockDim.x) A.decoded[C.dec_off + k] = dec[k];
  }
}

// the persistent decode: CIF items with whole blocks, then QCIF items with
// 256-thread groups
__global__ void __launch_bounds__(1024, 1) ldpca_batch_kernel(LdpcaBatch A) {
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ uint32_t s_ured[32];
  __shared__ int s_flag[4], s_item[4];
  __shared__ uint4 s_pdesc[XL_PHI_MAX_BINADES];
  xl_phi_stage(A.xt, s_pdesc);
  __syncthreads();
  {
    const LdGroup<1024, true> g{(int)threadIdx.x, 0};
    const LdSmem S = ld_carve(smem, A.L_cif.n, A.L_cif.e);
    for (;;) {
      if (g.t == 0) s_item[0] = A.n_cif ? pop_item(A, 0) : -1;
      g.sync();
      const int item = s_item[0];
      g.sync();
      if (item < 0) break;
      run_item<LdGroup<1024, true>, 7>(g, A, A.L_cif, item >> 8, item & 0xff, S, s_ured, &s_flag[0], s_pdesc);
    }
  }
  {
    const int gi = threadIdx.x >> 8;
    const LdGroup<256, false> g{(int)threadIdx.x & 255, 1 + gi};
    const size_t quarter = ldpca_smem_bytes(A.L_qcif.n, A.L_qcif.e);
    const LdSmem S = ld_carve(smem + gi * quarter, A.L_qcif.n, A.L_qcif.e);
    for (;;) {
      if (g.t == 0) s_item[gi] = A.n_qcif ? pop_item(A, 1) : -1;
      g.sync();
      const int item = s_item[gi];
      g.sync();
      if (item < 0) break;
      run_item<LdGroup<256, false>, 7>(g, A, A.L_qcif, item >> 8, item & 0xff, S, s_ured + 8 * gi, &s_flag[gi], s_pdesc);
    }
  }
}

size_t ldpca_batch_state_bytes(int count) {
  return (size_t)count * sizeof(LdpcaBatchState) + (size_t)count * kSlots * kWords * 4;
}

// dynamic shared memory of a batch block: one CIF codeword, or four QCIF ones
static size_t batch_smem_bytes() {
  const size_t cif = ldpca_smem_bytes(6336, 3 * 6336), qcif4 = 4 * ldpca_smem_bytes(1584, 3 * 1584);
  return cif > qcif4 ? cif : qcif4;
}

cudaError_t launch_ldpca_batch(LdpcaBatch A, int count, int grid, cudaStream_t s) {
  if (A.L_cif.n != 6336 || A.L_qcif.n != 1584) return cudaErrorInvalidValue;
  const size_t smem = batch_smem_bytes();
  static std::atomic<uint64_t> attr_set{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    e = cudaFuncSetAttribute(ldpca_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int pct = (int)(((smem + 4096) * 100 + 228 * 1024 - 1) / (228 * 1024));
    e = cudaFuncSetAttribute(ldpca_batch_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e != cudaSuccess) return e;
    attr_set.fetch_or(bit);
  }
  if ((e = cudaMemsetAsync(A.ctr, 0, 2 * sizeof(int), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(A.work, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
  // the entropy terms (n floats), later the full-rate syndrome, its words and the decoded bits
  ldpca_batch_prep_kernel<<<count, 256, 4 * LDPCA_MAX_N, s>>>(A);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(1024);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  cfg.attrs = attr;
  cfg.numAttrs = phi_window_attr(attr[0]);
  return cudaLaunchKernelEx(&cfg, ldpca_batch_kernel, A);
}

}  // namespace dvc
