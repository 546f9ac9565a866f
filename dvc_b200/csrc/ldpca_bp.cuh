// Device building blocks of LDPCA rate-adaptive decoding, shared by the
// frame-batch ladder kernel (k_ldpca.cu) and the persistent work-queue kernel
// (k_ldpca_batch.cu).
//
// Reference: DvcDec/src/LdpcaDecoder.cpp LdpcaDecoder (:646-771),
// beliefPropagation (:462-580), ComputeCE (:127-143), invH_mul (:624-643),
// bitplane.cpp putBitplaneToCoeff (:4-22).  The per-edge arithmetic, the order
// of every float sum (row sums in edge order, column sums in edge order, the
// entropy sum in block order) and the library functions (logf, tanhf via
// exact_libm) follow the reference exactly.
//
// A codeword is decoded by a group of NT threads: a whole thread block, or one
// of several equal parts of a block, each synchronising on its own named
// barrier (bar.sync id, NT), so that a block of 1024 threads can work on one
// CIF codeword (n = 6336) or on four QCIF codewords (n = 1584) at once with the
// same shared memory.  Each thread keeps the log-LRs of its columns
// (k = t, t + NT, ...) in registers: MAXC = ceil(n / NT) of them.
//
// Edge messages are kept in row order (each row's edges contiguous, in
// increasing edge index), so a row sum is a sequential pass over contiguous
// shared memory in the reference's summation order; columns (every column has
// degree 3) reach their edges through the per-code position array.  The
// parity check of an iteration's hard decision is folded into the next row
// pass.  The magnitude phi(y) = -logf(tanhf(y)) is one record read of the
// packed table (dvc_common.cuh), and the reads of a pass are issued in batches
// so that several are in flight per thread.
//
// Shared memory per codeword (n bits, e edges; CIF n=6336, e=19008: 125 KB;
// QCIF a quarter of it):
//   msg[e]  f32  edge messages by row-order position, in place:
//                phi(|v->c|) -> c->v -> next phi(|v->c|)
//   rowt[n] f32  row sums (after decoding: the decoded bits, one byte each)
//   sgd[e]  u8   bit 0: sign of the v->c message, bit 1: hard decision of its column
//   rpar[n] u8   bit 0: syndrome bit of the row, bit 1: sign parity of the row
//   accs[n/8]    the packed accumulated syndrome, staged once per codeword
#pragma once
#include <cuda_runtime.h>

#include "dvc_common.cuh"
#include "dvc_types.h"

namespace dvc {

#define LDPCA_LOG2 (0.693147181f)  // LdpcaDecoder.cpp:18
#define LDPCA_NONE 0x7f7f7f7f      // "no success yet" (memset pattern 0x7f)
#define LDPCA_MAX_N 6336           // largest codeword length

// columns per thread of a group of nt threads on codewords of n bits
#define LDPCA_COLS(n, nt) (((n) + (nt) - 1) / (nt))

// stage: the ladder code's index tables (rid, pos: 2 x e uint16) live in
// shared memory too (see ld_try_code)
__host__ __device__ inline size_t ldpca_smem_bytes(int n, int e, bool stage = false) {
  size_t b = (size_t)e * 4;       // msg
  if (stage) b += (size_t)e * 4;  // rid and pos of the code tried
  b += (size_t)n * 4;             // rowt
  b += (size_t)e;            // sgd
  b += (size_t)n;            // rpar
  b += (size_t)n / 8;        // accs
  return (b + 15) & ~(size_t)15;
}

// NT threads decoding one codeword; `t` is the thread's index in the group.
// BLOCK: the group is the whole thread block and synchronises with the block's
// barrier (__syncthreads); otherwise on the hardware barrier `bar` (1-15),
// which only its NT threads use.
template <int NT_, bool BLOCK>
struct LdGroup {
  static constexpr int NT = NT_;
  int t, bar;
  __device__ __forceinline__ void sync() const {
    if constexpr (BLOCK)
      __syncthreads();
    else
      asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(NT_) : "memory");
  }
  // barrier that also returns whether any thread of the group passed p != 0
  __device__ __forceinline__ int sync_or(int p) const {
    if constexpr (BLOCK) {
      return __syncthreads_or(p);
    } else {
      int r;
      asm volatile(
          "{\n\t.reg .pred q;\n\tsetp.ne.s32 q, %1, 0;\n\tbar.red.or.pred q, %2, %3, q;\n\tselp.s32 %0, 1, 0, q;\n\t}"
          : "=r"(r)
          : "r"(p), "r"(bar), "n"(NT_)
          : "memory");
      return r;
    }
  }
};

struct LdSmem {
  float *msg, *rowt;
  uint16_t *rid, *pos;  // staged index tables of the code tried (null: read from global memory)
  uint8_t *sgd, *rpar, *dec, *accs;
};

__device__ __forceinline__ LdSmem ld_carve(uint8_t *base, int n, int e, bool stage = false) {
  LdSmem S;
  S.msg = reinterpret_cast<float *>(base);
  S.rid = stage ? reinterpret_cast<uint16_t *>(S.msg + e) : nullptr;  // e is a multiple of 8: 16-byte aligned
  S.pos = stage ? S.rid + e : nullptr;
  S.rowt = stage ? reinterpret_cast<float *>(S.pos + e) : S.msg + e;
  S.sgd = reinterpret_cast<uint8_t *>(S.rowt + n);
  S.rpar = S.sgd + e;
  S.accs = S.rpar + n;                          // the codeword's packed accumulated syndrome
  S.dec = reinterpret_cast<uint8_t *>(S.rowt);  // decoded bits, once BP is over
  return S;
}

// the codeword's packed accumulated syndrome (n/8 bytes, MSB first) into
// shared memory, one coalesced byte per thread, for every ladder code it tries;
// the caller synchronises before use
template <class G>
__device__ __forceinline__ void ld_stage_acc(const G &g, const uint8_t *packed, int n, uint8_t *accs) {
  constexpr int NT = G::NT;
  for (int k = g.t; k < n / 8; k += NT) accs[k] = __ldg(packed + k);
}

// fused bitplane insertion (putBitplaneToCoeff, bitplane.cpp:4-22)
template <class G>
__device__ __forceinline__ void ld_put_bitplane(const G &g, const LdpcaJob &J, const uint8_t *dec, int n) {
  constexpr int NT = G::NT;
  const int b4w = J.w >> 2, b8w = J.w >> 3;
  const int row = J.index_in_blk >> 2, col = J.index_in_blk & 3;
  for (int k = g.t; k < n; k += NT) {
    const int i = k / b4w, j = k - i * b4w;
    if (J.mode[(i >> 1) * b8w + (j >> 1)] == DVC_WZ_B) {
      int *p = J.recons_trans + ((i << 2) + row) * J.w + (j << 2) + col;
      *p = (*p << 1) + (int)dec[k];
    }
  }
}

// decoded = inv(H) * syndrome of the full-rate code (LdpcaDecoder.cpp:695-716);
// syndrome words are built in `sw` (n/32 words of shared memory)
template <class G>
__device__ __forceinline__ void ld_invh_decode(const G &g, const LadderDev &L, const uint8_t *synd, uint8_t *dec,
                               uint32_t *sw) {
  constexpr int NT = G::NT;
  const int n = L.n, lane = g.t & 31, warp = g.t >> 5;
  for (int base = warp * 32; base < n; base += NT) {
    const int k = base + lane;
    const uint32_t b = __ballot_sync(0xffffffffu, k < n && (synd[k] & 1));
    if (lane == 0) sw[base >> 5] = b;
  }
  g.sync();
  for (int j = g.t; j < n; j += NT) {
    const uint32_t *row = L.invh + (size_t)j * L.invh_words;
    uint32_t x = 0;
    for (int w = 0; w < L.invh_words; w++) x ^= __ldg(row + w) & sw[w];
    dec[j] = (uint8_t)(__popc(x) & 1);
  }
  g.sync();
}

// one bit of the packed accumulated-syndrome bytes (MSB first, ByteToBit),
// from shared or global memory
__device__ __forceinline__ uint8_t ld_acc_bit(const uint8_t *packed, int i) {
  return (uint8_t)((packed[i >> 3] >> (7 - (i & 7))) & 1);
}

// syndrome of ladder code `code` from the accumulated syndrome (LdpcaDecoder.cpp:684-693):
// bit k of the code is accumulated bit idx[k % nb] + (k / nb) * period xor the
// same of k - 1.  Thread t takes k = t, t + NT, ...; the quotient and
// remainder of k by nb advance by those of NT, with no division per bit.
template <class G>
__device__ __forceinline__ void ld_build_syndrome(const G &g, const LadderDev &L, int code,
                                                  const uint8_t *packed, uint8_t *synd) {
  constexpr int NT = G::NT;
  const int m = L.synd_len[code], nb = L.bpp[code], P = L.period;
  const int *idx = L.idx + (size_t)code * P;
  const int dq = NT / nb, dr = NT - dq * nb;
  int q = g.t / nb, r = g.t - q * nb;
  for (int k = g.t; k < m; k += NT) {
    uint8_t s = ld_acc_bit(packed, __ldg(idx + r) + q * P);
    if (k > 0) s ^= ld_acc_bit(packed, r > 0 ? __ldg(idx + r - 1) + q * P : __ldg(idx + nb - 1) + (q - 1) * P);
    synd[k] = s;
    r += dr;
    q += dq;
    if (r >= nb) {
      r -= nb;
      q++;
    }
  }
}

// log LR of the group's columns into registers (LdpcaDecoder.cpp:665-666) and,
// when want_entropy, the entropy terms H_k = (P(-log P + log(1-P)) - log(1-P))
// / LOG2 with P = LR/(1+LR) (ComputeCE) into `terms` (n floats of shared memory).
template <class G, int MAXC>
__device__ __forceinline__ void ld_llr(const G &g, int n, const float *lr, const XlmDev &xt,
                                       const XlSmall &xs, float (&llr)[MAXC], float *terms, float *llr_out) {
  constexpr int NT = G::NT;
#pragma unroll
  for (int c = 0; c < MAXC; c++) {
    const int k = g.t + c * NT;
    llr[c] = 0.0f;
    if (k < n) {
      const float v = lr[k];
      if (terms) {
        const float pco = v / (1.0f + v);
        const float tmp = xl_logf(xt, xs, 1.0f - pco);
        terms[k] = (pco * (-xl_logf(xt, xs, pco) + tmp) - tmp) / LDPCA_LOG2;
      }
      llr[c] = xl_logf(xt, xs, v);
      if (llr_out) llr_out[k] = llr[c];
    }
  }
}

// the conditional-entropy bound: a sequential float sum of the terms in block
// order, divided by n (one thread; the caller synchronises before and after)
__device__ __forceinline__ float ld_entropy_sum(const float *terms, int n) {
  float h = 0.0f;
  int k = 0;
  for (; k + 8 <= n; k += 8) {
    const float v0 = terms[k], v1 = terms[k + 1], v2 = terms[k + 2], v3 = terms[k + 3];
    const float v4 = terms[k + 4], v5 = terms[k + 5], v6 = terms[k + 6], v7 = terms[k + 7];
    h += v0;
    h += v1;
    h += v2;
    h += v3;
    h += v4;
    h += v5;
    h += v6;
    h += v7;
  }
  for (; k < n; k++) h += terms[k];
  return h / (float)n;
}

// first ladder code whose rate reaches the bound (LdpcaDecoder.cpp:657-659)
__device__ __forceinline__ int ld_start_code(const LadderDev &L, float h) {
  int start = 0;
  while (start < L.num_codes - 1 && L.code_rate[start] < h) start++;
  return start;
}

// One ladder code below full rate: its syndrome (from the accumulated syndrome
// staged in S.accs by ld_stage_acc), sum-product BP until every
// parity check holds (success) or max_iter iterations ran or, when `bestp` is
// given, a lower code of the same codeword has succeeded (*bestp < code), then
// the CRC-8 of the hard decision (LdpcaDecoder.cpp:684-693, 718-758).
// Returns 1 when the code decodes with a matching CRC; the decoded bits are
// then in S.dec.  `iters` receives the BP iterations run.  s_ured holds NT/32
// words of shared memory, s_flag one int, both the group's own.
// an index table entry: a shared-memory read when staged, a read-only global one otherwise
template <bool STAGE>
__device__ __forceinline__ int ld_idx(const uint16_t *p) {
  if constexpr (STAGE) return *p;
  else return __ldg(p);
}

template <class G, int MAXC, bool STAGE = false>
__device__ __forceinline__ int ld_try_code(const G &g, const LadderDev &L, int code, const float (&llr)[MAXC],
                           int crc, const XlmDev &xt, const uint4 *pdesc, int max_iter,
                           const volatile int *bestp, const LdSmem &S, uint32_t *s_ured, int *s_flag, int &iters) {
  constexpr int NT = G::NT;
  constexpr int UNR = 8;                  // edge-pass table reads in flight per thread
  constexpr int CB = 1;  // column-pass columns per batch (3 reads each; more spill at 64 registers)
  const int n = L.n, E = L.e, t = g.t, lane = t & 31, warp = t >> 5;
  float *msg = S.msg, *rowt = S.rowt;
  uint8_t *sgd = S.sgd, *rpar = S.rpar, *dec = S.dec;
  const int m = L.synd_len[code];
  // STAGE: the code's index tables are copied to shared memory for the whole
  // try (e is a multiple of 8: 16-byte copies), which keeps a global round
  // trip off the chain leading to every table gather.  Only where the block
  // owns its SM and the copy leaves the shared-memory carveout (so the L1
  // that the in-flight table gathers allocate in) unchanged: QCIF codewords
  // on 1024 threads.  At CIF the 76 KB of tables would cut L1 to a fifth.
  const uint16_t *__restrict__ pos = L.pos + (size_t)code * E;
  const uint16_t *__restrict__ rid = L.rid + (size_t)code * E;
  if constexpr (STAGE) {
    const uint4 *gr = reinterpret_cast<const uint4 *>(rid), *gp = reinterpret_cast<const uint4 *>(pos);
    uint4 *sr = reinterpret_cast<uint4 *>(S.rid), *sp = reinterpret_cast<uint4 *>(S.pos);
    for (int i = t; i < E / 8; i += NT) {
      sr[i] = __ldg(gr + i);
      sp[i] = __ldg(gp + i);
    }
    pos = S.pos;
    rid = S.rid;
  }
  ld_build_syndrome(g, L, code, S.accs, rpar);
  g.sync();
  const int *rp = L.row_ptr + (size_t)code * (n + 1);
  // first magnitudes: phi(|LLR|) on the three edges of each column
  {
    float ph[MAXC];
#pragma unroll
    for (int c = 0; c < MAXC; c++)
      ph[c] = t + c * NT < n ? xl_phi(xt, pdesc, (fabsf(llr[c]) + 1e-9f) / 2.0f) : 0.0f;
#pragma unroll
    for (int c = 0; c < MAXC; c++) {
      const int k = t + c * NT;
      if (k < n) {
        const uint8_t ng = (uint8_t)(__float_as_uint(llr[c]) >> 31);
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const int p = ld_idx<STAGE>(pos + 3 * k + i);
          msg[p] = ph[c];
          sgd[p] = ng;
        }
      }
    }
  }
  g.sync();
  bool converged = false;
  int it = 0;
  for (;;) {
    // (R) rows: sum of the magnitudes in edge order and the sign parity with
    //     the syndrome bit, for the next edge pass; from the second pass on
    //     also the parity check of the previous hard decision
    int wrong = 0;
    for (int r = t; r < m; r += NT) {
      const int p0 = rp[r], p1 = rp[r + 1];
      float s = 0.0f;
      uint32_t x = 0;  // bit 0: xor of signs, bit 1: xor of decisions
      // low codes have few, long rows (up to ~200 edges): the loads of eight
      // edges are issued before their adds, which stay in edge order
      int p = p0;
      for (; p + 8 <= p1; p += 8) {
        float v[8];
        uint32_t b[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          v[q] = msg[p + q];
          b[q] = sgd[p + q];
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          s += v[q];
          x ^= b[q];
        }
      }
      for (; p < p1; p++) {
        s += msg[p];
        x ^= sgd[p];
      }
      const uint32_t syn = rpar[r] & 1u;
      rowt[r] = s;
      rpar[r] = (uint8_t)(syn | (((x & 1u) ^ syn) << 1));
      wrong |= (int)(((x >> 1) ^ syn) & 1u);
    }
    if (t == 0) *s_flag = bestp ? (int)(*bestp < code) : 0;
    const int any_wrong = g.sync_or(wrong);
    if (it > 0 && !any_wrong) {
      converged = true;
      break;
    }
    // abandon a code above a known success
    if (it == max_iter || *s_flag) break;
    it++;
    // (E) edges: c->v = phi(row sum - own magnitude) with the product of
    //     the other signs
    for (int p0 = t; p0 < E; p0 += UNR * NT) {
      float c[UNR];
      int rr[UNR];
#pragma unroll
      for (int q = 0; q < UNR; q++) {
        // lanes past the last edge repeat it (no branch, so that the UNR
        // table reads are in flight together) and store nothing
        const int p = min(p0 + q * NT, E - 1);
        rr[q] = ld_idx<STAGE>(rid + p);
        c[q] = xl_phi(xt, pdesc, (rowt[rr[q]] - msg[p] + 1e-9f) / 2.0f);
      }
#pragma unroll
      for (int q = 0; q < UNR; q++) {
        const int p = p0 + q * NT;
        if (p < E) msg[p] = c[q] * ((((uint32_t)rpar[rr[q]] >> 1) ^ (sgd[p] & 1u)) ? -1.0f : 1.0f);
      }
    }
    g.sync();
    // (C) columns: total in edge order, hard decision, extrinsic messages
    //     and their magnitudes for the next iteration
#pragma unroll
    for (int c0 = 0; c0 < MAXC; c0 += CB) {
      float ph[CB][3];
      uint32_t sb[CB][3];
      int pp[CB][3];
#pragma unroll
      for (int b = 0; b < CB; b++) {
        const int c = c0 + b, k = t + c * NT;
        if (c < MAXC && k < n) {
          float mv[3];
#pragma unroll
          for (int i = 0; i < 3; i++) {
            pp[b][i] = ld_idx<STAGE>(pos + 3 * k + i);
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
            ph[b][i] = xl_phi(xt, pdesc, (fabsf(v) + 1e-9f) / 2.0f);
          }
        }
      }
#pragma unroll
      for (int b = 0; b < CB; b++) {
        const int c = c0 + b, k = t + c * NT;
        if (c < MAXC && k < n)
#pragma unroll
          for (int i = 0; i < 3; i++) {
            msg[pp[b][i]] = ph[b][i];
            sgd[pp[b][i]] = (uint8_t)sb[b][i];
          }
      }
    }
    g.sync();
  }
  iters = it;
  if (!converged) {
    g.sync();  // every thread has read *s_flag: the caller may reuse it
    return 0;
  }
  // hard decision of each column (bit 1 of its edges' sgd) into dec, and the
  // CRC-8 of the decoded bitplane as the xor of single-bit CRCs (the CRC is
  // linear for a fixed length with zero initial value and no final xor)
  uint32_t cr = 0;
  for (int k = t; k < n; k += NT) {
    const uint8_t d = (uint8_t)((sgd[ld_idx<STAGE>(pos + 3 * k)] >> 1) & 1u);
    dec[k] = d;
    if (d) cr ^= __ldg(L.crc_tab + k);
  }
  for (int o = 16; o > 0; o >>= 1) cr ^= __shfl_xor_sync(0xffffffffu, cr, o);
  if (lane == 0) s_ured[warp] = cr;
  g.sync();
  if (t == 0) {
    uint32_t x = 0;
    for (int w = 0; w < NT / 32; w++) x ^= s_ured[w];
    *s_flag = (int)(x & 0xffu) == crc;
  }
  g.sync();
  const int ok = *s_flag;
  g.sync();
  return ok;
}

}  // namespace dvc
