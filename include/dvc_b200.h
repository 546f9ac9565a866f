/* dvc_b200: B200-native Wyner-Ziv decoder hot path (NTU DVC codec, DvcDec).
 *
 * C ABI of libdvc_b200.so: plain pointers and sizes, int status returns,
 * no exceptions, no process exit.  All entry points are synchronous with
 * respect to the host buffers they are given unless stated otherwise.
 *
 * The reference decoder's GPU plug-in (the functions DvcDec/src/DVC_Decoder.cpp
 * and LdpcaDecoder.cpp call when ParallelMode is 2 or 3) works on process-global
 * state (codingOption, Block44Num, ladder globals) and aborts on error.  This
 * library replaces it with an explicit context handle; each entry point below
 * names the reference interface it stands in for.
 */
#ifndef DVC_B200_H
#define DVC_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DVC_OK 0
#define DVC_E_ARG -1     /* invalid argument or malformed input */
#define DVC_E_CUDA -2    /* CUDA runtime error (message in dvc_last_error) */
#define DVC_E_NOMEM -3   /* device allocation failed or admission refused */
#define DVC_E_DATA -4    /* missing or inconsistent ladder/table data */

typedef struct dvc_ctx dvc_ctx;

/* Create a context on CUDA device `device`.  `data_dir` holds
 * ldpca_ladders.bin; `table_dir` caches the C-library correction tables and
 * the GF(2) inverses (built on first use when absent).
 * Replaces InitCUDA + LDPCA_CUDA_Init_Variable + *_Init_Buffer
 * (LDPCA_cuda.h:16-17, noiseModel_kernel.h:13, updateSI_kernel.h:13,
 * forwardME_kernel.h:11, motionLearning_kernel.h:11; called at main.cpp:92-103). */
int dvc_create(const char *data_dir, const char *table_dir, int device, dvc_ctx **out);

/* Release everything the context owns.  Replaces LDPCA_CUDA_Free_Variable and
 * the *_Free_Buffer calls (LDPCA_cuda.h:18, main.cpp:155-162). */
void dvc_destroy(dvc_ctx *ctx);

/* Message of the last failing call on this context (never NULL). */
const char *dvc_last_error(dvc_ctx *ctx);

/* Batched LDPCA decode of `count` bitplanes of codeword length n (1584 QCIF
 * or 6336 CIF), each through the full rate-adaptive ladder on the device.
 *   lr[count*n]         p0/p1 per 4x4 block (the condBitProb output)
 *   acc[count*n/8]      accumulated syndrome bytes, MSB first (bitstream layout)
 *   crc[count]          CRC-8 of each source bitplane
 *   decoded[count*n]    out: decoded bits (0/1), may be NULL
 *   results[count*4]    out: rate (m+8), first code tried, accepted code, BP iterations
 *   entropy[count]      out: conditional-entropy bound, may be NULL
 *   max_iter            BP iterations per ladder code (the reference uses 50)
 * Equivalent, per bitplane, to ComputeCE followed by LdpcaDecoder
 * (LdpcaDecoder.cpp:127-143, 646-771; called at DVC_Decoder.cpp:238,267),
 * and replaces beliefPropagation_CUDA / beliefPropagation_CUDA_earlyJump /
 * ComputeCE_FERMI (LDPCA_cuda.h:19-21). */
int dvc_ldpca_decode(dvc_ctx *ctx, int n, int count, const float *lr, const uint8_t *acc, const uint8_t *crc,
                     uint8_t *decoded, int *results, float *entropy, int max_iter);

/* Reference-shaped single-bitplane call: LdpcaDecoder(LR_intrinsic,
 * accumulatedSyndrome, decoded, &rate, crc, RateLowerBound) with the
 * accumulated syndrome as one bit per byte and the bound supplied by the
 * caller (LdpcaDecoder.cpp:646-649).  Like the reference, LR_intrinsic holds
 * log(p0/p1) on return. */
int dvc_LdpcaDecoder(dvc_ctx *ctx, int n, float *LR_intrinsic, const unsigned char *accumulatedSyndrome,
                     unsigned char *decoded, int *rate, unsigned char crc_encoder, float RateLowerBound);

#ifdef __cplusplus
}
#endif
#endif
