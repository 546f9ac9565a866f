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
 * forwardME_kernel.h:11, motionLearning_kernel.h:11; called at main.cpp:92-103).
 * Launch shape of the LDPCA ladder kernel, from the environment (the values
 * dvc_b200.autotune chooses by measurement; decoded output never depends on
 * them): DVC_LDPCA_THREADS = 512 or 1024 threads per CIF codeword block
 * (default 1024) and DVC_LDPCA_THREADS_QCIF = 256, 512 or 1024 per QCIF
 * codeword block (default 1024), DVC_SI_THREADS = 64, 128 or 256 threads per
 * updateSI search block (default 128) and DVC_FME_THREADS = 128, 256 or 512
 * per forward-search block (default 256), read here; DVC_LDPCA_SPEC_FLOOR = 1..32, the least number of
 * speculative blocks per codeword in a frame batch (default 4), and
 * DVC_LDPCA_SPEC = 1..32, a fixed number instead, both read when a batch is
 * prepared. */
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

/* JBIG (T.82) decoder for a skip or intra mode map of the WZ bitstream: the
 * coded stripe that follows a set skipMode / intraMode byte, decoded into
 * map[h*w] (1 = the 8x8 block has the mode), with *used = the bytes it
 * occupies (through the closing SDNORM/SDRST marker).  w x h = Block88Width x
 * Block88Height (22x18 QCIF, 44x36 CIF).  Replaces the reference's
 * simple_JBIG_dec over JBIG-KIT with the header it rebuilds
 * (DvcDec/src/wzbitstream.cpp:38-66, sJBIG.cpp:49-104).  Host code, no GPU.
 * DVC_E_DATA for a truncated stream or a stream with an adaptive-template move. */
int dvc_jbig_decode_mode_map(const uint8_t *data, size_t len, int w, int h, uint8_t *map, size_t *used);

/* JBIG (T.82) encoder for a skip or intra mode map: map[h*w] (nonzero = the
 * 8x8 block has the mode) coded as the reference encoder stores it after a set
 * skipMode / intraMode byte, the coded stripe closed by SDNORM, into out[cap];
 * *len = its length (also when cap is too small, which returns DVC_E_ARG).
 * Replaces simple_JBIG_enc over JBIG-KIT (DvcEnc/src/sJBIG.cpp:54-71, called
 * at wzbitstream.cpp:36-50) and gives the same bytes; the length is also what
 * the reference's skip-count rule uses (skipBlock.cpp:47-66).  Host code. */
int dvc_jbig_encode_mode_map(const uint8_t *map, int w, int h, uint8_t *out, size_t cap, size_t *len);

/* Intra blocks of one WZ frame (IntraMode 1), decoded from the sequence's
 * intra bitstream: CAVLC coefficients, de-quantisation with IntraQP, 4x4
 * inverse transform, DC prediction from intra neighbours; the pixels of every
 * 4x4 block inside an intra 8x8 block (mode[w*h/64] == 1) are written into
 * recon[w*h], other pixels are left alone.  *bit_offset is the position in
 * the bitstream, advanced past this frame's blocks (frames are read in the
 * reference's decoding order).  Replaces intraRecon (DvcDec/src/intra.cpp:
 * 187-268) with readCoeff4x4_CAVLC (vlc.cpp:613-761).  Host code, no GPU.
 * DVC_E_DATA on a malformed or exhausted bitstream. */
int dvc_intra_decode_frame(const uint8_t *stream, size_t stream_bytes, size_t *bit_offset, int width, int height,
                           int intra_qp, const uint8_t *mode, uint8_t *recon);

/* Intra blocks of one WZ frame into the intra bitstream: for every 4x4 block
 * inside an intra 8x8 block (mode[w*h/64] == 1), in raster order, DC
 * prediction from the reconstructed intra neighbours, the 4x4 core transform,
 * quantisation with IntraQP and CAVLC, appended at *bit_offset of
 * stream[stream_bytes] (advanced past the frame's blocks); recon[w*h] receives
 * the pixels dvc_intra_decode_frame will reconstruct, and block_bits (if not
 * NULL, one int per 4x4 block) the bits each intra block took.  The counterpart of the
 * reference encoder's real_intra (DvcEnc/src/intra.cpp, vlc.cpp), in the
 * stream format its decoder reads; this encoder's quantiser and the choice of
 * intra blocks are its own, so streams are valid but not byte-identical to
 * the reference encoder's.  Host code.  DVC_E_ARG when stream is too short. */
int dvc_intra_encode_frame(const uint8_t *ori, int width, int height, int intra_qp, const uint8_t *mode,
                           uint8_t *stream, size_t stream_bytes, size_t *bit_offset, uint8_t *recon,
                           int *block_bits);

/* Self-check of the belief-propagation magnitude table, host code, no GPU:
 * sweeps phi(y) = -logf(tanhf(y)) with this host's C library over every
 * float argument the decoder can form, packs it the way dvc_create does for
 * the device, and checks every packed entry against the sweep.  DVC_OK with
 * *packed_bytes = the device bytes of the packed table; DVC_E_DATA with the
 * reason in msg otherwise.  The reference has no counterpart: its decoder
 * calls the two library functions per edge (LdpcaDecoder.cpp:513,519). */
int dvc_phi_table_check(size_t *packed_bytes, char *msg, int msglen);

/* LDPCA encoder on the device: for `count` source bitplanes of n bits
 * (bits[count*n], one 0/1 byte per bit) the accumulated syndromes acc[count*n/8]
 * (full-rate syndrome H*x, prefix-xored over the rows, packed MSB first as in
 * the WZ bitstream) and crc[count] (CRC-8 of the bitplane).  Equivalent to
 * LdpcaEncoder (DvcEnc/src/LdpcaEncoder.cpp:64-95) plus CRC8 (crc8.h:57-67)
 * per bitplane; the decoder side of the reference has no counterpart. */
int dvc_ldpca_encode(dvc_ctx *ctx, int n, int count, const uint8_t *bits, uint8_t *acc, uint8_t *crc);

/* Reference-shaped single-bitplane call: LdpcaDecoder(LR_intrinsic,
 * accumulatedSyndrome, decoded, &rate, crc, RateLowerBound) with the
 * accumulated syndrome as one bit per byte and the bound supplied by the
 * caller (LdpcaDecoder.cpp:646-649).  Like the reference, LR_intrinsic holds
 * log(p0/p1) on return. */
int dvc_LdpcaDecoder(dvc_ctx *ctx, int n, float *LR_intrinsic, const unsigned char *accumulatedSyndrome,
                     unsigned char *decoded, int *rate, unsigned char crc_encoder, float RateLowerBound);

/* One Wyner-Ziv frame for dvc_decode_wz_frames (all buffers are host memory).
 * The fields are what the reference's decodeGOP reads for one frame
 * (DVC_Decoder.cpp:26-435): the two reconstructed reference frames, the parsed
 * WZ-bitstream data of the frame (wzbitstream.cpp:13-126) and, for intra
 * blocks, the pixels intraRecon produced. */
typedef struct {
  int width, height;           /* 176x144 or 352x288 */
  int qindex;                  /* 1..8 */
  int past_idx, future_idx, cur_idx; /* frame numbers (set the interpolation weights) */
  const uint8_t *past;         /* [w*h] reconstructed past reference (luma) */
  const uint8_t *future;       /* [w*h] reconstructed future reference */
  const uint8_t *mode;         /* [w*h/64] 8x8 block modes 0 WZ, 1 intra, 2 skip; NULL = all WZ */
  int skip_mode, intra_mode;   /* frame-level flags from the bitstream */
  const int *ac_range;         /* [16] AC dynamic range per coefficient index */
  const uint8_t *crc;          /* [qbits] CRC-8 per bitplane */
  const uint8_t *acc_synd;     /* [qbits * w*h/128] accumulated syndromes, bitstream byte layout */
  uint8_t *recon;              /* [w*h] in: intra-block pixels (if any); out: decoded frame before deblocking */
  int wz_bits;                 /* out: 10 per coded AC band + sum over bitplanes of (m+8) */
  int *plane_results;          /* out [qbits*4] or NULL: rate, first code, accepted code, and the BP
                                  iterations run (a work counter: it grows with the speculation width) */
  float *plane_entropy;        /* out [qbits] or NULL */
  uint8_t *deblock_flag;       /* out [w*h] or NULL: coefficients changed by reconstruction */
  int deblock;                 /* 1: deblocking filter after decoding (the stream header's mode) */
  int intra_qp;                /* IntraQP of the stream (deblocking thresholds) */
  const uint8_t *past_mode;    /* [w*h/64] block modes of the past reference when it is a WZ
                                  frame, NULL when it is a key frame (deblocking of skip blocks) */
} dvc_wz_frame;

/* Decode `count` WZ frames of one size as one batch on the device (frames
 * must not depend on each other).  Equivalent to running decodeGOP's body
 * (DVC_Decoder.cpp:39-435, without intraRecon and the deblocking filter) on
 * each frame; replaces the ParallelMode 2/3 calls forwardME_CUDA,
 * noiseDistribution_CUDA, condBitProb_CUDA, beliefPropagation_CUDA*,
 * updateSI_CUDA and updateSMF_CUDA (forwardME_kernel.h:13,
 * noiseModel_kernel.h:17-19, LDPCA_cuda.h:19-20, updateSI_kernel.h:16,
 * motionLearning_kernel.h:13) together with the CPU stages between them. */
int dvc_decode_wz_frames(dvc_ctx *ctx, int count, dvc_wz_frame *frames);

/* dvc_decode_wz_frames on one frame that also returns intermediate stages for
 * stage-level checks (each may be NULL): the side information after
 * createSideInfo and the intra copy (DVC_Decoder.cpp:54-56), the noise
 * parameters alpha (noiseParameter, :79) and the side information after the
 * last updateSI (:318).  No counterpart in the reference. */
int dvc_debug_wz_frame(dvc_ctx *ctx, dvc_wz_frame *frame, uint8_t *si_initial, float *alpha, uint8_t *si_final);

/* dvc_decode_wz_frames on one frame that also returns the likelihood ratios
 * p0/p1 of every bitplane as condBitProb computes them (noiseModel.cpp:191-310,
 * called at DVC_Decoder.cpp:210) and LdpcaDecoder receives them:
 * lr_planes[qbits][w*h/16], bitplanes in decoding order (band by band in
 * zig-zag order, most significant bit first), QbitsNumPerBlk bitplanes for the
 * frame's QIndex.  No counterpart in the reference. */
int dvc_debug_wz_frame_lr(dvc_ctx *ctx, dvc_wz_frame *frame, float *lr_planes);

/* Reconstruction steps (reconstruction.cpp:184-289) met so far on this
 * context's device whose rounding ROUND(x) could change if an exp result
 * differed by up to 2 units in the last place: the reference calls its C
 * library's double exp there and the device its own, so a count of 0 shows
 * that no decoded coefficient can depend on that difference.  No counterpart
 * in the reference. */
int dvc_recon_near_ties(dvc_ctx *ctx, long long *count);

/* Batched LDPCA decode of `count` codewords of mixed lengths in one
 * persistent launch (the batching form of the decoder): every codeword walks
 * the rate-adaptive ladder from its own start level, and the device schedules
 * (codeword, ladder code) pairs over all SMs from a work queue, so that
 * codewords of uneven length and request level share the GPU without
 * lockstep.  Results equal LdpcaDecoder's (LdpcaDecoder.cpp:646-771) for each
 * codeword with RateLowerBound = the rate of its start code.
 *   n[count]            codeword lengths, 1584 or 6336, in any order
 *   lr[sum n]           p0/p1 of every codeword, concatenated in order
 *   acc[sum n / 8]      accumulated syndrome bytes, MSB first, concatenated
 *   crc[count]          CRC-8 of each source codeword
 *   start[count]        first ladder code to try (0..64), or NULL: the
 *                       conditional-entropy bound picks it (ComputeCE)
 *   decoded[sum n]      out: decoded bits, concatenated (may be NULL)
 *   results[count*4]    out: rate (m+8), first code, accepted code, and the BP
 *                       iterations the sequential ladder runs
 *   entropy[count]      out: conditional-entropy bound (may be NULL)
 *   max_iter            BP iterations per ladder code (the reference uses 50)
 *   bp_iterations       out: BP iterations the launch ran, codes abandoned
 *                       above an earlier success included (may be NULL)
 *   kernel_ms           out: device time of the launch (may be NULL)
 * Replaces, for many codewords at once, the per-request host loop of
 * beliefPropagation_CUDA_earlyJump (LDPCA_cuda.cu:872-969). */
int dvc_ldpca_decode_batch(dvc_ctx *ctx, int count, const int *n, const float *lr, const uint8_t *acc,
                           const uint8_t *crc, const int *start, uint8_t *decoded, int *results, float *entropy,
                           int max_iter, long long *bp_iterations, double *kernel_ms);

/* Most codewords one dvc_ldpca_decode_noalloc call accepts. */
#define DVC_NOALLOC_MAX_CODEWORDS 1024

/* LDPCA ladder decode for callers that cannot allocate device memory at call
 * time (cudaMalloc may synchronise the whole device, cannot run under stream
 * capture, and fails when another framework's pool owns the memory).  Same
 * results as dvc_ldpca_decode, but every buffer is the caller's device memory
 * and the call only enqueues work on `stream` (a cudaStream_t; NULL is the
 * legacy default stream), returning before the device is done.  The
 * per-codeword descriptors the kernel reads are kept in a fixed array in the
 * library's device memory (DVC_NOALLOC_MAX_CODEWORDS entries, about 100 KB,
 * held on every GPU that loads the library until the process exits); more
 * codewords per call are rejected with DVC_E_ARG.  The first call on each
 * device sets that device up: it looks the array's address up, sets the LDPCA
 * kernel's shared-memory attributes and loads the kernels' module, so make it
 * before any stream capture.  The address is kept for the life of the process,
 * so a device reset (cudaDeviceReset) while the library is loaded is not
 * supported by this entry point.  All calls share the array: calls that
 * overlap on the GPU race.
 *   d_lr[count*n] f32, d_acc[count*n/8], d_crc[count]       inputs
 *   d_decoded[count*n] (may be NULL), d_results[count*4],    outputs
 *   d_entropy[count] (may be NULL)
 * No counterpart in the reference. */
int dvc_ldpca_decode_noalloc(dvc_ctx *ctx, int n, int count, const float *d_lr, const uint8_t *d_acc,
                             const uint8_t *d_crc, uint8_t *d_decoded, int *d_results, float *d_entropy,
                             int max_iter, void *stream);

/* Device-resident decoding session: the frames' inputs and reference frames
 * are uploaded once by dvc_session_create; every dvc_session_run decodes all
 * of them again from device memory, in batches of at most `max_batch` frames
 * spread over `streams` concurrent CUDA streams, and keeps the results on the
 * device until dvc_session_frame copies them out.  Frames of one session share
 * one size.  A frame whose past or future pointer equals another frame's
 * recon pointer takes that frame's decoded output as the reference (the GOP
 * recursion of DVC_Decoder.cpp:26-474 for GOP 4 and 8): frames are grouped
 * into levels and a batch starts when the batches it reads from are done,
 * with no host round trip.  No counterpart in the reference (its GPU path
 * copies every stage's data in and out). */
typedef struct dvc_session dvc_session;
int dvc_session_create(dvc_ctx *ctx, int count, const dvc_wz_frame *frames, int max_batch, int streams,
                       dvc_session **out);
/* Decode every frame of the session once; returns when the device is done.
 * *elapsed_ms: device time of the whole run from CUDA events (may be NULL).
 * profile != 0 also times each LDPCA launch (see dvc_session_profile).  The
 * first run issues its work stream by stream; the second unprofiled run
 * captures that work (every stream, joined) as one CUDA graph and later
 * unprofiled runs replay it; a profiled run always issues its work directly.
 * If the capture fails, every run stays direct. */
int dvc_session_run(dvc_session *ses, int profile, double *elapsed_ms);
/* How many runs so far replayed the captured graph. */
int dvc_session_replays(dvc_session *ses, long long *replays);
/* Results of the last run for frame `index` (any output may be NULL). */
int dvc_session_frame(dvc_session *ses, int index, uint8_t *recon, int *wz_bits, int *plane_results);
/* Accumulated profile since creation: [0] LDPCA kernel ms, [1] LDPCA launches,
 * [2] LDPCA codewords, [3] kernel launches, [4] runs. */
int dvc_session_profile(dvc_session *ses, double *out5);
void dvc_session_destroy(dvc_session *ses);

/* Continuous-batching decode server (no counterpart in the reference, which
 * decodes one frame at a time).  Requests from any number of streams are
 * queued by dvc_server_submit (inputs are copied, so the caller's buffers can
 * be reused at once) and scheduled by dvc_server_poll: each of `streams` CUDA
 * streams runs one cohort at a time, a cohort being up to `max_cohort` queued
 * frames of one size (quantisers may differ).  Frames are admitted while the estimated
 * device memory of the frames in flight stays within `mem_budget_bytes`; a
 * frame that alone exceeds the budget is refused with DVC_E_NOMEM.  Every
 * stage, including the per-bitplane syndrome-request feedback, stays on the
 * device; the host only submits, polls and collects.  The server must be polled
 * from one thread at a time.  Cohort buffers grow in stream order
 * (cudaMallocAsync), and dvc_server_create sets the release threshold of the
 * current device's default memory pool so that freed memory stays cached in
 * this process (other users of that pool in the process see the same). */
typedef struct dvc_server dvc_server;
int dvc_server_create(dvc_ctx *ctx, size_t mem_budget_bytes, int streams, int max_cohort, dvc_server **out);
int dvc_server_submit(dvc_server *srv, const dvc_wz_frame *frame, long long *ticket);
/* Retire finished cohorts and start new ones; *completed = frames finished by this call. */
int dvc_server_poll(dvc_server *srv, int *completed);
/* Result of a finished request (each output may be NULL); frees the request.
 * latency_ms: from dvc_server_submit to the poll that saw it finished. */
int dvc_server_result(dvc_server *srv, long long ticket, uint8_t *recon, int *wz_bits, int *plane_results,
                      double *latency_ms);
/* Tickets of finished requests not yet collected (up to cap of them, oldest
 * ticket first), so that a caller collects exactly those. */
int dvc_server_finished(dvc_server *srv, long long *tickets, int cap, int *count);
int dvc_server_stats(dvc_server *srv, long long *pending, long long *in_flight, size_t *bytes_in_flight);
/* Dynamic batching window: while another cohort is decoding, a cohort with
 * fewer than max_cohort frames waits up to this long for more (default 2000 us). */
int dvc_server_config(dvc_server *srv, int batch_window_us);
void dvc_server_destroy(dvc_server *srv);

#ifdef __cplusplus
}
#endif
#endif
