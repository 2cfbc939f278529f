/*
 * ldpc_b200.h - C ABI of the B200 (sm_100a) fixed-point LDPC decoding engine.
 *
 * Plain C types only (pointers, sizes, ints); no CUDA or torch types appear
 * in the signatures, so cgo / JNI / ctypes / C++ callers bind it directly.
 * Every entry point returns 0 on success or a negative LDPC_ERR_* code and
 * never exits the process; ldpc_last_error_string() describes the last
 * failure of the calling thread.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   - the compile-time H matrix: src/matrix/code.h:1 (#define CODE),
 *     src/matrix/<code>/constantes_gpu.h:6-16 (_N, _K, _M, NB_DEGRES, DEG_1,
 *     DEG_2, DEG_1_COMPUTATIONS, DEG_2_COMPUTATIONS) and
 *     src/matrix/<code>/constantes_decoder.h:3 (PosNoeudsVariable[_M])
 *     -> ldpc_code_create_from_table / ldpc_code_create / ldpc_code_load;
 *   - the plugin constructors CGPUDecoder::CGPUDecoder(nb_frames, n, k, m)
 *     (src/decoder_template/CGPUDecoder.cpp:14-38) and
 *     CGPU_Decoder_{MS,OMS,NMS,2NMS}_SIMD / CGPU_Decoder_MS_SIMD_v2
 *     (src/decoder_oms/CGPU_Decoder_OMS_SIMD.cu:20-90 and the same lines of the
 *     MS, NMS, 2NMS and oms_v2 plugins, selected in src/main.cpp:213-228)
 *     -> ldpc_decoder_create;
 *   - CGPU_Decoder_*::decode(float*, int*, int)
 *     (src/decoder_oms/CGPU_Decoder_OMS_SIMD.cu:97-147 and siblings)
 *     -> ldpc_decode_host;
 *   - the destructor (src/decoder_template/CGPUDecoder.cpp:41-54)
 *     -> ldpc_decoder_destroy;
 *   - ERROR_CHECK's print-then-exit(0) (src/custom_api/custom_cuda.cu:5-17)
 *     -> status codes + ldpc_last_error_string.
 */
#ifndef LDPC_B200_H
#define LDPC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define LDPC_OK 0
#define LDPC_ERR_ARG (-1)         /* bad argument: null pointer, size, range   */
#define LDPC_ERR_CUDA (-2)        /* a CUDA runtime call failed                */
#define LDPC_ERR_UNSUPPORTED (-3) /* valid request this build cannot serve     */
#define LDPC_ERR_NOMEM (-4)       /* device or host allocation failed          */
#define LDPC_ERR_SHAPE (-5)       /* batch shape not accepted                  */

/* decoder kinds = the reference's plugins (src/main.cpp:166-182 flags) */
#define LDPC_MS 0   /* -MS / -fMS : CGPU_Decoder_MS_SIMD                          */
#define LDPC_OMS 1  /* -OMS       : CGPU_Decoder_OMS_SIMD (offset 1)              */
#define LDPC_NMS 2  /* -NMS       : CGPU_Decoder_NMS_SIMD (x0.75)                 */
#define LDPC_2NMS 3 /* -2NMS      : CGPU_Decoder_2NMS_SIMD (x0.75/x0.875, early term.) */
#define LDPC_XMS 4  /* -xMS       : CGPU_Decoder_MS_SIMD_v2 (input already word-interleaved) */
#define LDPC_LEARNED 5 /* learned offset/scale min-sum (no reference counterpart), see
                          ldpc_decoder_set_learned */
#define LDPC_LEARNED_MAX_ITERS 32

/* frame packing of the on-chip decoder state */
/* LDPC_PACK_AUTO: the QC register kernel when the code is QC and one fits (info path 1);
 * else LDPC_PACK_F16X2 (2 frames per CTA, path 2) for MS / OMS / NMS / xMS without early
 * stop; else LDPC_PACK_SIMD4; LDPC_PACK_FRAME when no 4-frame state fits.  Every packing
 * gives the same decisions. */
#define LDPC_PACK_AUTO (-1)
#define LDPC_PACK_SIMD4 0 /* 4 frames per 32-bit word, saturating byte lanes      */
/* 2 frames per 32-bit word, integer-valued fp16 lanes.  On a QC code (ldpc_code_create_qc)
 * whose shape has no 4-frame register kernel (more than 8 block rows or an irregular
 * row degree, such as 24-column bases), an explicit LDPC_PACK_F16X2 selects the QC
 * kernel with 2 frames per CTA (info path 4); LDPC_PACK_AUTO keeps the level kernels
 * there.  With LDPC_FLAG_EARLY_STOP path 4 stops each frame pair (frames 4g, 4g+1 and
 * 4g+2, 4g+3) on its own and reports per word the larger of its two pairs' counts. */
#define LDPC_PACK_F16X2 1
#define LDPC_PACK_I8 2    /* 1 frame per thread lane, int8 storage, int32 math    */
/* 2 frames per CTA (1 where two do not fit): the frames' APP as int8 in shared memory
 * (2N bytes, one CTA per SM at N = 64800) and their c->v messages, one byte per edge and
 * frame, in a message scratch the decoder allocates in device memory, one slot per
 * resident CTA (about 58 MB for N = 64800 rate 1/2 on 148 SMs); row records and
 * messages reach shared memory by bulk copies two stages ahead of their use.
 * For long codes whose 4-frame state exceeds shared memory.  Row degree <= 14.
 * LDPC_PACK_AUTO falls back to it when nothing else fits.  Not for LDPC_2NMS
 * (whose early termination is per 4-frame word).  With LDPC_FLAG_EARLY_STOP each
 * frame stops on its own.  On this path d_iters_out always receives one count per
 * frame (4*n_words entries), and state dumps (ldpc_decode_device_state) are
 * unsupported. */
#define LDPC_PACK_FRAME 3
/* The 2-frame QC register kernel of path 4 (24-column bases, Z <= 128) with each check row
 * split over 4 lanes: every lane takes every 4th edge of the row and the lanes merge their
 * min1 / min2 / sign parity with warp shuffles, so a row of degree 24 costs 6 serial steps
 * and a CTA has Z * 4 threads.  Info path 7.  Same decisions, iteration counts (per pair, as
 * path 4) and restrictions as path 4. */
#define LDPC_PACK_F16X2_SPLIT 4

/* output formats of ldpc_decode_device */
#define LDPC_OUT_BYTES 0  /* frame-major 0/1 bytes [frames][n] (the reference's)  */
#define LDPC_OUT_PACKED 1 /* frame-major bits, LSB first, ceil(n/8) bytes/frame   */

typedef struct ldpc_code ldpc_code;
typedef struct ldpc_decoder ldpc_decoder;

/* ---- codes ------------------------------------------------------------- */

/* H in the reference's own form: PosNoeudsVariable[m_edges] listing, check
 * by check in layer order, the variable index of every edge; the first
 * deg1_rows rows have degree deg1, the next deg2_rows rows degree deg2
 * (nb_degres = 1 or 2).  Replaces src/matrix/<code>/constantes_gpu.h:6-16
 * and constantes_decoder.h:3. */
int ldpc_code_create_from_table(ldpc_code** out, int n, int k_checks, int m_edges,
                                int nb_degres, int deg1, int deg1_rows, int deg2,
                                int deg2_rows, const uint32_t* pos_noeuds_variable);

/* H as CSR rows in layer order.  row_class (nullable) marks rows of the
 * reference's second degree group (1) - the offset-min-sum kernel skips the
 * 31-clip on them in the first iteration (decoder_oms/cuda/CUDA_OMS_SIMD.cu:115-116). */
int ldpc_code_create(ldpc_code** out, int n_vars, int n_checks, const int32_t* row_ptr,
                     const int32_t* cols, const uint8_t* row_class);

/* Quasi-cyclic H from a base matrix: shifts[i*nb+j] is the circulant shift of
 * block (i, j) (row k of block row i meets variable j*z + (k+s) mod z), or -1
 * for a zero block.  Rows are block-row major (row i*z+k), a row's edges in
 * ascending block column.  Decoders of such codes may use the QC kernel that
 * keeps every message in registers.  No reference counterpart (the reference
 * only ships fixed tables). */
int ldpc_code_create_qc(ldpc_code** out, int z, int mb, int nb, const int32_t* shifts);

/* Loads a .ldpc table file (format: fast_ldpc_decoder_for_gpu_fixed_b200/codes.py). */
int ldpc_code_load(ldpc_code** out, const char* path);

/* info[0..7] = n, checks, edges, max row degree, schedule levels per
 * iteration, widest level, n_info (= n - checks), 0 */
int ldpc_code_info(const ldpc_code* code, int* info);

void ldpc_code_destroy(ldpc_code* code);

/* ---- decoders ---------------------------------------------------------- */

/* Syndrome early stop (no reference counterpart; not for LDPC_2NMS, which keeps
 * the reference's own rule): a 4-frame word stops after an iteration in which
 * at most `slack` (row, frame) pairs had odd extrinsic sign parity (the
 * quantity 2NMS tests, CUDA_2NMS_SIMD.cu, counted over the word's 4 frames) and
 * whose hard decisions (x > 0 is bit 1) of all 4 frames then satisfy every
 * check.  The count only decides when the syndrome is evaluated: a word never
 * stops on a non-codeword.  `iters` becomes the maximum; the iterations run
 * are reported per word through d_iters_out. */
#define LDPC_FLAG_EARLY_STOP 1
#define LDPC_EARLY_STOP_DEFAULT_SLACK 128

/* A slack of at least LDPC_EARLY_SLACK_ANY makes every iteration a candidate: a word
 * (or, with LDPC_FLAG_EARLY_STOP_PAIRS, a frame pair) stops after the first iteration
 * whose hard decisions are codewords.  The 4-frame QC register kernel (path 1) then
 * keeps no odd-row count: it checks the rows of the last layer from the APP it has
 * just updated, and the other layers' rows only when those all hold.  The other paths
 * check the syndrome after every iteration. */
#define LDPC_EARLY_SLACK_ANY 1073741824

/* Per-frame early stop (implies LDPC_FLAG_EARLY_STOP): the rule above applied to
 * each frame alone (its own odd rows against `slack`, its own syndrome).  Decoder
 * path 5: the QC register kernel with 4 frames per CTA (ldpc_code_create_qc, the
 * regular 8x16 base with Z a power of two, every kind but 2NMS) run as persistent CTAs
 * that refill a finished frame's slot with a prefetched frame; with LDPC_PACK_FRAME
 * (path 3) it is that path's own rule; on the level kernel with LDPC_PACK_SIMD4 (path 0,
 * what LDPC_PACK_AUTO gives a code without a QC register kernel) a frame that stops has
 * its decisions written at once while the other frames of its word go on.  Other
 * decoders fail with LDPC_ERR_UNSUPPORTED.  d_iters_out then receives one count per
 * frame (4*n_words entries); no state dumps; on path 5 iters <= 255 and no
 * ldpc_simulate.  The early stop of such a decoder cannot be turned off. */
#define LDPC_FLAG_EARLY_STOP_FRAMES 4

/* Flooding schedule (no reference counterpart; the reference is row-layered): every
 * check row of an iteration reads the a-posteriori values of the previous iteration,
 * and after all rows each variable's value is rebuilt as sat8(LLR + the sum of its
 * edges' new messages), the sum taken exactly and saturated once.  Two barriers per
 * iteration instead of one per level, at the price of more iterations to converge.
 * Decoder path 6: the 4-frame LDPC_PACK_F16X2 level kernel (AUTO selects it), with or
 * without LDPC_FLAG_EARLY_STOP; not with LDPC_FLAG_EARLY_STOP_FRAMES.  The CPU oracle
 * states the same schedule (oracle_set_schedule). */
#define LDPC_FLAG_FLOODING 8

/* Per-pair early stop (implies LDPC_FLAG_EARLY_STOP): the rule above applied to each
 * frame pair of a word (frames 4g, 4g+1 and 4g+2, 4g+3: their own odd rows against
 * `slack`, their own syndrome).  A stopped pair keeps its decisions while the other pair
 * of the word goes on; d_iters_out receives per word the larger of its pairs' counts.
 * Decoder path 1 (the 4-frame QC register kernel) and path 4 (whose early stop is per
 * pair anyway); other decoders fail with LDPC_ERR_UNSUPPORTED.  Not with
 * LDPC_FLAG_EARLY_STOP_FRAMES or LDPC_FLAG_FLOODING. */
#define LDPC_FLAG_EARLY_STOP_PAIRS 16

/* nb_frames counts 32-bit lanes like the reference's constructor argument:
 * a decoder serves up to 4*nb_frames codewords per call (src/main.cpp:309).
 * Unlike the reference (decoder_oms/CGPU_Decoder_OMS_SIMD.cu:101-105), any
 * nb_frames >= 1 is accepted.  The decoder owns its device buffers; the code
 * may be destroyed after this call.  pack = LDPC_PACK_*; flags = 0 or
 * LDPC_FLAG_EARLY_STOP, LDPC_FLAG_EARLY_STOP_FRAMES, LDPC_FLAG_EARLY_STOP_PAIRS,
 * LDPC_FLAG_FLOODING. */
int ldpc_decoder_create(ldpc_decoder** out, const ldpc_code* code, int kind, size_t nb_frames,
                        int pack, int flags);

/* Synchronous decode of 4*nb_frames codewords between host buffers, exactly
 * like CGPU_Decoder_*::decode(float* var_nodes, int* Rprime_fix, int iters):
 * llr = frame-major int8 [4*nb_frames][n] (LDPC_XMS: the word-interleaved
 * reading word[v*nb_frames+g], byte k = frame 4g+k, as CGPU_Decoder_MS_SIMD_v2
 * receives it), hard = frame-major 0/1 bytes [4*nb_frames][n].  Host buffers
 * may be pageable or pinned; copies are pipelined with the decoding. */
int ldpc_decode_host(ldpc_decoder* dec, const int8_t* llr, uint8_t* hard, int iters);

/* Like ldpc_decode_host, with the outputs the device call offers (no reference
 * counterpart beyond decode()): out_format = LDPC_OUT_PACKED returns ceil(n/8) bytes
 * per frame instead of n (an eighth of the copy back to the host); iters_out (host,
 * nullable) receives what d_iters_out of ldpc_decode_device would, for all nb_frames
 * words; syndrome_ok (host, nullable) the 4*nb_frames per-frame syndrome flags. */
int ldpc_decode_host_ex(ldpc_decoder* dec, const int8_t* llr, void* out, int iters, int out_format,
                        int32_t* iters_out, uint8_t* syndrome_ok);

/* Asynchronous decode between device buffers on `stream` (a cudaStream_t,
 * 0 = legacy default stream).  n_words <= nb_frames words (4*n_words
 * codewords) starting at llr; out_format = LDPC_OUT_*.  iters_out (nullable,
 * device, n_words int32) receives the iterations executed per word.
 * d_syndrome_ok (nullable, device, 4*n_words bytes) receives per frame 1 when
 * its hard decisions (x > 0 is bit 1) satisfy every check, else 0: the test the
 * reference's error analyser makes against the transmitted word
 * (src/ber_analyzer/CErrorAnalyzer.cpp:142-158), made without it.  Frames that
 * stopped early by the syndrome have passed it already; the others get one
 * syndrome pass in the kernel's epilogue. */
int ldpc_decode_device(ldpc_decoder* dec, const int8_t* d_llr, void* d_out, size_t n_words,
                       int iters, int out_format, int32_t* d_iters_out, uint8_t* d_syndrome_ok,
                       void* stream);

/* Like ldpc_decode_device, plus the final decoder state in the reference's
 * device layouts (nullable): d_app = device_V, n*n_words 32-bit words
 * word[v*n_words+g]; d_msg = d_MSG_C_2_V, edges*n_words words word[e*n_words+g]
 * with e the edge index in table order.  For parity checks. */
int ldpc_decode_device_state(ldpc_decoder* dec, const int8_t* d_llr, uint8_t* d_hard,
                             size_t n_words, int iters, int32_t* d_iters_out,
                             int8_t* d_app, int8_t* d_msg, void* stream);

/* Fused Monte-Carlo step on `stream`: the decoder's prologue draws the LLRs of
 * 4*n_words frames from the AWGN channel itself (bit-identical to
 * ldpc_channel_awgn with the same sigma, seed, offset and codewords), decodes
 * them, and its epilogue adds frames / bit errors / frame errors over the first
 * n_vars bits to d_counts[0..2] (as ldpc_count_errors).  d_hard (nullable)
 * also receives the 0/1 decisions.  Replaces the channel -> decode ->
 * analyser round trip through host memory of src/main.cpp:258-286.  Not for
 * LDPC_XMS (its input is the word-interleaved layout). */
int ldpc_simulate(ldpc_decoder* dec, size_t n_words, int iters, float sigma, uint64_t seed,
                  uint64_t offset, const uint8_t* d_codewords, size_t n_codewords, int n_vars,
                  int64_t* d_counts, uint8_t* d_hard, void* stream);

/* Decode with no allocation at all.  No counterpart in the reference.  For callers
 * that may not call cudaMalloc once running: real-time receive chains, which cannot
 * afford the stall of an allocation or the device-wide synchronisation of cudaFree,
 * and plugin hosts whose memory pool owns the GPU and may refuse a request.  The
 * caller passes `code`, the decoder `kind` and `pack` (LDPC_PACK_SIMD4 / F16X2 / I8;
 * AUTO means SIMD4) and its own device buffers: d_llr (frame-major int8, 4*n_words
 * frames; LDPC_XMS: word-interleaved) and d_hard (frame-major 0/1 bytes).  The hard
 * decisions equal those of ldpc_decode_device (LDPC_OUT_BYTES) for a decoder of the
 * same kind on the same code, since every packing decides identically; this entry
 * point always runs the 4-frame level-scheduled kernel of `pack`, which needs
 * 4*(n rounded up to 16 + max row degree * checks) bytes of shared memory (twice that
 * for LDPC_PACK_F16X2) and refuses larger codes with LDPC_ERR_UNSUPPORTED.  No early
 * stop, iteration counts or state dumps.
 * Instead of decoder-owned buffers the code's tables go into one static 256 KiB
 * device array inside the library, which every GPU that loads the library holds until
 * exit; codes whose tables exceed it return LDPC_ERR_UNSUPPORTED.  The tables travel
 * as kernel parameters, so the call neither reads host memory later nor waits for
 * earlier work in `stream`.  The first call on a device looks up the array's device
 * address (once per device, kept for the life of the process): make that first call
 * before any stream capture, and do not reset the device (cudaDeviceReset) between
 * calls.  Every call rewrites the array, so calls that overlap on the GPU (different
 * streams with no ordering between them) race: issue them on one stream or
 * synchronise between them. */
int ldpc_decode_noalloc(const ldpc_code* code, int kind, int pack, const int8_t* d_llr,
                        uint8_t* d_hard, size_t n_words, int iters, void* stream);

/* Constants of an LDPC_LEARNED decoder (no reference counterpart): for iteration
 * t < n_iters and row group g (the reference's DEG_1 / DEG_2 groups), offsets[2t+g]
 * (int8) and scales[2t+g] (Q1.7, 128 = 1.0) give the check-to-variable magnitude
 * clamp(floor(min * scale / 128) - offset, 0, 31); iterations past n_iters reuse
 * the last row.  scale 128 / offset 1 everywhere is OMS without its first-iteration
 * quirk.  LDPC_PACK_F16X2 decoders (and the QC path, which is fp16) compute the
 * magnitude arithmetically and accept scales that are multiples of 8 (a 1/16
 * grid) and offsets in [-31, 31] only (LDPC_ERR_UNSUPPORTED otherwise); the
 * other packings take any constants.  Trained by
 * fast_ldpc_decoder_for_gpu_fixed_b200/learned.py, which quantises to that grid. */
int ldpc_decoder_set_learned(ldpc_decoder* dec, int n_iters, const int8_t* offsets,
                             const uint8_t* scales);

/* Training of the LDPC_LEARNED constants (no reference counterpart): one FP32
 * forward pass of `iters` unrolled layered min-sum iterations over `frames`
 * frames (d_llr: frames*n floats in the int8 decoder's LLR units, frame-major),
 * with per-iteration, per-row-group real-valued alpha[2t+g] (scale) and
 * beta[2t+g] (offset): magnitude clamp(alpha*min - beta, 0, 31), or with
 * LDPC_TRAIN_QUANTIZED clamp(floor(alpha*min) - beta, 0, 31) (with integer
 * LLRs, alpha = s/128 and integer beta that is exactly the int8 LDPC_LEARNED
 * decoder).  With S_f(t) the sum over the frame's bits of the BCE of
 * sigmoid(d_kappa[f] * APP after iteration t) against d_bits (frames*n 0/1
 * bytes, or null = all-zero codeword), d_loss[0] += sum_t d_weights[t] *
 * mean_f S_f(t)/n, or with LDPC_TRAIN_FRAME_LOSS sum_t d_weights[t] *
 * mean_f (1 - exp(-S_f(t))) (a soft frame error rate); d_weights: `iters`
 * floats, or null = the last iteration only.  When d_grad_alpha, d_grad_beta
 * and d_stash (ldpc_train_stash_bytes) are given, the backward pass adds
 * d loss / d alpha and d loss / d beta (straight-through for min, sign, the
 * saturations and the floor) into them.  d_app_out (frames*n floats, optional)
 * receives the final APP.  The decoder supplies the code and its row schedule
 * (any kind); the kernel runs on `stream`. */
#define LDPC_TRAIN_QUANTIZED 1
#define LDPC_TRAIN_FRAME_LOSS 2
int ldpc_train_step(const ldpc_decoder* dec, const float* d_llr, const uint8_t* d_bits,
                    const float* d_kappa, size_t frames, int iters, int flags,
                    const float* d_alpha, const float* d_beta, const float* d_weights,
                    float* d_grad_alpha, float* d_grad_beta, float* d_loss, void* d_stash,
                    float* d_app_out, void* stream);
size_t ldpc_train_stash_bytes(const ldpc_decoder* dec, size_t frames, int iters);

/* Turns the syndrome early stop on or off and sets its slack (default
 * LDPC_EARLY_STOP_DEFAULT_SLACK).  Turning it on for a decoder created without
 * LDPC_FLAG_EARLY_STOP fails for the 2-frames-per-CTA kernel (path 2).  On path 5
 * turning it off keeps the per-frame scheduling: every frame runs `iters`. */
int ldpc_decoder_set_early_stop(ldpc_decoder* dec, int enabled, int slack);

/* info[0..7] = kind, pack, nb_frames (words), threads per CTA, shared bytes
 * per CTA, CTAs per SM, registers per thread, kernel path (0 = level
 * scheduled, 1 = QC register-message, 2 = level scheduled with 2 frames per
 * CTA: LDPC_PACK_F16X2 for every kind but 2NMS, 3 = one frame per CTA with
 * packed row state: LDPC_PACK_FRAME, 4 = QC register-message with 2 frames per
 * CTA, see LDPC_PACK_F16X2, 5 = QC register-message with per-frame early stop,
 * see LDPC_FLAG_EARLY_STOP_FRAMES, 6 = level kernel with the flooding schedule, see
 * LDPC_FLAG_FLOODING, 7 = QC register-message with 2 frames per CTA and split rows, see
 * LDPC_PACK_F16X2_SPLIT) */
int ldpc_decoder_info(const ldpc_decoder* dec, int* info);

int ldpc_decoder_destroy(ldpc_decoder* dec);

/* Kernel status of a decoder (no reference counterpart): *status = 1 when a kernel of
 * this decoder gave up waiting on a bulk copy since the last call (its frames' results
 * are then invalid), else 0; reading clears it.  Only the one-frame-per-CTA path
 * (LDPC_PACK_FRAME) waits on copies.  Call it after the decodes it should cover have
 * completed (for example after synchronizing their stream); ldpc_decode_host and
 * ldpc_decode_host_ex check it themselves and fail with LDPC_ERR_CUDA. */
int ldpc_decoder_status(ldpc_decoder* dec, int* status);

/* ---- batches of codes (no reference counterpart) ------------------------ */

/* A batch decodes frames of several codes (different lengths and rates) in one
 * persistent kernel launch: resident CTAs take 4-frame words of any code from a
 * shared counter, so uneven per-code frame counts and per-word iteration counts
 * (LDPC_FLAG_EARLY_STOP) keep every SM busy.  Arithmetic and results per word are
 * those of ldpc_decoder_create with the same kind and pack (level schedule).
 * kind: any but LDPC_XMS; pack: LDPC_PACK_SIMD4 / F16X2 / I8, or AUTO (the
 * smallest state that fits; ldpc_batch_autotune then picks the fastest).
 * flags: LDPC_FLAG_EARLY_STOP, LDPC_FLAG_EARLY_STOP_FRAMES (each frame stops on its own:
 * the persistent kernel with LDPC_PACK_SIMD4, and per code the SIMD4 level kernel or the
 * QC refill kernel; d_iters_out then holds one count per frame, 4*n_words[i] entries per
 * code), LDPC_BATCH_GRAPH (launches captured once in a CUDA
 * graph and replayed while buffers, sizes and settings stay the same; needs a
 * stream other than the legacy default stream).  The codes may be destroyed
 * after this call. */
typedef struct ldpc_batch ldpc_batch;
#define LDPC_BATCH_GRAPH 2
int ldpc_batch_create(ldpc_batch** out, const ldpc_code* const* codes, int n_codes, int kind, int pack, int flags);

/* Decodes n_words[c] 4-frame words of every code c: d_llr[c] frame-major int8
 * LLRs, d_out[c] hard decisions (LDPC_OUT_BYTES or LDPC_OUT_PACKED), optional
 * d_iters_out[c] (iterations per word) or d_iters_out null, optional
 * d_syndrome_ok[c] (per-frame syndrome flags, as ldpc_decode_device) or
 * d_syndrome_ok null.  Asynchronous on `stream`. */
int ldpc_batch_decode(ldpc_batch* batch, const int8_t* const* d_llr, void* const* d_out, const size_t* n_words,
                      int iters, int out_format, int32_t* const* d_iters_out,
                      uint8_t* const* d_syndrome_ok, void* stream);

/* Times, on these inputs (outputs are overwritten), the two strategies and keeps the
 * fastest, returning its time per decode in *best_ms:
 *  - one launch per code (shared memory sized per code, the launches side by side and,
 *    with LDPC_BATCH_GRAPH, in one graph), each code with its own kernel: first, per
 *    code, every candidate is timed alone - the level kernel of each packing (SIMD4,
 *    F16X2, I8: 4 or 2 frames per CTA), the QC register kernel (QC codes: 4 frames per
 *    CTA on the regular base, else 2 with early stop per frame pair), the same 2-frame
 *    kernel with split rows (LDPC_PACK_F16X2_SPLIT) and the flooding schedule
 *    (LDPC_FLAG_FLOODING) - and the
 *    fastest is kept among those whose frames failing the syndrome are no more than the
 *    layered SIMD4 kernel's (within 2 % and 2 frames), so that a faster schedule is
 *    never bought with a higher frame error rate;
 *  - the persistent kernel for each packing, CTA width (64, 128, 256) and residency
 *    (as many CTAs per SM as fit, or half).
 * ldpc_batch_code_info reports each code's choice. */
int ldpc_batch_autotune(ldpc_batch* batch, const int8_t* const* d_llr, void* const* d_out, const size_t* n_words,
                        int iters, int32_t* const* d_iters_out, double* best_ms, void* stream);

/* The per-code strategy's kernel of code `code`: info[0] = candidate (0 SIMD4, 1 F16X2,
 * 2 I8 level kernels, 3 the QC register kernel, 4 the flooding schedule, 5 the QC register
 * kernel with split rows, LDPC_PACK_F16X2_SPLIT), info[1] = its
 * decoder path (ldpc_decoder_info), info[2] = threads per CTA, info[3] = shared bytes per
 * CTA, info[4] = CTAs per SM; path -1 when that kernel has not been set up yet. */
int ldpc_batch_code_info(const ldpc_batch* batch, int code, int* info);

/* Gives code `code` the per-code kernel `candidate` (as ldpc_batch_code_info numbers them)
 * and selects the per-code strategy; LDPC_ERR_UNSUPPORTED when that kernel cannot serve
 * the code. */
int ldpc_batch_set_code_kernel(ldpc_batch* batch, int code, int candidate);

/* Sets the strategy by hand: per_code = 0: the persistent kernel with this pack,
 * CTA width (32..256) and resident CTAs per SM (0 = as many as fit); per_code = 1:
 * one launch of each code's own kernel with this pack, the launches forked onto the
 * batch's own streams from `stream` and joined back to it (they run side by side). */
int ldpc_batch_configure(ldpc_batch* batch, int per_code, int pack, int threads, int ctas_per_sm);

/* LDPC_LEARNED constants of the batch (all codes), as ldpc_decoder_set_learned. */
int ldpc_batch_set_learned(ldpc_batch* batch, int n_iters, const int8_t* offsets, const uint8_t* scales);

/* Early stop on/off and its slack, as ldpc_decoder_set_early_stop. */
int ldpc_batch_set_early_stop(ldpc_batch* batch, int enabled, int slack);

/* info[0..8] = kind, pack, threads per CTA, shared bytes per CTA, resident CTAs
 * per SM, grid (CTAs of the persistent launch), graph mode, number of codes,
 * strategy (0 = one persistent kernel, 1 = one launch per code; the CTA fields
 * are 0 then) */
int ldpc_batch_info(const ldpc_batch* batch, int* info);

int ldpc_batch_destroy(ldpc_batch* batch);

/* ---- channel and error counting (the simulation stages around the decoder) */

/* Noise deviation for an Eb/N0 (or Es/N0 when es_n0) in dB at code rate `rate`,
 * as CChanel_AWGN_SIMD::configure (src/awgn_channel/CChanel_AWGN_SIMD.cu:63-73). */
double ldpc_sigma(double ebn0, double rate, int es_n0);

/* AWGN channel on the GPU, replacing CChanel_AWGN_SIMD::generate
 * (src/awgn_channel/CChanel_AWGN_SIMD.cu:88-112): frames*n int8 LLRs,
 * frame-major, q = trunc(clamp(8*((2b-1) + sigma*g), -31, 31)) with g a
 * Box-Muller Gaussian from a Philox4x32-10 stream (seed, offset) indexed by
 * sample, b the codeword bit (d_codewords: n_codewords frame-major 0/1
 * codewords used cyclically, or null for the all-zero codeword). */
int ldpc_channel_awgn(int8_t* d_llr, size_t frames, int n, float sigma, uint64_t seed,
                      uint64_t offset, const uint8_t* d_codewords, size_t n_codewords,
                      void* stream);

/* Raw Philox4x32-10 words of stream (seed, offset), count of them (the
 * channel's uniforms are (word + 0.5) / 2^32).  No reference counterpart. */
int ldpc_philox(uint32_t* d_out, size_t count, uint64_t seed, uint64_t offset, void* stream);

/* Error counting on the GPU, replacing CErrorAnalyzer::generate
 * (src/ber_analyzer/CErrorAnalyzer.cpp:119-159): for each of `frames` decided
 * frames (0/1 bytes, frame-major, n per frame) the bits among the first n_vars
 * that differ from the transmitted codeword (null: all-zero) are counted;
 * d_counts[0] += frames, d_counts[1] += bit errors, d_counts[2] += frame errors. */
int ldpc_count_errors(const uint8_t* d_hard, size_t frames, int n, int n_vars,
                      const uint8_t* d_codewords, size_t n_codewords, int64_t* d_counts,
                      void* stream);

/* ---- misc -------------------------------------------------------------- */

const char* ldpc_last_error_string(void);
int ldpc_version(void);

/* Exhaustive check helper: applies the device's per-byte SIMD operation `op`
 * (ids as oracle_byte_op: 0 sat-sub, 1 sat-add, 2 abs, 3 minu, 4 maxu,
 * 5 subus, 6 gt-mask, 7 eq-mask, 8 neg, 9 gt-0/1) to n word pairs on the GPU. */
int ldpc_simd_selftest(int op, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_out,
                       size_t n, void* stream);

/* Measures this GPU's INT32 issue rate (lane operations per second, best of
 * independent LOP3 / IADD3 / mixed chains over all SMs): the denominator of
 * the integer decoder's roofline.  No reference counterpart. */
int ldpc_probe_int_peak(double* lane_ops_per_s, void* stream);

#ifdef __cplusplus
}
#endif
#endif
