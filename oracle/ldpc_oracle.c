/*
 * CPU oracle for the fixed-point LDPC decoders.  TEST INFRASTRUCTURE ONLY:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, as the checker.  The product path never calls it.
 *
 * It restates, frame by frame in plain C, what the reference GPU kernels
 * compute on one byte lane of their 4-frames-per-word SIMD packing:
 *
 *   MS    decoder_ms/cuda/CUDA_MS_SIMD.cu:25-248      (c = min(min,31))
 *   OMS   decoder_oms/cuda/CUDA_OMS_SIMD.cu:25-248    (c = min(subus(min,1),31);
 *                                                      no 31-clip on first-iteration
 *                                                      DEG_2 rows, :115-116)
 *   NMS   decoder_nms/cuda/CUDA_NMS_SIMD.cu:25-292    (c = (char)((float)min*0.75f))
 *   2NMS  decoder_2nms/cuda/CUDA_2NMS_SIMD.cu:17-292  (min1*0.75, min2*0.875,
 *                                                      EARLY_TERM 1)
 *   xMS   decoder_oms_v2/cuda/CUDA_OMS_SIMD_v2.cu:343-575 (OMS arithmetic with the
 *                                                      31-clip everywhere, EARLY_TERM 0;
 *                                                      plugin skips the input interleave,
 *                                                      CGPU_Decoder_MS_SIMD_v2.cu:187)
 *
 * Per-byte operation semantics follow the SIMD helper header the reference
 * vendors (decoder_oms/cuda/simd_functions.h:89-130): vabs4 wraps (|-128| is
 * 0x80), vaddss4/vsubss4 saturate to [-128,127], vsubus4 saturates at 0,
 * vminu4/vmaxu4 compare unsigned bytes, vcmpgts4 is a signed ">" per byte.
 *
 * The row loop is the reference's: rows in table order, the a-posteriori
 * value APP[v] rewritten in place right after each row (row-layered), the
 * first iteration reading APP directly (CUDA_OMS_SIMD.cu:40-134), later
 * iterations reading the extrinsic sat8(APP - msg) (:138-246).  Early
 * termination (2NMS) is decided per 32-bit word, i.e. jointly for the four
 * frames 4g..4g+3 that share a word, on the OR over rows of the extrinsic
 * sign parity, and only inside the "while (loops--)" iterations
 * (CUDA_2NMS_SIMD.cu:160-290).
 *
 * Layouts: the drop-in decode() takes frame-major int8 LLRs [4W][N] and
 * returns frame-major 0/1 bytes [4W][N]; the reference converts to and from
 * the word-interleaved layout word[v*W+g] (byte k = frame 4g+k) with
 * transpose/GPU_Transpose_uint8.cu:80-130 (Interleaver_uint8) and :9-78
 * (InvInterleaver_uint8, fused hard decision vsetgts4(x,0)).
 *
 * Parity pin: this restatement is checked against outputs of the reference
 * kernels themselves (compiled from the reference sources by
 * oracle/build_ref.sh and run on a B200 by tests/golden/make_golden.py); the
 * resulting fixtures live in tests/golden/.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define K_MS 0
#define K_OMS 1
#define K_NMS 2
#define K_2NMS 3
#define K_XMS 4
#define K_LEARNED 5

/* Learned min-sum (no reference counterpart): per iteration t and row group g an
 * int8 offset beta and a Q1.7 scale q; c = clamp(floor(min * q / 128) - beta, 0, 31).
 * scale 128 and offset 1 give OMS.  Iterations past the table reuse its last row. */
#define LEARNED_MAX_IT 64
static int g_learned_its = 0;
static int8_t g_learned_off[LEARNED_MAX_IT][2];
static uint8_t g_learned_scale[LEARNED_MAX_IT][2];

int oracle_set_learned(int n_iters, const int8_t* offsets, const uint8_t* scales)
{
    if (n_iters < 1 || n_iters > LEARNED_MAX_IT) return -1;
    g_learned_its = n_iters;
    for (int t = 0; t < n_iters; t++)
        for (int g = 0; g < 2; g++) {
            g_learned_off[t][g] = offsets[2 * t + g];
            g_learned_scale[t][g] = scales[2 * t + g];
        }
    return 0;
}

static inline int learned_mag(int it, int cls, int m)
{
    int t = it < g_learned_its ? it : g_learned_its - 1;
    int c = ((m * (int)g_learned_scale[t][cls]) >> 7) - g_learned_off[t][cls];
    return c < 0 ? 0 : (c > 31 ? 31 : c);
}

/* ---- per-byte semantics (simd_functions.h:89-130) ---------------------- */

static inline int sat8(int x) { return x < -128 ? -128 : (x > 127 ? 127 : x); }
/* vabs4 of one byte, as an unsigned byte: |-128| wraps to 0x80 = 128 */
static inline int vabs_u8(int x) { return (x < 0 ? -x : x) & 0xFF; }
static inline int minu(int a, int b) { return a < b ? a : b; } /* a,b in [0,255] */
static inline int maxu(int a, int b) { return a > b ? a : b; }
static inline int subus(int a, int b) { return a > b ? a - b : 0; }

/* vneg4 of one byte (wrap-around two's complement negate) */
static inline int vneg8(int x) { return (int8_t)(uint8_t)(-x); }

/* check-to-variable magnitudes c1 (for the minimum edge) and c2 (others) */
static inline void check_mags(int kind, int it, int row_class, int min1, int min2,
                              int* c1, int* c2)
{
    switch (kind) {
    case K_MS: /* CUDA_MS_SIMD.cu:73-74 */
        *c1 = minu(min2, 31);
        *c2 = minu(min1, 31);
        break;
    case K_OMS: /* CUDA_OMS_SIMD.cu:73-74; first-iteration DEG_2 rows :115-116 */
        if (it == 0 && row_class == 1) {
            *c1 = subus(min2, 1);
            *c2 = subus(min1, 1);
        } else {
            *c1 = minu(subus(min2, 1), 31);
            *c2 = minu(subus(min1, 1), 31);
        }
        break;
    case K_XMS: /* CUDA_OMS_SIMD_v2.cu:389-390, :433-434 */
        *c1 = minu(subus(min2, 1), 31);
        *c2 = minu(subus(min1, 1), 31);
        break;
    case K_NMS: /* CUDA_NMS_SIMD.cu:73-85: signed char -> float * 0.75f -> char */
        *c1 = (int8_t)((float)(int8_t)min2 * 0.750f);
        *c2 = (int8_t)((float)(int8_t)min1 * 0.750f);
        break;
    case K_2NMS: /* CUDA_2NMS_SIMD.cu:76-83 */
        *c1 = (int8_t)((float)(int8_t)min2 * 0.875f);
        *c2 = (int8_t)((float)(int8_t)min1 * 0.750f);
        break;
    case K_LEARNED:
        *c1 = learned_mag(it, row_class, min2);
        *c2 = learned_mag(it, row_class, min1);
        break;
    }
}

/*
 * Decode one word = 4 frames in lock-step (they share the early-termination
 * decision).  app: [4][n] int8 in/out; msg: [4][e] int8 scratch/out.
 * Returns the number of iterations executed.
 */
/* 1 when the hard decisions (x > 0) of all 4 frames satisfy every check */
static int word_syndrome_zero(int n, int m, const int32_t* row_ptr, const int32_t* cols, const int8_t* app, int nl)
{
    for (int lane = 0; lane < nl; lane++) {
        const int8_t* A = app + (size_t)lane * n;
        for (int r = 0; r < m; r++) {
            int p = 0;
            for (int k = row_ptr[r]; k < row_ptr[r + 1]; k++) p ^= (A[cols[k]] > 0);
            if (p) return 0;
        }
    }
    return 1;
}

/* Flooding schedule (LDPC_FLAG_FLOODING, no reference counterpart; set by
 * oracle_set_schedule): every row of an iteration reads the APP of the previous
 * iteration, computes its messages with the same check update as the layered
 * schedule, and only after all rows APP[v] = sat8(LLR[v] + sum of the new messages
 * of v's edges), the sum taken exactly and saturated once. */
static int g_flood = 0;

int oracle_set_schedule(int flooding)
{
    g_flood = flooding ? 1 : 0;
    return 0;
}

static int decode_word(int n, int m, const int32_t* row_ptr, const int32_t* cols,
                       const uint8_t* row_class, int kind, int iters,
                       int8_t* app, int8_t* msg, int early, int nl)
{
    int e_total = row_ptr[m];
    int et = (kind == K_2NMS);
    int dmax = 0;
    for (int r = 0; r < m; r++)
        if (row_ptr[r + 1] - row_ptr[r] > dmax) dmax = row_ptr[r + 1] - row_ptr[r];
    int* tv = (int*)malloc(sizeof(int) * (dmax > 0 ? dmax : 1));
    const int flood = g_flood;
    int8_t* llr0 = NULL; /* flooding: the channel values of the nl lanes */
    int* acc = NULL;     /* flooding: LLR + sum of the iteration's messages, per lane and variable */
    if (flood) {
        llr0 = (int8_t*)malloc((size_t)nl * n);
        acc = (int*)malloc(sizeof(int) * (size_t)nl * n);
        memcpy(llr0, app, (size_t)nl * n);
    }
    int executed = 0;
    for (int it = 0; it < iters; it++) {
        int ov_sign = 0; /* OR over rows and lanes of the extrinsic sign parity */
        int odd_rows = 0; /* (row, lane) pairs whose extrinsic sign parity was odd */
        if (flood)
            for (size_t i = 0; i < (size_t)nl * n; i++) acc[i] = llr0[i];
        for (int r = 0; r < m; r++) {
            int b = row_ptr[r], d = row_ptr[r + 1] - b;
            for (int lane = 0; lane < nl; lane++) {
                int8_t* A = app + (size_t)lane * n;
                int8_t* M = msg + (size_t)lane * e_total;
                int min1 = 127, min2 = 127, sgn = 0;
                for (int j = 0; j < d; j++) {
                    int v = cols[b + j];
                    int t = (it == 0) ? A[v] : sat8(A[v] - M[b + j]);
                    int a = vabs_u8(t);
                    tv[j] = t;
                    min2 = minu(min2, maxu(a, min1));
                    min1 = minu(min1, a);
                    sgn ^= (t > 0);
                }
                int c1, c2;
                check_mags(kind, it, row_class ? row_class[r] : 0, min1, min2, &c1, &c2);
                for (int j = 0; j < d; j++) {
                    int t = tv[j];
                    int a = vabs_u8(t);
                    int re = (a == min1) ? c1 : c2;
                    int s = sgn ^ (t > 0);
                    int out = s ? (int)(int8_t)re : vneg8(re);
                    M[b + j] = (int8_t)out;
                    if (flood)
                        acc[(size_t)lane * n + cols[b + j]] += out;
                    else
                        A[cols[b + j]] = (int8_t)sat8(t + out);
                }
                ov_sign |= sgn;
                odd_rows += sgn;
            }
        }
        if (flood)
            for (size_t i = 0; i < (size_t)nl * n; i++) app[i] = (int8_t)sat8(acc[i]);
        executed = it + 1;
        if (et && it >= 1 && ov_sign == 0) break;
        /* syndrome early stop (LDPC_FLAG_EARLY_STOP, no reference counterpart;
         * early = 1 + slack): after an iteration in which at most `slack` (row,
         * lane) pairs had odd extrinsic parity, stop if the hard decisions of all
         * 4 frames form codewords */
        if (early && odd_rows <= early - 1 && word_syndrome_zero(n, m, row_ptr, cols, app, nl)) break;
    }
    free(tv);
    free(llr0);
    free(acc);
    return executed;
}

/*
 * Decode nframes (multiple of 4) frames.
 *   llr  : if !interleaved, frame-major [nframes][n] int8 (the plugin's
 *          decode() input); if interleaved (xMS), the raw buffer is read as
 *          word[v*W+g], byte k = frame 4g+k, W = nframes/4.
 *   hard : [nframes][n] bytes 0/1, frame-major (InvInterleaver_uint8 output).
 *   app_out : optional, final APP in the word-interleaved layout
 *             [n][W] words (the reference's device_V), i.e. n*nframes bytes.
 *   msg_out : optional, final messages in the reference's device layout
 *             word[e*W+g] (d_MSG_C_2_V), e*nframes bytes.
 *   iters_out : optional, [W] iterations executed per word.
 */
/* group: frames that stop together under the early stop: 4 = a word (the level
 * kernels and the 4-frame QC kernel); 2 = a frame pair (the 2-frame QC kernel;
 * a word's count is the larger of its two pairs'); 1 = each frame alone (the
 * one-frame-per-CTA kernel, whose counts are per frame: iters_out holds nframes
 * entries) */
int oracle_decode_ex(int n, int m, const int32_t* row_ptr, const int32_t* cols,
                     const uint8_t* row_class, int kind, int iters, int nframes,
                     int interleaved, const int8_t* llr, uint8_t* hard,
                     int8_t* app_out, int8_t* msg_out, int32_t* iters_out, int nthreads, int early,
                     int group)
{
    if (nframes % 4 || iters < 1 || n <= 0 || m <= 0) return -1;
    int W = nframes / 4;
    int e_total = row_ptr[m];
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int g = 0; g < W; g++) {
        int8_t* app = (int8_t*)malloc((size_t)4 * n);
        int8_t* msg = (int8_t*)calloc((size_t)4 * e_total, 1);
        for (int lane = 0; lane < 4; lane++) {
            int f = 4 * g + lane;
            for (int v = 0; v < n; v++)
                app[(size_t)lane * n + v] = interleaved
                    ? llr[((size_t)v * W + g) * 4 + lane]
                    : llr[(size_t)f * n + v];
        }
        if (group == 1) {
            for (int lane = 0; lane < 4; lane++) {
                int ex = decode_word(n, m, row_ptr, cols, row_class, kind, iters, app + (size_t)lane * n,
                                     msg + (size_t)lane * e_total, early, 1);
                if (iters_out) iters_out[4 * g + lane] = ex;
            }
        } else if (group == 2) {
            int ex0 = decode_word(n, m, row_ptr, cols, row_class, kind, iters, app, msg, early, 2);
            int ex1 = decode_word(n, m, row_ptr, cols, row_class, kind, iters, app + (size_t)2 * n,
                                  msg + (size_t)2 * e_total, early, 2);
            if (iters_out) iters_out[g] = ex0 > ex1 ? ex0 : ex1;
        } else {
            int ex = decode_word(n, m, row_ptr, cols, row_class, kind, iters, app, msg, early, 4);
            if (iters_out) iters_out[g] = ex;
        }
        for (int lane = 0; lane < 4; lane++) {
            int f = 4 * g + lane;
            for (int v = 0; v < n; v++) {
                int8_t x = app[(size_t)lane * n + v];
                hard[(size_t)f * n + v] = (x > 0);
                if (app_out) app_out[((size_t)v * W + g) * 4 + lane] = x;
            }
            if (msg_out)
                for (int e = 0; e < e_total; e++)
                    msg_out[((size_t)e * W + g) * 4 + lane] = msg[(size_t)lane * e_total + e];
        }
        free(app);
        free(msg);
    }
    return 0;
}

int oracle_decode(int n, int m, const int32_t* row_ptr, const int32_t* cols,
                  const uint8_t* row_class, int kind, int iters, int nframes,
                  int interleaved, const int8_t* llr, uint8_t* hard,
                  int8_t* app_out, int8_t* msg_out, int32_t* iters_out, int nthreads)
{
    return oracle_decode_ex(n, m, row_ptr, cols, row_class, kind, iters, nframes, interleaved, llr, hard,
                            app_out, msg_out, iters_out, nthreads, 0, 4);
}

/* ---- layout restatements (transpose/GPU_Transpose_uint8.cu) ------------- */

/* Interleaver_uint8 (:80-130): frame-major [4W][n] -> word[v*W+g], byte k = frame 4g+k */
void oracle_interleave(int n, int W, const int8_t* in, int8_t* out)
{
    for (int g = 0; g < W; g++)
        for (int k = 0; k < 4; k++)
            for (int v = 0; v < n; v++)
                out[((size_t)v * W + g) * 4 + k] = in[(size_t)(4 * g + k) * n + v];
}

/* InvInterleaver_uint8 (:9-78): word layout -> frame-major 0/1 (vsetgts4(x,0), :29) */
void oracle_deinterleave_hd(int n, int W, const int8_t* in, uint8_t* out)
{
    for (int g = 0; g < W; g++)
        for (int k = 0; k < 4; k++)
            for (int v = 0; v < n; v++)
                out[(size_t)(4 * g + k) * n + v] = in[((size_t)v * W + g) * 4 + k] > 0;
}

/* ---- per-byte op table, for exhaustive checks of device SIMD helpers ---- */

/* op ids: 0 sat-sub, 1 sat-add, 2 abs(wrap), 3 minu, 4 maxu, 5 subus, 6 gt0(0xFF),
 * 7 eq(0xFF), 8 neg(wrap), 9 setgt0 (0/1) */
int oracle_byte_op(int op, int a, int b)
{
    int8_t x = (int8_t)a, y = (int8_t)b;
    uint8_t ux = (uint8_t)a, uy = (uint8_t)b;
    switch (op) {
    case 0: return (uint8_t)sat8(x - y);
    case 1: return (uint8_t)sat8(x + y);
    case 2: return (uint8_t)vabs_u8(x);
    case 3: return ux < uy ? ux : uy;
    case 4: return ux > uy ? ux : uy;
    case 5: return ux > uy ? ux - uy : 0;
    case 6: return x > y ? 0xFF : 0;
    case 7: return ux == uy ? 0xFF : 0;
    case 8: return (uint8_t)(-x);
    case 9: return x > y ? 1 : 0;
    }
    return -1;
}

/* ---- error analyser restatement (ber_analyzer/CErrorAnalyzer.cpp:142-158) --
 * counts, for each frame, the non-zero decisions among its first n_vars
 * bytes (all-zero codeword), n_vars = N - #checks (trame/CTrame.cpp:65-67). */
void oracle_count_errors(int n, int n_vars, int nframes, const uint8_t* hard,
                         int64_t* bit_errors, int64_t* frame_errors, int32_t* per_frame)
{
    int64_t be = 0, fe = 0;
    for (int f = 0; f < nframes; f++) {
        int e = 0;
        for (int i = 0; i < n_vars; i++) e += hard[(size_t)f * n + i] != 0;
        if (per_frame) per_frame[f] = e;
        be += e;
        fe += (e != 0);
    }
    *bit_errors = be;
    *frame_errors = fe;
}

/* ---- channel quantiser restatement (awgn_channel/CChanel_AWGN_SIMD.cu:17-24)
 * v = -1 + (x * trig) * sigma, q = (char) fminf(fmaxf(8v, -31), 31) with
 * truncation toward zero; computed here in float like the reference. */
int oracle_quantize(float x_times_trig, float sigma)
{
    float v = (-1.0f + x_times_trig * sigma);
    return (int8_t)fminf(fmaxf(8.0f * v, -31.0f), 31.0f);
}

/* sigma from Eb/N0 (CChanel_AWGN_SIMD.cu:63-73) */
double oracle_sigma(double ebn0, double rate, int es_n0)
{
    double eb = es_n0 ? ebn0 - 10.0 * log10(2 * rate) : ebn0;
    double interm = 10.0 * log10(rate);
    interm = -0.1 * (eb + interm);
    return sqrt(pow(10.0, interm) / 2);
}

/* ---- channel restatement in double precision ----------------------------
 * Philox4x32-10 (Salmon et al., SC'11, the counter-based generator the
 * project's GPU channel uses in place of the reference's cuRAND XORWOW), then
 * Box-Muller and the reference quantiser
 * q = (char) clamp(8 * (mean + sigma * g), -31, 31)
 * (awgn_channel/CChanel_AWGN_SIMD.cu:17-24) evaluated in double. */
static void philox10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

void oracle_philox(uint32_t* out, size_t count, uint64_t seed, uint64_t offset)
{
    for (size_t q = 0; 4 * q < count; q++) {
        uint32_t c[4] = {(uint32_t)q, (uint32_t)(q >> 32), (uint32_t)offset, (uint32_t)(offset >> 32)};
        philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        for (int i = 0; i < 4 && 4 * q + i < count; i++) out[4 * q + i] = c[i];
    }
}

/* also returns, per sample, the pre-quantisation value 8y in y8 (nullable) */
void oracle_awgn(int8_t* out, double* y8, size_t frames, int n, double sigma, uint64_t seed,
                 uint64_t offset, const uint8_t* cw, size_t n_cw)
{
    const double PI = 3.14159265358979323846;
    size_t total = frames * (size_t)n;
    for (size_t q = 0; 4 * q < total; q++) {
        uint32_t c[4] = {(uint32_t)q, (uint32_t)(q >> 32), (uint32_t)offset, (uint32_t)(offset >> 32)};
        philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        double u[4], g[4];
        for (int i = 0; i < 4; i++) u[i] = ((double)c[i] + 0.5) / 4294967296.0;
        for (int p = 0; p < 2; p++) {
            double r = sqrt(-2.0 * log(u[2 * p]));
            g[2 * p] = r * cos(2.0 * PI * u[2 * p + 1]);
            g[2 * p + 1] = r * sin(2.0 * PI * u[2 * p + 1]);
        }
        for (int i = 0; i < 4 && 4 * q + i < total; i++) {
            size_t s = 4 * q + i;
            double mean = -1.0;
            if (cw) {
                size_t f = s / n, v = s % n;
                mean = cw[(f % n_cw) * n + v] ? 1.0 : -1.0;
            }
            double y = 8.0 * (mean + sigma * g[i]);
            if (y8) y8[s] = y;
            out[s] = (int8_t)trunc(fmin(fmax(y, -31.0), 31.0));
        }
    }
}
