/*
 * Batched CPU decoder used as the timed CPU baseline.  TEST INFRASTRUCTURE
 * ONLY (bench.py's CPU-baseline leg and tests/ load it; the product path
 * never does).
 *
 * Same arithmetic as ldpc_oracle.c (the restatement of the reference kernels
 * decoder_{ms,oms,nms,oms_v2}/cuda/ kernels, row-layered, byte semantics of
 * decoder_oms/cuda/simd_functions.h:89-130), but 32 frames run in lock-step in
 * one AVX2 register per value, the way the reference runs 4 frames in one
 * 32-bit word: _mm256_subs_epi8 / _mm256_adds_epi8 saturate like vsubss4 /
 * vaddss4, _mm256_abs_epi8 wraps |-128| to 0x80 like vabs4, and the unsigned
 * byte min/max match vminu4/vmaxu4.  Early-terminating kinds (2NMS) are not
 * batched; the caller uses the scalar oracle for those.  OpenMP spreads the
 * frame groups over the host threads.  Where the CPU has AVX-512BW the groups
 * are 64 frames in one __m512i per value (the same byte operations, with mask
 * registers for the selects); AVX2 stays the fallback.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <immintrin.h>

#define K_MS 0
#define K_OMS 1
#define K_NMS 2
#define K_2NMS 3
#define K_XMS 4
#define LANES 32

__attribute__((target("avx2"))) static inline __m256i scale_floor(__m256i x, int num, int shift)
{
    /* floor(x * num / 2^shift) per unsigned byte x <= 127, through 16-bit lanes */
    __m256i lo = _mm256_unpacklo_epi8(x, _mm256_setzero_si256());
    __m256i hi = _mm256_unpackhi_epi8(x, _mm256_setzero_si256());
    __m256i k = _mm256_set1_epi16((short)num);
    lo = _mm256_srli_epi16(_mm256_mullo_epi16(lo, k), shift);
    hi = _mm256_srli_epi16(_mm256_mullo_epi16(hi, k), shift);
    return _mm256_packus_epi16(lo, hi);
}

__attribute__((target("avx2"))) static void decode_group(
    int n, int m, const int32_t* row_ptr, const int32_t* cols, const uint8_t* row_class,
    int kind, int iters, __m256i* app, __m256i* msg, __m256i* tv)
{
    const __m256i zero = _mm256_setzero_si256();
    const __m256i one = _mm256_set1_epi8(1);
    const __m256i c31 = _mm256_set1_epi8(31);
    const __m256i c127 = _mm256_set1_epi8(127);
    for (int it = 0; it < iters; it++) {
        for (int r = 0; r < m; r++) {
            int b = row_ptr[r], d = row_ptr[r + 1] - b;
            __m256i min1 = c127, min2 = c127, sgn = zero;
            for (int j = 0; j < d; j++) {
                __m256i a_v = app[cols[b + j]];
                __m256i t = (it == 0) ? a_v : _mm256_subs_epi8(a_v, msg[b + j]);
                __m256i a = _mm256_abs_epi8(t);
                tv[j] = t;
                min2 = _mm256_min_epu8(min2, _mm256_max_epu8(a, min1));
                min1 = _mm256_min_epu8(min1, a);
                sgn = _mm256_xor_si256(sgn, _mm256_cmpgt_epi8(t, zero));
            }
            __m256i c1, c2;
            int cls = row_class ? row_class[r] : 0;
            if (kind == K_MS) {
                c1 = _mm256_min_epu8(min2, c31);
                c2 = _mm256_min_epu8(min1, c31);
            } else if (kind == K_NMS) {
                c1 = scale_floor(min2, 3, 2);
                c2 = scale_floor(min1, 3, 2);
            } else {
                c1 = _mm256_subs_epu8(min2, one);
                c2 = _mm256_subs_epu8(min1, one);
                if (!(kind == K_OMS && it == 0 && cls == 1)) {
                    c1 = _mm256_min_epu8(c1, c31);
                    c2 = _mm256_min_epu8(c2, c31);
                }
            }
            for (int j = 0; j < d; j++) {
                __m256i t = tv[j];
                __m256i a = _mm256_abs_epi8(t);
                __m256i re = _mm256_blendv_epi8(c2, c1, _mm256_cmpeq_epi8(a, min1));
                __m256i s = _mm256_xor_si256(sgn, _mm256_cmpgt_epi8(t, zero));
                /* s = 0xFF -> +re, else -re */
                __m256i out = _mm256_blendv_epi8(_mm256_sub_epi8(zero, re), re, s);
                msg[b + j] = out;
                app[cols[b + j]] = _mm256_adds_epi8(t, out);
            }
        }
    }
}

__attribute__((target("avx512bw"))) static inline __m512i scale_floor512(__m512i x, int num, int shift)
{
    __m512i lo = _mm512_unpacklo_epi8(x, _mm512_setzero_si512());
    __m512i hi = _mm512_unpackhi_epi8(x, _mm512_setzero_si512());
    __m512i k = _mm512_set1_epi16((short)num);
    lo = _mm512_srli_epi16(_mm512_mullo_epi16(lo, k), shift);
    hi = _mm512_srli_epi16(_mm512_mullo_epi16(hi, k), shift);
    return _mm512_packus_epi16(lo, hi);
}

/* decode_group with 64 frames per register (AVX-512BW) */
__attribute__((target("avx512bw"))) static void decode_group512(
    int n, int m, const int32_t* row_ptr, const int32_t* cols, const uint8_t* row_class,
    int kind, int iters, __m512i* app, __m512i* msg, __m512i* tv)
{
    const __m512i zero = _mm512_setzero_si512();
    const __m512i one = _mm512_set1_epi8(1);
    const __m512i c31 = _mm512_set1_epi8(31);
    const __m512i c127 = _mm512_set1_epi8(127);
    (void)n;
    for (int it = 0; it < iters; it++) {
        for (int r = 0; r < m; r++) {
            int b = row_ptr[r], d = row_ptr[r + 1] - b;
            __m512i min1 = c127, min2 = c127;
            __mmask64 sgn = 0;
            for (int j = 0; j < d; j++) {
                __m512i a_v = app[cols[b + j]];
                __m512i t = (it == 0) ? a_v : _mm512_subs_epi8(a_v, msg[b + j]);
                __m512i a = _mm512_abs_epi8(t);
                tv[j] = t;
                min2 = _mm512_min_epu8(min2, _mm512_max_epu8(a, min1));
                min1 = _mm512_min_epu8(min1, a);
                sgn ^= _mm512_cmpgt_epi8_mask(t, zero);
            }
            __m512i c1, c2;
            int cls = row_class ? row_class[r] : 0;
            if (kind == K_MS) {
                c1 = _mm512_min_epu8(min2, c31);
                c2 = _mm512_min_epu8(min1, c31);
            } else if (kind == K_NMS) {
                c1 = scale_floor512(min2, 3, 2);
                c2 = scale_floor512(min1, 3, 2);
            } else {
                c1 = _mm512_subs_epu8(min2, one);
                c2 = _mm512_subs_epu8(min1, one);
                if (!(kind == K_OMS && it == 0 && cls == 1)) {
                    c1 = _mm512_min_epu8(c1, c31);
                    c2 = _mm512_min_epu8(c2, c31);
                }
            }
            for (int j = 0; j < d; j++) {
                __m512i t = tv[j];
                __m512i a = _mm512_abs_epi8(t);
                __m512i re = _mm512_mask_blend_epi8(_mm512_cmpeq_epi8_mask(a, min1), c2, c1);
                __mmask64 s = sgn ^ _mm512_cmpgt_epi8_mask(t, zero);
                /* s set -> +re, else -re */
                __m512i out = _mm512_mask_blend_epi8(s, _mm512_sub_epi8(zero, re), re);
                msg[b + j] = out;
                app[cols[b + j]] = _mm512_adds_epi8(t, out);
            }
        }
    }
}

int oracle_batch_supported(void)
{
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx2") ? 1 : 0;
}

/* 2: AVX-512BW (64 frames per group), 1: AVX2 (32 frames per group), 0: neither */
int oracle_batch_isa(void)
{
    __builtin_cpu_init();
    if (__builtin_cpu_supports("avx512bw")) return 2;
    return __builtin_cpu_supports("avx2") ? 1 : 0;
}

static int g_force_avx2 = 0;

/* forces the AVX2 path (1) or lets the CPU's best run (0); for tests of both paths */
void oracle_batch_force_avx2(int on) { g_force_avx2 = on; }

/*
 * nframes must be a multiple of 32.  llr: frame-major [nframes][n] (or the
 * word-interleaved reading of the buffer when interleaved != 0, as xMS);
 * hard: frame-major 0/1 [nframes][n].  Returns 0, or -1 when not supported.
 */
int oracle_decode_batch(int n, int m, const int32_t* row_ptr, const int32_t* cols,
                        const uint8_t* row_class, int kind, int iters, int nframes,
                        int interleaved, const int8_t* llr, uint8_t* hard, int nthreads)
{
    if (!oracle_batch_supported() || kind == K_2NMS || nframes % LANES || iters < 1) return -1;
    int W = nframes / 4;
    int e_total = row_ptr[m], dmax = 1;
    for (int r = 0; r < m; r++)
        if (row_ptr[r + 1] - row_ptr[r] > dmax) dmax = row_ptr[r + 1] - row_ptr[r];
    /* 64-frame groups with AVX-512BW, then the remaining 32 frames (if any) with AVX2 */
    const int wide = !g_force_avx2 && oracle_batch_isa() == 2;
    int groups512 = wide ? nframes / 64 : 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int g = 0; g < groups512; g++) {
        __m512i* app = (__m512i*)aligned_alloc(64, sizeof(__m512i) * (size_t)n);
        __m512i* msg = (__m512i*)aligned_alloc(64, sizeof(__m512i) * (size_t)e_total);
        __m512i* tv = (__m512i*)aligned_alloc(64, sizeof(__m512i) * (size_t)dmax);
        memset(msg, 0, sizeof(__m512i) * (size_t)e_total);
        int8_t* A = (int8_t*)app;
        for (int l = 0; l < 64; l++) {
            int f = g * 64 + l;
            for (int v = 0; v < n; v++)
                A[(size_t)v * 64 + l] = interleaved ? llr[((size_t)v * W + f / 4) * 4 + (f & 3)]
                                                    : llr[(size_t)f * n + v];
        }
        decode_group512(n, m, row_ptr, cols, row_class, kind, iters, app, msg, tv);
        for (int l = 0; l < 64; l++) {
            int f = g * 64 + l;
            for (int v = 0; v < n; v++) hard[(size_t)f * n + v] = A[(size_t)v * 64 + l] > 0;
        }
        free(app);
        free(msg);
        free(tv);
    }
    const int first = groups512 * 64 / LANES, groups = nframes / LANES;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int g = first; g < groups; g++) {
        __m256i* app = (__m256i*)aligned_alloc(32, sizeof(__m256i) * (size_t)n);
        __m256i* msg = (__m256i*)aligned_alloc(32, sizeof(__m256i) * (size_t)e_total);
        __m256i* tv = (__m256i*)aligned_alloc(32, sizeof(__m256i) * (size_t)dmax);
        memset(msg, 0, sizeof(__m256i) * (size_t)e_total);
        int8_t* A = (int8_t*)app;
        for (int l = 0; l < LANES; l++) {
            int f = g * LANES + l;
            for (int v = 0; v < n; v++)
                A[(size_t)v * LANES + l] = interleaved
                    ? llr[((size_t)v * W + f / 4) * 4 + (f & 3)]
                    : llr[(size_t)f * n + v];
        }
        decode_group(n, m, row_ptr, cols, row_class, kind, iters, app, msg, tv);
        for (int l = 0; l < LANES; l++) {
            int f = g * LANES + l;
            for (int v = 0; v < n; v++) hard[(size_t)f * n + v] = A[(size_t)v * LANES + l] > 0;
        }
        free(app);
        free(msg);
        free(tv);
    }
    return 0;
}
