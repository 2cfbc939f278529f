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
 * 32-frame groups over the host threads.
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

int oracle_batch_supported(void)
{
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx2") ? 1 : 0;
}

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
    int groups = nframes / LANES, W = nframes / 4;
    int e_total = row_ptr[m], dmax = 1;
    for (int r = 0; r < m; r++)
        if (row_ptr[r + 1] - row_ptr[r] > dmax) dmax = row_ptr[r + 1] - row_ptr[r];
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int g = 0; g < groups; g++) {
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
