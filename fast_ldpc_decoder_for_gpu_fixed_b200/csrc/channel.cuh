// Device helpers of the AWGN channel (Philox4x32-10 uniforms, Box-Muller,
// the reference quantiser), shared by the stand-alone channel kernel and the
// decoder prologue that generates its own LLRs.  See channel.cu.
#pragma once
#include <cstdint>

namespace ldpc {

__host__ __device__ inline void philox_round(uint32_t (&c)[4], const uint32_t (&k)[2])
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k[0], n2 = hi0 ^ c[3] ^ k[1];
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

// Philox4x32 with 10 rounds; counter (c0..c3), key (k0, k1)
__host__ __device__ inline void philox4x32_10(uint32_t (&c)[4], uint32_t k0, uint32_t k1)
{
    uint32_t k[2] = {k0, k1};
#pragma unroll
    for (int r = 0; r < 10; r++) {
        philox_round(c, k);
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
}

// 4 uniforms in (0, 1) for the 4 consecutive samples 4q..4q+3 of stream (seed, offset)
__device__ __forceinline__ void uniforms4(uint64_t q, uint64_t seed, uint64_t offset, float (&u)[4])
{
    uint32_t c[4] = {(uint32_t)q, (uint32_t)(q >> 32), (uint32_t)offset, (uint32_t)(offset >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
    for (int i = 0; i < 4; i++) u[i] = ((float)c[i] + 0.5f) * 2.3283064365386963e-10f;  // (x + 1/2) / 2^32
}

__device__ __forceinline__ int8_t quantise(float y)
{
    return (int8_t)truncf(fminf(fmaxf(8.0f * y, -31.0f), 31.0f));
}

// Box-Muller: (u0, u1) -> (r cos, r sin), (u2, u3) -> (r cos, r sin)
__device__ __forceinline__ void box_muller4(const float (&u)[4], float (&g)[4])
{
#pragma unroll
    for (int p = 0; p < 2; p++) {
        float r = sqrtf(-2.0f * logf(u[2 * p]));
        float sn, cs;
        sincospif(2.0f * u[2 * p + 1], &sn, &cs);
        g[2 * p] = r * cs;
        g[2 * p + 1] = r * sn;
    }
}

// LLR of sample s (frame-major index frame * n + v): its Box-Muller pair comes from
// the 4 uniforms of Philox counter s / 4, exactly as the stand-alone channel kernel
__device__ __forceinline__ int8_t awgn_sample(unsigned long long s, unsigned long long seed, unsigned long long offset,
                                              float sigma, float mean)
{
    float u[4];
    uniforms4(s >> 2, seed, offset, u);
    const int i = (int)(s & 3), p = i >> 1;
    float r = sqrtf(-2.0f * logf(u[2 * p]));
    float sn, cs;
    sincospif(2.0f * u[2 * p + 1], &sn, &cs);
    float gss = (i & 1) ? r * sn : r * cs;
    return quantise(mean + sigma * gss);
}

}  // namespace ldpc
