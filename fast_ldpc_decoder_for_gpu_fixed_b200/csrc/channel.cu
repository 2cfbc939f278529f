// AWGN channel and error counting on the GPU: the stages either side of the
// decoder in the reference's simulation loop (src/main.cpp:258-294).
//
// Channel (replaces awgn_channel/CChanel_AWGN_SIMD.cu, which draws cuRAND
// XORWOW uniforms and quantises them in GenerateNoiseAndTransform, :7-30):
//   * uniforms from a counter-based Philox4x32-10 generator (Salmon, Moraes,
//     Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), so any
//     frame of any batch can be regenerated from (seed, sample index) alone;
//   * Box-Muller pairs n = sqrt(-2 ln u1) * (cos, sin)(2 pi u2);
//   * BPSK y = (2b - 1) + sigma * n for codeword bit b (b = 0: y = -1 + sigma n,
//     the reference's all-zero transmission, CChanel_AWGN_SIMD.cu:21-22);
//   * the reference quantiser q = (char) clamp(8y, -31, 31) (truncation toward
//     zero, CChanel_AWGN_SIMD.cu:23-24), written frame-major as int8.
// Error counting (replaces ber_analyzer/CErrorAnalyzer.cpp:142-158, a CPU loop):
//   per frame, the number of decided bits among the first n_vars that differ
//   from the transmitted codeword (all-zero when none is given); counts[0..2]
//   accumulate frames, bit errors and frame errors.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ldpc_b200.h"
#include "channel.cuh"

namespace ldpc {

// one thread = 4 consecutive samples of the flattened [frames][n] array
__global__ void awgn_kernel(int8_t* out, uint64_t total, int n, float sigma, uint64_t seed, uint64_t offset,
                            const uint8_t* cw, uint64_t n_cw)
{
    uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t s0 = 4 * q;
    if (s0 >= total) return;
    float u[4], g[4];
    uniforms4(q, seed, offset, u);
    box_muller4(u, g);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        uint64_t s = s0 + i;
        if (s >= total) break;
        float mean = -1.0f;
        if (cw) {
            uint64_t f = s / (uint64_t)n, v = s - f * (uint64_t)n;
            mean = cw[(f % n_cw) * (uint64_t)n + v] ? 1.0f : -1.0f;
        }
        out[s] = quantise(mean + sigma * g[i]);
    }
}

__global__ void philox_kernel(uint32_t* out, uint64_t count, uint64_t seed, uint64_t offset)
{
    uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (4 * q >= count) return;
    uint32_t c[4] = {(uint32_t)q, (uint32_t)(q >> 32), (uint32_t)offset, (uint32_t)(offset >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    for (int i = 0; i < 4 && 4 * q + i < count; i++) out[4 * q + i] = c[i];
}

// one CTA per frame
__global__ void count_errors_kernel(const uint8_t* hard, int n, int n_vars, const uint8_t* cw, uint64_t n_cw,
                                    unsigned long long* counts)
{
    const uint64_t f = blockIdx.x;
    const uint8_t* h = hard + f * (uint64_t)n;
    const uint8_t* c = cw ? cw + (f % n_cw) * (uint64_t)n : nullptr;
    int e = 0;
    for (int i = threadIdx.x; i < n_vars; i += blockDim.x) e += (h[i] != 0) != (c ? (c[i] != 0) : false);
#pragma unroll
    for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    __shared__ int part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) tot += part[w];
        atomicAdd(counts + 0, 1ull);
        atomicAdd(counts + 1, (unsigned long long)tot);
        atomicAdd(counts + 2, tot ? 1ull : 0ull);
    }
}

}  // namespace ldpc

using namespace ldpc;

int ldpc_internal_fail(int code, const char* msg);

extern "C" int ldpc_channel_awgn(int8_t* d_llr, size_t frames, int n, float sigma, uint64_t seed, uint64_t offset,
                                 const uint8_t* d_codewords, size_t n_codewords, void* stream)
{
    if (!d_llr || n <= 0 || sigma < 0 || (d_codewords && n_codewords == 0))
        return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_channel_awgn: bad argument");
    uint64_t total = (uint64_t)frames * n;
    if (total == 0) return LDPC_OK;
    uint64_t threads = (total + 3) / 4;
    awgn_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_llr, total, n, sigma, seed,
                                                                                    offset, d_codewords, n_codewords);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LDPC_OK : ldpc_internal_fail(LDPC_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" int ldpc_philox(uint32_t* d_out, size_t count, uint64_t seed, uint64_t offset, void* stream)
{
    if (!d_out) return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_philox: null pointer");
    if (!count) return LDPC_OK;
    uint64_t threads = (count + 3) / 4;
    philox_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_out, count, seed, offset);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LDPC_OK : ldpc_internal_fail(LDPC_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" int ldpc_count_errors(const uint8_t* d_hard, size_t frames, int n, int n_vars, const uint8_t* d_codewords,
                                 size_t n_codewords, int64_t* d_counts, void* stream)
{
    if (!d_hard || !d_counts || n <= 0 || n_vars < 0 || n_vars > n || (d_codewords && n_codewords == 0))
        return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_count_errors: bad argument");
    if (!frames) return LDPC_OK;
    count_errors_kernel<<<(unsigned)frames, 256, 0, (cudaStream_t)stream>>>(
        d_hard, n, n_vars, d_codewords, n_codewords, reinterpret_cast<unsigned long long*>(d_counts));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LDPC_OK : ldpc_internal_fail(LDPC_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" double ldpc_sigma(double ebn0, double rate, int es_n0)
{
    // CChanel_AWGN_SIMD::configure (awgn_channel/CChanel_AWGN_SIMD.cu:63-73)
    double eb = es_n0 ? ebn0 - 10.0 * log10(2 * rate) : ebn0;
    double interm = -0.1 * (eb + 10.0 * log10(rate));
    return sqrt(pow(10.0, interm) / 2);
}
