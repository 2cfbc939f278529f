// Training of the LDPC_LEARNED constants: FP32 forward and backward passes
// through the unrolled row-layered min-sum decoder, one CTA per frame.
//
// Forward model, per frame, iterations t = 0..T-1, rows in the decoder's level
// order, g = the row's class (degree group), j over the row's d edges, v_j its
// variables (the int8 decoders' semantics, with real-valued constants):
//   t_j   = clamp(a[v_j] - m_j, -128, 127)               (m_j = this edge's last message, 0 at t = 0)
//   u_j   = [t_j > 0]   (bit 1),  P = xor_j u_j
//   mag_j = min(|t_j|, 127);  min1 = mag_i1 <= min2 = mag_i2 <= the others
//   y(x)  = alpha[t][g] * x - beta[t][g]    or, with `quantized`, floor(alpha * x) - beta
//   c(x)  = clamp(y(x), 0, 31)
//   m_j   = (P ^ u_j ? +1 : -1) * (j == i1 ? c(min2) : c(min1))
//   a[v_j] = clamp(t_j + m_j, -128, 127)
// a starts as the channel LLRs in the int8 decoders' units.  With integer LLRs,
// alpha = s / 128 and integer beta, the quantized forward pass is exactly the
// LDPC_LEARNED int8 decoder (offsets beta, Q1.7 scales s): every value is an
// integer below 2^24, so FP32 holds it exactly.  Every forward operation is one
// IEEE FP32 operation rounded to nearest (no contraction into FMA), so a float32
// emulation reproduces the forward pass bit for bit.
//
// Loss, with w[t] the weight of iteration t (default: the last iteration only),
// a(t) the APP after iteration t, b the transmitted bits (a positive LLR means
// bit 1), kappa_f the frame's factor from the decoder's LLR units to natural
// log-likelihood ratios and S_f(t) = sum_v BCE(sigmoid(kappa_f a_v(t)), b_v):
//   bit loss   (LDPC_TRAIN_BIT_LOSS):   sum_t w[t] * mean_f S_f(t) / n
//   frame loss (LDPC_TRAIN_FRAME_LOSS): sum_t w[t] * mean_f (1 - exp(-S_f(t)))
// exp(-S_f) is the probability, under the soft output, that every bit of the
// frame is right, so the frame loss is a soft frame error rate.
//
// Backward: the reverse row sequence (levels in reverse order, the rows of a
// level in parallel, as in the forward pass).  Gradients are straight-through
// for min and sign (the argmins and signs found in the forward pass are held
// fixed), for the two saturations and for the floor; c's clamp passes the
// gradient only where 0 < y < 31.  The forward pass records {min1, min2,
// i1 | i2 << 8, sign bits} per row and iteration (16 bytes), and for weighted
// iterations before the last the APP (4 bytes per variable) and S_f(t), in a
// caller-provided stash.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ldpc_b200.h"
#include "decode_kernel.cuh"

namespace ldpc {

struct TrainArgs {
    const float* llr;      // [frames][n]
    const uint8_t* bits;   // [frames][n] transmitted bits, or null for the all-zero codeword
    const float* kappa;    // [frames]
    const float* alpha;    // [T][2]
    const float* beta;     // [T][2]
    float* grad_alpha;     // [T][2] accumulated
    float* grad_beta;      // [T][2] accumulated
    float* loss;           // [1] accumulated
    uint4* stash;          // [frames][T][m]
    float* stash_app;      // [frames][T][n]
    float* stash_s;        // [frames][T]
    const float* weights;  // [T] loss weight per iteration, or null (last only)
    float* app_out;        // [frames][n] final soft output, or null
    int T;
    int quantized;
    int frame_loss;
    int backward;
    float inv_frames;      // 1 / frames
    float inv_n;           // 1 / n
};

__device__ __forceinline__ float warp_sum(float x)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// sum over the CTA (blockDim.x a multiple of 32, at most 256), returned to every thread
__device__ __forceinline__ float block_sum(float x, float* scratch)
{
    x = warp_sum(x);
    __syncthreads();  // scratch may still be read from a previous call
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = x;
    __syncthreads();
    float s = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += scratch[w];
    return s;
}

__device__ __forceinline__ float pre_mag(float al, float be, float x, int quantized)
{
    const float p = __fmul_rn(al, x);
    return __fsub_rn(quantized ? floorf(p) : p, be);
}

// BCE(sigmoid(z), b) = softplus(z) - b z, and its derivative sigmoid(z) - b
__device__ __forceinline__ float bce(float z, float b) { return fmaxf(z, 0.f) + log1pf(expf(-fabsf(z))) - b * z; }
__device__ __forceinline__ float bce_grad(float z, float b) { return 1.f / (1.f + expf(-z)) - b; }

__device__ __forceinline__ float iter_weight(const TrainArgs& A, int t)
{
    return A.weights ? A.weights[t] : (t == A.T - 1 ? 1.f : 0.f);
}

// the loss term of iteration t for this frame from S = S_f(t), and the factor
// that multiplies kappa * (sigmoid - b) in its gradient
__device__ __forceinline__ float term_loss(const TrainArgs& A, float w, float S)
{
    return A.frame_loss ? w * (1.f - expf(-S)) * A.inv_frames : w * S * A.inv_n * A.inv_frames;
}
__device__ __forceinline__ float term_grad(const TrainArgs& A, float w, float S)
{
    return A.frame_loss ? w * expf(-S) * A.inv_frames : w * A.inv_n * A.inv_frames;
}

__global__ void __launch_bounds__(256) train_kernel(const Plan P, const TrainArgs A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* a = reinterpret_cast<float*>(smem_raw);    // APP, then its gradient
    float* msg = a + P.npad;                          // messages [dmax][m], then their gradients
    __shared__ float gpar[4 * LDPC_LEARNED_MAX_ITERS];  // [t][g][d alpha, d beta]
    __shared__ float scratch[8];
    const long long f = blockIdx.x;
    const int T = A.T;

    for (int i = threadIdx.x; i < 4 * LDPC_LEARNED_MAX_ITERS; i += blockDim.x) gpar[i] = 0.f;
    for (int v = threadIdx.x; v < P.n; v += blockDim.x) a[v] = A.llr[f * P.n + v];
    for (int i = threadIdx.x; i < P.dmax * P.m; i += blockDim.x) msg[i] = 0.f;
    __syncthreads();

    const float kap = A.kappa[f];
    float floss = 0.f;  // this frame's loss (thread 0)
    auto bit = [&](int v) { return A.bits ? (float)A.bits[f * P.n + v] : 0.f; };

    // ---------------- forward ----------------
    for (int t = 0; t < T; t++) {
        for (int l = 0; l < P.nlevels; l++) {
            const int2 lv = __ldg(P.levels + l);
            for (int r = lv.x + threadIdx.x; r < lv.x + lv.y; r += blockDim.x) {
                const int d = __ldg(P.rowdeg + r), g = __ldg(P.rowcls + r);
                const float al = A.alpha[2 * t + g], be = A.beta[2 * t + g];
                float tv[32];
                float m1 = 127.f, m2 = 127.f;
                int i1 = 0, i2 = 1;
                uint32_t pos = 0;
                for (int j = 0; j < d; j++) {
                    const int v = __ldg(P.cols + j * P.m + r);
                    const float x = fminf(fmaxf(__fsub_rn(a[v], msg[j * P.m + r]), -128.f), 127.f);
                    tv[j] = x;
                    const float ax = fminf(fabsf(x), 127.f);
                    pos |= (x > 0.f ? 1u : 0u) << j;
                    if (ax < m1) {
                        m2 = m1; i2 = i1; m1 = ax; i1 = j;
                    } else if (ax < m2) {
                        m2 = ax; i2 = j;
                    }
                }
                if (i2 == i1) i2 = (i1 + 1) % d;  // all magnitudes 127: any second edge
                const uint32_t par = __popc(pos) & 1;
                const float c1 = fminf(fmaxf(pre_mag(al, be, m2, A.quantized), 0.f), 31.f);
                const float c2 = fminf(fmaxf(pre_mag(al, be, m1, A.quantized), 0.f), 31.f);
                for (int j = 0; j < d; j++) {
                    const int v = __ldg(P.cols + j * P.m + r);
                    const float c = j == i1 ? c1 : c2;
                    const float mj = (par ^ ((pos >> j) & 1)) ? c : -c;
                    msg[j * P.m + r] = mj;
                    a[v] = fminf(fmaxf(__fadd_rn(tv[j], mj), -128.f), 127.f);
                }
                if (A.backward)
                    A.stash[((size_t)f * T + t) * P.m + r] =
                        make_uint4(__float_as_uint(m1), __float_as_uint(m2), (uint32_t)(i1 | (i2 << 8)), pos);
            }
            __syncthreads();
        }
        // intermediate loss terms: their APPs and S_f(t) are kept for the backward pass
        const float w = iter_weight(A, t);
        if (t < T - 1 && w != 0.f) {
            float part = 0.f;
            for (int v = threadIdx.x; v < P.n; v += blockDim.x) {
                part += bce(kap * a[v], bit(v));
                if (A.backward) A.stash_app[((size_t)f * T + t) * P.n + v] = a[v];
            }
            const float S = block_sum(part, scratch);  // also orders the reads of a before iteration t+1
            floss += term_loss(A, w, S);
            if (A.backward && threadIdx.x == 0) A.stash_s[(size_t)f * T + t] = S;
        }
    }

    // ---------------- final loss term and its gradient ----------------
    {
        float part = 0.f;
        for (int v = threadIdx.x; v < P.n; v += blockDim.x) {
            if (A.app_out) A.app_out[f * P.n + v] = a[v];
            part += bce(kap * a[v], bit(v));
        }
        const float w = iter_weight(A, T - 1);
        const float S = block_sum(part, scratch);
        floss += term_loss(A, w, S);
        const float coef = term_grad(A, w, S);
        for (int v = threadIdx.x; v < P.n; v += blockDim.x) a[v] = coef * kap * bce_grad(kap * a[v], bit(v));
        for (int i = threadIdx.x; i < P.dmax * P.m; i += blockDim.x) msg[i] = 0.f;
        if (threadIdx.x == 0) atomicAdd(A.loss, floss);
        __syncthreads();
    }
    if (!A.backward) return;

    // ---------------- backward ----------------
    for (int t = T - 1; t >= 0; t--) {
        float ga[2] = {0.f, 0.f}, gb[2] = {0.f, 0.f};
        const float w = iter_weight(A, t);
        if (t < T - 1 && w != 0.f) {  // the loss term on the APP after iteration t
            const float* keep = A.stash_app + ((size_t)f * T + t) * P.n;
            const float coef = term_grad(A, w, A.stash_s[(size_t)f * T + t]);
            for (int v = threadIdx.x; v < P.n; v += blockDim.x) a[v] += coef * kap * bce_grad(kap * keep[v], bit(v));
            __syncthreads();
        }
        for (int l = P.nlevels - 1; l >= 0; l--) {
            const int2 lv = __ldg(P.levels + l);
            for (int r = lv.x + threadIdx.x; r < lv.x + lv.y; r += blockDim.x) {
                const int d = __ldg(P.rowdeg + r), g = __ldg(P.rowcls + r);
                const float al = A.alpha[2 * t + g], be = A.beta[2 * t + g];
                const uint4 st = A.stash[((size_t)f * T + t) * P.m + r];
                const float m1 = __uint_as_float(st.x), m2 = __uint_as_float(st.y);
                const int i1 = st.z & 0xff, i2 = (st.z >> 8) & 0xff;
                const uint32_t pos = st.w, par = __popc(pos) & 1;
                float gt[32];
                float gc1 = 0.f, gc2 = 0.f;
                for (int j = 0; j < d; j++) {
                    const int v = __ldg(P.cols + j * P.m + r);
                    const float gav = a[v];                    // d/d a[v] after this row
                    const float gm = gav + msg[j * P.m + r];   // d/d m_j: the APP and the next iteration
                    gt[j] = gav;
                    const float s = (par ^ ((pos >> j) & 1)) ? gm : -gm;
                    if (j == i1) gc1 += s; else gc2 += s;
                }
                float gm1 = 0.f, gm2 = 0.f;
                const float y1 = pre_mag(al, be, m2, A.quantized), y2 = pre_mag(al, be, m1, A.quantized);
                if (y1 > 0.f && y1 < 31.f) {
                    ga[g] += m2 * gc1;
                    gb[g] -= gc1;
                    gm2 = al * gc1;
                }
                if (y2 > 0.f && y2 < 31.f) {
                    ga[g] += m1 * gc2;
                    gb[g] -= gc2;
                    gm1 = al * gc2;
                }
                // min1 = |t_i1|, min2 = |t_i2|; d|t|/dt = +1 for t > 0, -1 otherwise
                gt[i1] += ((pos >> i1) & 1) ? gm1 : -gm1;
                gt[i2] += ((pos >> i2) & 1) ? gm2 : -gm2;
                for (int j = 0; j < d; j++) {
                    const int v = __ldg(P.cols + j * P.m + r);
                    a[v] = gt[j];                // d/d a[v] before this row
                    msg[j * P.m + r] = -gt[j];   // d/d (this edge's message of iteration t-1)
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int g = 0; g < 2; g++) {
            const float x = warp_sum(ga[g]), y = warp_sum(gb[g]);
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(&gpar[(2 * t + g) * 2 + 0], x);
                atomicAdd(&gpar[(2 * t + g) * 2 + 1], y);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * T; i += blockDim.x) {
        atomicAdd(A.grad_alpha + i, gpar[2 * i + 0]);
        atomicAdd(A.grad_beta + i, gpar[2 * i + 1]);
    }
}

}  // namespace ldpc

using namespace ldpc;

int ldpc_internal_fail(int code, const char* msg);
int ldpc_internal_plan(const ldpc_decoder* dec, Plan* plan, int* threads);
cudaError_t ldpc_internal_raise_smem(const void* fn, size_t bytes);

static size_t stash_rows(const Plan& P, size_t frames, int iters) { return frames * (size_t)iters * P.m * sizeof(uint4); }
static size_t stash_apps(const Plan& P, size_t frames, int iters) { return frames * (size_t)iters * P.n * sizeof(float); }

extern "C" size_t ldpc_train_stash_bytes(const ldpc_decoder* dec, size_t frames, int iters)
{
    Plan P;
    int threads = 0;
    if (!dec || iters < 1 || ldpc_internal_plan(dec, &P, &threads)) return 0;
    return stash_rows(P, frames, iters) + stash_apps(P, frames, iters) + frames * (size_t)iters * sizeof(float);
}

extern "C" int ldpc_train_step(const ldpc_decoder* dec, const float* d_llr, const uint8_t* d_bits,
                               const float* d_kappa, size_t frames, int iters, int flags,
                               const float* d_alpha, const float* d_beta, const float* d_weights,
                               float* d_grad_alpha, float* d_grad_beta, float* d_loss, void* d_stash,
                               float* d_app_out, void* stream)
{
    if (!dec || !d_llr || !d_kappa || !d_alpha || !d_beta || !d_loss)
        return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_train_step: null pointer");
    if (flags & ~(LDPC_TRAIN_QUANTIZED | LDPC_TRAIN_FRAME_LOSS))
        return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_train_step: unknown flags");
    const bool backward = d_grad_alpha || d_grad_beta || d_stash;
    if (backward && !(d_grad_alpha && d_grad_beta && d_stash))
        return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_train_step: gradients need grad_alpha, grad_beta and stash");
    if (iters < 1 || iters > LDPC_LEARNED_MAX_ITERS)
        return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_train_step: iterations must be in [1, 32]");
    if (frames < 1 || frames > 0x7fffffffu) return ldpc_internal_fail(LDPC_ERR_SHAPE, "ldpc_train_step: frames");
    Plan P;
    int threads = 0;
    if (ldpc_internal_plan(dec, &P, &threads))
        return ldpc_internal_fail(LDPC_ERR_ARG, "ldpc_train_step: decoder has no row schedule");
    if (P.dmax > 32 || P.dmax < 2)
        return ldpc_internal_fail(LDPC_ERR_UNSUPPORTED, "ldpc_train_step: row degrees must be in [2, 32]");
    const size_t smem = 4 * ((size_t)P.npad + (size_t)P.dmax * P.m);
    int dev = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem + 16 * LDPC_LEARNED_MAX_ITERS + 64 > (size_t)smem_max)
        return ldpc_internal_fail(LDPC_ERR_UNSUPPORTED,
                                  "ldpc_train_step: one frame's FP32 state does not fit in shared memory");
    TrainArgs A;
    A.llr = d_llr;
    A.bits = d_bits;
    A.kappa = d_kappa;
    A.alpha = d_alpha;
    A.beta = d_beta;
    A.grad_alpha = d_grad_alpha;
    A.grad_beta = d_grad_beta;
    A.loss = d_loss;
    char* sb = reinterpret_cast<char*>(d_stash);
    A.stash = reinterpret_cast<uint4*>(sb);
    A.stash_app = sb ? reinterpret_cast<float*>(sb + stash_rows(P, frames, iters)) : nullptr;
    A.stash_s = sb ? reinterpret_cast<float*>(sb + stash_rows(P, frames, iters) + stash_apps(P, frames, iters))
                   : nullptr;
    A.weights = d_weights;
    A.app_out = d_app_out;
    A.T = iters;
    A.quantized = (flags & LDPC_TRAIN_QUANTIZED) ? 1 : 0;
    A.frame_loss = (flags & LDPC_TRAIN_FRAME_LOSS) ? 1 : 0;
    A.backward = backward ? 1 : 0;
    A.inv_frames = (float)(1.0 / (double)frames);
    A.inv_n = (float)(1.0 / (double)P.n);
    cudaError_t e = ldpc_internal_raise_smem((const void*)train_kernel, smem);
    if (e == cudaSuccess) {
        train_kernel<<<(unsigned)frames, threads, smem, (cudaStream_t)stream>>>(P, A);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? LDPC_OK : ldpc_internal_fail(LDPC_ERR_CUDA, cudaGetErrorString(e));
}
