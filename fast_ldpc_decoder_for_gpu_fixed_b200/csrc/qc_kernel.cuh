// Layered decoder for quasi-cyclic codes with every c->v message in registers.
//
// A QC code is a base matrix of L block rows ("layers") whose nonzero entries
// are Z x Z circulant permutations: row k of layer l connects variable
// c*Z + (k + s) mod Z for every nonzero (c, s) of the layer.  The Z rows of a
// layer touch disjoint variables, so the reference's serial row order
// (decoder_oms/cuda/CUDA_OMS_SIMD.cu:138-246) is reproduced exactly by
// updating a whole layer at once and ordering the layers.
//
// Mapping: CTA = Z threads; thread k owns row k of every layer, so its L*D
// messages per pair-word never leave registers, and the APP (biased fp16 pairs)
// is the only shared-memory state.  One barrier per layer.  WPT = 2: the CTA holds
// the 4 frames of reference word g (two fp16x2 pair-words, 8 bytes per variable),
// so 2NMS early termination (per 32-bit word) is a __syncthreads_or.  WPT = 1:
// the CTA holds frames 2h, 2h+1 of word g (blockIdx.x = 2 * (g - word0) + h), 4
// bytes per variable and half the registers, for codes with many layers or
// high row degrees (24-column bases); its early stop is per frame pair.
#pragma once
#include "decode_kernel.cuh"

namespace ldpc {

constexpr int QC_MAX_LAYERS = 16;
constexpr int QC_MAX_DEG = 24;

struct QCParams {
    int z;                   // circulant size = threads per CTA
    int n;                   // variables = nb * z
    int layers;
    int zb;                  // bytes of one block column of the APP = vb * z (vb = 4 * WPT bytes per variable)
    int deg[QC_MAX_LAYERS];  // row degree of each layer
    int cls[QC_MAX_LAYERS];  // reference degree group of each layer (OMS quirk)
    // per (layer, edge): byte offset of the block column in the APP array and the shift
    int cz4[QC_MAX_LAYERS * QC_MAX_DEG];  // vb * c * z
    int s[QC_MAX_LAYERS * QC_MAX_DEG];    // vb * shift
};

// byte offset (vb bytes per variable) of the variable of edge `idx` of row k, from
// kb = vb * k: ((kb + vb*s) mod zb) + vb*c*z; for a power-of-two z the mod is a mask
// and the block offset an OR (its low bits are zero)
template <bool POW2>
__device__ __forceinline__ int qc_var_off(const QCParams& Q, int idx, int kb)
{
    int u = kb + Q.s[idx];
    if (POW2) return (u & (Q.zb - 1)) | Q.cz4[idx];
    u = min((unsigned)u, (unsigned)(u - Q.zb));
    return Q.cz4[idx] + u;
}

// hard-decision parity masks of one biased pair-word: bit 15 / 31 set iff that
// frame's decision is 0 (b >= 127.0; (b | 0x8000) - 0x57f0 has bit 15 set iff so)
__device__ __forceinline__ uint32_t qc_zero_bits(uint32_t b) { return ((b | 0x80008000u) - 0x57f057f0u) & 0x80008000u; }

// true when row k of some layer in [L0, L1) has odd hard-decision parity in one of
// the CTA's frames (see the early stop in decode_qc_kernel)
template <int DT, bool EXACT, int L0, int L1, bool POW2, int WPT>
__device__ __noinline__ bool qc_rows_unsatisfied(const QCParams& Q, const char* appb, int k)
{
    bool bad = false;
    const int kb = 4 * WPT * k;
#pragma unroll
    for (int l = L0; l < L1; l++) {
        const int d = EXACT ? DT : Q.deg[l];
        uint32_t acc0 = (d & 1) ? 0x80008000u : 0u, acc1 = acc0;
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                const int off = qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kb);
                if (WPT == 2) {
                    const uint2 v = *reinterpret_cast<const uint2*>(appb + off);
                    acc0 ^= qc_zero_bits(v.x);
                    acc1 ^= qc_zero_bits(v.y);
                } else {
                    acc0 ^= qc_zero_bits(*reinterpret_cast<const uint32_t*>(appb + off));
                }
            }
        }
        bad |= (WPT == 2 ? (acc0 | acc1) : acc0) != 0;
    }
    return bad;
}

// ET: the syndrome early stop compiled in (J.early is then always set); without
// it the extrinsic-parity count is dead code for every kind but 2NMS
template <int KIND, int DT, bool EXACT, int L, bool POW2, bool ET, int WPT>
__global__ void __launch_bounds__(256, WPT == 2 ? 2 : 1) decode_qc_kernel(const __grid_constant__ QCParams Q, const Job J)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint2* app = reinterpret_cast<uint2*>(smem_raw);     // WPT = 2: [n] (pair-word 0, pair-word 1)
    uint32_t* app1 = reinterpret_cast<uint32_t*>(smem_raw);  // WPT = 1: [n] pair-word of frames 2h, 2h+1
    char* appb = reinterpret_cast<char*>(smem_raw);
    uint16_t* slut = reinterpret_cast<uint16_t*>(smem_raw + (size_t)Q.n * 4 * WPT);  // KIND_LEARNED
    const long long g = J.word0 + (WPT == 2 ? blockIdx.x : blockIdx.x >> 1);
    const int h = WPT == 2 ? 0 : (blockIdx.x & 1);
    const int k = threadIdx.x;
    __shared__ unsigned s_odd[2];
    if (k < 2) s_odd[k] = 0;

    Plan P;  // only n is used by the shared prologue / epilogue helpers
    P.n = Q.n;
    read_group(P, J, g, [&](int v, uint32_t w) {
        if (WPT == 2)
            app[v] = make_uint2(Access<PackF16x2>::pair(w, 0), Access<PackF16x2>::pair(w, 2));
        else
            app1[v] = Access<PackF16x2>::pair(w, 2 * h);
    });
    __syncthreads();

    uint32_t msg[WPT][L][DT];
#pragma unroll
    for (int w = 0; w < WPT; w++)
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int j = 0; j < DT; j++) msg[w][l][j] = 0;

    int executed = 0;
    for (int it = 0; it < J.iters; it++) {
        uint32_t ov = 0;
        if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int d = EXACT ? DT : Q.deg[l];
            const bool noclip = J.quirk && it == 0 && Q.cls[l];
            // recompute the 2-instruction addresses each layer instead of pinning
            // L*D of them in registers across iterations (a shared-memory table of
            // them measured slower: the dependent load costs more than it saves)
            int kk = 4 * WPT * k;
            asm volatile("" : "+r"(kk));
            int off[DT];
            uint32_t b0[DT], b1[DT];
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    off[j] = qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kk);
                    if (WPT == 2) {
                        uint2 v = *reinterpret_cast<const uint2*>(appb + off[j]);
                        b0[j] = v.x;
                        b1[j] = v.y;
                    } else {
                        b0[j] = *reinterpret_cast<const uint32_t*>(appb + off[j]);
                    }
                }
            }
            uint32_t lk, lb;  // LEARNED constants of this layer's class (registers only within the layer)
            h2::learned_kb<KIND>(slut + 128 * Q.cls[l], lk, lb);
            h2::row<KIND, DT, EXACT>(b0, msg[0][l], d, noclip, ov, lk, lb);
            if (WPT == 2) h2::row<KIND, DT, EXACT>(b1, msg[WPT - 1][l], d, noclip, ov, lk, lb);
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    if (WPT == 2)
                        *reinterpret_cast<uint2*>(appb + off[j]) = make_uint2(b0[j], b1[j]);
                    else
                        *reinterpret_cast<uint32_t*>(appb + off[j]) = b0[j];
                }
            }
            // with the early stop, the barrier of the odd-row count closes the last layer
            if (!(ET && KIND != KIND_2NMS && l == L - 1)) __syncthreads();
        }
        executed = it + 1;
        if (KIND == KIND_2NMS && it >= 1) {
            if (!__syncthreads_or(ov != 0)) break;
        }
        // syndrome early stop (odd_rows_within_slack): thread k checks row k of
        // every layer.  For a biased APP b (x = 127 - b, an fp16 in [0, 255]),
        // ((b | 0x8000) - 0x57f0) has bit 15 set iff b >= 127.0, i.e. iff the
        // hard decision is 0; a row is satisfied when its count of 1s is even.
        if (KIND != KIND_2NMS && ET) {
            if (odd_rows_within_slack(J, ov, it, s_odd)) {
                // staged: the first layers alone reject most words that are not codewords yet
                constexpr int LS = L > 2 ? 2 : L;
                bool done = !__syncthreads_or(qc_rows_unsatisfied<DT, EXACT, 0, LS, POW2, WPT>(Q, appb, k));
                if (LS < L && done)
                    done = !__syncthreads_or(qc_rows_unsatisfied<DT, EXACT, LS, L, POW2, WPT>(Q, appb, k));
                if (done) break;
            }
        }
    }

    if (WPT == 1) {
        // frames 2h, 2h+1 only; the word's iteration count is the larger of its two pairs
        // (the host zeroes d_iters_out before the launch)
        write_group(P, J, g, [&](int v) { return AccessHalf::get(app1, v, h); }, 3 << (2 * h));
        if (J.iters_out && threadIdx.x == 0) atomicMax(J.iters_out + (g - J.word0), executed);
        return;
    }
    write_group(P, J, g, [&](int v) { uint2 a = app[v]; return Access<PackF16x2>::unbias(a.x, a.y); });
    if (J.iters_out && threadIdx.x == 0) J.iters_out[g - J.word0] = executed;
    if (J.app_out) {
        uint32_t* ao = reinterpret_cast<uint32_t*>(J.app_out);
        for (int v = threadIdx.x; v < Q.n; v += blockDim.x) {
            uint2 a = app[v];
            ao[(long long)v * J.total_words + g] = Access<PackF16x2>::unbias(a.x, a.y);
        }
    }
    if (J.msg_out) {
        // edge index in table order: rows are layer-major (row = l*z + k), each row's
        // edges in the order of the layer's entries; e = first edge of the layer + k*d + j
        uint32_t* mo = reinterpret_cast<uint32_t*>(J.msg_out);
        long long e0 = 0;
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int d = EXACT ? DT : Q.deg[l];
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    auto x = [](uint32_t h) { return (uint32_t)(uint8_t)(int8_t)(-__half2int_rn(__ushort_as_half((uint16_t)h))); };
                    uint32_t lo = msg[0][l][j], hi = msg[WPT - 1][l][j];
                    uint32_t wv = x(lo & 0xffff) | (x(lo >> 16) << 8) | (x(hi & 0xffff) << 16) | (x(hi >> 16) << 24);
                    mo[(e0 + (long long)k * d + j) * J.total_words + g] = wv;
                }
            }
            e0 += (long long)Q.z * d;
        }
    }
}

}  // namespace ldpc
