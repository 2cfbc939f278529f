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
constexpr int QC_LUT_ITS = 32;  // LDPC_LEARNED iteration rows (LDPC_LEARNED_MAX_ITERS)

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

// hard decisions of one biased pair-word as sign bits, one fp16 add for both frames on
// the FMA pipe: the integer b is below 127 (decision 1, x > 0) exactly when b - 126.5 is
// negative.  XORed over a row, bits 15 / 31 are the row's parity of 1s in each frame; the
// other bits are don't-care.
__device__ __forceinline__ uint32_t qc_one_signs(uint32_t b) { return h2::add(b, 0xd7e8d7e8u); }

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
        uint32_t acc0 = 0, acc1 = 0;
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                const int off = qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kb);
                if (WPT == 2) {
                    const uint2 v = *reinterpret_cast<const uint2*>(appb + off);
                    acc0 ^= qc_one_signs(v.x);
                    acc1 ^= qc_one_signs(v.y);
                } else {
                    acc0 ^= qc_one_signs(*reinterpret_cast<const uint32_t*>(appb + off));
                }
            }
        }
        bad |= ((WPT == 2 ? (acc0 | acc1) : acc0) & 0x80008000u) != 0;
    }
    return bad;
}

// bit i set when the CTA's frame i (lanes of the pair-words: WPT = 2: frames 0..3 of the
// word; WPT = 1: frames 2h, 2h + 1 in bits 0, 1) has a row of odd hard-decision parity
// among rows k of layers [L0, L1)
template <int DT, bool EXACT, int L0, int L1, bool POW2, int WPT>
__device__ __noinline__ unsigned qc_rows_unsat_mask(const QCParams& Q, const char* appb, int k)
{
    uint32_t bad0 = 0, bad1 = 0;
    const int kb = 4 * WPT * k;
#pragma unroll
    for (int l = L0; l < L1; l++) {
        const int d = EXACT ? DT : Q.deg[l];
        uint32_t acc0 = 0, acc1 = 0;
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                const int off = qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kb);
                if (WPT == 2) {
                    const uint2 v = *reinterpret_cast<const uint2*>(appb + off);
                    acc0 ^= qc_one_signs(v.x);
                    acc1 ^= qc_one_signs(v.y);
                } else {
                    acc0 ^= qc_one_signs(*reinterpret_cast<const uint32_t*>(appb + off));
                }
            }
        }
        bad0 |= acc0;
        if (WPT == 2) bad1 |= acc1;
    }
    bad0 &= 0x80008000u;
    bad1 &= 0x80008000u;
    return ((bad0 >> 15) & 1u) | ((bad0 >> 30) & 2u) | ((bad1 >> 13) & 4u) | ((bad1 >> 28) & 8u);
}

// ET: the syndrome early stop compiled in (J.early is then always set): 1 = the CTA's
// frames stop together, 2 (WPT = 2 only) = each frame pair (frames 0, 1 and 2, 3 of the
// word) stops on its own: a stopped pair's rows are no longer updated and its APP stays
// as it was, and the word reports the larger of its pairs' counts.  Without it the
// extrinsic-parity count is dead code for every kind but 2NMS.
// 3 = the CTA's frames stop together at the first iteration whose hard decisions are
// codewords (the rule of modes 1 and 2 with an unbounded slack, LDPC_EARLY_SLACK_ANY).
// No odd-row count: the rows of the last layer are checked from the registers that hold
// their freshly updated APP (no later layer of the iteration touches those variables, so
// their parity is final), reduced by the barrier that closes the layer; only when every
// one of them holds are the other layers' rows checked from shared memory.
template <int KIND, int DT, bool EXACT, int L, bool POW2, int ET, int WPT>
__global__ void __launch_bounds__(256, WPT == 2 ? 2 : 1) decode_qc_kernel(const __grid_constant__ QCParams Q, const Job J)
{
    static_assert(ET != 2 || WPT == 2, "per-pair early stop: 4 frames per CTA");
    static_assert(ET != 3 || KIND != KIND_2NMS, "2NMS has its own early termination");
    constexpr bool PAIRS = ET == 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint2* app = reinterpret_cast<uint2*>(smem_raw);     // WPT = 2: [n] (pair-word 0, pair-word 1)
    uint32_t* app1 = reinterpret_cast<uint32_t*>(smem_raw);  // WPT = 1: [n] pair-word of frames 2h, 2h+1
    char* appb = reinterpret_cast<char*>(smem_raw);
    const long long g = J.word0 + (WPT == 2 ? blockIdx.x : blockIdx.x >> 1);
    const int h = WPT == 2 ? 0 : (blockIdx.x & 1);
    const int k = threadIdx.x;
    __shared__ unsigned s_odd[2];
    // KIND_LEARNED: the (k, k) and (b, b) words of every iteration and row group, loaded
    // once (the head of each [iteration][group] table, see ldpc_decoder_set_learned), so
    // that no iteration waits on a global load and a barrier for its constants
    constexpr bool LRN = KIND == KIND_LEARNED || KIND == KIND_LEARNED_OFS;
    __shared__ uint2 s_kb[LRN ? QC_LUT_ITS : 1][2];
    if (k < 2) s_odd[k] = 0;
    if (LRN && k < 2 * J.lut_its) {
        uint2 kb = *reinterpret_cast<const uint2*>(J.lut + (k >> 1) * 256 + (k & 1) * 128);
        if (KIND == KIND_LEARNED_OFS) kb.y = h2::add(kb.y, 0x37803780u);  // b + 15/32 = -offset (scale 1)
        s_kb[k >> 1][k & 1] = kb;
    }
    // the odd-row count of the early stop: a +-1 accumulator on the FMA pipe (row(), CMODE 2);
    // 2NMS keeps the exact popcount, which its own rule tests against zero
    constexpr int CM = ((ET == 1 || ET == 2) && KIND != KIND_2NMS) ? 2 : 0;

    // The LLRs of the word that will take this CTA's place, about one wave of resident CTAs
    // (2 per SM) later, go into L2 by one TMA bulk prefetch, so that its prologue loads hit L2:
    // a CTA that stops early starts its successor sooner, and the prologue's HBM latency
    // would otherwise fall on every one of them.
    if (WPT == 2 && threadIdx.x == 0 && !J.gen && !J.interleaved && (Q.n & 3) == 0) {
        unsigned nsm;
        asm("mov.u32 %0, %%nsmid;" : "=r"(nsm));
        const long long gn = g + 2 * (long long)nsm;
        if (gn < J.word0 + (long long)gridDim.x) {
            const int8_t* src = J.llr + 4 * (gn - J.word0) * (long long)Q.n;
            if (((uintptr_t)src & 15) == 0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(4u * (unsigned)Q.n) : "memory");
        }
    }
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
    bool passed = false;  // stopped by the syndrome early stop: every check of every frame holds
    unsigned live = 3;    // PAIRS: bit p set while pair p is decoding (the same in every thread)
    for (int it = 0; it < J.iters; it++) {
        bool last_ok = false;  // ET 3: every row of the last layer holds in every frame
        uint32_t ov = 0, ov1 = 0;  // PAIRS: ov1 is pair 1's odd-row accumulator
        const int lt = LRN ? min(it, J.lut_its - 1) : 0;  // constants of this iteration
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
            uint32_t lk = 0, lb = 0;  // LEARNED constants of this layer's class (registers only within the layer)
            if (KIND == KIND_LEARNED || KIND == KIND_LEARNED_OFS) {
                const uint2 kb = s_kb[lt][Q.cls[l]];
                lk = kb.x;
                lb = kb.y;
            }
            // a stopped pair's words are stored back unchanged
            if (!PAIRS || (live & 1u)) h2::row<KIND, DT, EXACT, CM>(b0, msg[0][l], d, noclip, ov, lk, lb);
            if (WPT == 2 && (!PAIRS || (live & 2u)))
                h2::row<KIND, DT, EXACT, CM>(b1, msg[WPT - 1][l], d, noclip, PAIRS ? ov1 : ov, lk, lb);
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    if (WPT == 2)
                        *reinterpret_cast<uint2*>(appb + off[j]) = make_uint2(b0[j], b1[j]);
                    else
                        *reinterpret_cast<uint32_t*>(appb + off[j]) = b0[j];
                }
            }
            if (ET == 3 && l == L - 1) {
                // the parity of row k of the last layer in each frame, from the updated APP
                uint32_t p0 = 0, p1 = 0;
#pragma unroll
                for (int j = 0; j < DT; j++) {
                    if (EXACT || j < d) {
                        p0 ^= qc_one_signs(b0[j]);
                        if (WPT == 2) p1 ^= qc_one_signs(b1[j]);
                    }
                }
                last_ok = !__syncthreads_or(((p0 | p1) & 0x80008000u) != 0);
            } else if (!(ET && KIND != KIND_2NMS && l == L - 1)) {
                // with the early stop (modes 1, 2), the barrier of the odd-row count closes the last layer
                __syncthreads();
            }
        }
        executed = it + 1;
        if (KIND == KIND_2NMS && it >= 1) {
            if (!__syncthreads_or(ov != 0)) break;
        }
        // syndrome early stop (odd_rows_within_slack): thread k checks row k of
        // every layer.  For a biased APP b (x = 127 - b, an fp16 in [0, 255]),
        // b - 126.5 is negative iff the hard decision is 1 (qc_one_signs); a row is
        // satisfied when its count of 1s is even.
        if (KIND != KIND_2NMS && PAIRS) {
            // both pairs' counts in one word (each at most 2 * L * 256 < 2^16)
            const unsigned tot = odd_rows_total(h2::odd_count(ov, L) | (h2::odd_count(ov1, L) << 16), it, s_odd);
            unsigned gate = live & (((tot & 0xffffu) <= J.early_slack ? 1u : 0u) | ((tot >> 16) <= J.early_slack ? 2u : 0u));
            if (gate) {
                // staged as below; bit p of a thread's mask: pair p has an odd row among its rows k
                constexpr int LS = L > 2 ? 2 : L;
                unsigned m = qc_rows_unsat_mask<DT, EXACT, 0, LS, POW2, 2>(Q, appb, k);
                if ((gate & 1u) && __syncthreads_or(m & 3u)) gate &= ~1u;
                if ((gate & 2u) && __syncthreads_or(m & 12u)) gate &= ~2u;
                if (LS < L && gate) {
                    m = qc_rows_unsat_mask<DT, EXACT, LS, L, POW2, 2>(Q, appb, k);
                    if ((gate & 1u) && __syncthreads_or(m & 3u)) gate &= ~1u;
                    if ((gate & 2u) && __syncthreads_or(m & 12u)) gate &= ~2u;
                }
                live &= ~gate;  // the pairs whose frames are codewords stop here
                if (!live) {
                    passed = true;
                    break;
                }
            }
        } else if (ET == 3) {
            if (last_ok) {
                // staged like mode 1: the first layers alone reject most words that are not codewords yet
                constexpr int LS = L > 3 ? 2 : 1;
                bool done = true;
                if (L > 1) done = !__syncthreads_or(qc_rows_unsatisfied<DT, EXACT, 0, (L > 1 ? LS : 0), POW2, WPT>(Q, appb, k));
                if (LS < L - 1 && done)
                    done = !__syncthreads_or(qc_rows_unsatisfied<DT, EXACT, LS, (L > 1 ? L - 1 : 0), POW2, WPT>(Q, appb, k));
                if (done) {
                    passed = true;
                    break;
                }
            }
        } else if (KIND != KIND_2NMS && ET) {
            if (odd_rows_within_slack(J, h2::odd_count(ov, L * WPT), it, s_odd)) {
                // staged: the first layers alone reject most words that are not codewords yet
                constexpr int LS = L > 2 ? 2 : L;
                bool done = !__syncthreads_or(qc_rows_unsatisfied<DT, EXACT, 0, LS, POW2, WPT>(Q, appb, k));
                if (LS < L && done)
                    done = !__syncthreads_or(qc_rows_unsatisfied<DT, EXACT, LS, L, POW2, WPT>(Q, appb, k));
                if (done) {
                    passed = true;
                    break;
                }
            }
        }
    }

    if (WPT == 1) {
        // frames 2h, 2h+1 only; the word's iteration count is the larger of its two pairs
        // (the host zeroes d_iters_out before the launch)
        write_group(P, J, g, [&](int v) { return AccessHalf::get(app1, v, h); }, 3 << (2 * h));
        if (J.iters_out && threadIdx.x == 0) atomicMax(J.iters_out + (g - J.word0), executed);
        if (J.synd_out) {
            const unsigned bad = passed ? 0u : qc_rows_unsat_mask<DT, EXACT, 0, L, POW2, 1>(Q, appb, k);
            write_syndrome_flags(J, 4 * (g - J.word0) + 2 * h, bad, 3, true);
        }
        return;
    }
    write_group(P, J, g, [&](int v) { uint2 a = app[v]; return Access<PackF16x2>::unbias(a.x, a.y); });
    if (J.iters_out && threadIdx.x == 0) J.iters_out[g - J.word0] = executed;
    if (J.synd_out) {
        const unsigned bad = passed ? 0u : qc_rows_unsat_mask<DT, EXACT, 0, L, POW2, 2>(Q, appb, k);
        write_syndrome_flags(J, 4 * (g - J.word0), bad, 0xF, true);
    }
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

// ---- 2 frames per CTA with each check row split over SPLIT lanes (decoder path 7) ----
//
// The layout of the WPT = 1 kernel (CTA 2(g - word0) + h holds frames 2h, 2h + 1 of word g,
// one fp16x2 pair-word per variable), but row k of a layer belongs to the SPLIT lanes
// k*SPLIT .. k*SPLIT + SPLIT - 1 of the CTA: lane s takes the row's edges s, s + SPLIT, ...
// (DL = ceil(DT / SPLIT) of them, their messages in its registers), and the lanes merge their
// partial min1 / min2 / sign parity with warp shuffles (h2::row_split).  High-degree rows
// (the rate-3/4 and 5/6 bases reach 18 and 24) then cost DL serial steps instead of DT, a
// CTA has SPLIT times the threads, and each thread holds 1/SPLIT of the messages.  Every
// kind but 2NMS; the early stop is per frame pair, as on path 4.
template <int KIND, int DT, int L, int SPLIT, bool ET>
__global__ void __launch_bounds__(512) decode_qc_split_kernel(const __grid_constant__ QCParams Q, const Job J)
{
    constexpr int DL = (DT + SPLIT - 1) / SPLIT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* app1 = reinterpret_cast<uint32_t*>(smem_raw);  // [n] pair-word of frames 2h, 2h+1
    char* appb = reinterpret_cast<char*>(smem_raw);
    const long long g = J.word0 + (blockIdx.x >> 1);
    const int h = blockIdx.x & 1;
    const int k = threadIdx.x / SPLIT, s = threadIdx.x % SPLIT;
    const bool lead = s == 0;
    // the lanes of this warp (a CTA of Z * SPLIT threads may end in a partial warp; a row's
    // lanes are never split between warps because SPLIT divides 32)
    const unsigned wmask = __activemask();
    __shared__ unsigned s_odd[2];
    constexpr bool LRN = KIND == KIND_LEARNED;
    __shared__ uint2 s_kb[LRN ? QC_LUT_ITS : 1][2];
    if (threadIdx.x < 2) s_odd[threadIdx.x] = 0;
    if (LRN && threadIdx.x < 2 * J.lut_its) {
        const int t = threadIdx.x;
        s_kb[t >> 1][t & 1] = *reinterpret_cast<const uint2*>(J.lut + (t >> 1) * 256 + (t & 1) * 128);
    }
    constexpr int CM = ET ? 2 : 0;

    Plan P;
    P.n = Q.n;
    read_group(P, J, g, [&](int v, uint32_t w) { app1[v] = Access<PackF16x2>::pair(w, 2 * h); });
    __syncthreads();

    uint32_t msg[L][DL];
#pragma unroll
    for (int l = 0; l < L; l++)
#pragma unroll
        for (int i = 0; i < DL; i++) msg[l][i] = 0;

    int executed = 0;
    bool passed = false;
    for (int it = 0; it < J.iters; it++) {
        uint32_t ov = 0;
        const int lt = LRN ? min(it, J.lut_its - 1) : 0;
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int d = Q.deg[l];
            const int nv = d > s ? (d - s + SPLIT - 1) / SPLIT : 0;  // this lane's edges of the row
            const bool noclip = J.quirk && it == 0 && Q.cls[l];
            int kk = 4 * k;
            asm volatile("" : "+r"(kk));
            int off[DL];
            uint32_t b[DL];
#pragma unroll
            for (int i = 0; i < DL; i++) {
                if (i < nv) {
                    off[i] = qc_var_off<false>(Q, l * QC_MAX_DEG + s + SPLIT * i, kk);
                    b[i] = *reinterpret_cast<const uint32_t*>(appb + off[i]);
                }
            }
            uint32_t lk = 0, lb = 0;
            if (LRN) {
                const uint2 kb = s_kb[lt][Q.cls[l]];
                lk = kb.x;
                lb = kb.y;
            }
            h2::row_split<KIND, DL, SPLIT, CM>(b, msg[l], nv, noclip, ov, lk, lb, wmask, lead);
#pragma unroll
            for (int i = 0; i < DL; i++)
                if (i < nv) *reinterpret_cast<uint32_t*>(appb + off[i]) = b[i];
            if (!(ET && l == L - 1)) __syncthreads();
        }
        executed = it + 1;
        if (ET) {
            // the lead lane of each row counts and checks it (the other lanes add nothing)
            if (odd_rows_within_slack(J, lead ? h2::odd_count(ov, L) : 0u, it, s_odd) &&
                !__syncthreads_or(lead && qc_rows_unsatisfied<DT, false, 0, L, false, 1>(Q, appb, k))) {
                passed = true;
                break;
            }
        }
    }
    // frames 2h, 2h+1 only; the word's iteration count is the larger of its two pairs
    // (the host zeroes d_iters_out before the launch)
    write_group(P, J, g, [&](int v) { return AccessHalf::get(app1, v, h); }, 3 << (2 * h));
    if (J.iters_out && threadIdx.x == 0) atomicMax(J.iters_out + (g - J.word0), executed);
    if (J.synd_out) {
        const unsigned bad = passed || !lead ? 0u : qc_rows_unsat_mask<DT, false, 0, L, false, 1>(Q, appb, k);
        write_syndrome_flags(J, 4 * (g - J.word0) + 2 * h, bad, 3, true);
    }
}

// ---- per-frame early stop with lane refill (decoder path 5) ----
//
// The 4 frames of a CTA (the fp16 halves of its two pair-words, "lanes" 0..3) are
// independent: nothing in the row update mixes lanes.  So each lane can run its own
// frame on its own schedule: the odd-row count, the syndrome check and the iteration
// limit are evaluated per lane, the learned constants and the OMS first-iteration
// clip follow each lane's own iteration number, and when a lane's frame stops the
// CTA writes that frame's decisions and iteration count, puts its next frame into the
// lane and zeroes the lane's messages.  CTAs are persistent: CTA c of G decodes
// frames c, c + G, c + 2G, ... (static, so no atomics; at tens of frames per CTA the
// per-frame iteration counts average out), and keeps its next QC_STAGE frames' LLRs
// in shared memory, copied with cp.async when the previous ones were taken, so that a
// refill does not wait on global memory.  A CTA exits when every lane is idle.  Each
// frame's decisions and iteration count are those of decoding it alone, with the
// early-stop rule (odd rows within the slack, then the syndrome) applied to that
// frame only.

constexpr int QC_STAGE = 4;     // staged frames per CTA (a refill takes at most 4)

// CTA-wide OR of a lane mask through the shared slot *s (zero on entry); every thread calls it
__device__ __forceinline__ unsigned cta_or_lanes(unsigned m, unsigned* s)
{
    const unsigned lanes = __activemask();
    const unsigned w = __reduce_or_sync(lanes, m);
    if (w && (int)(threadIdx.x & 31) == __ffs(lanes) - 1) atomicOr(s, w);
    __syncthreads();
    return *s;
}

// one frame's int8 LLRs (src: global memory, or a staging slot in shared memory) into
// lane `lane` of the biased APP (apph[4 v + lane]), 4 variables per thread and step
template <bool GLOBAL>
__device__ __forceinline__ void qc_put_lane(const int8_t* src, uint16_t* apph, int n, int lane)
{
    if ((n & 3) == 0) {
        const uint32_t* s4 = reinterpret_cast<const uint32_t*>(src);
        for (int q = threadIdx.x; q < (n >> 2); q += blockDim.x) {
            const uint32_t y = (GLOBAL ? __ldg(s4 + q) : s4[q]) ^ 0x7f7f7f7fu;  // see Access<PackF16x2>::pair
            const uint32_t lo = h2::add(__byte_perm(y, 0x6464u, 0x4140), h2::CNEG1024);
            const uint32_t hi = h2::add(__byte_perm(y, 0x6464u, 0x4342), h2::CNEG1024);
            uint16_t* p = apph + 16 * q + lane;
            p[0] = (uint16_t)lo;
            p[4] = (uint16_t)(lo >> 16);
            p[8] = (uint16_t)hi;
            p[12] = (uint16_t)(hi >> 16);
        }
    } else {
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            const uint32_t y = (uint32_t)(uint8_t)(GLOBAL ? __ldg(src + v) : src[v]) ^ 0x7fu;
            apph[4 * v + lane] = (uint16_t)h2::add(__byte_perm(y, 0x6464u, 0x4140), h2::CNEG1024);
        }
    }
}

// starts the copy of frame f's LLRs into a staging slot: cp.async (16-byte pieces,
// completed by cp.async.wait_all) when source and size allow it, else plain copies
__device__ __forceinline__ void qc_stage_frame(const Job& J, int8_t* slot, int n, long long f, bool async16)
{
    const int8_t* src = J.llr + f * n;
    if (async16) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(slot);
        for (int c = threadIdx.x; c < (n >> 4); c += blockDim.x)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16 * c), "l"(src + 16 * c) : "memory");
        asm volatile("cp.async.commit_group;" ::: "memory");
    } else {
        for (int v = threadIdx.x; v < n; v += blockDim.x) slot[v] = __ldg(src + v);
    }
}

// lane `lane`'s hard decisions (x > 0, i.e. biased b < 127) as frame f of the output
__device__ __forceinline__ void qc_store_lane(const Job& J, const uint16_t* apph, int n, long long f, int lane)
{
    if (!J.out) return;
    auto bit = [&](int v) { return (uint32_t)((apph[4 * v + lane] & 0x7fffu) < 0x57f0u); };
    if (!J.out_packed) {
        uint8_t* o = reinterpret_cast<uint8_t*>(J.out) + f * n;
        if ((n & 3) == 0) {
            uint32_t* o4 = reinterpret_cast<uint32_t*>(o);
            for (int q = threadIdx.x; q < (n >> 2); q += blockDim.x)
                o4[q] = bit(4 * q) | (bit(4 * q + 1) << 8) | (bit(4 * q + 2) << 16) | (bit(4 * q + 3) << 24);
        } else {
            for (int v = threadIdx.x; v < n; v += blockDim.x) o[v] = (uint8_t)bit(v);
        }
    } else {
        const int nb = (n + 7) >> 3;
        uint8_t* o = reinterpret_cast<uint8_t*>(J.out) + f * nb;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            uint32_t acc = 0;
            for (int j = 0; j < 8; j++) {
                const int v = 8 * b + j;
                if (v < n) acc |= bit(v) << j;
            }
            o[b] = (uint8_t)acc;
        }
    }
}

// ---- exact-gate early stop per frame pair (4 frames per CTA) ----
//
// true when row k of some layer in [L0, L1) has odd hard-decision parity in one of the two
// frames of one pair-word of the 8-byte-per-variable APP; appb points at that pair's half
// (byte 0 or 4 of each variable)
template <int DT, bool EXACT, int L0, int L1, bool POW2>
__device__ __noinline__ bool qc_rows_unsat_half(const QCParams& Q, const char* appb, int k)
{
    bool bad = false;
    const int kb = 8 * k;
#pragma unroll
    for (int l = L0; l < L1; l++) {
        const int d = EXACT ? DT : Q.deg[l];
        uint32_t acc = 0;
#pragma unroll
        for (int j = 0; j < DT; j++)
            if (EXACT || j < d)
                acc ^= qc_one_signs(*reinterpret_cast<const uint32_t*>(appb + qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kb)));
        bad |= (acc & 0x80008000u) != 0;
    }
    return bad;
}

// OR over the CTA of a 2-bit value (bit p: pair p): one barrier reduction per pair
__device__ __forceinline__ unsigned cta_or_pairs(unsigned bits)
{
    const unsigned b0 = __syncthreads_or(bits & 1u) ? 1u : 0u;
    return b0 | (__syncthreads_or(bits & 2u) ? 2u : 0u);
}

// The remaining pair of decode_qc_pairs_kernel decoding alone: its messages m, its APP
// half at byte hoff of each 8-byte variable; runs from iteration it until the pair's
// decisions are codewords (live = 0) or J.iters.  Every thread of the CTA calls it.
template <int KIND, int DT, bool EXACT, int L, bool POW2>
__device__ __forceinline__ void qc_one_pair(const QCParams& Q, const Job& J, char* appb, int hoff,
                                            uint32_t (&m)[L][DT], const uint2 (*s_kb)[2], int& it, unsigned& live)
{
    constexpr bool LRN = KIND == KIND_LEARNED || KIND == KIND_LEARNED_OFS;
    constexpr int LS = L > 3 ? 2 : 1;
    const int k = threadIdx.x;
    uint32_t ov = 0;  // unused extrinsic count of row()
    while (live && it < J.iters) {
        const int lt = LRN ? min(it, J.lut_its - 1) : 0;
        bool last_bad = false;
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int d = EXACT ? DT : Q.deg[l];
            const bool noclip = J.quirk && it == 0 && Q.cls[l];
            int kk = 8 * k;
            asm volatile("" : "+r"(kk));
            int off[DT];
            uint32_t b0[DT];
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    off[j] = qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kk) + hoff;
                    b0[j] = *reinterpret_cast<const uint32_t*>(appb + off[j]);
                }
            }
            uint32_t lk = 0, lb = 0;
            if (LRN) {
                const uint2 kb = s_kb[lt][Q.cls[l]];
                lk = kb.x;
                lb = kb.y;
            }
            h2::row<KIND, DT, EXACT, 0>(b0, m[l], d, noclip, ov, lk, lb);
#pragma unroll
            for (int j = 0; j < DT; j++)
                if (EXACT || j < d) *reinterpret_cast<uint32_t*>(appb + off[j]) = b0[j];
            if (l == L - 1) {
                uint32_t p0 = 0;
#pragma unroll
                for (int j = 0; j < DT; j++)
                    if (EXACT || j < d) p0 ^= qc_one_signs(b0[j]);
                last_bad = __syncthreads_or((p0 & 0x80008000u) != 0);
            } else {
                __syncthreads();
            }
        }
        it++;
        if (!last_bad) {
            bool done = true;
            if (L > 1) done = !__syncthreads_or(qc_rows_unsat_half<DT, EXACT, 0, (L > 1 ? LS : 0), POW2>(Q, appb + hoff, k));
            if (done && LS < L - 1)
                done = !__syncthreads_or(qc_rows_unsat_half<DT, EXACT, LS, (L > 1 ? L - 1 : 0), POW2>(Q, appb + hoff, k));
            if (done) live = 0;
        }
    }
}

// The 4-frame QC decoder with each frame pair (frames 0, 1 and 2, 3 of word g: the two
// fp16x2 pair-words) stopping on its own at the first iteration whose decisions are
// codewords in both of its frames (the oracle's pair rule with an unbounded slack,
// LDPC_EARLY_SLACK_ANY).  While both pairs decode, each layer updates both rows as in
// decode_qc_kernel and the last layer's rows are checked from registers (per pair); the
// other layers' rows only when a pair's last-layer rows all hold.  When one pair stops,
// its APP and messages stay as they were and the CTA goes on with the other pair alone:
// one row per layer, about 0.55 of a two-pair iteration (qc_one_pair, inlined once for
// each pair so that its messages stay in their own registers).
// The word's count is the iteration at which its last pair stopped.  Every kind but 2NMS.
template <int KIND, int DT, bool EXACT, int L, bool POW2>
__global__ void __launch_bounds__(256, 2) decode_qc_pairs_kernel(const __grid_constant__ QCParams Q, const Job J)
{
    static_assert(KIND != KIND_2NMS, "2NMS has its own early termination");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint2* app = reinterpret_cast<uint2*>(smem_raw);
    char* appb = reinterpret_cast<char*>(smem_raw);
    const long long g = J.word0 + blockIdx.x;
    const int k = threadIdx.x;
    constexpr bool LRN = KIND == KIND_LEARNED || KIND == KIND_LEARNED_OFS;
    __shared__ uint2 s_kb[LRN ? QC_LUT_ITS : 1][2];
    if (LRN && k < 2 * J.lut_its) {
        uint2 kb = *reinterpret_cast<const uint2*>(J.lut + (k >> 1) * 256 + (k & 1) * 128);
        if (KIND == KIND_LEARNED_OFS) kb.y = h2::add(kb.y, 0x37803780u);  // b + 15/32 = -offset (scale 1)
        s_kb[k >> 1][k & 1] = kb;
    }
    // the successor word's LLRs into L2, as in decode_qc_kernel
    if (threadIdx.x == 0 && !J.gen && !J.interleaved && (Q.n & 3) == 0) {
        unsigned nsm;
        asm("mov.u32 %0, %%nsmid;" : "=r"(nsm));
        const long long gn = g + 2 * (long long)nsm;
        if (gn < J.word0 + (long long)gridDim.x) {
            const int8_t* src = J.llr + 4 * (gn - J.word0) * (long long)Q.n;
            if (((uintptr_t)src & 15) == 0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(4u * (unsigned)Q.n) : "memory");
        }
    }
    Plan P;
    P.n = Q.n;
    read_group(P, J, g, [&](int v, uint32_t w) {
        app[v] = make_uint2(Access<PackF16x2>::pair(w, 0), Access<PackF16x2>::pair(w, 2));
    });
    __syncthreads();

    uint32_t msg[2][L][DT];
#pragma unroll
    for (int w = 0; w < 2; w++)
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int j = 0; j < DT; j++) msg[w][l][j] = 0;

    constexpr int LS = L > 3 ? 2 : 1;  // staged check: layers [0, LS), then [LS, L - 1)
    unsigned live = 3;  // bit p set while pair p is decoding (the same in every thread)
    int it = 0;
    uint32_t ov = 0;    // unused extrinsic count of row()
    // both pairs
    while (it < J.iters) {
        const int lt = LRN ? min(it, J.lut_its - 1) : 0;
        unsigned last_bad = 0;
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int d = EXACT ? DT : Q.deg[l];
            const bool noclip = J.quirk && it == 0 && Q.cls[l];
            int kk = 8 * k;
            asm volatile("" : "+r"(kk));
            int off[DT];
            uint32_t b0[DT], b1[DT];
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    off[j] = qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kk);
                    const uint2 v = *reinterpret_cast<const uint2*>(appb + off[j]);
                    b0[j] = v.x;
                    b1[j] = v.y;
                }
            }
            uint32_t lk = 0, lb = 0;
            if (LRN) {
                const uint2 kb = s_kb[lt][Q.cls[l]];
                lk = kb.x;
                lb = kb.y;
            }
            h2::row<KIND, DT, EXACT, 0>(b0, msg[0][l], d, noclip, ov, lk, lb);
            h2::row<KIND, DT, EXACT, 0>(b1, msg[1][l], d, noclip, ov, lk, lb);
#pragma unroll
            for (int j = 0; j < DT; j++)
                if (EXACT || j < d) *reinterpret_cast<uint2*>(appb + off[j]) = make_uint2(b0[j], b1[j]);
            if (l == L - 1) {
                uint32_t p0 = 0, p1 = 0;
#pragma unroll
                for (int j = 0; j < DT; j++) {
                    if (EXACT || j < d) {
                        p0 ^= qc_one_signs(b0[j]);
                        p1 ^= qc_one_signs(b1[j]);
                    }
                }
                last_bad = cta_or_pairs(((p0 & 0x80008000u) ? 1u : 0u) | ((p1 & 0x80008000u) ? 2u : 0u));
            } else {
                __syncthreads();
            }
        }
        it++;
        unsigned gate = ~last_bad & 3u;  // pairs whose last-layer rows all hold
        if (gate && L > 1) {
            unsigned m = qc_rows_unsat_mask<DT, EXACT, 0, (L > 1 ? LS : 0), POW2, 2>(Q, appb, k);
            gate &= ~cta_or_pairs(((m & 3u) ? 1u : 0u) | ((m & 12u) ? 2u : 0u));
            if (gate && LS < L - 1) {
                m = qc_rows_unsat_mask<DT, EXACT, LS, (L > 1 ? L - 1 : 0), POW2, 2>(Q, appb, k);
                gate &= ~cta_or_pairs(((m & 3u) ? 1u : 0u) | ((m & 12u) ? 2u : 0u));
            }
        }
        live &= ~gate;
        if (live != 3) break;
    }
    // one pair left: it goes on alone with its own message registers and APP half
    if (live == 1u)
        qc_one_pair<KIND, DT, EXACT, L, POW2>(Q, J, appb, 0, msg[0], s_kb, it, live);
    else if (live == 2u)
        qc_one_pair<KIND, DT, EXACT, L, POW2>(Q, J, appb, 4, msg[1], s_kb, it, live);

    write_group(P, J, g, [&](int v) { uint2 a = app[v]; return Access<PackF16x2>::unbias(a.x, a.y); });
    if (J.iters_out && threadIdx.x == 0) J.iters_out[g - J.word0] = it;
    if (J.synd_out) {
        // a stopped pair holds codewords; the rest are checked on their final APP
        const unsigned bad = live ? qc_rows_unsat_mask<DT, EXACT, 0, L, POW2, 2>(Q, appb, k) : 0u;
        write_syndrome_flags(J, 4 * (g - J.word0), bad, 0xF, true);
    }
    if (J.app_out) {
        uint32_t* ao = reinterpret_cast<uint32_t*>(J.app_out);
        for (int v = threadIdx.x; v < Q.n; v += blockDim.x) {
            uint2 a = app[v];
            ao[(long long)v * J.total_words + g] = Access<PackF16x2>::unbias(a.x, a.y);
        }
    }
    if (J.msg_out) {
        uint32_t* mo = reinterpret_cast<uint32_t*>(J.msg_out);
        long long e0 = 0;
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int d = EXACT ? DT : Q.deg[l];
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    auto x = [](uint32_t h) { return (uint32_t)(uint8_t)(int8_t)(-__half2int_rn(__ushort_as_half((uint16_t)h))); };
                    const uint32_t lo = msg[0][l][j], hi = msg[1][l][j];
                    const uint32_t wv = x(lo & 0xffff) | (x(lo >> 16) << 8) | (x(hi & 0xffff) << 16) | (x(hi >> 16) << 24);
                    mo[(e0 + (long long)k * d + j) * J.total_words + g] = wv;
                }
            }
            e0 += (long long)Q.z * d;
        }
    }
}

// frames: 4 * words of this launch.  Dynamic shared memory: the APP (8n bytes) and
// QC_STAGE staging slots of n bytes.  J.iters <= 255 (per-lane iteration counts are
// byte fields).  J.iters_out, when set, receives one count per frame.
template <int KIND, int DT, bool EXACT, int L, bool POW2>
__global__ void __launch_bounds__(256, 2) decode_qc_refill_kernel(const __grid_constant__ QCParams Q, const Job J,
                                                                  long long frames)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint16_t* apph = reinterpret_cast<uint16_t*>(smem_raw);  // [n][4 lanes]
    char* appb = reinterpret_cast<char*>(smem_raw);
    int8_t* stage = reinterpret_cast<int8_t*>(smem_raw + 8 * (size_t)Q.n);  // [QC_STAGE][n]
    const int k = threadIdx.x;
    const long long G = gridDim.x;
    const bool async16 = ((reinterpret_cast<uintptr_t>(J.llr) | (uintptr_t)Q.n) & 15) == 0;
    __shared__ unsigned s_cnt[2][2];   // odd rows per lane (16-bit fields of pair-words 0, 1), by iteration parity
    __shared__ unsigned s_bad[2][2];   // unsatisfied lanes of the two check stages, by iteration parity
    __shared__ long long s_frame[4];   // frame of each lane, -1 = idle
    __shared__ long long s_slot[QC_STAGE];  // frame staged in each slot, -1 = none (the frames run out)
    __shared__ int s_src[4];           // refill: the slot each done lane takes
    __shared__ int s_head;             // the slot holding the earliest staged frame
    __shared__ __align__(16) uint32_t s_kb[2][4];  // LEARNED, per row group: k words of pair-words 0, 1, then b words
    __shared__ uint32_t s_clip[2];     // OMS: clip words of second-group rows (per lane: 31, or none in iteration 0)
    __shared__ uint16_t s_tab[QC_LUT_ITS][2][2];  // LEARNED: fp16 (k, b) per iteration and row group

    if (k < 2) {
        s_cnt[0][k] = s_cnt[1][k] = 0;
        s_bad[0][k] = s_bad[1][k] = 0;
    }
    if (KIND == KIND_LEARNED)
        for (int i = k; i < 4 * J.lut_its; i += blockDim.x)
            s_tab[i >> 2][(i >> 1) & 1][i & 1] = J.lut[(i >> 2) * 256 + ((i >> 1) & 1) * 128 + 2 * (i & 1)];
    if (k == 0) {
        // this CTA's frames: blockIdx.x + G j; lanes take j = 0..3, the slots j = 4..7
        for (int i = 0; i < 4; i++) {
            const long long f = blockIdx.x + G * i;
            s_frame[i] = f < frames ? f : -1;
        }
        for (int i = 0; i < QC_STAGE; i++) {
            const long long f = blockIdx.x + G * (4 + i);
            s_slot[i] = f < frames ? f : -1;
        }
        s_head = 0;
    }
    __syncthreads();
    long long next = blockIdx.x + G * (4 + QC_STAGE);  // the next frame to stage (uniform)
#pragma unroll
    for (int i = 0; i < QC_STAGE; i++)
        if (s_slot[i] >= 0) qc_stage_frame(J, stage + (size_t)i * Q.n, Q.n, s_slot[i], async16);
    unsigned act = 0;  // lanes holding a frame (uniform across the CTA, like itp)
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const long long f = s_frame[i];
        if (f >= 0) {
            act |= 1u << i;
            qc_put_lane<true>(J.llr + f * Q.n, apph, Q.n, i);
        }
    }
    if (!act) {
        if (async16) asm volatile("cp.async.wait_all;" ::: "memory");
        return;
    }
    uint32_t itp = 0;  // iterations run by each lane's frame, byte i = lane i

    uint32_t msg[2][L][DT];
#pragma unroll
    for (int w = 0; w < 2; w++)
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int j = 0; j < DT; j++) msg[w][l][j] = 0;

    int par = 0;
    for (;;) {
        // this iteration's per-lane constants (the barrier also publishes refilled lanes)
        if (k < 4) {
            const int it = (itp >> (8 * k)) & 0xff;
            uint16_t* h = reinterpret_cast<uint16_t*>(s_kb);
            if (KIND == KIND_LEARNED) {
                const int t = it < J.lut_its ? it : J.lut_its - 1;
#pragma unroll
                for (int g = 0; g < 2; g++) {
                    h[8 * g + k] = s_tab[t][g][0];
                    h[8 * g + 4 + k] = s_tab[t][g][1];
                }
            }
            if (KIND == KIND_OMS)
                reinterpret_cast<uint16_t*>(s_clip)[k] = (J.quirk && it == 0) ? 0x7bffu : 0x4fc0u;
        }
        __syncthreads();

        uint32_t ov0 = 0, ov1 = 0;
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int d = EXACT ? DT : Q.deg[l];
            int kk = 8 * k;
            asm volatile("" : "+r"(kk));
            int off[DT];
            uint32_t b0[DT], b1[DT];
#pragma unroll
            for (int j = 0; j < DT; j++) {
                if (EXACT || j < d) {
                    off[j] = qc_var_off<POW2>(Q, l * QC_MAX_DEG + j, kk);
                    const uint2 v = *reinterpret_cast<const uint2*>(appb + off[j]);
                    b0[j] = v.x;
                    b1[j] = v.y;
                }
            }
            uint32_t lk0 = 0, lk1 = 0, lb0 = 0, lb1 = 0;
            if (KIND == KIND_LEARNED) {
                const uint4 q = reinterpret_cast<const uint4*>(s_kb)[Q.cls[l]];
                lk0 = q.x;
                lk1 = q.y;
                lb0 = q.z;
                lb1 = q.w;
            }
            uint32_t cl0 = h2::C31, cl1 = h2::C31;
            if (KIND == KIND_OMS && Q.cls[l]) {
                cl0 = s_clip[0];
                cl1 = s_clip[1];
            }
            h2::row<KIND, DT, EXACT, 1>(b0, msg[0][l], d, false, ov0, lk0, lb0, cl0);
            h2::row<KIND, DT, EXACT, 1>(b1, msg[1][l], d, false, ov1, lk1, lb1, cl1);
#pragma unroll
            for (int j = 0; j < DT; j++)
                if (EXACT || j < d) *reinterpret_cast<uint2*>(appb + off[j]) = make_uint2(b0[j], b1[j]);
            if (l < L - 1) __syncthreads();  // the count's barrier closes the last layer
        }
        {
            const unsigned lanes = __activemask();
            const unsigned w0 = __reduce_add_sync(lanes, ov0), w1 = __reduce_add_sync(lanes, ov1);
            if ((int)(threadIdx.x & 31) == __ffs(lanes) - 1) {
                if (w0) atomicAdd(&s_cnt[par][0], w0);
                if (w1) atomicAdd(&s_cnt[par][1], w1);
            }
        }
        __syncthreads();
        const unsigned cnt01 = s_cnt[par][0], cnt23 = s_cnt[par][1];
        if (k == 0) {  // slots of the next iteration (their last readers are past this iteration's barriers)
            s_cnt[par ^ 1][0] = s_cnt[par ^ 1][1] = 0;
            s_bad[par ^ 1][0] = s_bad[par ^ 1][1] = 0;
        }
        itp += (act & 1u) | ((act & 2u) << 7) | ((act & 4u) << 14) | ((act & 8u) << 21);

        unsigned cand = 0, limit = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (!((act >> i) & 1u)) continue;
            const unsigned c = ((i < 2 ? cnt01 : cnt23) >> (16 * (i & 1))) & 0xffffu;
            if (J.early && c <= J.early_slack) cand |= 1u << i;
            if ((int)((itp >> (8 * i)) & 0xffu) >= J.iters) limit |= 1u << i;
        }
        unsigned pass = 0;
        if (cand) {
            // staged like the per-word kernel: the first layers reject most non-codewords
            constexpr int LS = L > 2 ? 2 : L;
            pass = cand & ~cta_or_lanes(qc_rows_unsat_mask<DT, EXACT, 0, LS, POW2, 2>(Q, appb, k) & cand, &s_bad[par][0]);
            if (LS < L && pass)
                pass &= ~cta_or_lanes(qc_rows_unsat_mask<DT, EXACT, LS, L, POW2, 2>(Q, appb, k) & pass, &s_bad[par][1]);
        }
        const unsigned done = pass | limit;
        if (done) {
            // syndrome flags: lanes that passed the check satisfy every row; lanes stopped by
            // the iteration limit alone are checked here (uniform: limit and pass are)
            unsigned unsat = 0;
            const unsigned chk = J.synd_out ? limit & ~pass : 0u;
            if (chk) {
                const unsigned lm = qc_rows_unsat_mask<DT, EXACT, 0, L, POW2, 2>(Q, appb, k) & chk;
#pragma unroll
                for (int i = 0; i < 4; i++)
                    if (((chk >> i) & 1u) && __syncthreads_or((lm >> i) & 1u)) unsat |= 1u << i;
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                if (!((done >> i) & 1u)) continue;
                const long long f = s_frame[i];
                qc_store_lane(J, apph, Q.n, f, i);
                if (k == 0 && J.iters_out) J.iters_out[f] = (int32_t)((itp >> (8 * i)) & 0xffu);
                if (k == 0 && J.synd_out) J.synd_out[f] = ((unsat >> i) & 1u) ? 0 : 1;
            }
            if (async16) asm volatile("cp.async.wait_all;" ::: "memory");
            __syncthreads();  // staged frames landed; decisions and s_frame read before they are replaced
            const int head = s_head;
            const int nd = __popc(done);
            if (k == 0) {
                // done lanes take the staged frames in order (the earliest first)
                int c = 0;
                for (int i = 0; i < 4; i++)
                    if ((done >> i) & 1u) {
                        const int sl = (head + c++) % QC_STAGE;
                        s_src[i] = sl;
                        s_frame[i] = s_slot[sl];
                    }
            }
            __syncthreads();
            uint32_t keep0 = 0xffffffffu, keep1 = 0xffffffffu;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                if (!((done >> i) & 1u)) continue;
                if (s_frame[i] >= 0)
                    qc_put_lane<false>(stage + (size_t)s_src[i] * Q.n, apph, Q.n, i);
                else
                    act &= ~(1u << i);
                itp &= ~(0xffu << (8 * i));
                if (i < 2)
                    keep0 &= (i & 1) ? 0x0000ffffu : 0xffff0000u;
                else
                    keep1 &= (i & 1) ? 0x0000ffffu : 0xffff0000u;
            }
            if (!act) break;
            __syncthreads();  // the taken slots are read before new frames are copied into them
            if (k == 0) s_head = (head + nd) % QC_STAGE;
            for (int c = 0; c < nd; c++) {
                const int sl = (head + c) % QC_STAGE;
                const long long f = next < frames ? next : -1;
                next += G;
                if (k == 0) s_slot[sl] = f;  // read again only after the next refill's barriers
                if (f >= 0) qc_stage_frame(J, stage + (size_t)sl * Q.n, Q.n, f, async16);
            }
#pragma unroll
            for (int l = 0; l < L; l++)
#pragma unroll
                for (int j = 0; j < DT; j++) {
                    msg[0][l][j] &= keep0;
                    msg[1][l][j] &= keep1;
                }
        }
        par ^= 1;
    }
}

}  // namespace ldpc
