// Row-layered decoder for long codes (DVB-S2 size, N = 64800): one frame per CTA,
// everything on chip.
//
// The 4-frame state of a long code does not fit in one CTA's shared memory
// (N = 64800 needs 259 KB of APP alone for 4 frames), and per-edge c->v messages
// would add E bytes per frame (194 KB for the rate-1/2 IRA code).  But every
// message of a min-sum check row is a function of four row quantities: the
// magnitude c1 sent on the minimum edge, the magnitude c2 sent on the others,
// the index of the minimum edge and one sign bit per edge.  Stored as one
// 32-bit word per row (7 + 7 + 4 + 14 bits: degree <= 14, magnitudes <= 127,
// which every kind but 2NMS satisfies), a frame's whole decoder state is
// N + 4M bytes: 194 KB for N = 64800, M = 32400, inside one SM's shared memory.
// No message crosses HBM; the prologue reads N LLR bytes and the epilogue
// writes the hard decisions.
//
// The state reproduces the reference's per-edge messages exactly: edges whose
// |t| equals min1 receive c1 in the reference (CUDA_OMS_SIMD.cu:73-90), and
// when two edges tie at min1, min2 = min1 and c1 = c2, so one stored index
// suffices.
//
// Early stop (ET) is per frame: the frame stops after an iteration in which at
// most J.early_slack of its rows had odd extrinsic parity and its hard decisions
// then satisfy every check.  Iteration counts are reported per frame.
#pragma once
#include "decode_kernel.cuh"

namespace ldpc {

constexpr int FRAME_MAX_THREADS = 512;
constexpr int FRAME_MAX_DEGREE = 14;

// Reads frame f (batch index) and calls put(v, x) with its int8 LLR of variable v.
template <class F>
__device__ __forceinline__ void read_frame(const Plan& P, const Job& J, long long f, F put)
{
    const int n = P.n;
    if (J.gen) {
        float mean = -1.0f;
        const uint8_t* cw = J.cw ? J.cw + ((unsigned long long)f % (unsigned long long)J.n_cw) * n : nullptr;
        if ((n & 3) == 0) {
            for (int q = threadIdx.x; q < (n >> 2); q += blockDim.x) {
                float u[4], gs[4];
                uniforms4(((unsigned long long)f * n + 4 * q) >> 2, J.seed, J.offset, u);
                box_muller4(u, gs);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (cw) mean = cw[4 * q + i] ? 1.0f : -1.0f;
                    put(4 * q + i, quantise(mean + J.sigma * gs[i]));
                }
            }
        } else {
            for (int v = threadIdx.x; v < n; v += blockDim.x) {
                if (cw) mean = cw[v] ? 1.0f : -1.0f;
                put(v, awgn_sample((unsigned long long)f * n + v, J.seed, J.offset, J.sigma, mean));
            }
        }
        return;
    }
    if (J.interleaved) {  // word[v * W + g], byte k = frame 4g + k
        const int8_t* src = J.llr + (f & 3);
        const long long g = f >> 2;
        for (int v = threadIdx.x; v < n; v += blockDim.x) put(v, __ldg(src + 4 * ((long long)v * J.total_words + g)));
        return;
    }
    const int8_t* src = J.llr + (f - 4 * J.word0) * (long long)n;
    if ((n & 15) == 0 && (reinterpret_cast<uintptr_t>(J.llr) & 15) == 0) {
        const int4* s16 = reinterpret_cast<const int4*>(src);
        for (int q = threadIdx.x; q < (n >> 4); q += blockDim.x) {
            const int4 w = __ldg(s16 + q);
            const uint32_t ws[4] = {(uint32_t)w.x, (uint32_t)w.y, (uint32_t)w.z, (uint32_t)w.w};
#pragma unroll
            for (int i = 0; i < 16; i++) put(16 * q + i, (int8_t)(ws[i >> 2] >> (8 * (i & 3))));
        }
    } else {
        for (int v = threadIdx.x; v < n; v += blockDim.x) put(v, __ldg(src + v));
    }
}

// Hard decisions (x > 0) and error counts of frame f; x(v) returns the APP of v.
template <class F>
__device__ __forceinline__ void write_frame(const Plan& P, const Job& J, long long f, F x)
{
    const int n = P.n;
    const long long lf = f - 4 * J.word0;
    if (J.counts) {
        __shared__ int part[FRAME_MAX_THREADS / 32];
        int e = 0;
        const uint8_t* cw = J.cw ? J.cw + ((unsigned long long)f % (unsigned long long)J.n_cw) * n : nullptr;
        for (int v = threadIdx.x; v < J.n_vars; v += blockDim.x) e += (x(v) > 0) != (cw ? cw[v] != 0 : false);
#pragma unroll
        for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
            atomicAdd(J.counts + 0, 1ull);
            atomicAdd(J.counts + 1, (unsigned long long)t);
            atomicAdd(J.counts + 2, (unsigned long long)(t != 0));
        }
    }
    if (!J.out) return;
    if (!J.out_packed) {
        uint8_t* o = reinterpret_cast<uint8_t*>(J.out) + lf * n;
        if ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(J.out) & 3) == 0) {
            uint32_t* o32 = reinterpret_cast<uint32_t*>(o);
            for (int q = threadIdx.x; q < (n >> 2); q += blockDim.x) {
                uint32_t w = 0;
#pragma unroll
                for (int i = 0; i < 4; i++) w |= (uint32_t)(x(4 * q + i) > 0) << (8 * i);
                o32[q] = w;
            }
        } else {
            for (int v = threadIdx.x; v < n; v += blockDim.x) o[v] = x(v) > 0;
        }
    } else {
        const int nb = (n + 7) >> 3;
        uint8_t* o = reinterpret_cast<uint8_t*>(J.out) + lf * nb;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            uint32_t acc = 0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int v = 8 * b + j;
                if (v < n) acc |= (uint32_t)(x(v) > 0) << j;
            }
            o[b] = (uint8_t)acc;
        }
    }
}

// true in some thread when a check of the frame has odd hard-decision parity
__device__ __forceinline__ bool frame_rows_unsatisfied(const int8_t* app, const Plan& P)
{
    bool bad = false;
    for (int r = threadIdx.x; r < P.m; r += blockDim.x) {
        const int d = __ldg(P.rowdeg + r);
        int p = 0;
        for (int j = 0; j < d; j++) p ^= app[__ldg(P.cols + j * P.m + r)] > 0;
        bad |= p != 0;
    }
    return bad;
}

// The row a thread updates in one level: its record (columns, degree, class;
// see Plan::rowrec) and its index.  Records do not depend on the frame's
// state, so they are loaded two levels ahead: with one CTA per SM nothing else
// hides the L2 latency of a table too large for L1 (1 MB for M = 32400).
struct FrameRow {
    uint4 c0, c1;
    int r, end;  // row, end of its level
    __device__ __forceinline__ int deg() const { return (c1.w >> 16) & 0xff; }
    __device__ __forceinline__ int cls() const { return c1.w >> 24; }
    __device__ __forceinline__ int col(int j) const  // j a compile-time constant after unrolling
    {
        const uint4& q = j < 8 ? c0 : c1;
        const int k = (j & 7) >> 1;
        const uint32_t w = k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
        return (j & 1) ? (int)(w >> 16) : (int)(w & 0xffff);
    }
};

__device__ __forceinline__ void load_row(const Plan& P, int r, FrameRow& x)
{
    x.c0 = __ldg(P.rowrec + 2 * r);
    x.c1 = __ldg(P.rowrec + 2 * r + 1);
}

__device__ __forceinline__ void fetch_row(const Plan& P, int l, FrameRow& x)
{
    const int2 lv = __ldg(P.levels + l);
    x.r = lv.x + threadIdx.x;
    x.end = lv.x + lv.y;
    if (x.r < x.end) {
        load_row(P, x.r, x);
    } else {
        x.c1.w = 0;  // degree 0: no row for this thread
    }
}

// One check row of one frame (the reference's per-byte update, CUDA_OMS_SIMD.cu:40-134)
// with its messages held as the packed row state st: c1 | c2 << 7 | i1 << 14 | signs << 18,
// sign bit j set when edge j's message is positive.  D: the row's degree (fully
// unrolled).  Returns the new state.
//
// Two edges per 32-bit word: edges 2p and 2p+1 are the fp16 halves of pair p, in the
// biased negated form of the F16X2 packing (b = 127 - x in [0, 255], integer-valued,
// so every step is exact; see namespace h2).  Each half keeps its own running
// (min1, min2, sign parity) over its edges; the halves are merged once per row.  An
// odd degree's last pair carries a dummy edge x = -127 with no message: |u| = 127
// equals the initial min1 and min2 and its sign is positive, so it changes nothing.
// All edges whose |t| equals min1 get c1 (as in the reference); ties give c1 = c2 for
// every kind served here, so the stored index (the first such edge) is exact.
template <int KIND, int D>
__device__ __forceinline__ uint32_t frame_row(int8_t* app, const FrameRow& row, uint32_t st, bool first, bool noclip,
                                              int& odd, const uint16_t* lut)
{
    using namespace h2;
    constexpr int NP = (D + 1) / 2;
    uint32_t bt[NP], ut[NP];
    // old messages: magnitude oc1 on edge oi, oc2 on the others, as fp16 pairs
    const uint32_t oc1 = st & 0x7f, oc2 = (st >> 7) & 0x7f, oi = (st >> 14) & 0xf;
    const uint32_t h22 = add(0x64006400u | oc2 | (oc2 << 16), CNEG1024);
    const uint32_t h12 = add(0x64006400u | oc1 | (oc2 << 16), CNEG1024);
    const uint32_t h21 = add(0x64006400u | oc2 | (oc1 << 16), CNEG1024);
    uint32_t mn1 = C127, mn2 = C127;
#pragma unroll
    for (int p = 0; p < NP; p++) {
        const int j0 = 2 * p, j1 = 2 * p + 1;
        // bytes x of the two edges; 127 - x as an unsigned byte is x ^ 0x7f (Access<PackF16x2>::pair)
        uint32_t w = (uint32_t)(uint8_t)app[row.col(j0)];
        w |= (j1 < D ? (uint32_t)(uint8_t)app[row.col(j1)] : 0x81u) << 16;
        const uint32_t b = add((w ^ 0x007f007fu) | 0x64006400u, CNEG1024);
        uint32_t m = 0;  // negated old messages (h2 convention: t = clamp(b - m))
        if (!first) {
            const uint32_t sb = st >> (18 + j0);  // bit 0: edge j0's message positive, bit 1: edge j1's
            m = (oi == (uint32_t)j0 ? h12 : (oi == (uint32_t)j1 ? h21 : h22)) | ((sb & 1u) << 15) | ((sb & 2u) << 30);
            if (j1 >= D) m &= 0xffffu;
        }
        bt[p] = hmin(fma_relu(m, NEG1, b), C255);
        ut[p] = add(bt[p], CNEG127);
        const uint32_t mx = max_xs(ut[p], mn1);
        mn1 = min_xs(mn1, ut[p]);
        mn2 = min_xs(mn2, mx);
    }
    // merge the halves: min1 of both, min2 = min(max of the two min1s, both min2s), parity of both
    const uint32_t s1 = __byte_perm(mn1, 0, 0x1032), s2 = __byte_perm(mn2, 0, 0x1032);
    const uint32_t m1 = min_xs(mn1, s1);  // |min1| in both halves, sign: the row's parity
    const uint32_t m2 = min_xs(min_xs(mn2, s2), max_xs(mn1, s1));
    const uint32_t a1 = habs(m1), a2 = habs(m2);
    uint32_t c1, c2, ic1, ic2;
    if (KIND == KIND_LEARNED) {
        // the integer tables of the I8 packing (any constants): c1 = lut[min2], c2 = lut[min1]
        ic1 = lut[add(a2, C1024) & 0x7fu];
        ic2 = lut[add(a1, C1024) & 0x7fu];
        c1 = add(0x64006400u | ic1 | (ic1 << 16), CNEG1024);
        c2 = add(0x64006400u | ic2 | (ic2 << 16), CNEG1024);
    } else {
        h2::mags<KIND>(a1, a2, noclip, c1, c2, 0u, 0u);
        ic1 = add(c1, C1024) & 0x7fu;
        ic2 = add(c2, C1024) & 0x7fu;
    }
    const uint32_t c1s = c1 | (m1 & SIGN), c2s = c2 | (m1 & SIGN);
    const uint32_t dcs = sub(c2s, c1s), na1 = a1 ^ SIGN;
    uint32_t notmin = 0, sgn = 0;
#pragma unroll
    for (int p = 0; p < NP; p++) {
        const int j0 = 2 * p, j1 = 2 * p + 1;
        const uint32_t fl = add_sat(habs(ut[p]), na1);  // 0.0 on minimum edges, 1.0 elsewhere
        const uint32_t mo = fma(fl, dcs, c1s) ^ (ut[p] & SIGN);
        const uint32_t bn = add(hmin(fma_relu(mo, ONE, bt[p]), C255), C1024);  // 1024 + b: b in the low byte
        app[row.col(j0)] = (int8_t)(bn ^ 0x7fu);
        notmin |= ((fl >> 13) & 1u) << j0;
        sgn |= ((mo >> 15) & 1u) << j0;  // the message -mo is positive
        if (j1 < D) {
            app[row.col(j1)] = (int8_t)((bn >> 16) ^ 0x7fu);
            notmin |= ((fl >> 29) & 1u) << j1;
            sgn |= (mo >> 31) << j1;
        }
    }
    const uint32_t mins = ~notmin & ((1u << D) - 1u);
    const uint32_t i1 = mins ? (uint32_t)(__ffs(mins) - 1) : 0u;
    odd += (m1 >> 15) & 1u;
    return ic1 | (ic2 << 7) | (i1 << 14) | (sgn << 18);
}

// Dispatches a row to the unrolled update for its degree.  Rows of a level are
// sorted by degree, so the warps of a level mostly take one case.
template <int KIND, int DT, bool EXACT>
__device__ __forceinline__ uint32_t frame_row_any(int8_t* app, const FrameRow& row, uint32_t st, bool first,
                                                  bool noclip, int& odd, const uint16_t* lut)
{
    if (EXACT) return frame_row<KIND, DT>(app, row, st, first, noclip, odd, lut);
#define LDPC_FRAME_CASE(D) \
    case D:                \
        if (D <= DT) return frame_row<KIND, (D <= DT ? D : DT)>(app, row, st, first, noclip, odd, lut);
    switch (row.deg()) {
        LDPC_FRAME_CASE(1) LDPC_FRAME_CASE(2) LDPC_FRAME_CASE(3) LDPC_FRAME_CASE(4) LDPC_FRAME_CASE(5)
        LDPC_FRAME_CASE(6) LDPC_FRAME_CASE(7) LDPC_FRAME_CASE(8) LDPC_FRAME_CASE(9) LDPC_FRAME_CASE(10)
        LDPC_FRAME_CASE(11) LDPC_FRAME_CASE(12) LDPC_FRAME_CASE(13) LDPC_FRAME_CASE(14)
    }
#undef LDPC_FRAME_CASE
    return st;  // not reached: degrees are 1..FRAME_MAX_DEGREE
}

// Launched with at most FRAME_MAX_THREADS (512) threads, so 128 registers a thread always
// fit; a plain launch bound let the compiler settle at 64 and spill the degree-14 update.
template <int KIND, int DT, bool EXACT, bool ET>
__global__ void __maxnreg__(128) decode_frame_kernel(const Plan P, const Job J)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int8_t* app = reinterpret_cast<int8_t*>(smem_raw);                                  // [npad]
    uint32_t* state = reinterpret_cast<uint32_t*>(smem_raw + P.npad);                   // [m]
    uint16_t* slut = reinterpret_cast<uint16_t*>(smem_raw + P.npad + 4 * (size_t)P.m);  // KIND_LEARNED
    __shared__ unsigned s_odd[2];
    const long long lf = blockIdx.x;
    const long long f = 4 * J.word0 + lf;

    read_frame(P, J, f, [&](int v, int x) { app[v] = (int8_t)x; });
    if (threadIdx.x < 2) s_odd[threadIdx.x] = 0;
    __syncthreads();

    const int nl = P.nlevels;
    FrameRow next1, next2;  // the rows of levels l+1 and l+2 (cyclically)
    fetch_row(P, 0, next1);
    fetch_row(P, nl > 1 ? 1 : 0, next2);
    int lf2 = nl > 2 ? 2 : 2 % nl;  // level fetched next
    int executed = 0;
    bool passed = false;  // stopped by the syndrome early stop: every check holds
    for (int it = 0; it < J.iters; it++) {
        int odd = 0;
        if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
        for (int l = 0; l < nl; l++) {
            const FrameRow cur = next1;
            next1 = next2;
            fetch_row(P, lf2, next2);
            lf2 = lf2 + 1 == nl ? 0 : lf2 + 1;
            if (cur.r < cur.end) {
                const bool noclip = J.quirk && it == 0 && cur.cls();
                state[cur.r] = frame_row_any<KIND, DT, EXACT>(app, cur, it == 0 ? 0u : state[cur.r], it == 0, noclip,
                                                              odd, slut + 128 * cur.cls());
            }
            // levels wider than the CTA: the remaining rows load their records directly
            for (int r = cur.r + blockDim.x; r < cur.end; r += blockDim.x) {
                FrameRow x;
                load_row(P, r, x);
                const bool noclip = J.quirk && it == 0 && x.cls();
                state[r] = frame_row_any<KIND, DT, EXACT>(app, x, it == 0 ? 0u : state[r], it == 0, noclip, odd,
                                                          slut + 128 * x.cls());
            }
            __syncthreads();
        }
        executed = it + 1;
        if (ET) {
            if (odd_rows_within_slack(J, (unsigned)odd, it, s_odd) && !__syncthreads_or(frame_rows_unsatisfied(app, P))) {
                passed = true;
                break;
            }
        }
    }

    write_frame(P, J, f, [&](int v) { return (int)app[v]; });
    if (J.iters_out && threadIdx.x == 0) J.iters_out[lf] = executed;
    if (J.synd_out) {
        int odd = 0;
        if (!passed) odd = __syncthreads_or(frame_rows_unsatisfied(app, P));
        if (threadIdx.x == 0) J.synd_out[lf] = odd ? 0 : 1;
    }
}

}  // namespace ldpc
