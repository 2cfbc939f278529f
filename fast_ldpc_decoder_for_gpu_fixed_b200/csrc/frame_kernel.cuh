// Row-layered decoder for long codes (DVB-S2 size, N = 64800): one frame per CTA,
// its APP in shared memory, its c->v messages in a global scratch.
//
// The 4-frame state of a long code does not fit in one CTA's shared memory
// (N = 64800 needs 259 KB of APP alone for 4 frames).  One frame's APP as int8 is
// N bytes (64.8 KB), so two CTAs, two frames, fit on an SM.  The frame's E
// messages (194 K for the rate-1/2 IRA code) go to the decoder's scratch in global
// memory, one byte per edge, 8 bytes per check row for its edges 0-7 (and 8 more for
// edges 8-15): the thread that updates a row reads and writes its row words
// coalesced with the other rows of the level, a level ahead of their use, so the
// latency hides behind the level in between.  (Two levels ahead spilled the
// prefetched registers under the two-CTAs-per-SM register budget, and a spill waits
// for its load.)  Per frame and iteration that is 2E
// bytes of message traffic, the HBM-bound case of this decoder.
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

// The row a thread updates in one level: its record (columns, degree, class; see
// Plan::rowrec), its index, and its c->v messages.  Records and messages do not depend
// on the frame's APP, so they are loaded a level ahead: the record table (1 MB for
// M = 32400) lives in L2 and the messages in the decoder's scratch in HBM.
struct FrameRow {
    uint4 c0, c1;
    uint2 m0, m1;  // messages of edges 0-7 and 8-15, one byte each (see frame_row)
    int r, end;    // row, end of its level
    __device__ __forceinline__ int deg() const { return (c1.w >> 16) & 0xff; }
    __device__ __forceinline__ int cls() const { return c1.w >> 24; }
    __device__ __forceinline__ int col(int j) const  // j a compile-time constant after unrolling
    {
        const uint4& q = j < 8 ? c0 : c1;
        const int k = (j & 7) >> 1;
        const uint32_t w = k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
        return (j & 1) ? (int)(w >> 16) : (int)(w & 0xffff);
    }
    // the 32-bit word of the messages that holds edges 2p and 2p+1 (bytes 2(p&1), +1)
    __device__ __forceinline__ uint32_t& mword(int p)
    {
        return p < 4 ? ((p >> 1) ? m0.y : m0.x) : ((p >> 1) & 1 ? m1.y : m1.x);
    }
};

// The decoder's message scratch: one slot per resident CTA, M rows of 8 bytes for edges
// 0-7 and, for row degrees above 8, a second array of M rows for edges 8-15.
struct FrameMsgs {
    uint2* lo;
    uint2* hi;
};

// Loads issued where they stand: the compiler may not move a volatile asm across the
// level barriers, so a load issued a level ahead stays a level ahead instead of being
// sunk next to its use to save registers.
__device__ __forceinline__ uint4 ld_nc_v4(const uint4* p)
{
    uint4 v;
    asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

__device__ __forceinline__ uint2 ld_v2(const uint2* p)
{
    uint2 v;
    asm volatile("ld.global.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void load_row(const Plan& P, int r, FrameRow& x)
{
    x.c0 = ld_nc_v4(P.rowrec + 2 * r);
    x.c1 = ld_nc_v4(P.rowrec + 2 * r + 1);
}

template <int DT>
__device__ __forceinline__ void load_msgs(const FrameMsgs& M, FrameRow& x)
{
    x.m0 = ld_v2(M.lo + x.r);
    if (DT > 8) x.m1 = ld_v2(M.hi + x.r);
}

template <int DT>
__device__ __forceinline__ void store_msgs(const FrameMsgs& M, const FrameRow& x)
{
    // ordered with the volatile loads of the same words (a row's words are written and
    // read back by the same thread)
    asm volatile("st.global.v2.u32 [%0], {%1, %2};" ::"l"(M.lo + x.r), "r"(x.m0.x), "r"(x.m0.y) : "memory");
    if (DT > 8)
        asm volatile("st.global.v2.u32 [%0], {%1, %2};" ::"l"(M.hi + x.r), "r"(x.m1.x), "r"(x.m1.y) : "memory");
}

// the row of level l this thread updates first (records and, with msgs, messages)
template <int DT>
__device__ __forceinline__ void fetch_row(const Plan& P, const FrameMsgs& M, int l, FrameRow& x, bool msgs)
{
    const int2 lv = __ldg(P.levels + l);
    x.r = lv.x + threadIdx.x;
    x.end = lv.x + lv.y;
    if (x.r < x.end) {
        load_row(P, x.r, x);
        if (msgs) load_msgs<DT>(M, x);
    } else {
        x.c1.w = 0;  // degree 0: no row for this thread
    }
}

// f16x2 of 1152 and -1152: a message byte y = 128 + u (u the negated message, |u| <= 127)
// under the byte 0x64 is the fp16 1024 + y, so adding -1152 gives u, and adding 1152 to u
// puts y back in the low byte
constexpr uint32_t FRAME_C1152 = 0x64806480u, FRAME_CNEG1152 = 0xe480e480u;

// One check row of one frame (the reference's per-byte update, CUDA_OMS_SIMD.cu:40-134):
// APP bytes in shared memory, this row's messages in row.m0 / row.m1 (in / out), one byte
// per edge holding 128 - msg.  D: the row's degree (fully unrolled).
//
// Two edges per 32-bit word: edges 2p and 2p+1 are the fp16 halves of pair p, in the
// biased negated form of the F16X2 packing (b = 127 - x in [0, 255], integer-valued,
// so every step is exact; see namespace h2).  Each half keeps its own running
// (min1, min2, sign parity) over its edges; the halves are merged once per row.  An
// odd degree's last pair carries a dummy edge x = -127 with no message: |u| = 127
// equals the initial min1 and min2 and its sign is positive, so it changes nothing.
template <int KIND, int D>
__device__ __forceinline__ void frame_row(int8_t* app, FrameRow& row, bool first, bool noclip, int& odd,
                                          const uint16_t* lut)
{
    using namespace h2;
    constexpr int NP = (D + 1) / 2;
    uint32_t bt[NP];  // the extrinsics t = 127 - bt are recomputed where needed (registers)
    uint32_t mn1 = C127, mn2 = C127;
#pragma unroll
    for (int p = 0; p < NP; p++) {
        const int j0 = 2 * p, j1 = 2 * p + 1;
        // bytes x of the two edges; 127 - x as an unsigned byte is x ^ 0x7f (Access<PackF16x2>::pair)
        uint32_t w = (uint32_t)(uint8_t)app[row.col(j0)];
        w |= (j1 < D ? (uint32_t)(uint8_t)app[row.col(j1)] : 0x81u) << 16;
        const uint32_t b = add((w ^ 0x007f007fu) | 0x64006400u, CNEG1024);
        uint32_t u = 0;  // negated old messages (h2 convention: t = clamp(b - u))
        if (!first) {
            u = add(__byte_perm(row.mword(p), 0x64646464u, (p & 1) ? 0x4342 : 0x4140), FRAME_CNEG1152);
            if (j1 >= D) u &= 0xffffu;
        }
        bt[p] = hmin(fma_relu(u, NEG1, b), C255);
        const uint32_t ut = add(bt[p], CNEG127);
        const uint32_t mx = max_xs(ut, mn1);
        mn1 = min_xs(mn1, ut);
        mn2 = min_xs(mn2, mx);
    }
    // merge the halves: min1 of both, min2 = min(max of the two min1s, both min2s), parity of both
    const uint32_t s1 = __byte_perm(mn1, 0, 0x1032), s2 = __byte_perm(mn2, 0, 0x1032);
    const uint32_t m1 = min_xs(mn1, s1);  // |min1| in both halves, sign: the row's parity
    const uint32_t m2 = min_xs(min_xs(mn2, s2), max_xs(mn1, s1));
    const uint32_t a1 = habs(m1), a2 = habs(m2);
    uint32_t c1, c2;
    if (KIND == KIND_LEARNED) {
        // the integer tables of the I8 packing (any constants): c1 = lut[min2], c2 = lut[min1]
        const uint32_t ic1 = lut[add(a2, C1024) & 0x7fu];
        const uint32_t ic2 = lut[add(a1, C1024) & 0x7fu];
        c1 = add(0x64006400u | ic1 | (ic1 << 16), CNEG1024);
        c2 = add(0x64006400u | ic2 | (ic2 << 16), CNEG1024);
    } else {
        h2::mags<KIND>(a1, a2, noclip, c1, c2, 0u, 0u);
    }
    const uint32_t c1s = c1 | (m1 & SIGN), c2s = c2 | (m1 & SIGN);
    const uint32_t dcs = sub(c2s, c1s), na1 = a1 ^ SIGN;
#pragma unroll
    for (int p = 0; p < NP; p++) {
        const int j0 = 2 * p, j1 = 2 * p + 1;
        const uint32_t ut = add(bt[p], CNEG127);
        const uint32_t fl = add_sat(habs(ut), na1);  // 0.0 on minimum edges, 1.0 elsewhere
        const uint32_t mo = fma(fl, dcs, c1s) ^ (ut & SIGN);
        const uint32_t bn = add(hmin(fma_relu(mo, ONE, bt[p]), C255), C1024) ^ 0x007f007fu;  // x bytes
        app[row.col(j0)] = (int8_t)bn;
        if (j1 < D) app[row.col(j1)] = (int8_t)(bn >> 16);
        uint32_t& mw = row.mword(p);
        mw = __byte_perm(mw, add(mo, FRAME_C1152), (p & 1) ? 0x6410 : 0x3264);
    }
    odd += (m1 >> 15) & 1u;
}

// Dispatches a row to the unrolled update for its degree.  Rows of a level are
// sorted by degree, so the warps of a level mostly take one case.
template <int KIND, int DT, bool EXACT>
__device__ __forceinline__ void frame_row_any(int8_t* app, FrameRow& row, bool first, bool noclip, int& odd,
                                              const uint16_t* lut)
{
    if (EXACT) return frame_row<KIND, DT>(app, row, first, noclip, odd, lut);
#define LDPC_FRAME_CASE(D)                                                                        \
    case D:                                                                                       \
        if (D <= DT) frame_row<KIND, (D <= DT ? D : DT)>(app, row, first, noclip, odd, lut);      \
        return;
    switch (row.deg()) {
        LDPC_FRAME_CASE(1) LDPC_FRAME_CASE(2) LDPC_FRAME_CASE(3) LDPC_FRAME_CASE(4) LDPC_FRAME_CASE(5)
        LDPC_FRAME_CASE(6) LDPC_FRAME_CASE(7) LDPC_FRAME_CASE(8) LDPC_FRAME_CASE(9) LDPC_FRAME_CASE(10)
        LDPC_FRAME_CASE(11) LDPC_FRAME_CASE(12) LDPC_FRAME_CASE(13) LDPC_FRAME_CASE(14)
    }
#undef LDPC_FRAME_CASE
}

// Persistent CTAs: CTA c decodes frames c, c + G, c + 2G, ... of the launch (G = gridDim.x),
// one at a time, with slot c of the message scratch (J.fmsg: J.fslots slots of P.m rows,
// then as many again for edges 8-15 when DT > 8).  Shared memory: the frame's APP
// (npad bytes) and, for KIND_LEARNED, the iteration's tables.
template <int KIND, int DT, bool EXACT, bool ET>
__global__ void __maxnreg__(80) decode_frame_kernel(const Plan P, const Job J, long long frames)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int8_t* app = reinterpret_cast<int8_t*>(smem_raw);                     // [npad]
    uint16_t* slut = reinterpret_cast<uint16_t*>(smem_raw + P.npad);       // KIND_LEARNED
    __shared__ unsigned s_odd[2];
    const FrameMsgs M = {J.fmsg + (long long)blockIdx.x * P.m, J.fmsg + (J.fslots + blockIdx.x) * (long long)P.m};
    const int nl = P.nlevels;
    // messages are fetched with the records one level ahead; a row's messages are written
    // back when its level is updated, so with a single level per iteration the fetch would
    // come before that write: such codes load them when the row is updated
    const bool pf = nl >= 2;
    for (long long lf = blockIdx.x; lf < frames; lf += gridDim.x) {
        const long long f = 4 * J.word0 + lf;
        if (threadIdx.x < 2) s_odd[threadIdx.x] = 0;
        read_frame(P, J, f, [&](int v, int x) { app[v] = (int8_t)x; });
        __syncthreads();

        FrameRow next;  // the row of level l+1 (cyclically)
        fetch_row<DT>(P, M, 0, next, pf);
        int lnext = nl > 1 ? 1 : 0;  // level fetched next
        int executed = 0;
        bool passed = false;  // stopped by the syndrome early stop: every check holds
        for (int it = 0; it < J.iters; it++) {
            int odd = 0;
            const bool first = it == 0, keep = it + 1 < J.iters;  // the last iteration's messages are not needed
            if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
            for (int l = 0; l < nl; l++) {
                FrameRow cur = next;
                fetch_row<DT>(P, M, lnext, next, pf);
                lnext = lnext + 1 == nl ? 0 : lnext + 1;
                if (cur.r < cur.end) {
                    if (!pf && !first) load_msgs<DT>(M, cur);
                    const bool noclip = J.quirk && first && cur.cls();
                    frame_row_any<KIND, DT, EXACT>(app, cur, first, noclip, odd, slut + 128 * cur.cls());
                    if (keep) store_msgs<DT>(M, cur);
                }
                // levels wider than the CTA: the remaining rows load their records directly
                for (int r = cur.r + blockDim.x; r < cur.end; r += blockDim.x) {
                    FrameRow x;
                    x.r = r;
                    x.end = cur.end;
                    load_row(P, r, x);
                    if (!first) load_msgs<DT>(M, x);
                    const bool noclip = J.quirk && first && x.cls();
                    frame_row_any<KIND, DT, EXACT>(app, x, first, noclip, odd, slut + 128 * x.cls());
                    if (keep) store_msgs<DT>(M, x);
                }
                __syncthreads();
            }
            executed = it + 1;
            if (ET) {
                if (odd_rows_within_slack(J, (unsigned)odd, it, s_odd) &&
                    !__syncthreads_or(frame_rows_unsatisfied(app, P))) {
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
        __syncthreads();  // the APP is refilled by the next frame
    }
}

}  // namespace ldpc
