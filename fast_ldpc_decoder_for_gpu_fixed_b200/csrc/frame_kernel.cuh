// Row-layered decoder for long codes (DVB-S2 size, N = 64800): one frame per CTA,
// its APP in shared memory, its c->v messages in a global scratch.
//
// The 4-frame state of a long code does not fit in one CTA's shared memory
// (N = 64800 needs 259 KB of APP alone for 4 frames).  One frame's APP as int8 is
// N bytes (64.8 KB), so two CTAs, two frames, fit on an SM.  The frame's E
// messages (194 K for the rate-1/2 IRA code) live in the decoder's scratch in global
// memory, one byte per edge.
//
// Stages: the host cuts every schedule level into chunks of at most blockDim.x rows
// (FrameStage); each thread updates at most one row of a stage.  A stage's record
// (row words, then the rows' columns) and its messages are contiguous, 16-byte aligned
// blocks in global memory, which the TMA engine copies (cp.async.bulk, completion on
// an mbarrier) into a ring of FRAME_RING shared-memory slots two stages ahead of their
// use; after a stage its updated messages go back with a bulk store from the slot.
// So no thread waits on a global load inside the iteration loop, no register holds a
// prefetched row, and message traffic is exactly one byte per edge (plus one per odd
// row degree) each way per iteration.
//
// Early stop (ET) is per frame: the frame stops after an iteration in which at
// most J.early_slack of its rows had odd extrinsic parity and its hard decisions
// then satisfy every check.  Iteration counts are reported per frame.
#pragma once
#include "decode_kernel.cuh"

namespace ldpc {

constexpr int FRAME_MAX_THREADS = 512;  // rows of a stage at most; the CTA adds one producer warp
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
        __shared__ int part[FRAME_MAX_THREADS / 32 + 1];
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

// One stage of the schedule: at most blockDim.x rows of one level (consecutive rows of the
// level, whose rows are sorted by decreasing degree).  Record (copied to shared memory):
//   a 32-byte header: word 0 = rows, word 1 = the record's bytes (where the stage's messages
//     follow it in the ring slot); bytes 16..31 = pair-slot offsets poff[0..7] (u16, in
//     pairs): pair slot p holds pair p (edges 2p, 2p+1) of every row of degree > 2p, the
//     stage's row t at poff[p] + t;
//   the row words, u32 per row (degree | class << 8), padded to 16 bytes;
//   the column pairs, u32 per pair slot entry (column of edge 2p | column of edge 2p+1 << 16).
// Messages: one u16 per pair slot entry (the two edges' bytes 128 - msg), same indexing.
// Rows t of a warp read consecutive words of each pair slot: no bank conflicts.
struct FrameStage {
    int rec_off;    // byte offset of the record in FrameStages::rec (16-aligned)
    int rec_bytes;  // multiple of 16
    int msg_off;    // byte offset of the messages in a CTA's scratch slot (16-aligned)
    int msg_bytes;  // multiple of 16
};

constexpr int FRAME_STAGE_HEADER = 32;

struct FrameStages {
    const FrameStage* st;     // [nst], one iteration's stages in order
    const unsigned char* rec;
    unsigned char* msg;       // fslots scratch slots of slot_bytes, one per resident CTA
    long long slot_bytes;
    int nst;
    int slot_sz;              // bytes of a ring slot: the largest record plus its messages
    int* status;              // set to 1 when a wait on the copy engine gave up
};

constexpr int FRAME_RING = 4;
// a wait on a bulk copy gives up after this many clock cycles (about a second)
constexpr long long FRAME_WAIT_CYCLES = 2000000000ll;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

// thread-scope try_wait loop with a cycle limit; false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > FRAME_WAIT_CYCLES) return false;
    }
}

// the bulk copies of stage `st` (its messages too when msgs) into ring slot `slot`,
// completing on bar; issued by one thread
__device__ __forceinline__ void stage_load(const FrameStages& S, const FrameStage& st, unsigned char* slot,
                                           const unsigned char* gmsg, bool msgs, unsigned long long* bar)
{
    const uint32_t b = smem_u32(bar);
    const uint32_t bytes = st.rec_bytes + (msgs ? st.msg_bytes : 0);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(slot)),
                 "l"(S.rec + st.rec_off), "r"(st.rec_bytes), "r"(b)
                 : "memory");
    if (msgs)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_u32(slot + st.rec_bytes)),
                     "l"(gmsg + st.msg_off), "r"(st.msg_bytes), "r"(b)
                     : "memory");
}

// f16x2 of 1152 and -1152: a message byte y = 128 + u (u the negated message, |u| <= 127)
// under the byte 0x64 is the fp16 1024 + y, so adding -1152 gives u, and adding 1152 to u
// puts y back in the low byte
constexpr uint32_t FRAME_C1152 = 0x64806480u, FRAME_CNEG1152 = 0xe480e480u;

// One check row of one frame (the reference's per-byte update, CUDA_OMS_SIMD.cu:40-134):
// APP bytes in shared memory, the row's columns (cp: u32 pairs) and messages (mp: u16
// pairs, in / out, one byte per edge holding 128 - msg) in the stage's ring slot.
// D: the row's degree (fully unrolled).
//
// Two edges per 32-bit word: edges 2p and 2p+1 are the fp16 halves of pair p, in the
// biased negated form of the F16X2 packing (b = 127 - x in [0, 255], integer-valued,
// so every step is exact; see namespace h2).  Each half keeps its own running
// (min1, min2, sign parity) over its edges; the halves are merged once per row.  An
// odd degree's last pair carries a dummy edge x = -127 with no message: |u| = 127
// equals the initial min1 and min2 and its sign is positive, so it changes nothing.
template <int KIND, int D>
__device__ __forceinline__ void frame_row(int8_t* app, const uint32_t* cp, uint16_t* mp, const uint4& po, bool first,
                                          bool noclip, int& odd, const uint16_t* lut)
{
    using namespace h2;
    constexpr int NP = (D + 1) / 2;
    uint32_t bt[NP];  // the extrinsics t = 127 - bt are recomputed where needed (registers)
    uint32_t cw[NP];  // column pairs
    int pi[NP];       // this row's entry of each pair slot
    uint32_t mn1 = C127, mn2 = C127;
#pragma unroll
    for (int p = 0; p < NP; p++) {
        const uint32_t w = p < 2 ? po.x : (p < 4 ? po.y : (p < 6 ? po.z : po.w));
        pi[p] = (int)((p & 1) ? (w >> 16) : (w & 0xffffu));
        cw[p] = cp[pi[p]];
    }
#pragma unroll
    for (int p = 0; p < NP; p++) {
        const bool two = 2 * p + 1 < D;
        // bytes x of the two edges; 127 - x as an unsigned byte is x ^ 0x7f (Access<PackF16x2>::pair)
        uint32_t w = (uint32_t)(uint8_t)app[cw[p] & 0xffffu];
        w |= (two ? (uint32_t)(uint8_t)app[cw[p] >> 16] : 0x81u) << 16;
        const uint32_t b = add((w ^ 0x007f007fu) | 0x64006400u, CNEG1024);
        uint32_t u = 0;  // negated old messages (h2 convention: t = clamp(b - u))
        if (!first) {
            u = add(__byte_perm((uint32_t)mp[pi[p]], 0x64646464u, 0x4140), FRAME_CNEG1152);
            if (!two) u &= 0xffffu;
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
        const uint32_t ut = add(bt[p], CNEG127);
        const uint32_t fl = add_sat(habs(ut), na1);  // 0.0 on minimum edges, 1.0 elsewhere
        const uint32_t mo = fma(fl, dcs, c1s) ^ (ut & SIGN);
        const uint32_t bn = add(hmin(fma_relu(mo, ONE, bt[p]), C255), C1024) ^ 0x007f007fu;  // x bytes
        app[cw[p] & 0xffffu] = (int8_t)bn;
        if (2 * p + 1 < D) app[cw[p] >> 16] = (int8_t)(bn >> 16);
        mp[pi[p]] = (uint16_t)__byte_perm(add(mo, FRAME_C1152), 0, 0x0020);
    }
    odd += (m1 >> 15) & 1u;
}

// Dispatches a row to the unrolled update for its degree.  Rows of a level are
// sorted by degree, so the warps of a stage mostly take one case.
template <int KIND, int DT, bool EXACT>
__device__ __forceinline__ void frame_row_any(int deg, int8_t* app, const uint32_t* cp, uint16_t* mp, const uint4& po,
                                              bool first, bool noclip, int& odd, const uint16_t* lut)
{
    if (EXACT) return frame_row<KIND, DT>(app, cp, mp, po, first, noclip, odd, lut);
#define LDPC_FRAME_CASE(D)                                                                            \
    case D:                                                                                           \
        if (D <= DT) frame_row<KIND, (D <= DT ? D : DT)>(app, cp, mp, po, first, noclip, odd, lut);   \
        return;
    switch (deg) {
        LDPC_FRAME_CASE(1) LDPC_FRAME_CASE(2) LDPC_FRAME_CASE(3) LDPC_FRAME_CASE(4) LDPC_FRAME_CASE(5)
        LDPC_FRAME_CASE(6) LDPC_FRAME_CASE(7) LDPC_FRAME_CASE(8) LDPC_FRAME_CASE(9) LDPC_FRAME_CASE(10)
        LDPC_FRAME_CASE(11) LDPC_FRAME_CASE(12) LDPC_FRAME_CASE(13) LDPC_FRAME_CASE(14)
    }
#undef LDPC_FRAME_CASE
}

// Persistent CTAs: CTA c decodes frames c, c + G, c + 2G, ... of the launch (G = gridDim.x),
// one at a time, with slot c of the message scratch.  Shared memory: the frame's APP
// (npad bytes), for KIND_LEARNED the iteration's tables (512 bytes), then the ring of
// FRAME_RING stage slots (S.slot_sz bytes each).
//
// Copy protocol (the last thread of the CTA, in a warp of its own after the rows' warps, is
// the producer):
//   * stage g of the frame lives in ring slot (G0 + g) % FRAME_RING, whose mbarrier
//     completes its phase ((G0 + g) / FRAME_RING) & 1 when the stage's bytes landed;
//   * with at least FRAME_RING stages per iteration the producer issues stage g + 2 at
//     the start of stage g, after cp.async.bulk.wait_group 1: every message store but
//     stage g-1's has then completed, in particular stage g-2's (the slot being
//     refilled) and the store of the same stage one iteration earlier (the messages
//     being loaded); with fewer stages it issues stage g itself after wait_group 0;
//   * every stage stores its messages back (one bulk group per stage, the last
//     iteration included), and a frame ends with wait_group 0 and the wait for any
//     stage it had already issued, so the next frame starts with an idle ring.
template <int KIND, int DT, bool EXACT, bool ET>
__global__ void __maxnreg__(80) decode_frame_kernel(const Plan P, const Job J,
                                                                        const FrameStages S, long long frames)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int8_t* app = reinterpret_cast<int8_t*>(smem_raw);                       // [npad]
    uint16_t* slut = reinterpret_cast<uint16_t*>(smem_raw + P.npad);         // KIND_LEARNED
    unsigned char* ring = smem_raw + P.npad + (KIND == KIND_LEARNED ? 512 : 0);
    const int slot_sz = S.slot_sz;
    __shared__ __align__(8) unsigned long long bars[FRAME_RING];
    __shared__ unsigned s_odd[2];
    __shared__ int s_abort;
    const bool producer = threadIdx.x == blockDim.x - 1;
    const unsigned char* gmsg_c = S.msg + (long long)blockIdx.x * S.slot_bytes;
    unsigned char* gmsg = S.msg + (long long)blockIdx.x * S.slot_bytes;
    const int nst = S.nst;
    const int pd = nst >= FRAME_RING ? 2 : 0;  // stages issued ahead of their use
    if (threadIdx.x == 0) {
        for (int i = 0; i < FRAME_RING; i++) mbar_init(&bars[i]);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned long long G0 = 0;  // stages this CTA issued before the current frame
    for (long long lf = blockIdx.x; lf < frames; lf += gridDim.x) {
        const long long f = 4 * J.word0 + lf;
        const long long total = (long long)J.iters * nst;  // stages of the frame at most
        if (threadIdx.x < 2) s_odd[threadIdx.x] = 0;
        if (producer && pd)
            for (int g = 0; g < pd && g < total; g++)
                stage_load(S, S.st[g], ring + ((G0 + g) % FRAME_RING) * slot_sz, gmsg_c, false,
                           &bars[(G0 + g) % FRAME_RING]);
        long long issued = pd ? (total < pd ? total : pd) : 0;  // stages of this frame issued so far
        read_frame(P, J, f, [&](int v, int x) { app[v] = (int8_t)x; });
        __syncthreads();

        int executed = 0;
        bool passed = false;  // stopped by the syndrome early stop: every check holds
        long long g = 0;      // stage of the frame
        for (int it = 0; it < J.iters; it++) {
            int odd = 0;
            const bool first = it == 0;
            if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
            for (int l = 0; l < nst; l++, g++) {
                const unsigned long long gg = G0 + g;
                unsigned char* slot = ring + (gg % FRAME_RING) * slot_sz;
                // every thread keeps the same count of issued stages (G0 must agree); the
                // producer alone issues
                if (pd) {
                    if (g + pd < total) {
                        const long long gn = g + pd;
                        if (producer) {
                            asm volatile("cp.async.bulk.wait_group 1;" ::: "memory");
                            stage_load(S, S.st[gn % nst], ring + ((G0 + gn) % FRAME_RING) * slot_sz, gmsg_c,
                                       gn >= nst, &bars[(G0 + gn) % FRAME_RING]);
                        }
                        issued = gn + 1;
                    }
                } else {
                    if (producer) {
                        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
                        stage_load(S, S.st[l], slot, gmsg_c, !first, &bars[gg % FRAME_RING]);
                    }
                    issued = g + 1;
                }
                if (!mbar_wait(&bars[gg % FRAME_RING], (uint32_t)((gg / FRAME_RING) & 1))) s_abort = 1;
                const int t = threadIdx.x;
                const int2 hd = *reinterpret_cast<const int2*>(slot);  // rows, record bytes
                const int rows = hd.x;
                if (t < rows) {
                    const uint4 po = reinterpret_cast<const uint4*>(slot)[1];  // pair-slot offsets
                    const uint32_t rw = reinterpret_cast<const uint32_t*>(slot + FRAME_STAGE_HEADER)[t];
                    const int cols_off = FRAME_STAGE_HEADER + (4 * rows + 15) / 16 * 16;
                    const uint32_t* cp = reinterpret_cast<const uint32_t*>(slot + cols_off) + t;
                    uint16_t* mp = reinterpret_cast<uint16_t*>(slot + hd.y) + t;
                    const int cls = (int)(rw >> 8);
                    const bool noclip = J.quirk && first && cls;
                    frame_row_any<KIND, DT, EXACT>((int)(rw & 0xffu), app, cp, mp, po, first, noclip, odd,
                                                   slut + 128 * cls);
                }
                // the slot's messages, written by this CTA's threads, are read next by the
                // copy engine's store
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (s_abort) break;
                if (producer) {
                    const FrameStage st = S.st[l];
                    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gmsg + st.msg_off),
                                 "r"(smem_u32(slot + st.rec_bytes)), "r"(st.msg_bytes)
                                 : "memory");
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            }
            if (s_abort) break;
            executed = it + 1;
            if (ET) {
                if (odd_rows_within_slack(J, (unsigned)odd, it, s_odd) &&
                    !__syncthreads_or(frame_rows_unsatisfied(app, P))) {
                    passed = true;
                    break;
                }
            }
        }
        // the stages issued ahead that the frame did not use, and the message stores
        for (long long q = g; q < issued; q++) {
            const unsigned long long gg = G0 + q;
            if (!mbar_wait(&bars[gg % FRAME_RING], (uint32_t)((gg / FRAME_RING) & 1))) s_abort = 1;
        }
        if (producer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        G0 += issued;
        __syncthreads();
        if (s_abort) {
            if (threadIdx.x == 0) atomicExch(S.status, 1);
            return;
        }

        write_frame(P, J, f, [&](int v) { return (int)app[v]; });
        if (J.iters_out && threadIdx.x == 0) J.iters_out[lf] = executed;
        if (J.synd_out) {
            int bad = 0;
            if (!passed) bad = __syncthreads_or(frame_rows_unsatisfied(app, P));
            if (threadIdx.x == 0) J.synd_out[lf] = bad ? 0 : 1;
        }
        __syncthreads();  // the APP is refilled by the next frame
    }
}

// ---- two frames per CTA (decoder path 3 when two frames' APP fit) ----
//
// The same stages, ring, producer warp and copy protocol as decode_frame_kernel, but the CTA
// holds frames 2p and 2p + 1 of the launch as the two fp16 lanes of every word: its APP is
// one u16 per variable (the two frames' int8 values), and each thread updates its row for
// both frames at once, one edge per fp16x2 word, so the per-row work (record, dispatch,
// minima, magnitudes) is shared by two frames.  Stage record: a 64-byte header (word 0 =
// rows, word 1 = the record's bytes; bytes 32..63 = edge-slot offsets eoff[0..15], u16:
// edge slot j holds edge j of every row of degree > j, the stage's row t at eoff[j] + t),
// the row words (u32: degree | class << 8) padded to 16 bytes, then the columns, u16 per
// edge-slot entry, padded to 16.  Messages: u16 per edge-slot entry (the two frames'
// bytes 128 - msg), same index.  Each frame stops on its own: when it does, its decisions
// and count are written at once; its lane then keeps running beside the other frame (the
// lanes never mix, so that changes nothing the frame wrote).

constexpr int FRAME2_HEADER = 64;

// One check row of two frames (fp16 lanes 0 and 1 = frames 2p, 2p+1): the reference's
// per-byte update (CUDA_OMS_SIMD.cu:40-134) in the biased negated arithmetic of namespace
// h2, one edge per word.  cp / mp: this row's entry of edge slot 0 of the columns / the
// messages; eo: the edge-slot offsets (u16 pairs).  odd: odd rows of frame 0 | frame 1 << 16.
template <int KIND, int D>
__device__ __forceinline__ void frame2_row(uint16_t* app, const uint16_t* cp, uint16_t* mp, const uint32_t (&eo)[8],
                                           bool first, bool noclip, uint32_t& odd, const uint16_t* lut)
{
    using namespace h2;
    uint32_t bt[D];
    int ci[D], ei[D];
    uint32_t mn1 = C127, mn2 = C127;
#pragma unroll
    for (int j = 0; j < D; j++) {
        ei[j] = (int)((j & 1) ? (eo[j >> 1] >> 16) : (eo[j >> 1] & 0xffffu));
        ci[j] = cp[ei[j]];
    }
#pragma unroll
    for (int j = 0; j < D; j++) {
        // x bytes of the two frames; 127 - x as an unsigned byte is x ^ 0x7f
        const uint32_t w = (uint32_t)app[ci[j]] ^ 0x7f7fu;
        const uint32_t b = add(__byte_perm(w, 0x6464u, 0x5140), CNEG1024);
        uint32_t u = 0;  // negated old messages
        if (!first) u = add(__byte_perm((uint32_t)mp[ei[j]], 0x6464u, 0x5140), FRAME_CNEG1152);
        bt[j] = hmin(fma_relu(u, NEG1, b), C255);
        const uint32_t ut = add(bt[j], CNEG127);
        const uint32_t mx = max_xs(ut, mn1);
        mn1 = min_xs(mn1, ut);
        mn2 = min_xs(mn2, mx);
    }
    const uint32_t a1 = habs(mn1), a2 = habs(mn2);
    uint32_t c1, c2;
    if (KIND == KIND_LEARNED) {
        // the integer tables of the I8 packing, one lookup per frame: c1 = lut[min2], c2 = lut[min1]
        const uint32_t i2 = add(a2, C1024), i1 = add(a1, C1024);
        const uint32_t c1l = lut[i2 & 0x7fu], c1h = lut[(i2 >> 16) & 0x7fu];
        const uint32_t c2l = lut[i1 & 0x7fu], c2h = lut[(i1 >> 16) & 0x7fu];
        c1 = add(0x64006400u | c1l | (c1h << 16), CNEG1024);
        c2 = add(0x64006400u | c2l | (c2h << 16), CNEG1024);
    } else {
        h2::mags<KIND>(a1, a2, noclip, c1, c2, 0u, 0u);
    }
    const uint32_t c1s = c1 | (mn1 & SIGN), c2s = c2 | (mn1 & SIGN);
    const uint32_t dcs = sub(c2s, c1s), na1 = a1 ^ SIGN;
#pragma unroll
    for (int j = 0; j < D; j++) {
        const uint32_t ut = add(bt[j], CNEG127);
        const uint32_t fl = add_sat(habs(ut), na1);  // 0.0 on minimum edges, 1.0 elsewhere
        const uint32_t mo = fma(fl, dcs, c1s) ^ (ut & SIGN);
        const uint32_t bn = add(hmin(fma_relu(mo, ONE, bt[j]), C255), C1024) ^ 0x007f007fu;  // x bytes 0, 2
        app[ci[j]] = (uint16_t)__byte_perm(bn, 0, 0x0020);
        mp[ei[j]] = (uint16_t)__byte_perm(add(mo, FRAME_C1152), 0, 0x0020);
    }
    odd += ((mn1 >> 15) & 1u) | ((mn1 >> 31) << 16);
}

template <int KIND, int DT, bool EXACT>
__device__ __forceinline__ void frame2_row_any(int deg, uint16_t* app, const uint16_t* cp, uint16_t* mp,
                                               const uint32_t (&eo)[8], bool first, bool noclip, uint32_t& odd,
                                               const uint16_t* lut)
{
    if (EXACT) return frame2_row<KIND, DT>(app, cp, mp, eo, first, noclip, odd, lut);
#define LDPC_FRAME2_CASE(D)                                                                           \
    case D:                                                                                           \
        if (D <= DT) frame2_row<KIND, (D <= DT ? D : DT)>(app, cp, mp, eo, first, noclip, odd, lut);  \
        return;
    switch (deg) {
        LDPC_FRAME2_CASE(1) LDPC_FRAME2_CASE(2) LDPC_FRAME2_CASE(3) LDPC_FRAME2_CASE(4) LDPC_FRAME2_CASE(5)
        LDPC_FRAME2_CASE(6) LDPC_FRAME2_CASE(7) LDPC_FRAME2_CASE(8) LDPC_FRAME2_CASE(9) LDPC_FRAME2_CASE(10)
        LDPC_FRAME2_CASE(11) LDPC_FRAME2_CASE(12) LDPC_FRAME2_CASE(13) LDPC_FRAME2_CASE(14)
    }
#undef LDPC_FRAME2_CASE
}

// Byte k of the result is nonzero in some thread when frame k (lane k of the APP words) has
// a check of odd hard-decision parity (x > 0 is bit 1)
__device__ __forceinline__ uint32_t frame2_rows_odd(const uint16_t* app, const Plan& P)
{
    uint32_t bad = 0;
    for (int r = threadIdx.x; r < P.m; r += blockDim.x) {
        const int d = __ldg(P.rowdeg + r);
        uint32_t acc = 0;
        for (int j = 0; j < d; j++) acc ^= __vcmpgts4((uint32_t)app[__ldg(P.cols + j * P.m + r)], 0u);
        bad |= acc;
    }
    return bad & 0xffffu;
}

// Persistent CTAs: CTA c decodes frame pairs c, c + G, ... (pair p = frames 2p, 2p + 1 of the
// launch), with slot c of the message scratch.  Shared memory: the pair's APP (2 npad bytes),
// for KIND_LEARNED the iteration's tables (512 bytes), then the ring.  The copy protocol is
// decode_frame_kernel's.
template <int KIND, int DT, bool EXACT, bool ET>
__global__ void __maxnreg__(120) decode_frame2_kernel(const Plan P, const Job J, const FrameStages S, long long frames)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint16_t* app = reinterpret_cast<uint16_t*>(smem_raw);                   // [npad]
    int8_t* app8 = reinterpret_cast<int8_t*>(smem_raw);                      // byte 2v + k: frame k
    uint16_t* slut = reinterpret_cast<uint16_t*>(smem_raw + 2 * P.npad);     // KIND_LEARNED
    unsigned char* ring = smem_raw + 2 * P.npad + (KIND == KIND_LEARNED ? 512 : 0);
    const int slot_sz = S.slot_sz;
    __shared__ __align__(8) unsigned long long bars[FRAME_RING];
    __shared__ unsigned s_odd[2];
    __shared__ int s_abort;
    const bool producer = threadIdx.x == blockDim.x - 1;
    const unsigned char* gmsg_c = S.msg + (long long)blockIdx.x * S.slot_bytes;
    unsigned char* gmsg = S.msg + (long long)blockIdx.x * S.slot_bytes;
    const int nst = S.nst;
    const int pd = nst >= FRAME_RING ? 2 : 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < FRAME_RING; i++) mbar_init(&bars[i]);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned long long G0 = 0;
    const long long pairs = frames >> 1;
    for (long long lp = blockIdx.x; lp < pairs; lp += gridDim.x) {
        const long long lf0 = 2 * lp, f0 = 4 * J.word0 + lf0;
        const long long total = (long long)J.iters * nst;
        if (threadIdx.x < 2) s_odd[threadIdx.x] = 0;
        if (producer && pd)
            for (int g = 0; g < pd && g < total; g++)
                stage_load(S, S.st[g], ring + ((G0 + g) % FRAME_RING) * slot_sz, gmsg_c, false,
                           &bars[(G0 + g) % FRAME_RING]);
        long long issued = pd ? (total < pd ? total : pd) : 0;
        read_frame(P, J, f0, [&](int v, int x) { app8[2 * v] = (int8_t)x; });
        read_frame(P, J, f0 + 1, [&](int v, int x) { app8[2 * v + 1] = (int8_t)x; });
        __syncthreads();

        unsigned live = 3u;  // frames of the pair still decoding (the same in every thread)
        int its[2] = {0, 0};
        int executed = 0;
        long long g = 0;
        for (int it = 0; it < J.iters; it++) {
            uint32_t odd = 0;
            const bool first = it == 0;
            if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
            for (int l = 0; l < nst; l++, g++) {
                const unsigned long long gg = G0 + g;
                unsigned char* slot = ring + (gg % FRAME_RING) * slot_sz;
                if (pd) {
                    if (g + pd < total) {
                        const long long gn = g + pd;
                        if (producer) {
                            asm volatile("cp.async.bulk.wait_group 1;" ::: "memory");
                            stage_load(S, S.st[gn % nst], ring + ((G0 + gn) % FRAME_RING) * slot_sz, gmsg_c,
                                       gn >= nst, &bars[(G0 + gn) % FRAME_RING]);
                        }
                        issued = gn + 1;
                    }
                } else {
                    if (producer) {
                        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
                        stage_load(S, S.st[l], slot, gmsg_c, !first, &bars[gg % FRAME_RING]);
                    }
                    issued = g + 1;
                }
                if (!mbar_wait(&bars[gg % FRAME_RING], (uint32_t)((gg / FRAME_RING) & 1))) s_abort = 1;
                const int t = threadIdx.x;
                const int2 hd = *reinterpret_cast<const int2*>(slot);  // rows, record bytes
                if (t < hd.x) {
                    const uint4 e0 = reinterpret_cast<const uint4*>(slot)[2], e1 = reinterpret_cast<const uint4*>(slot)[3];
                    const uint32_t eo[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
                    const uint32_t rw = reinterpret_cast<const uint32_t*>(slot + FRAME2_HEADER)[t];
                    const int cols_off = FRAME2_HEADER + (4 * hd.x + 15) / 16 * 16;
                    const uint16_t* cp = reinterpret_cast<const uint16_t*>(slot + cols_off) + t;
                    uint16_t* mp = reinterpret_cast<uint16_t*>(slot + hd.y) + t;
                    const int cls = (int)(rw >> 8);
                    const bool noclip = J.quirk && first && cls;
                    frame2_row_any<KIND, DT, EXACT>((int)(rw & 0xffu), app, cp, mp, eo, first, noclip, odd,
                                                    slut + 128 * cls);
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (s_abort) break;
                if (producer) {
                    const FrameStage st = S.st[l];
                    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gmsg + st.msg_off),
                                 "r"(smem_u32(slot + st.rec_bytes)), "r"(st.msg_bytes)
                                 : "memory");
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            }
            if (s_abort) break;
            executed = it + 1;
            if (ET) {
                const unsigned tot = odd_rows_total(odd, it, s_odd);
                unsigned gate = live & (((tot & 0xffffu) <= J.early_slack ? 1u : 0u) |
                                        ((tot >> 16) <= J.early_slack ? 2u : 0u));
                if (gate) {
                    const uint32_t bad = frame2_rows_odd(app, P);
                    if ((gate & 1u) && __syncthreads_or(bad & 0xffu)) gate &= ~1u;
                    if ((gate & 2u) && __syncthreads_or(bad & 0xff00u)) gate &= ~2u;
                    for (int k = 0; k < 2; k++) {
                        if (!((gate >> k) & 1u)) continue;
                        // frame k stops here: its decisions, its count, its syndrome flag
                        write_frame(P, J, f0 + k, [&](int v) { return (int)app8[2 * v + k]; });
                        its[k] = it + 1;
                        if (threadIdx.x == 0) {
                            if (J.iters_out) J.iters_out[lf0 + k] = it + 1;
                            if (J.synd_out) J.synd_out[lf0 + k] = 1;
                        }
                    }
                    live &= ~gate;
                    if (!live) break;
                    if (gate) __syncthreads();  // write_frame read the APP the next stage updates
                }
            }
        }
        for (long long q = g; q < issued; q++) {
            const unsigned long long gg = G0 + q;
            if (!mbar_wait(&bars[gg % FRAME_RING], (uint32_t)((gg / FRAME_RING) & 1))) s_abort = 1;
        }
        if (producer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        G0 += issued;
        __syncthreads();
        if (s_abort) {
            if (threadIdx.x == 0) atomicExch(S.status, 1);
            return;
        }
        // the frames still live ran every iteration
        uint32_t bad = 0;
        if (live && J.synd_out) bad = frame2_rows_odd(app, P);
        for (int k = 0; k < 2; k++) {
            if (!((live >> k) & 1u)) continue;
            write_frame(P, J, f0 + k, [&](int v) { return (int)app8[2 * v + k]; });
            if (J.iters_out && threadIdx.x == 0) J.iters_out[lf0 + k] = executed;
            if (J.synd_out) {
                const int o = __syncthreads_or((bad >> (8 * k)) & 0xffu);
                if (threadIdx.x == 0) J.synd_out[lf0 + k] = o ? 0 : 1;
            }
        }
        (void)its;
        __syncthreads();  // the APP is refilled by the next pair
    }
}

}  // namespace ldpc
