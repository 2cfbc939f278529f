// Level-scheduled, row-layered fixed-point LDPC decoder kernel for sm_100a.
//
// One CTA decodes one group of 4 frames (the 4 frames 4g..4g+3 that the
// reference packs into 32-bit word g), with the whole decoder state on chip:
// the APP array and every c->v message of the group live in shared memory for
// all iterations.  The reference instead gives one thread per word and walks
// every check row serially with APP and messages in global memory
// (decoder_oms/cuda/CUDA_OMS_SIMD.cu:25-248, launched with nb_frames/128 CTAs
// of 128 threads, decoder_oms/CGPU_Decoder_OMS_SIMD.cu:119).
//
// Bit-exactness with the reference's strictly row-serial, update-in-place
// order comes from the schedule built on the host (ldpc_b200.cu): rows are
// grouped into "levels" such that a row's level is one more than the highest
// level of any earlier row sharing a variable with it.  Rows of one level touch
// disjoint variables, so the CTA's threads update them concurrently and the
// result equals the serial order; a barrier separates levels and iterations.
// Rows are renumbered in schedule order (r'), so the threads of a level read
// consecutive entries of the column table and of the message store.
//
// Per-word early termination (2NMS): the OR over rows of the extrinsic sign
// parity decides, from the second iteration on, whether the word stops
// (decoder_2nms/cuda/CUDA_2NMS_SIMD.cu:160-290); here that OR is reduced over
// the CTA with __syncthreads_or.
#pragma once
#include <cstdint>
#include "channel.cuh"
#include "packs.cuh"

namespace ldpc {

struct Plan {
    int n;           // variables
    int npad;        // n rounded up to 16 (APP row stride in shared memory)
    int m;           // rows (checks)
    int dmax;        // largest row degree
    int nlevels;     // levels per iteration
    const uint16_t* cols;   // [dmax][m] variable of edge j of row r' (schedule order)
    const uint8_t* rowdeg;  // [m]
    const uint8_t* rowcls;  // [m] 1 = reference's second degree group
    const int2* levels;     // [nlevels] (first r', row count)
    const int32_t* edge_orig;  // [dmax][m] edge index in table order (state dumps)
    // the flooding schedule: variable v's edges as message indices j * m + r' (schedule
    // order), vedge[vptr[v] .. vptr[v + 1])
    const int32_t* vptr;
    const int32_t* vedge;
};

struct Job {
    const int8_t* llr;    // frame-major int8 [4*words][n] (or word-interleaved, see interleaved)
    void* out;            // hard decisions (LDPC_OUT_BYTES or LDPC_OUT_PACKED)
    int out_packed;
    int interleaved;      // 1: llr is word[v*total_words + g] (xMS input)
    long long total_words;  // word stride of the interleaved layout and of the state dumps
    long long word0;      // first word of this launch within the batch
    int iters;
    int quirk;            // 1: OMS first-iteration no-clip on second-group rows
    int early;            // 1: syndrome early stop per word (LDPC_FLAG_EARLY_STOP)
    unsigned early_slack;  // evaluate the syndrome when at most this many (row, frame) pairs were odd
    int32_t* iters_out;   // [words] or null
    uint8_t* synd_out;    // [4 * words] per-frame syndrome flags (1: every check satisfied) or null
    int8_t* app_out;      // state dumps (reference device layouts) or null
    int8_t* msg_out;
    // fused simulation (llr == null): the channel generates the LLRs in the
    // prologue and the epilogue counts errors instead of (or as well as) writing
    // hard decisions
    int gen;              // 1: generate LLRs (AWGN channel) instead of reading llr
    float sigma;
    unsigned long long seed, offset;
    const uint8_t* cw;    // transmitted codewords (frame-major 0/1), null = all-zero
    long long n_cw;
    unsigned long long* counts;  // [3] frames, bit errors, frame errors (or null)
    int n_vars;           // bits counted per frame
    // KIND_LEARNED: magnitude tables [lut_its][2 row groups][128] (see packs.cuh)
    const uint16_t* lut;
    int lut_its;
};

// KIND_LEARNED: loads the tables of iteration `it` into shared memory (256 entries);
// called by every thread at the top of an iteration, ends with a barrier
__device__ __forceinline__ void load_iteration_lut(const Job& J, int it, uint16_t* slut)
{
    const int t = it < J.lut_its ? it : J.lut_its - 1;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) slut[i] = J.lut[t * 256 + i];
    __syncthreads();
}

// ---- prologue / epilogue: frame-major global <-> packed shared memory ----

// 4x4 byte transpose: in[k] = 4 consecutive bytes of frame k; out[j] = byte j of all 4 frames
__device__ __forceinline__ void transpose4x4(const uint32_t (&a)[4], uint32_t (&w)[4])
{
    uint32_t t0 = __byte_perm(a[0], a[1], 0x5140), t1 = __byte_perm(a[2], a[3], 0x5140);
    uint32_t t2 = __byte_perm(a[0], a[1], 0x7362), t3 = __byte_perm(a[2], a[3], 0x7362);
    w[0] = __byte_perm(t0, t1, 0x5410);
    w[1] = __byte_perm(t0, t1, 0x7632);
    w[2] = __byte_perm(t2, t3, 0x5410);
    w[3] = __byte_perm(t2, t3, 0x7632);
}

// Reads the group's 4 frames; calls put(v, word) with the 4-frame byte word of variable v.
template <class F>
__device__ __forceinline__ void read_group(const Plan& P, const Job& J, long long g, F put)
{
    const int n = P.n;
    if (J.gen) {
        // frames 4g..4g+3 of the channel stream: sample s = frame * n + v
        if ((n & 3) == 0) {
            // 4 consecutive samples of a frame share one Philox call (counter s / 4)
            for (int q = threadIdx.x; q < (n >> 2); q += blockDim.x) {
                uint32_t a[4], w[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const unsigned long long f = 4ull * g + k;
                    const unsigned long long s0 = f * (unsigned long long)n + 4 * q;
                    float u[4], gs[4];
                    uniforms4(s0 >> 2, J.seed, J.offset, u);
                    box_muller4(u, gs);
                    uint32_t x = 0;
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        float mean = -1.0f;
                        if (J.cw) mean = J.cw[(f % (unsigned long long)J.n_cw) * n + 4 * q + i] ? 1.0f : -1.0f;
                        x |= (uint32_t)(uint8_t)quantise(mean + J.sigma * gs[i]) << (8 * i);
                    }
                    a[k] = x;
                }
                transpose4x4(a, w);
#pragma unroll
                for (int j = 0; j < 4; j++) put(4 * q + j, w[j]);
            }
        } else {
            for (int v = threadIdx.x; v < n; v += blockDim.x) {
                uint32_t w = 0;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const unsigned long long f = 4ull * g + k, s = f * (unsigned long long)n + v;
                    float mean = -1.0f;
                    if (J.cw) mean = J.cw[(f % (unsigned long long)J.n_cw) * n + v] ? 1.0f : -1.0f;
                    w |= (uint32_t)(uint8_t)awgn_sample(s, J.seed, J.offset, J.sigma, mean) << (8 * k);
                }
                put(v, w);
            }
        }
        return;
    }
    if (J.interleaved) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(J.llr);
        for (int v = threadIdx.x; v < n; v += blockDim.x) put(v, __ldg(src + (long long)v * J.total_words + g));
    } else if ((n & 3) == 0) {
        const uint32_t* f0 = reinterpret_cast<const uint32_t*>(J.llr + (4 * (g - J.word0)) * (long long)n);
        const int n4 = n >> 2;
        // the loads of B loop trips are issued before any of them is used, so that one
        // global latency, not B, starts each word
        constexpr int B = 4;
        for (int q0 = threadIdx.x; q0 < n4; q0 += B * blockDim.x) {
            uint32_t a[B][4];
#pragma unroll
            for (int t = 0; t < B; t++) {
                const int q = q0 + t * blockDim.x;
                if (q < n4)
#pragma unroll
                    for (int k = 0; k < 4; k++) a[t][k] = __ldg(f0 + k * n4 + q);
            }
#pragma unroll
            for (int t = 0; t < B; t++) {
                const int q = q0 + t * blockDim.x;
                if (q < n4) {
                    uint32_t w[4];
                    transpose4x4(a[t], w);
#pragma unroll
                    for (int j = 0; j < 4; j++) put(4 * q + j, w[j]);
                }
            }
        }
    } else {
        const int8_t* f0 = J.llr + (4 * (g - J.word0)) * (long long)n;
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) w |= (uint32_t)(uint8_t)__ldg(f0 + k * n + v) << (8 * k);
            put(v, w);
        }
    }
}

// Error counting of the group's 4 frames against the transmitted codewords
// (ber_analyzer/CErrorAnalyzer.cpp:142-158): bits among the first n_vars whose
// decision (x > 0) differs from the codeword bit.  Every thread of the CTA calls it.
template <class F>
__device__ __forceinline__ void count_group_errors(const Plan& P, const Job& J, long long g, F get, int kmask)
{
    __shared__ int part[4][32];
    int e[4] = {0, 0, 0, 0};
    for (int v = threadIdx.x; v < J.n_vars; v += blockDim.x) {
        uint32_t h = __vsetgts4(get(v), 0u);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!((kmask >> k) & 1)) continue;
            int bit = (h >> (8 * k)) & 1;
            int ref = J.cw ? (J.cw[((4ull * g + k) % (unsigned long long)J.n_cw) * P.n + v] != 0) : 0;
            e[k] += bit != ref;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
#pragma unroll
        for (int o = 16; o; o >>= 1) e[k] += __shfl_xor_sync(0xffffffffu, e[k], o);
    }
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; k++) part[k][threadIdx.x >> 5] = e[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long be = 0, fe = 0, nf = 0;
        for (int k = 0; k < 4; k++) {
            if (!((kmask >> k) & 1)) continue;
            int t = 0;
            for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) t += part[k][w];
            be += t;
            fe += t != 0;
            nf++;
        }
        atomicAdd(J.counts + 0, nf);
        atomicAdd(J.counts + 1, be);
        atomicAdd(J.counts + 2, fe);
    }
}

// Writes hard decisions; get(v) returns the 4-frame byte word (values as x) of variable v.
template <class F>
__device__ __forceinline__ void write_group(const Plan& P, const Job& J, long long g, F get, int kmask = 0xF)
{
    const int n = P.n;
    const long long lg = g - J.word0;
    if (J.counts) count_group_errors(P, J, g, get, kmask);
    if (!J.out) return;
    if (!J.out_packed) {
        uint8_t* o = reinterpret_cast<uint8_t*>(J.out) + 4 * lg * n;
        if ((n & 3) == 0) {
            const int n4 = n >> 2;
            uint32_t* o32 = reinterpret_cast<uint32_t*>(o);
            for (int q = threadIdx.x; q < n4; q += blockDim.x) {
                uint32_t a[4], w[4];
#pragma unroll
                for (int j = 0; j < 4; j++) a[j] = __vsetgts4(get(4 * q + j), 0u);
                transpose4x4(a, w);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if ((kmask >> k) & 1) o32[k * n4 + q] = w[k];
            }
        } else {
            for (int v = threadIdx.x; v < n; v += blockDim.x) {
                uint32_t h = __vsetgts4(get(v), 0u);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if ((kmask >> k) & 1) o[k * n + v] = (h >> (8 * k)) & 1;
            }
        }
    } else {
        const int nb = (n + 7) >> 3;
        uint8_t* o = reinterpret_cast<uint8_t*>(J.out) + 4 * lg * nb;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            uint32_t acc = 0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                int v = 8 * b + j;
                if (v < n) acc |= __vsetgts4(get(v), 0u) << j;
            }
#pragma unroll
            for (int k = 0; k < 4; k++)
                if ((kmask >> k) & 1) o[k * nb + b] = (acc >> (8 * k)) & 0xff;
        }
    }
}

// ---- pack-specific state access (x values as 4-frame byte words) ----

template <class PK> struct Access;

template <> struct Access<PackSIMD4> {
    __device__ __forceinline__ static void put(uint32_t* app, int npad, int v, uint32_t w) { app[v] = w; }
    __device__ __forceinline__ static uint32_t get(const uint32_t* app, int npad, int v) { return app[v]; }
    __device__ __forceinline__ static uint32_t get_msg(const uint32_t* msg, int stride, int idx) { return msg[idx]; }
};

template <> struct Access<PackF16x2> {
    // x bytes of frames k0, k0+1 -> biased negated pair b = 127 - x.  As an unsigned
    // byte, 127 - x is x ^ 0x7f for every int8 x; under the byte 0x64 it becomes the
    // fp16 bit pattern of 1024 + (127 - x), and subtracting 1024 is exact.
    __device__ __forceinline__ static uint32_t pair(uint32_t w, int k0)
    {
        const uint32_t y = w ^ 0x7f7f7f7fu;
        return h2::add(__byte_perm(y, 0x6464u, k0 == 0 ? 0x4140 : 0x4342), h2::CNEG1024);
    }
    __device__ __forceinline__ static void put(uint32_t* app, int npad, int v, uint32_t w)
    {
        app[v] = pair(w, 0);
        app[npad + v] = pair(w, 2);
    }
    // the inverse of pair() for both pair-words: b + 1024 has the integer b in its low
    // byte (b is an integer in [0, 255]), and x = 127 - b is that byte ^ 0x7f
    __device__ __forceinline__ static uint32_t unbias(uint32_t lo, uint32_t hi)
    {
        return __byte_perm(h2::add(lo, h2::C1024), h2::add(hi, h2::C1024), 0x6420) ^ 0x7f7f7f7fu;
    }
    __device__ __forceinline__ static uint32_t get(const uint32_t* app, int npad, int v)
    {
        return unbias(app[v], app[npad + v]);
    }
    __device__ __forceinline__ static uint32_t get_msg(const uint32_t* msg, int stride, int idx)
    {
        auto x = [](uint16_t h) { return (uint32_t)(uint8_t)(int8_t)(-__half2int_rn(__ushort_as_half(h))); };
        uint32_t lo = msg[idx], hi = msg[stride + idx];
        return x(lo & 0xffff) | (x(lo >> 16) << 8) | (x(hi & 0xffff) << 16) | (x(hi >> 16) << 24);
    }
};

// one pair-word (frames 2h, 2h+1 of the word); get/get_msg leave the other 2 bytes 0
struct AccessHalf {
    __device__ __forceinline__ static void put(uint32_t* app, int v, uint32_t w, int h)
    {
        app[v] = Access<PackF16x2>::pair(w, 2 * h);
    }
    __device__ __forceinline__ static uint32_t spread(uint32_t two, int h) { return two << (16 * h); }
    __device__ __forceinline__ static uint32_t get(const uint32_t* app, int v, int h)
    {
        return spread(Access<PackF16x2>::unbias(app[v], 0x57f057f0u) & 0xffffu, h);
    }
    __device__ __forceinline__ static uint32_t get_msg(const uint32_t* msg, int idx, int h)
    {
        auto x = [](uint16_t hv) { return (uint32_t)(uint8_t)(int8_t)(-__half2int_rn(__ushort_as_half(hv))); };
        uint32_t lo = msg[idx];
        return spread(x(lo & 0xffff) | (x(lo >> 16) << 8), h);
    }
};

template <> struct Access<PackI8> {
    __device__ __forceinline__ static void put(int8_t* app, int npad, int v, uint32_t w)
    {
#pragma unroll
        for (int k = 0; k < 4; k++) app[k * npad + v] = (int8_t)(w >> (8 * k));
    }
    __device__ __forceinline__ static uint32_t get(const int8_t* app, int npad, int v)
    {
        uint32_t w = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) w |= (uint32_t)(uint8_t)app[k * npad + v] << (8 * k);
        return w;
    }
    __device__ __forceinline__ static uint32_t get_msg(const int8_t* msg, int stride, int idx)
    {
        uint32_t w = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) w |= (uint32_t)(uint8_t)(int8_t)(-msg[k * stride + idx]) << (8 * k);
        return w;
    }
};

// ---- syndrome early stop ----
// After iteration `it`, the word stops when at most J.early_slack (row, frame)
// pairs had odd extrinsic sign parity during the iteration (each thread's `odd`
// counts its own; the row updates compute the parities anyway) and the hard
// decisions of its frames then satisfy every check.  The count goes through a
// double-buffered shared counter, so one barrier serves both the sum and the
// reset for the next iteration.  Uniform across the CTA.
// The CTA's sum of `odd` in iteration it (s_odd: two words, zeroed before the first
// iteration; each iteration clears the other's word).  Every thread of the CTA calls it.
__device__ __forceinline__ unsigned odd_rows_total(unsigned odd, int it, unsigned* s_odd)
{
    // one shared atomic per warp, not per thread
    const unsigned lanes = __activemask();
    const unsigned w = __reduce_add_sync(lanes, odd);
    if (w && (int)(threadIdx.x & 31) == __ffs(lanes) - 1) atomicAdd(&s_odd[it & 1], w);
    __syncthreads();
    const unsigned total = s_odd[it & 1];
    if (threadIdx.x == 0) s_odd[(it + 1) & 1] = 0;
    return total;
}

__device__ __forceinline__ bool odd_rows_within_slack(const Job& J, unsigned odd, int it, unsigned* s_odd)
{
    return odd_rows_total(odd, it, s_odd) <= J.early_slack;
}

// true in some thread when a check has odd hard-decision parity (x > 0 is bit 1)
// in one of the CTA's frames; rows are spread over the CTA's threads
template <class PK>
__device__ __forceinline__ bool rows_unsatisfied(const typename PK::S* app, const Plan& P)
{
    bool bad = false;
    for (int r = threadIdx.x; r < P.m; r += blockDim.x) {
        const int d = __ldg(P.rowdeg + r);
        uint32_t acc = 0;
        for (int j = 0; j < d; j++) acc ^= __vcmpgts4(Access<PK>::get(app, P.npad, __ldg(P.cols + j * P.m + r)), 0u);
        bad |= acc != 0;
    }
    return bad;
}

// Per-byte odd-parity mask of the CTA's checks: byte k is nonzero in some thread when
// frame k has a check of odd hard-decision parity (x > 0 is bit 1); get(v) returns the
// 4-frame byte word (values as x) of variable v.  Rows are spread over the CTA's threads.
template <class F>
__device__ __forceinline__ uint32_t rows_odd_mask(const Plan& P, F get)
{
    uint32_t bad = 0;
    for (int r = threadIdx.x; r < P.m; r += blockDim.x) {
        const int d = __ldg(P.rowdeg + r);
        uint32_t acc = 0;
        for (int j = 0; j < d; j++) acc ^= __vcmpgts4(get(__ldg(P.cols + j * P.m + r)), 0u);
        bad |= acc;
    }
    return bad;
}

// Writes the syndrome flags of frames first + k (k in kmask): 1 when no thread saw an odd
// check of frame k in its `bad` mask (byte k, or bit k with bits set).  Every thread of the
// CTA calls it (one barrier per frame of kmask).
__device__ __forceinline__ void write_syndrome_flags(const Job& J, long long first, uint32_t bad, int kmask,
                                                     bool bits = false)
{
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (!((kmask >> k) & 1)) continue;
        const int odd = __syncthreads_or(bits ? (bad >> k) & 1u : (bad >> (8 * k)) & 0xffu);
        if (threadIdx.x == 0) J.synd_out[first + k] = odd ? 0 : 1;
    }
}

// ---- one check row over all storage words of the group ----

template <class PK, int KIND, int DT, bool EXACT>
__device__ __forceinline__ void row_update(typename PK::S* app, typename PK::S* msg, const Plan& P,
                                           int r, int d, bool noclip, typename PK::R& ov, const uint16_t* lut)
{
    using R = typename PK::R;
    int v[DT];
#pragma unroll
    for (int j = 0; j < DT; j++)
        if (EXACT || j < d) v[j] = __ldg(P.cols + j * P.m + r);
    const int mstride = P.dmax * P.m;
#pragma unroll
    for (int w = 0; w < PK::WPC; w++) {
        typename PK::S* A = app + w * P.npad;
        typename PK::S* M = msg + w * mstride;
        R x[DT], mm[DT];
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                x[j] = PK::ld_app(A + v[j]);
                mm[j] = PK::ld_msg(M + j * P.m + r);
            }
        }
        PK::template update<KIND, DT, EXACT>(x, mm, d, noclip, ov, lut);
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                PK::st_msg(M + j * P.m + r, mm[j]);
                PK::st_app(A + v[j], x[j]);
            }
        }
    }
}

// row_update() for PackSIMD4 with the odd rows counted per frame (PackSIMD4::update_lanes)
template <int KIND, int DT, bool EXACT>
__device__ __forceinline__ void row_update_lanes(uint32_t* app, uint32_t* msg, const Plan& P, int r, int d,
                                                 bool noclip, uint32_t& oc01, uint32_t& oc23, const uint16_t* lut)
{
    int v[DT];
    uint32_t x[DT], mm[DT];
#pragma unroll
    for (int j = 0; j < DT; j++) {
        if (EXACT || j < d) {
            v[j] = __ldg(P.cols + j * P.m + r);
            x[j] = app[v[j]];
            mm[j] = msg[j * P.m + r];
        }
    }
    PackSIMD4::template update_lanes<KIND, DT, EXACT>(x, mm, d, noclip, oc01, oc23, lut);
#pragma unroll
    for (int j = 0; j < DT; j++) {
        if (EXACT || j < d) {
            msg[j * P.m + r] = mm[j];
            app[v[j]] = x[j];
        }
    }
}

// The CTA's per-frame odd-row totals of iteration it: a holds frames 0 and 1 in its 16-bit
// halves, b frames 2 and 3 (each total at most m < 2^16).  s4: four words, zeroed before the
// first iteration; each iteration uses one pair and clears the other.  Every thread calls it.
__device__ __forceinline__ uint2 odd_rows_total_lanes(uint32_t a, uint32_t b, int it, unsigned* s4)
{
    const unsigned lanes = __activemask();
    const unsigned wa = __reduce_add_sync(lanes, a), wb = __reduce_add_sync(lanes, b);
    unsigned* cur = s4 + 2 * (it & 1);
    if ((int)(threadIdx.x & 31) == __ffs(lanes) - 1) {
        if (wa) atomicAdd(cur, wa);
        if (wb) atomicAdd(cur + 1, wb);
    }
    __syncthreads();
    const uint2 t = make_uint2(cur[0], cur[1]);
    if (threadIdx.x == 0) {
        unsigned* nxt = s4 + 2 * ((it + 1) & 1);
        nxt[0] = 0;
        nxt[1] = 0;
    }
    return t;
}

// Decodes word g (4 frames) with the level schedule, all state in the CTA's shared
// memory (smem_raw: APP, messages, then the LEARNED table).  Every thread of the
// CTA calls it; it has no barrier after its last shared-memory access, so a
// caller that reuses the memory synchronises first.
// PF (PackSIMD4 only, LDPC_FLAG_EARLY_STOP_FRAMES): each frame (byte lane) stops on its own:
// after an iteration in which at most J.early_slack of its rows had odd extrinsic parity
// and its hard decisions satisfy every check, its decisions are written and its count is
// recorded (d_iters_out: one count per frame); the lanes are independent, so what it writes
// is what decoding that frame alone gives.  The CTA goes on while a frame is live.
// s_odd: two words, four with PF.
template <class PK, int KIND, int DT, bool EXACT, bool PF = false>
__device__ __forceinline__ void decode_word_levels(const Plan& P, const Job& J, long long g, unsigned char* smem_raw,
                                                   unsigned* s_odd)
{
    static_assert(!PF || (PK::ID == 0 && KIND != KIND_2NMS), "per-frame early stop: PackSIMD4, not 2NMS");
    using S = typename PK::S;
    using R = typename PK::R;
    S* app = reinterpret_cast<S*>(smem_raw);
    S* msg = app + PK::WPC * P.npad;
    uint16_t* slut = reinterpret_cast<uint16_t*>(smem_raw + PK::WPC * sizeof(S) * ((size_t)P.npad + (size_t)P.dmax * P.m));
    if (threadIdx.x < (PF ? 4 : 2)) s_odd[threadIdx.x] = 0;

    read_group(P, J, g, [&](int v, uint32_t w) { Access<PK>::put(app, P.npad, v, w); });
    {
        const int msg_bytes = PK::WPC * P.dmax * P.m * (int)sizeof(S);
        uint32_t* mz = reinterpret_cast<uint32_t*>(msg);
        for (int i = threadIdx.x; i < msg_bytes / 4; i += blockDim.x) mz[i] = 0;
    }
    __syncthreads();

    int executed = 0;
    bool passed = false;  // stopped by the syndrome early stop: every check of every frame holds
    unsigned live = 0xFu;        // PF: frames still decoding (the same in every thread)
    int its[4] = {0, 0, 0, 0};   // PF: iterations of the frames that stopped
    const auto get = [&](int v) { return Access<PK>::get(app, P.npad, v); };
    for (int it = 0; it < J.iters; it++) {
        R ov = 0;
        uint32_t oc01 = 0, oc23 = 0;  // PF: odd rows per frame (16-bit halves)
        const bool first = (it == 0);
        if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
        for (int l = 0; l < P.nlevels; l++) {
            const int2 lv = __ldg(P.levels + l);
            for (int r = lv.x + threadIdx.x; r < lv.x + lv.y; r += blockDim.x) {
                const int d = EXACT ? DT : __ldg(P.rowdeg + r);
                const int cls = __ldg(P.rowcls + r);
                const bool noclip = J.quirk && first && cls;
                if (PF)
                    row_update_lanes<KIND, DT, EXACT>(reinterpret_cast<uint32_t*>(app), reinterpret_cast<uint32_t*>(msg),
                                                      P, r, d, noclip, oc01, oc23, slut + 128 * cls);
                else
                    row_update<PK, KIND, DT, EXACT>(app, msg, P, r, d, noclip, ov, slut + 128 * cls);
            }
            __syncthreads();
        }
        executed = it + 1;
        if (PF) {
            const uint2 t = odd_rows_total_lanes(oc01, oc23, it, s_odd);
            const unsigned cnt[4] = {t.x & 0xffffu, t.x >> 16, t.y & 0xffffu, t.y >> 16};
            unsigned gate = 0;
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (((live >> k) & 1u) && cnt[k] <= J.early_slack) gate |= 1u << k;
            if (gate) {
                const uint32_t bad = rows_odd_mask(P, get);  // 0xff in byte k: frame k has an odd check
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (((gate >> k) & 1u) && __syncthreads_or((bad >> (8 * k)) & 0xffu)) gate &= ~(1u << k);
                if (gate) {
                    // these frames stop here: their decisions now, their count
                    write_group(P, J, g, get, (int)gate);
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if ((gate >> k) & 1u) its[k] = it + 1;
                    live &= ~gate;
                    if (!live) break;
                    __syncthreads();  // write_group read the APP that the next iteration updates
                }
            }
            continue;
        }
        if (KIND == KIND_2NMS && it >= 1) {
            if (!__syncthreads_or(ov != 0)) break;
        }
        if (KIND != KIND_2NMS && J.early) {
            if (odd_rows_within_slack(J, ov, it, s_odd) && !__syncthreads_or(rows_unsatisfied<PK>(app, P))) {
                passed = true;
                break;
            }
        }
    }

    if (PF) {
        // the frames still live ran every iteration
        if (live) write_group(P, J, g, get, (int)live);
        if (J.iters_out && threadIdx.x == 0)
            for (int k = 0; k < 4; k++) J.iters_out[4 * (g - J.word0) + k] = ((live >> k) & 1u) ? executed : its[k];
        if (J.synd_out) {
            if (threadIdx.x == 0)
                for (int k = 0; k < 4; k++)
                    if (!((live >> k) & 1u)) J.synd_out[4 * (g - J.word0) + k] = 1;
            if (live) write_syndrome_flags(J, 4 * (g - J.word0), rows_odd_mask(P, get), (int)live);
        }
        return;
    }
    write_group(P, J, g, get);
    if (J.iters_out && threadIdx.x == 0) J.iters_out[g - J.word0] = executed;
    if (J.synd_out) {
        const uint32_t bad = passed ? 0u : rows_odd_mask(P, get);
        write_syndrome_flags(J, 4 * (g - J.word0), bad, 0xF);
    }
    if (J.app_out) {
        uint32_t* ao = reinterpret_cast<uint32_t*>(J.app_out);
        for (int v = threadIdx.x; v < P.n; v += blockDim.x)
            ao[(long long)v * J.total_words + g] = Access<PK>::get(app, P.npad, v);
    }
    if (J.msg_out) {
        uint32_t* mo = reinterpret_cast<uint32_t*>(J.msg_out);
        const int mstride = P.dmax * P.m;
        for (int i = threadIdx.x; i < P.dmax * P.m; i += blockDim.x) {
            const int j = i / P.m, r = i - j * P.m;
            if (j < P.rowdeg[r])
                mo[(long long)P.edge_orig[i] * J.total_words + g] = Access<PK>::get_msg(msg, mstride, i);
        }
    }
}

// ---- the flooding schedule (LDPC_FLAG_FLOODING; no reference counterpart) ----
//
// Every row of an iteration reads the APP of the previous iteration and stores only its
// new messages; then every variable's APP is rebuilt from its channel value and the new
// messages of its edges, x = sat8(LLR + sum of messages), the sum exact (integer-valued
// fp16 below 2048) and saturated once.  Two barriers per iteration whatever the level
// structure.  PackF16x2 only (4 frames, two pair-words): APP [2][npad], messages
// [2][dmax*m], the channel values [2][npad] (biased like the APP), then the LEARNED table.

template <int KIND, int DT, bool EXACT>
__device__ __forceinline__ void row_update_flood(uint32_t* app, uint32_t* msg, const Plan& P, int r, int d,
                                                 bool noclip, uint32_t& ov, const uint16_t* lut)
{
    int v[DT];
#pragma unroll
    for (int j = 0; j < DT; j++)
        if (EXACT || j < d) v[j] = __ldg(P.cols + j * P.m + r);
    const int mstride = P.dmax * P.m;
#pragma unroll
    for (int w = 0; w < 2; w++) {
        const uint32_t* A = app + w * P.npad;
        uint32_t* M = msg + w * mstride;
        uint32_t x[DT], mm[DT];
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                x[j] = A[v[j]];
                mm[j] = M[j * P.m + r];
            }
        }
        PackF16x2::update<KIND, DT, EXACT>(x, mm, d, noclip, ov, lut);
#pragma unroll
        for (int j = 0; j < DT; j++)
            if (EXACT || j < d) M[j * P.m + r] = mm[j];
    }
}

template <int KIND, int DT, bool EXACT>
__global__ void __launch_bounds__(256) decode_flood_kernel(const Plan P, const Job J)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_odd[2];
    using PK = PackF16x2;
    const long long g = J.word0 + blockIdx.x;
    const int mstride = P.dmax * P.m;
    uint32_t* app = reinterpret_cast<uint32_t*>(smem_raw);
    uint32_t* msg = app + 2 * P.npad;
    uint32_t* llrb = msg + 2 * mstride;
    uint16_t* slut = reinterpret_cast<uint16_t*>(llrb + 2 * P.npad);
    if (threadIdx.x < 2) s_odd[threadIdx.x] = 0;

    read_group(P, J, g, [&](int v, uint32_t w) {
        Access<PK>::put(app, P.npad, v, w);
        Access<PK>::put(llrb, P.npad, v, w);
    });
    for (int i = threadIdx.x; i < 2 * mstride; i += blockDim.x) msg[i] = 0;
    __syncthreads();

    int executed = 0;
    bool passed = false;
    for (int it = 0; it < J.iters; it++) {
        uint32_t ov = 0;
        const bool first = (it == 0);
        if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
        for (int r = threadIdx.x; r < P.m; r += blockDim.x) {
            const int d = EXACT ? DT : __ldg(P.rowdeg + r);
            const int cls = __ldg(P.rowcls + r);
            const bool noclip = J.quirk && first && cls;
            row_update_flood<KIND, DT, EXACT>(app, msg, P, r, d, noclip, ov, slut + 128 * cls);
        }
        __syncthreads();
        for (int v = threadIdx.x; v < P.n; v += blockDim.x) {
            const int e0 = __ldg(P.vptr + v), e1 = __ldg(P.vptr + v + 1);
            uint32_t a0 = llrb[v], a1 = llrb[P.npad + v];
            for (int e = e0; e < e1; e++) {
                const int i = __ldg(P.vedge + e);
                a0 = h2::add(a0, msg[i]);
                a1 = h2::add(a1, msg[mstride + i]);
            }
            app[v] = h2::hmin(h2::fma_relu(a0, h2::ONE, 0u), h2::C255);
            app[P.npad + v] = h2::hmin(h2::fma_relu(a1, h2::ONE, 0u), h2::C255);
        }
        __syncthreads();
        executed = it + 1;
        if (KIND == KIND_2NMS && it >= 1) {
            if (!__syncthreads_or(ov != 0)) break;
        }
        if (KIND != KIND_2NMS && J.early) {
            if (odd_rows_within_slack(J, ov, it, s_odd) && !__syncthreads_or(rows_unsatisfied<PK>(app, P))) {
                passed = true;
                break;
            }
        }
    }

    write_group(P, J, g, [&](int v) { return Access<PK>::get(app, P.npad, v); });
    if (J.iters_out && threadIdx.x == 0) J.iters_out[g - J.word0] = executed;
    if (J.synd_out) {
        const uint32_t bad = passed ? 0u : rows_odd_mask(P, [&](int v) { return Access<PK>::get(app, P.npad, v); });
        write_syndrome_flags(J, 4 * (g - J.word0), bad, 0xF);
    }
    if (J.app_out) {
        uint32_t* ao = reinterpret_cast<uint32_t*>(J.app_out);
        for (int v = threadIdx.x; v < P.n; v += blockDim.x)
            ao[(long long)v * J.total_words + g] = Access<PK>::get(app, P.npad, v);
    }
    if (J.msg_out) {
        uint32_t* mo = reinterpret_cast<uint32_t*>(J.msg_out);
        for (int i = threadIdx.x; i < mstride; i += blockDim.x) {
            const int j = i / P.m, r = i - j * P.m;
            if (j < P.rowdeg[r])
                mo[(long long)P.edge_orig[i] * J.total_words + g] = Access<PK>::get_msg(msg, mstride, i);
        }
    }
}

template <class PK, int KIND, int DT, bool EXACT, bool PF = false>
__global__ void __launch_bounds__(256) decode_levels_kernel(const Plan P, const Job J)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_odd[4];
    decode_word_levels<PK, KIND, DT, EXACT, PF>(P, J, J.word0 + blockIdx.x, smem_raw, s_odd);
}

// The level-scheduled kernel for PackF16x2h: a CTA holds frames 2h, 2h+1 of word g
// (blockIdx.x = 2 * (g - word0) + h).  Same schedule and arithmetic as above.
template <int KIND, int DT, bool EXACT>
__global__ void __launch_bounds__(256) decode_levels_half_kernel(const Plan P, const Job J)
{
    using PK = PackF16x2h;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* app = reinterpret_cast<uint32_t*>(smem_raw);
    uint32_t* msg = app + P.npad;
    uint16_t* slut = reinterpret_cast<uint16_t*>(msg + (size_t)P.dmax * P.m);
    const long long g = J.word0 + (blockIdx.x >> 1);
    const int h = blockIdx.x & 1;

    read_group(P, J, g, [&](int v, uint32_t w) { AccessHalf::put(app, v, w, h); });
    for (int i = threadIdx.x; i < P.dmax * P.m; i += blockDim.x) msg[i] = 0;
    __syncthreads();

    uint32_t ov = 0;
    for (int it = 0; it < J.iters; it++) {
        const bool first = (it == 0);
        if (KIND == KIND_LEARNED) load_iteration_lut(J, it, slut);
        for (int l = 0; l < P.nlevels; l++) {
            const int2 lv = __ldg(P.levels + l);
            for (int r = lv.x + threadIdx.x; r < lv.x + lv.y; r += blockDim.x) {
                const int d = EXACT ? DT : __ldg(P.rowdeg + r);
                const int cls = __ldg(P.rowcls + r);
                const bool noclip = J.quirk && first && cls;
                row_update<PK, KIND, DT, EXACT>(app, msg, P, r, d, noclip, ov, slut + 128 * cls);
            }
            __syncthreads();
        }
    }

    const int kmask = 3 << (2 * h);
    write_group(P, J, g, [&](int v) { return AccessHalf::get(app, v, h); }, kmask);
    if (J.iters_out && threadIdx.x == 0 && h == 0) J.iters_out[g - J.word0] = J.iters;
    if (J.synd_out)
        write_syndrome_flags(J, 4 * (g - J.word0), rows_odd_mask(P, [&](int v) { return AccessHalf::get(app, v, h); }),
                             kmask);
    if (J.app_out) {
        uint8_t* ao = reinterpret_cast<uint8_t*>(J.app_out);
        for (int v = threadIdx.x; v < P.n; v += blockDim.x) {
            uint32_t w = AccessHalf::get(app, v, h);
            for (int k = 2 * h; k < 2 * h + 2; k++) ao[((long long)v * J.total_words + g) * 4 + k] = w >> (8 * k);
        }
    }
    if (J.msg_out) {
        uint8_t* mo = reinterpret_cast<uint8_t*>(J.msg_out);
        for (int i = threadIdx.x; i < P.dmax * P.m; i += blockDim.x) {
            const int j = i / P.m, r = i - j * P.m;
            if (j < P.rowdeg[r]) {
                uint32_t w = AccessHalf::get_msg(msg, i, h);
                for (int k = 2 * h; k < 2 * h + 2; k++)
                    mo[((long long)P.edge_orig[i] * J.total_words + g) * 4 + k] = w >> (8 * k);
            }
        }
    }
}

}  // namespace ldpc

// Kernel variants: EXACT<D> for codes whose rows all have degree D, else the
// smallest bucket DT >= the largest row degree (rows shorter than DT predicate
// the unused edge slots off).
#define LDPC_DEGREE_VARIANTS(X, PK, KIND) \
    X(PK, KIND, 6, true) X(PK, KIND, 7, true) X(PK, KIND, 8, false) X(PK, KIND, 16, false) X(PK, KIND, 32, false)
