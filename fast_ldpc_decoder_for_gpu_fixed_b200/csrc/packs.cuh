// Frame packings of the decoder state and their check-node arithmetic.
//
// A "pack" decides how the per-frame int8 values of the reference decoder
// (APP in [-128,127], c->v messages) are laid out in shared memory and
// registers, and implements one check-row update over them.  All three give
// bit-identical results to the reference's byte lanes
// (decoder_oms/cuda/CUDA_OMS_SIMD.cu:64-87 and :164-187; per-byte semantics
// of the SIMD helper header decoder_oms/cuda/simd_functions.h:89-130):
//
//   PackSIMD4  4 frames per 32-bit word, one byte per frame, CUDA's per-byte
//              SIMD intrinsics (__vsubss4, __vabs4, __vminu4, ...).  Same
//              packing as the reference; word g holds frames 4g..4g+3.
//   PackF16x2  2 frames per 32-bit word as two fp16 lanes holding the integer
//              values exactly.  Every value is NEGATED (u = -x): then the
//              reference's "bit 1" test x > 0 is exactly the sign bit of u
//              (x = 0 gives u = +0, sign 0), so sign products are XORs of sign
//              bits and conditional negations are sign-bit XORs; the
//              saturations become clamps to [-127, 128].  -0 can appear only
//              in messages, where x - (-0) = x keeps it harmless.  APP is
//              stored biased by +127 (see namespace h2).
//   PackI8     1 frame per thread lane: int8 in shared memory, int32 math.
//              APP kept as x, messages kept negated (u = -m, |u| <= 127).
//
// Check magnitudes (c1 for the minimum edge, c2 for the others):
//   MS   min(m, 31)                          decoder_ms/cuda/CUDA_MS_SIMD.cu:73-74
//   OMS  min(max(m-1, 0), 31); no 31-clip on first-iteration rows of the second
//        degree group                        decoder_oms/cuda/CUDA_OMS_SIMD.cu:73-74,115-116
//   NMS  floor(0.75 m) for both              decoder_nms/cuda/CUDA_NMS_SIMD.cu:73-85
//   2NMS floor(0.875 min2), floor(0.75 min1) decoder_2nms/cuda/CUDA_2NMS_SIMD.cu:76-83
// (the reference's float multiply followed by the char conversion truncates a
// non-negative exact product, i.e. floors it).
#pragma once
#include <cstdint>
#include <cuda_fp16.h>

namespace ldpc {

enum { KIND_MS = 0, KIND_OMS = 1, KIND_NMS = 2, KIND_2NMS = 3, KIND_XMS = 4, KIND_LEARNED = 5 };

// KIND_LEARNED with every scale 1.0 (a learned-offset decoder): the magnitude is
// clamp(min - offset, 0, 31), no floor step, the arithmetic of OMS with the offset of
// the iteration.  Used by the fp16 QC register kernel, which the host switches to it
// when the constants allow; the (k, b) words then carry b = -offset.
constexpr int KIND_LEARNED_OFS = 6;

// KIND_LEARNED (no reference counterpart): the magnitude of a check's outgoing
// messages is c = clamp(floor(min * scale_q7 / 128) - offset, 0, 31) with the
// trained int8 offset and Q1.7 scale of the current iteration and row group.
// PackSIMD4 / PackI8 read it from a 128-entry table of plain integers built on
// the host; PackF16x2 computes it from (k, b) pairs stored at the head of the
// same table (h2::mags).

// ------------------------------------------------------------------------
// 4 frames per word, per-byte saturating SIMD
// ------------------------------------------------------------------------
struct PackSIMD4 {
    using S = uint32_t;  // shared-memory element
    using R = uint32_t;  // register value
    static constexpr int WPC = 1;  // storage words per 4-frame group
    static constexpr int ID = 0;

    __device__ __forceinline__ static R ld_app(const S* p) { return *p; }
    __device__ __forceinline__ static R ld_msg(const S* p) { return *p; }
    __device__ __forceinline__ static void st_app(S* p, R v) { *p = v; }
    __device__ __forceinline__ static void st_msg(S* p, R v) { *p = v; }

    __device__ __forceinline__ static R lut4(R m, const uint16_t* lut)
    {
        return (R)lut[m & 0xff] | ((R)lut[(m >> 8) & 0xff] << 8) | ((R)lut[(m >> 16) & 0xff] << 16) |
               ((R)lut[m >> 24] << 24);
    }

    template <int KIND>
    __device__ __forceinline__ static void mags(R mn1, R mn2, bool noclip, R& c1, R& c2, const uint16_t* lut)
    {
        if (KIND == KIND_LEARNED) {
            c1 = lut4(mn2, lut);
            c2 = lut4(mn1, lut);
        } else if (KIND == KIND_MS) {
            c1 = __vminu4(mn2, 0x1f1f1f1fu);
            c2 = __vminu4(mn1, 0x1f1f1f1fu);
        } else if (KIND == KIND_OMS) {
            c1 = __vsubus4(mn2, 0x01010101u);
            c2 = __vsubus4(mn1, 0x01010101u);
            if (!noclip) {
                c1 = __vminu4(c1, 0x1f1f1f1fu);
                c2 = __vminu4(c2, 0x1f1f1f1fu);
            }
        } else {
            // floor(3m/4) = m - ceil(m/4); bytes <= 127 so no carry crosses a byte
            c2 = mn1 - (((mn1 + 0x03030303u) >> 2) & 0x3f3f3f3fu);
            if (KIND == KIND_NMS)
                c1 = mn2 - (((mn2 + 0x03030303u) >> 2) & 0x3f3f3f3fu);
            else  // floor(7m/8) = m - ceil(m/8)
                c1 = mn2 - (((mn2 + 0x07070707u) >> 3) & 0x1f1f1f1fu);
        }
    }

    // x[j]: APP in / APP out; m[j]: message in / out (all 4 byte lanes)
    template <int KIND, int DT, bool EXACT>
    __device__ __forceinline__ static void update(R (&x)[DT], R (&m)[DT], int d, bool noclip, R& ov,
                                                  const uint16_t* lut)
    {
        const R s = update_row<KIND, DT, EXACT>(x, m, d, noclip, lut);
        ov += __popc(s) >> 3;  // odd (row, frame) pairs: s is 0xff in each odd byte
    }

    // update() with the odd rows counted per frame: lanes 0 and 1 in the 16-bit halves of
    // oc01, lanes 2 and 3 in those of oc23 (the per-frame early stop)
    template <int KIND, int DT, bool EXACT>
    __device__ __forceinline__ static void update_lanes(R (&x)[DT], R (&m)[DT], int d, bool noclip, R& oc01,
                                                        R& oc23, const uint16_t* lut)
    {
        const R s = update_row<KIND, DT, EXACT>(x, m, d, noclip, lut);
        oc01 += __byte_perm(s, 0, 0x4140) & 0x00010001u;
        oc23 += __byte_perm(s, 0, 0x4342) & 0x00010001u;
    }

    // the row update; returns the row's extrinsic sign parity, 0xff in each odd byte lane
    template <int KIND, int DT, bool EXACT>
    __device__ __forceinline__ static R update_row(R (&x)[DT], R (&m)[DT], int d, bool noclip, const uint16_t* lut)
    {
        R mn1 = 0x7f7f7f7fu, mn2 = 0x7f7f7f7fu, s = 0;
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                R t = __vsubss4(x[j], m[j]);
                x[j] = t;
                R a = __vabs4(t);
                mn2 = __vminu4(mn2, __vmaxu4(a, mn1));
                mn1 = __vminu4(mn1, a);
                s ^= __vcmpgts4(t, 0u);
            }
        }
        R c1, c2;
        mags<KIND>(mn1, mn2, noclip, c1, c2, lut);
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                R t = x[j];
                R eq = __vcmpeq4(__vabs4(t), mn1);
                R re = (eq & c1) | (~eq & c2);
                R sg = s ^ __vcmpgts4(t, 0u);
                R out = (re & sg) | (__vneg4(re) & ~sg);
                m[j] = out;
                x[j] = __vaddss4(t, out);
            }
        }
        return s;
    }
};

// ------------------------------------------------------------------------
// 2 frames per word, integer-valued fp16 lanes, negated values
// ------------------------------------------------------------------------
//
// Values: u = -x (so the sign bit of u is the reference's "x > 0" test), every
// integer in [-128, 256] is exact in fp16.  APP is kept biased, b = u + 127 in
// [0, 255], so the saturation of the extrinsic and of the new APP is one
// fma.relu (lower bound, FMA pipe) plus one min (upper bound, ALU pipe).
// min.xorsign.abs folds the running min1 and the XOR of the sign bits of the
// row into one instruction: its result has magnitude min(|a|,|b|) and sign
// sign(a) ^ sign(b).
__device__ __forceinline__ uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

namespace h2 {
constexpr uint32_t SIGN = 0x80008000u, MAG = 0x7fff7fffu;
constexpr uint32_t ONE = 0x3c003c00u, NEG1 = 0xbc00bc00u, C127 = 0x57f057f0u, CNEG127 = 0xd7f0d7f0u,
                   C255 = 0x5bf85bf8u, C31 = 0x4fc04fc0u, C1024 = 0x64006400u, CNEG1024 = 0xe400e400u,
                   C075 = 0x3a003a00u, CNEG0375 = 0xb600b600u, C0875 = 0x3b003b00u, CNEG04375 = 0xb700b700u;
__device__ __forceinline__ uint32_t fma_relu(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("fma.rn.relu.f16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ uint32_t fma(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ uint32_t add(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("add.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t add_sat(uint32_t a, uint32_t b)  // clamp(a + b, 0, 1)
{
    uint32_t d;
    asm("add.rn.sat.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t sub(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("sub.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t hmin(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("min.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t min_xs(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("min.xorsign.abs.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t habs(uint32_t a)
{
    uint32_t d;
    asm("abs.f16x2 %0, %1;" : "=r"(d) : "r"(a));
    return d;
}
__device__ __forceinline__ uint32_t max_xs(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("max.xorsign.abs.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
// floor(m * k) for integer m in [0,127], k with few fraction bits (3/4, 7/8, s/16):
// m*k - (1/2 - 2^-(bits+1)) is exact, within 1/2 of the floor and never on a tie,
// so adding 1024 rounds it there.
__device__ __forceinline__ uint32_t floor_scale(uint32_t m, uint32_t k, uint32_t bias)
{
    return add(add(fma_relu(m, k, bias), C1024), CNEG1024);
}

// row magnitudes from |min1| (a1) and |min2| (a2); lk, lb: the LEARNED (k, k), (b, b) words
template <int KIND>
__device__ __forceinline__ void mags(uint32_t a1, uint32_t a2, bool noclip, uint32_t& c1, uint32_t& c2, uint32_t lk,
                                     uint32_t lb, uint32_t clip = C31)
{
    if (KIND == KIND_LEARNED_OFS) {
        // scale 1: clamp(a - offset, 0, 31) with lb = (-offset, -offset), exact on integers
        c1 = hmin(fma_relu(a2, ONE, lb), C31);
        c2 = hmin(fma_relu(a1, ONE, lb), C31);
    } else if (KIND == KIND_LEARNED) {
        // clamp(floor(a * k) - offset, 0, 31) = min(round(relu(a * k + b)), 31), b = -offset - 15/32:
        // with k on a 1/16 grid, a * k + b is exact below 64 and never within 1/32 of a tie
        // (ldpc_decoder_set_learned stores (k, k) and (b, b) at the head of the class's table)
        c1 = hmin(floor_scale(a2, lk, lb), C31);
        c2 = hmin(floor_scale(a1, lk, lb), C31);
    } else if (KIND == KIND_MS) {
        c1 = hmin(a2, C31);
        c2 = hmin(a1, C31);
    } else if (KIND == KIND_OMS) {
        c1 = fma_relu(a2, ONE, NEG1);
        c2 = fma_relu(a1, ONE, NEG1);
        if (!noclip) {  // clip: C31, or per lane C31 / no clip (the first iteration of a lane's frame)
            c1 = hmin(c1, clip);
            c2 = hmin(c2, clip);
        }
    } else {
        c2 = floor_scale(a1, C075, CNEG0375);
        c1 = (KIND == KIND_NMS) ? floor_scale(a2, C075, CNEG0375) : floor_scale(a2, C0875, CNEG04375);
    }
}

// one row over one pair-word: b[j] biased APP in/out, m[j] negated message in/out
// the LEARNED (k, b) words at the head of a class's table (zero for other kinds)
template <int KIND>
__device__ __forceinline__ void learned_kb(const uint16_t* lut, uint32_t& lk, uint32_t& lb)
{
    lk = lb = 0;
    if (KIND == KIND_LEARNED) {
        lk = reinterpret_cast<const uint32_t*>(lut)[0];
        lb = reinterpret_cast<const uint32_t*>(lut)[1];
    }
}

// CMODE 0: ov counts odd (row, frame) pairs; 1: ov counts odd rows per fp16 lane (bit 0 and
// bit 16 fields), and clip is the per-lane OMS clip word; 2: ov is a count_parity
// accumulator (+1 per even row, -1 per odd row and lane, on the FMA pipe)
template <int KIND, int DT, bool EXACT, int CMODE = 0>
__device__ __forceinline__ void row(uint32_t (&b)[DT], uint32_t (&m)[DT], int d, bool noclip, uint32_t& ov,
                                    uint32_t lk, uint32_t lb, uint32_t clip = C31)
{
    uint32_t ut[DT];
    uint32_t mn1 = C127, mn2 = C127;
    if (EXACT && DT >= 4) {
        // Rows of a known degree: the two smallest |t| by a tournament (pairs sorted, then
        // merged: min1 = min(m1, l), min2 = min(max(m1, l), min(m2, h))), 3.5 min/max per
        // two edges instead of 3 per edge.  The xorsign forms carry the sign parity of
        // the row into min1 as in the running form below.
#pragma unroll
        for (int j = 0; j < DT; j++) {
            const uint32_t bt = hmin(fma_relu(m[j], NEG1, b[j]), C255);  // clamp(b - m, 0, 255)
            b[j] = bt;
            ut[j] = add(bt, CNEG127);
        }
        mn1 = min_xs(ut[0], ut[1]);
        mn2 = max_xs(ut[0], ut[1]);
#pragma unroll
        for (int j = 2; j + 1 < DT; j += 2) {
            const uint32_t lo = min_xs(ut[j], ut[j + 1]), hi = max_xs(ut[j], ut[j + 1]);
            const uint32_t m2 = min_xs(max_xs(mn1, lo), min_xs(mn2, hi));
            mn1 = min_xs(mn1, lo);
            mn2 = m2;
        }
        if (DT & 1) {
            const uint32_t mx = max_xs(ut[DT - 1], mn1);
            mn1 = min_xs(mn1, ut[DT - 1]);
            mn2 = min_xs(mn2, mx);
        }
        // The reference starts both minima at 127; |t| reaches 128 only for x = -128.  That
        // changes a magnitude only where the magnitude is not clipped to 31 (NMS, 2NMS,
        // LEARNED, the OMS first-iteration no-clip), so only those cap.
        if (KIND == KIND_NMS || KIND == KIND_2NMS || KIND == KIND_LEARNED || KIND == KIND_LEARNED_OFS ||
            (KIND == KIND_OMS && (noclip || clip != C31))) {
            mn1 = min_xs(mn1, C127);
            mn2 = min_xs(mn2, C127);
        }
    } else {
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                uint32_t bt = hmin(fma_relu(m[j], NEG1, b[j]), C255);  // clamp(b - m, 0, 255)
                b[j] = bt;
                ut[j] = add(bt, CNEG127);
                uint32_t mx = max_xs(ut[j], mn1);
                mn1 = min_xs(mn1, ut[j]);
                mn2 = min_xs(mn2, mx);
            }
        }
    }
    const uint32_t a1 = habs(mn1), a2 = habs(mn2);
    uint32_t c1, c2;
    mags<KIND>(a1, a2, noclip, c1, c2, lk, lb, clip);
    const uint32_t c1s = c1 | (mn1 & SIGN), c2s = c2 | (mn1 & SIGN);
    const uint32_t dcs = sub(c2s, c1s), na1 = a1 ^ SIGN;
#pragma unroll
    for (int j = 0; j < DT; j++) {
        if (EXACT || j < d) {
            // |t| >= min1 on every edge, so sat(|t| - min1) is 0 on the minimum edge(s)
            // and 1 elsewhere: r = c1s there, c2s elsewhere (one FMA instead of a
            // compare and a select)
            // (abs.f16x2 rather than a mask: the abs folds into the saturating add)
            uint32_t r = fma(add_sat(habs(ut[j]), na1), dcs, c1s);
            uint32_t mo = r ^ (ut[j] & SIGN);                   // flip by this edge's own sign
            m[j] = mo;
            b[j] = hmin(fma_relu(mo, ONE, b[j]), C255);         // clamp(bt + m, 0, 255)
        }
    }
    if (CMODE == 1)
        ov += (mn1 & SIGN) >> 15;  // odd rows of each lane's frame
    else if (CMODE == 2)
        ov = add(ov, (mn1 & SIGN) | ONE);
    else
        ov += __popc(mn1 & SIGN);  // odd (row, frame) pairs
}

// row() for a check row split over SPLIT lanes of a warp (lanes k*SPLIT .. k*SPLIT+SPLIT-1):
// this lane holds nv (<= DL) of the row's edges.  Each lane takes the running min1 / min2 /
// sign parity of its own edges, then the lanes merge them with log2(SPLIT) butterfly
// shuffles: min1 = min of both (xorsign: the parities combine), min2 = min(both min2s, max of
// the two min1s).  A lane without edges contributes (127, 127, +), the reference's initial
// minima, so it changes nothing.  The reference's min1 / min2 / parity do not depend on the
// order of the edges, so every lane ends with the row's values and computes its own edges'
// messages.  wmask: the warp's lanes (all of them take part in every call); lead: the lane
// that counts the row (CMODE 2).
template <int KIND, int DL, int SPLIT, int CMODE>
__device__ __forceinline__ void row_split(uint32_t (&b)[DL], uint32_t (&m)[DL], int nv, bool noclip, uint32_t& ov,
                                          uint32_t lk, uint32_t lb, unsigned wmask, bool lead)
{
    uint32_t ut[DL];
    uint32_t mn1 = C127, mn2 = C127;
#pragma unroll
    for (int i = 0; i < DL; i++) {
        if (i < nv) {
            const uint32_t bt = hmin(fma_relu(m[i], NEG1, b[i]), C255);  // clamp(b - m, 0, 255)
            b[i] = bt;
            ut[i] = add(bt, CNEG127);
            const uint32_t mx = max_xs(ut[i], mn1);
            mn1 = min_xs(mn1, ut[i]);
            mn2 = min_xs(mn2, mx);
        }
    }
#pragma unroll
    for (int o = 1; o < SPLIT; o <<= 1) {
        const uint32_t p1 = __shfl_xor_sync(wmask, mn1, o), p2 = __shfl_xor_sync(wmask, mn2, o);
        mn2 = min_xs(min_xs(mn2, p2), max_xs(mn1, p1));
        mn1 = min_xs(mn1, p1);
    }
    const uint32_t a1 = habs(mn1), a2 = habs(mn2);
    uint32_t c1, c2;
    mags<KIND>(a1, a2, noclip, c1, c2, lk, lb);
    const uint32_t c1s = c1 | (mn1 & SIGN), c2s = c2 | (mn1 & SIGN);
    const uint32_t dcs = sub(c2s, c1s), na1 = a1 ^ SIGN;
#pragma unroll
    for (int i = 0; i < DL; i++) {
        if (i < nv) {
            const uint32_t r = fma(add_sat(habs(ut[i]), na1), dcs, c1s);
            const uint32_t mo = r ^ (ut[i] & SIGN);
            m[i] = mo;
            b[i] = hmin(fma_relu(mo, ONE, b[i]), C255);
        }
    }
    if (CMODE == 2 && lead) ov = add(ov, (mn1 & SIGN) | ONE);
}

// The number of odd rows from a CMODE 2 accumulator of row() after `rows` rows per lane:
// each row added +1 (even) or -1 (odd) per lane, so 2 * rows - sum is twice that number.
__device__ __forceinline__ unsigned odd_count(uint32_t acc, int rows)
{
    const __half2 h = *reinterpret_cast<const __half2*>(&acc);
    const int sum = __half2int_rn(__low2half(h)) + __half2int_rn(__high2half(h));
    return (unsigned)((2 * rows - sum) >> 1);
}
}  // namespace h2

struct PackF16x2 {
    using S = uint32_t;
    using R = uint32_t;
    static constexpr int WPC = 2;
    static constexpr int ID = 1;

    __device__ __forceinline__ static R ld_app(const S* p) { return *p; }
    __device__ __forceinline__ static R ld_msg(const S* p) { return *p; }
    __device__ __forceinline__ static void st_app(S* p, R v) { *p = v; }
    __device__ __forceinline__ static void st_msg(S* p, R v) { *p = v; }

    template <int KIND, int DT, bool EXACT>
    __device__ __forceinline__ static void update(R (&x)[DT], R (&m)[DT], int d, bool noclip, R& ov,
                                                  const uint16_t* lut)
    {
        uint32_t lk, lb;
        h2::learned_kb<KIND>(lut, lk, lb);
        h2::row<KIND, DT, EXACT>(x, m, d, noclip, ov, lk, lb);
    }
};

// The same packing for a CTA that holds only 2 of the 4 frames of a word (one
// pair-word): half the shared memory per CTA, twice the CTAs.  Not for 2NMS,
// whose early termination is decided per 4-frame word.
struct PackF16x2h : PackF16x2 {
    static constexpr int WPC = 1;
    static constexpr int ID = 3;
};

// ------------------------------------------------------------------------
// 1 frame per lane, int8 storage, int32 arithmetic
// ------------------------------------------------------------------------
struct PackI8 {
    using S = int8_t;
    using R = int;
    static constexpr int WPC = 4;
    static constexpr int ID = 2;

    __device__ __forceinline__ static R ld_app(const S* p) { return *p; }
    __device__ __forceinline__ static R ld_msg(const S* p) { return *p; }
    __device__ __forceinline__ static void st_app(S* p, R v) { *p = (S)v; }
    __device__ __forceinline__ static void st_msg(S* p, R v) { *p = (S)v; }

    template <int KIND>
    __device__ __forceinline__ static void mags(int mn1, int mn2, bool noclip, int& c1, int& c2, const uint16_t* lut)
    {
        if (KIND == KIND_LEARNED) {
            c1 = lut[mn2];
            c2 = lut[mn1];
        } else if (KIND == KIND_MS) {
            c1 = min(mn2, 31);
            c2 = min(mn1, 31);
        } else if (KIND == KIND_OMS) {
            c1 = max(mn2 - 1, 0);
            c2 = max(mn1 - 1, 0);
            if (!noclip) {
                c1 = min(c1, 31);
                c2 = min(c2, 31);
            }
        } else {
            c2 = (3 * mn1) >> 2;
            c1 = (KIND == KIND_NMS) ? (3 * mn2) >> 2 : (7 * mn2) >> 3;
        }
    }

    // x[j]: APP (as x) in/out; m[j]: message stored negated (u = -msg) in/out
    template <int KIND, int DT, bool EXACT>
    __device__ __forceinline__ static void update(R (&x)[DT], R (&m)[DT], int d, bool noclip, R& ov,
                                                  const uint16_t* lut)
    {
        int mn1 = 127, mn2 = 127, s = 0;
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                int ut = min(max(-x[j] - m[j], -127), 128);  // u_t = -(sat8(app - msg))
                x[j] = ut;
                int a = abs(ut);
                mn2 = min(mn2, max(a, mn1));
                mn1 = min(mn1, a);
                s ^= ut;
            }
        }
        int c1, c2;
        mags<KIND>(mn1, mn2, noclip, c1, c2, lut);
        const int sm = s >> 31;  // all ones when the parity of "x > 0" edges is odd
        c1 = (c1 ^ sm) - sm;
        c2 = (c2 ^ sm) - sm;
#pragma unroll
        for (int j = 0; j < DT; j++) {
            if (EXACT || j < d) {
                int ut = x[j];
                int re = (abs(ut) == mn1) ? c1 : c2;
                int tm = ut >> 31;
                int um = (re ^ tm) - tm;  // negated message: sign flips with this edge's bit
                m[j] = um;
                x[j] = min(max(-(ut + um), -128), 127);
            }
        }
        ov += (uint32_t)s >> 31;  // odd (row, frame) pairs
    }
};

}  // namespace ldpc
