// Instantiations of the QC register-message decoder for the code shapes in use,
// each with and without the syndrome early stop compiled in:
//   4 frames per CTA (WPT = 2): the regular (3,6) rate-1/2 8x16 base (row degree 6,
//     8 layers, Z a power of two), every kind and the offset-only learned kind, the
//     early stop per word or per frame pair (et = 1, 2);
//   2 frames per CTA (WPT = 1): 24-column irregular bases (802.11n-like) at rates
//     1/2, 2/3, 3/4, 5/6, i.e. 12, 8, 6, 4 layers of row degree up to 10, 14, 18, 24,
//     any Z.  Not for 2NMS, whose early termination is per 4-frame word;
//   the exact-gate early stop (LDPC_EARLY_SLACK_ANY) per word (et = 3) and per frame
//     pair (decode_qc_pairs_kernel) for the 4-frame kernels, every kind but 2NMS;
//   the per-frame early stop with lane refill (decode_qc_refill_kernel) for the
//     regular base, every kind but 2NMS.
#include "qc_kernel.cuh"

namespace ldpc {

#define LDPC_QC(KIND, D, EX, L, P2, W)                                                                  \
    if (kind == KIND && dt == D && exact == EX && layers == L && pow2 == P2 && wpt == W)                \
        return et == 3 && W == 2 && KIND != KIND_2NMS                                                    \
                   ? (const void*)decode_qc_kernel<KIND, D, EX, L, P2, (W == 2 && KIND != KIND_2NMS ? 3 : 1), W> \
               : et == 2 && W == 2 ? (const void*)decode_qc_kernel<KIND, D, EX, L, P2, (W == 2 ? 2 : 1), W> \
               : et              ? (const void*)decode_qc_kernel<KIND, D, EX, L, P2, 1, W>                  \
                                 : (const void*)decode_qc_kernel<KIND, D, EX, L, P2, 0, W>;
#define LDPC_QC_KINDS(D, EX, L, P2)                                                                    \
    LDPC_QC(KIND_MS, D, EX, L, P2, 2) LDPC_QC(KIND_OMS, D, EX, L, P2, 2)                                \
    LDPC_QC(KIND_NMS, D, EX, L, P2, 2) LDPC_QC(KIND_2NMS, D, EX, L, P2, 2) LDPC_QC(KIND_LEARNED, D, EX, L, P2, 2) \
    LDPC_QC(KIND_LEARNED_OFS, D, EX, L, P2, 2)
#define LDPC_QC_PAIR(D, L) \
    LDPC_QC(KIND_MS, D, false, L, false, 1) LDPC_QC(KIND_OMS, D, false, L, false, 1) \
    LDPC_QC(KIND_NMS, D, false, L, false, 1) LDPC_QC(KIND_LEARNED, D, false, L, false, 1)

const void* kernel_table_qc(int kind, int dt, bool exact, int layers, bool pow2, int et, int wpt)
{
    LDPC_QC_KINDS(6, true, 8, true)  // regular (3,6) rate-1/2 QC, 8x16 base (Z = 2^k)
    LDPC_QC_PAIR(10, 12) LDPC_QC_PAIR(14, 8) LDPC_QC_PAIR(18, 6) LDPC_QC_PAIR(24, 4)
    return nullptr;
}

// The exact-gate twin of a 4-frame QC kernel with the early stop per word (et = 1 ->
// et = 3) or per frame pair (et = 2 -> decode_qc_pairs_kernel), or null when f is neither
const void* kernel_qc_exact_of(const void* f)
{
#define LDPC_QC_X(KIND)                                                          \
    if (f == (const void*)decode_qc_kernel<KIND, 6, true, 8, true, 1, 2>)          \
        return (const void*)decode_qc_kernel<KIND, 6, true, 8, true, 3, 2>;        \
    if (f == (const void*)decode_qc_kernel<KIND, 6, true, 8, true, 2, 2>)          \
        return (const void*)decode_qc_pairs_kernel<KIND, 6, true, 8, true>;
    LDPC_QC_X(KIND_MS) LDPC_QC_X(KIND_OMS) LDPC_QC_X(KIND_NMS) LDPC_QC_X(KIND_LEARNED) LDPC_QC_X(KIND_LEARNED_OFS)
#undef LDPC_QC_X
    return nullptr;
}

// per-frame early stop with lane refill (4 frames per CTA): the regular (3,6) base
#define LDPC_QC_REFILL(KIND, D, EX, L, P2)                                          \
    if (kind == KIND && dt == D && exact == EX && layers == L && pow2 == P2)           \
        return (const void*)decode_qc_refill_kernel<KIND, D, EX, L, P2>;

const void* kernel_table_qc_refill(int kind, int dt, bool exact, int layers, bool pow2)
{
    LDPC_QC_REFILL(KIND_MS, 6, true, 8, true) LDPC_QC_REFILL(KIND_OMS, 6, true, 8, true)
    LDPC_QC_REFILL(KIND_NMS, 6, true, 8, true) LDPC_QC_REFILL(KIND_LEARNED, 6, true, 8, true)
    return nullptr;
}

}  // namespace ldpc
