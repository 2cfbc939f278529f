// Instantiations of the 2-frames-per-CTA level-scheduled decoder (PackF16x2h).
#include "decode_kernel.cuh"

namespace ldpc {

#define LDPC_HENTRY(PK, KIND, D, EX) (const void*)decode_levels_half_kernel<KIND, D, EX>,
#define LDPC_HROW(KIND) {LDPC_DEGREE_VARIANTS(LDPC_HENTRY, PackF16x2h, KIND)},

// [kind: MS, OMS, NMS, LEARNED][variant: exact 6, exact 7, <=8, <=16, <=32]; no 2NMS (per-word early termination)
const void* kernel_table_f16x2h(int kind, int variant)
{
    static const void* table[4][5] = {LDPC_HROW(KIND_MS) LDPC_HROW(KIND_OMS) LDPC_HROW(KIND_NMS) LDPC_HROW(KIND_LEARNED)};
    if (kind < 0 || kind > 3 || variant < 0 || variant > 4) return nullptr;
    return table[kind][variant];
}

}  // namespace ldpc
