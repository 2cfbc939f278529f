// Instantiations of the level-scheduled decoder for PackF16x2 (one file per
// pack so that nvcc compiles the packs in parallel).
#include "decode_kernel.cuh"

namespace ldpc {

#define LDPC_ENTRY(PK, KIND, D, EX) (const void*)decode_levels_kernel<PK, KIND, D, EX>,
#define LDPC_ROW(KIND) {LDPC_DEGREE_VARIANTS(LDPC_ENTRY, PackF16x2, KIND)},

// [kind: MS, OMS, NMS, 2NMS, LEARNED][variant: exact 6, exact 7, <=8, <=16, <=32]
const void* kernel_table_f16x2(int kind, int variant)
{
    static const void* table[5][5] = {LDPC_ROW(KIND_MS) LDPC_ROW(KIND_OMS) LDPC_ROW(KIND_NMS) LDPC_ROW(KIND_2NMS)
                                      LDPC_ROW(KIND_LEARNED)};
    if (kind < 0 || kind > 4 || variant < 0 || variant > 4) return nullptr;
    return table[kind][variant];
}

// the flooding schedule (decode_flood_kernel), same table shape
#define LDPC_FLOOD_ENTRY(PK, KIND, D, EX) (const void*)decode_flood_kernel<KIND, D, EX>,
#define LDPC_FLOOD_ROW(KIND) {LDPC_DEGREE_VARIANTS(LDPC_FLOOD_ENTRY, PackF16x2, KIND)},

const void* kernel_table_flood(int kind, int variant)
{
    static const void* table[5][5] = {LDPC_FLOOD_ROW(KIND_MS) LDPC_FLOOD_ROW(KIND_OMS) LDPC_FLOOD_ROW(KIND_NMS)
                                      LDPC_FLOOD_ROW(KIND_2NMS) LDPC_FLOOD_ROW(KIND_LEARNED)};
    if (kind < 0 || kind > 4 || variant < 0 || variant > 4) return nullptr;
    return table[kind][variant];
}

}  // namespace ldpc
