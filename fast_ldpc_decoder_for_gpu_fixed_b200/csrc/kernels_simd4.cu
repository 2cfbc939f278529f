// Instantiations of the level-scheduled decoder for PackSIMD4 (one file per
// pack so that nvcc compiles the packs in parallel).
#include "decode_kernel.cuh"

namespace ldpc {

#define LDPC_ENTRY(PK, KIND, D, EX) (const void*)decode_levels_kernel<PK, KIND, D, EX>,
#define LDPC_ROW(KIND) {LDPC_DEGREE_VARIANTS(LDPC_ENTRY, PackSIMD4, KIND)},

// [kind: MS, OMS, NMS, 2NMS, LEARNED][variant: exact 6, exact 7, <=8, <=16, <=32]
const void* kernel_table_simd4(int kind, int variant)
{
    static const void* table[5][5] = {LDPC_ROW(KIND_MS) LDPC_ROW(KIND_OMS) LDPC_ROW(KIND_NMS) LDPC_ROW(KIND_2NMS)
                                      LDPC_ROW(KIND_LEARNED)};
    if (kind < 0 || kind > 4 || variant < 0 || variant > 4) return nullptr;
    return table[kind][variant];
}

// the per-frame early stop (LDPC_FLAG_EARLY_STOP_FRAMES): [kind: MS, OMS, NMS, -, LEARNED][variant]
#define LDPC_ENTRY_PF(PK, KIND, D, EX) (const void*)decode_levels_kernel<PK, KIND, D, EX, true>,
#define LDPC_ROW_PF(KIND) {LDPC_DEGREE_VARIANTS(LDPC_ENTRY_PF, PackSIMD4, KIND)},

const void* kernel_table_simd4_pf(int kind, int variant)
{
    static const void* table[4][5] = {LDPC_ROW_PF(KIND_MS) LDPC_ROW_PF(KIND_OMS) LDPC_ROW_PF(KIND_NMS)
                                      LDPC_ROW_PF(KIND_LEARNED)};
    const int row = kind == KIND_LEARNED ? 3 : kind;
    if (kind == KIND_2NMS || row < 0 || row > 3 || variant < 0 || variant > 4) return nullptr;
    return table[row][variant];
}

}  // namespace ldpc
