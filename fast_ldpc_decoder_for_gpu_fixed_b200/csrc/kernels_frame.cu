// Instantiations of the one-frame-per-CTA decoder with packed row state
// (frame_kernel.cuh), for every kind but 2NMS, the degree variants up to 14 and
// both early-stop settings.
#include "frame_kernel.cuh"

namespace ldpc {

#define LDPC_FRAME_ENTRIES(ET, KIND)                                                                   \
    {(const void*)decode_frame_kernel<KIND, 6, true, ET>, (const void*)decode_frame_kernel<KIND, 7, true, ET>, \
     (const void*)decode_frame_kernel<KIND, 8, false, ET>,                                             \
     (const void*)decode_frame_kernel<KIND, FRAME_MAX_DEGREE, false, ET>},

// [early stop][kind: MS, OMS, NMS, LEARNED][variant: exact 6, exact 7, <=8, <=14]
const void* kernel_table_frame(int kind, int variant, bool et)
{
    static const void* table[2][4][4] = {
        {LDPC_FRAME_ENTRIES(false, KIND_MS) LDPC_FRAME_ENTRIES(false, KIND_OMS) LDPC_FRAME_ENTRIES(false, KIND_NMS)
             LDPC_FRAME_ENTRIES(false, KIND_LEARNED)},
        {LDPC_FRAME_ENTRIES(true, KIND_MS) LDPC_FRAME_ENTRIES(true, KIND_OMS) LDPC_FRAME_ENTRIES(true, KIND_NMS)
             LDPC_FRAME_ENTRIES(true, KIND_LEARNED)}};
    const int row = kind == KIND_LEARNED ? 3 : kind;
    if (kind == KIND_2NMS || row < 0 || row > 3 || variant < 0 || variant > 3) return nullptr;
    return table[et ? 1 : 0][row][variant];
}

#define LDPC_FRAME2_ENTRIES(ET, KIND)                                                                  \
    {(const void*)decode_frame2_kernel<KIND, 6, true, ET>, (const void*)decode_frame2_kernel<KIND, 7, true, ET>, \
     (const void*)decode_frame2_kernel<KIND, 8, false, ET>,                                            \
     (const void*)decode_frame2_kernel<KIND, FRAME_MAX_DEGREE, false, ET>},

// two frames per CTA: [early stop][kind: MS, OMS, NMS, LEARNED][variant]
const void* kernel_table_frame2(int kind, int variant, bool et)
{
    static const void* table[2][4][4] = {
        {LDPC_FRAME2_ENTRIES(false, KIND_MS) LDPC_FRAME2_ENTRIES(false, KIND_OMS) LDPC_FRAME2_ENTRIES(false, KIND_NMS)
             LDPC_FRAME2_ENTRIES(false, KIND_LEARNED)},
        {LDPC_FRAME2_ENTRIES(true, KIND_MS) LDPC_FRAME2_ENTRIES(true, KIND_OMS) LDPC_FRAME2_ENTRIES(true, KIND_NMS)
             LDPC_FRAME2_ENTRIES(true, KIND_LEARNED)}};
    const int row = kind == KIND_LEARNED ? 3 : kind;
    if (kind == KIND_2NMS || row < 0 || row > 3 || variant < 0 || variant > 3) return nullptr;
    return table[et ? 1 : 0][row][variant];
}

}  // namespace ldpc
