// Instantiations of the 2-frame QC register-message decoder whose check rows are split over
// 4 lanes (decode_qc_split_kernel, decoder path 7; Z <= 128), for the 24-column irregular bases
// at rates 1/2, 2/3, 3/4, 5/6 (12, 8, 6, 4 layers of row degree up to 10, 14, 18, 24), any
// Z, every kind but 2NMS, with and without the syndrome early stop.
#include "qc_kernel.cuh"

namespace ldpc {

#define LDPC_QCS(KIND, D, L, S)                                                                  \
    if (kind == KIND && dt == D && layers == L && split == S)                                      \
        return et ? (const void*)decode_qc_split_kernel<KIND, D, L, S, true>                       \
                  : (const void*)decode_qc_split_kernel<KIND, D, L, S, false>;
#define LDPC_QCS_KINDS(D, L, S) \
    LDPC_QCS(KIND_MS, D, L, S) LDPC_QCS(KIND_OMS, D, L, S) LDPC_QCS(KIND_NMS, D, L, S) LDPC_QCS(KIND_LEARNED, D, L, S)

const void* kernel_table_qc_split(int kind, int dt, int layers, int split, bool et)
{
    LDPC_QCS_KINDS(10, 12, 4) LDPC_QCS_KINDS(14, 8, 4) LDPC_QCS_KINDS(18, 6, 4) LDPC_QCS_KINDS(24, 4, 4)
    return nullptr;
}

}  // namespace ldpc
