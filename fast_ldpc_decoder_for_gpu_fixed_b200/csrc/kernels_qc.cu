// Instantiations of the QC register-message decoder for the code shapes in use:
// (row degree, exact, layers, power-of-two Z), each with and without the
// syndrome early stop compiled in.
#include "qc_kernel.cuh"

namespace ldpc {

#define LDPC_QC(KIND, D, EX, L, P2)                                                                  \
    if (kind == KIND && dt == D && exact == EX && layers == L && pow2 == P2)                         \
        return et ? (const void*)decode_qc_kernel<KIND, D, EX, L, P2, true>                          \
                  : (const void*)decode_qc_kernel<KIND, D, EX, L, P2, false>;
#define LDPC_QC_KINDS(D, EX, L, P2) \
    LDPC_QC(KIND_MS, D, EX, L, P2) LDPC_QC(KIND_OMS, D, EX, L, P2) \
    LDPC_QC(KIND_NMS, D, EX, L, P2) LDPC_QC(KIND_2NMS, D, EX, L, P2) LDPC_QC(KIND_LEARNED, D, EX, L, P2)

const void* kernel_table_qc(int kind, int dt, bool exact, int layers, bool pow2, bool et)
{
    LDPC_QC_KINDS(6, true, 8, true)  // regular (3,6) rate-1/2 QC, 8x16 base (Z = 2^k)
    return nullptr;
}

}  // namespace ldpc
