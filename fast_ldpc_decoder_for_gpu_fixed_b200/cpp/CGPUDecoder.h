// C++ decoder plugin classes with the reference's names and signatures,
// forwarding to the C ABI of libldpc_b200.so.
//
// Reference: src/decoder_template/CGPUDecoder.h:19-35 (abstract base) and the
// five plugins selected in src/main.cpp:213-228:
//   CGPU_Decoder_MS_SIMD   (-MS, -fMS)   decoder_ms/CGPU_Decoder_MS_SIMD.h
//   CGPU_Decoder_OMS_SIMD  (-OMS)        decoder_oms/CGPU_Decoder_OMS_SIMD.h
//   CGPU_Decoder_NMS_SIMD  (-NMS)        decoder_nms/CGPU_Decoder_NMS_SIMD.h
//   CGPU_Decoder_2NMS_SIMD (-2NMS)       decoder_2nms/CGPU_Decoder_2NMS_SIMD.h
//   CGPU_Decoder_MS_SIMD_v2 (-xMS)       decoder_oms_v2/CGPU_Decoder_MS_SIMD_v2.h
// Same constructor arguments (nb_frames = 32-bit lanes = codewords / 4; n, k, m =
// variables, checks, edges of the H matrix), same decode(float*, int*, int)
// contract (frame-major int8 LLRs in, frame-major 0/1 bytes out, host
// buffers).  Differences: the H matrix is chosen at run time with
// CGPUDecoder::select_code instead of src/matrix/code.h; errors do not exit(0)
// the process: decode() records a status readable with last_status().
#ifndef LDPC_B200_CGPUDECODER_H
#define LDPC_B200_CGPUDECODER_H

#include <cstddef>
#include <string>

#include "ldpc_b200.h"

class CGPUDecoder {
protected:
    ldpc_decoder* dec_;
    size_t nb_frames;
    size_t sz_nodes;
    size_t sz_checks;
    size_t sz_msgs;
    int status_;

    CGPUDecoder(size_t _nb_frames, size_t n, size_t k, size_t m, int kind);
    void run(float var_nodes[], int Rprime_fix[], int nombre_iterations);

public:
    virtual ~CGPUDecoder();
    virtual void initialize() = 0;
    virtual void decode(float var_nodes[], int Rprime_fix[], int nombre_iterations) = 0;

    int last_status() const { return status_; }
    std::string last_error() const;

    // The H matrix the plugins are built for (the reference's compile-time CODE).
    static void select_code(ldpc_code* code);
    static ldpc_code* selected_code();
};

#define LDPC_B200_PLUGIN(NAME, KIND)                                                        \
    class NAME : public CGPUDecoder {                                                       \
    public:                                                                                 \
        NAME(size_t _nb_frames, size_t n, size_t k, size_t m) : CGPUDecoder(_nb_frames, n, k, m, KIND) {} \
        ~NAME() {}                                                                          \
        void initialize() {}                                                                \
        void decode(float var_nodes[], int Rprime_fix[], int nombre_iterations)             \
        {                                                                                   \
            run(var_nodes, Rprime_fix, nombre_iterations);                                  \
        }                                                                                   \
    };

LDPC_B200_PLUGIN(CGPU_Decoder_MS_SIMD, LDPC_MS)
LDPC_B200_PLUGIN(CGPU_Decoder_OMS_SIMD, LDPC_OMS)
LDPC_B200_PLUGIN(CGPU_Decoder_NMS_SIMD, LDPC_NMS)
LDPC_B200_PLUGIN(CGPU_Decoder_2NMS_SIMD, LDPC_2NMS)
LDPC_B200_PLUGIN(CGPU_Decoder_MS_SIMD_v2, LDPC_XMS)

#endif
