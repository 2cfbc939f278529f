// Plugin classes over the C ABI (see CGPUDecoder.h).
#include "CGPUDecoder.h"

#include <cstdio>
#include <stdexcept>

static ldpc_code* g_code = nullptr;

void CGPUDecoder::select_code(ldpc_code* code) { g_code = code; }
ldpc_code* CGPUDecoder::selected_code() { return g_code; }

CGPUDecoder::CGPUDecoder(size_t _nb_frames, size_t n, size_t k, size_t m, int kind)
    : dec_(nullptr), nb_frames(_nb_frames), sz_nodes(n * _nb_frames), sz_checks(k * _nb_frames),
      sz_msgs(m * _nb_frames), status_(LDPC_OK)
{
    int info[8];
    if (!g_code) throw std::runtime_error("CGPUDecoder: no code selected (CGPUDecoder::select_code)");
    ldpc_code_info(g_code, info);
    if ((size_t)info[0] != n || (size_t)info[1] != k || (size_t)info[2] != m) {
        char buf[160];
        snprintf(buf, sizeof buf, "CGPUDecoder: (N,K,M)=(%zu,%zu,%zu) but the selected code is (%d,%d,%d)", n, k, m,
                 info[0], info[1], info[2]);
        throw std::runtime_error(buf);
    }
    status_ = ldpc_decoder_create(&dec_, g_code, kind, nb_frames, LDPC_PACK_AUTO, 0);
    if (status_ != LDPC_OK) throw std::runtime_error(std::string("CGPUDecoder: ") + ldpc_last_error_string());
}

CGPUDecoder::~CGPUDecoder() { ldpc_decoder_destroy(dec_); }

void CGPUDecoder::run(float var_nodes[], int Rprime_fix[], int nombre_iterations)
{
    status_ = ldpc_decode_host(dec_, reinterpret_cast<const int8_t*>(var_nodes), reinterpret_cast<uint8_t*>(Rprime_fix),
                               nombre_iterations);
}

std::string CGPUDecoder::last_error() const { return ldpc_last_error_string(); }
