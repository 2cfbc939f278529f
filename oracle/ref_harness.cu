/*
 * Harness that drives the reference's own, unmodified GPU kernels so that the
 * CPU oracle can be pinned against real reference outputs.  TEST
 * INFRASTRUCTURE ONLY: built by oracle/build_ref.sh into oracle/_ref/ (git
 * ignored) together with the reference sources it launches, and used by
 * oracle/make_golden.py.  Nothing in the product links it.
 *
 * It reproduces the body of the reference plugins' decode()
 * (decoder_oms/CGPU_Decoder_OMS_SIMD.cu:97-147 and the other four plugins;
 * decoder_oms_v2/CGPU_Decoder_MS_SIMD_v2.cu:120-266 for xMS) without the
 * plugin constructors, whose register-count guard exit(0)s for the NMS,
 * 2NMS and xMS kernels on sm_100a.  Buffers are sized so that every access
 * of the reference kernels stays inside an allocation: the inverse
 * interleaver reads variables up to round_up(N,128)-1 and the interleaver
 * reads up to 31 words past the last frame, so APP is padded to
 * round_up(N,128) rows and the staging buffer holds max(M, N+pad) rows.
 */
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "matrix/constantes_gpu.h"
#include "decoder_ms/cuda/CUDA_MS_SIMD.h"
#include "decoder_oms/cuda/CUDA_OMS_SIMD.h"
#include "decoder_nms/cuda/CUDA_NMS_SIMD.h"
#include "decoder_2nms/cuda/CUDA_2NMS_SIMD.h"
#include "decoder_oms_v2/cuda/CUDA_OMS_SIMD_v2.h"
#include "transpose/GPU_Transpose_uint8.h"

#ifndef DEG_2
#define DEG_2 0
#define DEG_2_COMPUTATIONS 0
#endif

extern "C" int ref_info(int* out)
{
    out[0] = _N;
    out[1] = _K;
    out[2] = _M;
    out[3] = NB_DEGRES;
    out[4] = DEG_1;
    out[5] = DEG_1_COMPUTATIONS;
    out[6] = DEG_2;
    out[7] = DEG_2_COMPUTATIONS;
    return 0;
}

#define CK(x)                                                                        \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            fprintf(stderr, "ref_harness: %s (%s:%d)\n", cudaGetErrorString(e_),   \
                    __FILE__, __LINE__);                                             \
            return -1;                                                               \
        }                                                                            \
    } while (0)

/*
 * kind: 0 MS, 1 OMS, 2 NMS, 3 2NMS, 4 xMS.  W = 32-bit words per variable
 * (= frames / 4), multiple of 32 and of `block`.  llr: 4W*N bytes as the
 * plugin receives them; hard: 4W*N bytes; app: N*W words; msg: M*W words.
 * Returns the kernel time in microseconds (>= 0) or -1.
 */
extern "C" double ref_decode(int kind, const int8_t* llr, int W, int iters, int block,
                             uint8_t* hard, int8_t* app, int8_t* msg)
{
    if (W % 32 || W % block || iters < 1) return -1;
    const size_t npad = ((size_t)_N + 127) / 128 * 128;
    const size_t stage_rows = (size_t)_M > npad + 32 ? (size_t)_M : npad + 32;
    unsigned int *d_pos = 0, *d_app = 0, *d_stage = 0;
    CK(cudaMalloc(&d_pos, sizeof(unsigned int) * _M));
    CK(cudaMalloc(&d_app, sizeof(unsigned int) * npad * W));
    CK(cudaMalloc(&d_stage, sizeof(unsigned int) * stage_rows * W));
    CK(cudaMemset(d_app, 0, sizeof(unsigned int) * npad * W));
    CK(cudaMemset(d_stage, 0, sizeof(unsigned int) * stage_rows * W));
    CK(cudaMemcpy(d_pos, PosNoeudsVariable, sizeof(unsigned int) * _M, cudaMemcpyHostToDevice));
    const size_t in_bytes = (size_t)_N * W * 4;
    dim3 tgrid(1, W / 32), tthreads(32, 32);
    if (kind == 4) {
        CK(cudaMemcpy(d_app, llr, in_bytes, cudaMemcpyHostToDevice));
    } else {
        CK(cudaMemcpy(d_stage, llr, in_bytes, cudaMemcpyHostToDevice));
        Interleaver_uint8<<<tgrid, tthreads>>>((int*)d_stage, (int*)d_app, _N, W);
        CK(cudaGetLastError());
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    unsigned nb = W / block;
    switch (kind) {
    case 0: LDPC_Sched_Stage_1_MS_SIMD<<<nb, block>>>(d_app, d_stage, d_pos, iters); break;
    case 1: LDPC_Sched_Stage_1_OMS_SIMD<<<nb, block>>>(d_app, d_stage, d_pos, iters); break;
    case 2: LDPC_Sched_Stage_1_NMS_SIMD<<<nb, block>>>(d_app, d_stage, d_pos, iters); break;
    case 3: LDPC_Sched_Stage_1_2NMS_SIMD<<<nb, block>>>(d_app, d_stage, d_pos, iters); break;
    case 4:
#if NB_DEGRES != 1
        LDPC_Sched_Stage_1_MS_SIMD_Two_CN_Degs<<<nb, block>>>(d_app, d_stage, d_pos, iters);
#elif DEG_1 == 6
        LDPC_Sched_Stage_1_MS_SIMD_Deg_6_Only<<<nb, block>>>(d_app, d_stage, d_pos, iters);
#elif DEG_1 == 7
        LDPC_Sched_Stage_1_MS_SIMD_Deg_7_Only<<<nb, block>>>(d_app, d_stage, d_pos, iters);
#endif
        break;
    default: return -1;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(e1));
    CK(cudaDeviceSynchronize());
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (app) CK(cudaMemcpy(app, d_app, (size_t)_N * W * 4, cudaMemcpyDeviceToHost));
    if (msg) CK(cudaMemcpy(msg, d_stage, (size_t)_M * W * 4, cudaMemcpyDeviceToHost));
    InvInterleaver_uint8<<<tgrid, tthreads>>>((int*)d_app, (int*)d_stage, _N, W);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(hard, d_stage, in_bytes, cudaMemcpyDeviceToHost));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_pos);
    cudaFree(d_app);
    cudaFree(d_stage);
    return ms * 1000.0;
}
