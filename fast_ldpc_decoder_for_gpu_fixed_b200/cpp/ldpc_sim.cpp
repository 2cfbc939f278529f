// Monte-Carlo BER/FER simulator: the reference's src/main.cpp pipeline
// (AWGN channel -> decoder plugin -> error analyser, swept over Eb/N0) on top
// of libldpc_b200.so.
//
// Same command-line flags as src/main.cpp:120-192 (-min -max -pas -timer -iter
// -fer -qef -bpsk -qpsk -Eb/N0 -Es/N0 -n -fMS -xMS -MS -OMS -NMS -2NMS -info),
// plus -code <table name or .ldpc path> (the reference picks its H matrix at
// compile time in src/matrix/code.h), -seed <u64> and -json (one JSON line per
// Eb/N0 point).  The channel runs on the GPU (Philox4x32-10 instead of cuRAND
// XORWOW, same quantiser) and its LLRs land in pinned host memory, so every
// decode() call goes through the reference-facing host-buffer path with both
// PCIe copies inside the timed window, as src/main.cpp:266-268 times it.  The
// error analyser counts, like ber_analyzer/CErrorAnalyzer.cpp:142-158, the
// non-zero decisions among the first N-K bytes of each frame.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "CGPUDecoder.h"

namespace {

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Counters {  // CErrorAnalyzer totals
    long long frames = 0, bit_errors = 0, frame_errors = 0;
    double ber(int n_vars) const { return frames ? (double)bit_errors / frames / n_vars : 0; }
    double fer() const { return frames ? (double)frame_errors / frames : 0; }
};

void count_errors(const uint8_t* hard, long long frames, int n, int n_vars, Counters& c)
{
    for (long long f = 0; f < frames; f++) {
        const uint8_t* h = hard + f * n;
        int e = 0;
        for (int i = 0; i < n_vars; i++) e += h[i] != 0;
        c.bit_errors += e;
        c.frame_errors += (e != 0);
        c.frames += 1;
    }
}

std::string find_table(const std::string& name, const char* argv0)
{
    if (name.find('/') != std::string::npos || name.find(".ldpc") != std::string::npos) return name;
    std::string exe = argv0;
    size_t p = exe.rfind('/');
    std::string dir = (p == std::string::npos) ? "." : exe.substr(0, p);
    return dir + "/../codes/" + name + ".ldpc";
}

void show_info()
{
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, 0);
    printf("(II) GPU                              : %s\n", prop.name);
    printf("(II) Nombre de Multi-Processor        : %d\n", prop.multiProcessorCount);
    printf("(II) + totalGlobalMem                 : %zu Mo\n", prop.totalGlobalMem / 1024 / 1024);
    printf("(II) + sharedMemPerBlockOptin         : %zu Ko\n", prop.sharedMemPerBlockOptin / 1024);
    printf("(II) + regsPerMultiprocessor          : %d\n", prop.regsPerMultiprocessor);
    printf("(II) library version                  : %d\n", ldpc_version());
}

}  // namespace

int main(int argc, char* argv[])
{
    double min_snr = 0.50, max_snr = 3.01, step_snr = 0.10;
    int iters = 20, stop_timer_s = -1, fe_limit = 200, nb_lanes = 1024;
    bool es_n0 = false, qef = false, json = false;
    double qef_limit = 1e-7;
    uint64_t seed = 1234;
    std::string type = "fMS", code_name = "4000x2000";
    for (int p = 1; p < argc; p++) {
        std::string a = argv[p];
        auto next = [&]() -> const char* {
            if (p + 1 >= argc) {
                printf("(EE) Missing value after %s\n", argv[p]);
                exit(1);
            }
            return argv[++p];
        };
        if (a == "-min") min_snr = atof(next());
        else if (a == "-max") max_snr = atof(next());
        else if (a == "-pas") step_snr = atof(next());
        else if (a == "-timer") stop_timer_s = atoi(next());
        else if (a == "-iter") iters = atoi(next());
        else if (a == "-fer") fe_limit = atoi(next());
        else if (a == "-qef") { qef = true; qef_limit = atof(next()); }
        else if (a == "-bpsk" || a == "-qpsk") { /* the reference channel ignores the modulation flag */ }
        else if (a == "-Eb/N0") es_n0 = false;
        else if (a == "-Es/N0") es_n0 = true;
        else if (a == "-n") nb_lanes = atoi(next());
        else if (a == "-fMS" || a == "-xMS" || a == "-MS" || a == "-OMS" || a == "-NMS" || a == "-2NMS") type = a.substr(1);
        else if (a == "-code") code_name = next();
        else if (a == "-seed") seed = strtoull(next(), nullptr, 10);
        else if (a == "-json") json = true;
        else if (a == "-info") { show_info(); return 0; }
        else {
            printf("(EE) Unknown argument (%d) => [%s]\n", p, argv[p]);
            return 1;
        }
    }

    ldpc_code* code = nullptr;
    std::string path = find_table(code_name, argv[0]);
    if (ldpc_code_load(&code, path.c_str()) != LDPC_OK) {
        printf("(EE) %s\n", ldpc_last_error_string());
        return 1;
    }
    int ci[8];
    ldpc_code_info(code, ci);
    const int N = ci[0], K = ci[1], M = ci[2], n_vars = ci[6];
    const double rate = (double)n_vars / N;
    CGPUDecoder::select_code(code);
    printf("(II) LDPC DECODER - layered schedule (B200 engine)\n");
    printf("(II) Code LDPC (N, K)     : (%d,%d)  [%s]\n", N, K, path.c_str());
    printf("(II) Rendement du code    : %.3f\n", rate);
    printf("(II) # ITERATIONs du CODE : %d\n", iters);
    printf("(II) FER LIMIT FOR SIMU   : %d\n", fe_limit);
    printf("(II) SIMULATION  RANGE    : [%.2f, %.2f], STEP = %.2f\n", min_snr, max_snr, step_snr);
    printf("(II) MODE EVALUATION      : %s\n", es_n0 ? "Es/N0" : "Eb/N0");
    printf("(II) MIN-SUM ALGORITHM    : %s\n", type.c_str());

    const size_t frames = 4 * (size_t)nb_lanes, bytes = frames * N;
    int8_t* noise = nullptr;      // CTrame::t_noise_data (pinned)
    uint8_t* decoded = nullptr;   // CTrame::t_decode_data (pinned)
    int8_t* d_noise = nullptr;
    if (cudaMallocHost(&noise, bytes) != cudaSuccess || cudaMallocHost(&decoded, bytes) != cudaSuccess ||
        cudaMalloc(&d_noise, bytes) != cudaSuccess) {
        printf("(EE) allocation of %zu-byte buffers failed\n", bytes);
        return 1;
    }

    CGPUDecoder* decoder = nullptr;
    try {
        if (type == "fMS" || type == "MS") decoder = new CGPU_Decoder_MS_SIMD(nb_lanes, N, K, M);
        else if (type == "OMS") decoder = new CGPU_Decoder_OMS_SIMD(nb_lanes, N, K, M);
        else if (type == "NMS") decoder = new CGPU_Decoder_NMS_SIMD(nb_lanes, N, K, M);
        else if (type == "2NMS") decoder = new CGPU_Decoder_2NMS_SIMD(nb_lanes, N, K, M);
        else decoder = new CGPU_Decoder_MS_SIMD_v2(nb_lanes, N, K, M);
    } catch (const std::exception& e) {
        printf("(EE) %s\n", e.what());
        return 1;
    }
    decoder->initialize();

    uint64_t batch = 0;
    auto generate = [&](double sigma) {  // CChanel_AWGN_SIMD::generate, on the GPU
        ldpc_channel_awgn(d_noise, frames, N, (float)sigma, seed, batch++, nullptr, 0, nullptr);
        cudaMemcpy(noise, d_noise, bytes, cudaMemcpyDeviceToHost);
    };

    const double t_start = now_s();
    double temps_ms = 0;
    long long fdecoding = 0;
    bool timed_out = false;
    for (double ebn0 = min_snr; ebn0 <= max_snr; ebn0 += step_snr) {
        const double sigma = ldpc_sigma(ebn0, rate, es_n0);
        const double t_point = now_s();
        double t_refresh = now_s();
        Counters err;
        generate(sigma);
        while (true) {
            double t0 = now_s();
            decoder->decode(reinterpret_cast<float*>(noise), reinterpret_cast<int*>(decoded), iters);
            temps_ms += (now_s() - t0) * 1e3;
            fdecoding += 1;
            if (decoder->last_status() != LDPC_OK) {
                printf("(EE) decode failed: %s\n", decoder->last_error().c_str());
                return 1;
            }
            generate(sigma);
            count_errors(decoded, frames, N, n_vars, err);
            if (err.frame_errors >= fe_limit) break;
            if (now_s() - t_refresh >= 1) {
                t_refresh = now_s();
                printf("(RT) FRA: %8lld | FE: %3lld | FER: %2.2e | BE : %5lld | BER: %2.2e\r", err.frames,
                       err.frame_errors, err.fer(), err.bit_errors, err.ber(n_vars));
                fflush(stdout);
            }
            if (stop_timer_s != -1 && now_s() - t_start >= stop_timer_s) {
                double ms = temps_ms / fdecoding;
                printf("(II) THE SIMULATION HAS STOP DUE TO THE (USER) TIME CONTRAINT.\n");
                printf("(II) PERFORMANCE EVALUATION WAS PERFORMED ON %lld RUNS, TOTAL TIME = %.0fms\n", fdecoding,
                       temps_ms);
                printf("(II) + TIME / RUN = %.3fms\n", ms);
                printf("(II) + DECODER THROUGHPUT (Mbps)= %.1f   [coded bits, copies included]\n",
                       frames * (double)N / ms / 1e3);
                printf("(II) + DECODED INFO THROUGHPUT (Gbit/s) = %.3f\n", frames * (double)n_vars / ms / 1e6);
                timed_out = true;
                break;
            }
        }
        double runtime = now_s() - t_point;
        printf("SNR = %.2f | BER =  %2.3e | FER =  %2.3e | BPS =  %2.2f | MATRICES = %10lld| FE = %lld | BE = %lld | "
               "RUNTIME = %.1fs\n",
               ebn0, err.ber(n_vars), err.fer(), err.frames * (double)N / runtime / 1e6, err.frames,
               err.frame_errors, err.bit_errors, runtime);
        if (json)
            printf("{\"ebn0\": %.3f, \"ber\": %.6e, \"fer\": %.6e, \"frames\": %lld, \"frame_errors\": %lld, "
                   "\"bit_errors\": %lld, \"decoder\": \"%s\", \"iters\": %d, \"code\": \"%s\"}\n",
                   ebn0, err.ber(n_vars), err.fer(), err.frames, err.frame_errors, err.bit_errors, type.c_str(), iters,
                   code_name.c_str());
        fflush(stdout);
        if (timed_out) break;
        if (qef && err.ber(n_vars) < qef_limit) {
            printf("(II) THE SIMULATION HAS STOP DUE TO THE (USER) QUASI-ERROR FREE CONTRAINT.\n");
            break;
        }
    }
    delete decoder;
    ldpc_code_destroy(code);
    cudaFreeHost(noise);
    cudaFreeHost(decoded);
    cudaFree(d_noise);
    return 0;
}
