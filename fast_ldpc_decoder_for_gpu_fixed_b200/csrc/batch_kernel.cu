// Batched decoding of several codes of different length and rate in one
// persistent launch (no reference counterpart: the reference decodes one
// compile-time H per process).
//
// Work items are 4-frame words, numbered code after code.  Each resident CTA
// takes the next item from a global counter, finds its code from the prefix
// counts, and decodes the word with that code's level schedule
// (decode_word_levels: the same arithmetic and early stop as the per-code
// kernels), so every CTA stays busy until the batch is empty whatever the mix of
// code sizes and per-word iteration counts.  Shared memory is sized for the
// largest code of the batch.
#include "decode_kernel.cuh"

namespace ldpc {

struct BatchCode {
    Plan plan;
    const int8_t* llr;      // frame-major int8, 4 * words frames
    void* out;              // 0/1 bytes (or packed bits), frame-major
    int32_t* iters_out;     // [words] or null
    uint8_t* synd_out;      // [4 * words] per-frame syndrome flags or null
    long long words;
    long long first_item;   // items of the codes before this one
    int quirk;              // OMS first-iteration quirk (row classes of this code)
    int out_packed;
    int variant;            // this code's row-degree class: 0 <= 8, 1 <= 16, 2 <= 32
};

// VMAX: the largest degree class of the batch; each word runs the unrolled update
// of its own code's class
// PF: the per-frame early stop (PackSIMD4; iters_out then holds one count per frame)
template <class PK, int KIND, int VMAX, bool PF = false>
__global__ void __launch_bounds__(256) decode_batch_kernel(const BatchCode* __restrict__ codes, int n_codes,
                                                           unsigned long long* counter, long long total, const Job base)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_odd[4];
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long item = s_item;
        if (item >= total) break;  // uniform
        int c = 0;
        while (c + 1 < n_codes && item >= codes[c + 1].first_item) c++;
        const BatchCode& bc = codes[c];
        Job J = base;
        J.llr = bc.llr;
        J.out = bc.out;
        J.out_packed = bc.out_packed;
        J.iters_out = bc.iters_out;
        J.synd_out = bc.synd_out;
        J.total_words = bc.words;
        J.word0 = 0;
        J.quirk = bc.quirk;
        const Plan P = bc.plan;
        const long long g = item - bc.first_item;
        if (VMAX == 0 || bc.variant == 0)
            decode_word_levels<PK, KIND, 8, false, PF>(P, J, g, smem_raw, s_odd);
        else if (VMAX == 1 || bc.variant == 1)
            decode_word_levels<PK, KIND, (VMAX >= 1 ? 16 : 8), false, PF>(P, J, g, smem_raw, s_odd);
        else
            decode_word_levels<PK, KIND, (VMAX >= 2 ? 32 : 8), false, PF>(P, J, g, smem_raw, s_odd);
        __syncthreads();  // shared memory and s_item are reused by the next item
    }
}

#define LDPC_BATCH_ROW(PK, KIND)                                                                  \
    {(const void*)decode_batch_kernel<PK, KIND, 0>, (const void*)decode_batch_kernel<PK, KIND, 1>, \
     (const void*)decode_batch_kernel<PK, KIND, 2>},
#define LDPC_BATCH_PACK(PK)                                                                                         \
    {LDPC_BATCH_ROW(PK, KIND_MS) LDPC_BATCH_ROW(PK, KIND_OMS) LDPC_BATCH_ROW(PK, KIND_NMS) LDPC_BATCH_ROW(PK, KIND_2NMS) \
         LDPC_BATCH_ROW(PK, KIND_LEARNED)},

// [pack: SIMD4, F16X2, I8][kind: MS, OMS, NMS, 2NMS, LEARNED][largest degree class: <= 8, 16, 32]
const void* kernel_table_batch(int pack, int kind, int variant)
{
    static const void* table[3][5][3] = {LDPC_BATCH_PACK(PackSIMD4) LDPC_BATCH_PACK(PackF16x2) LDPC_BATCH_PACK(PackI8)};
    const int row = kind == KIND_LEARNED ? 4 : kind;
    if (pack < 0 || pack > 2 || row < 0 || row > 4 || variant < 0 || variant > 2) return nullptr;
    return table[pack][row][variant];
}

#define LDPC_BATCH_ROW_PF(KIND)                                                                                \
    {(const void*)decode_batch_kernel<PackSIMD4, KIND, 0, true>, (const void*)decode_batch_kernel<PackSIMD4, KIND, 1, true>, \
     (const void*)decode_batch_kernel<PackSIMD4, KIND, 2, true>},

// the per-frame early stop, PackSIMD4: [kind: MS, OMS, NMS, LEARNED][largest degree class]
const void* kernel_table_batch_pf(int kind, int variant)
{
    static const void* table[4][3] = {LDPC_BATCH_ROW_PF(KIND_MS) LDPC_BATCH_ROW_PF(KIND_OMS) LDPC_BATCH_ROW_PF(KIND_NMS)
                                          LDPC_BATCH_ROW_PF(KIND_LEARNED)};
    const int row = kind == KIND_LEARNED ? 3 : kind;
    if (kind == KIND_2NMS || row < 0 || row > 3 || variant < 0 || variant > 2) return nullptr;
    return table[row][variant];
}

size_t batch_code_bytes() { return sizeof(BatchCode); }

// fills one BatchCode record on the host (the struct stays private to this file)
void batch_code_fill(void* rec, const Plan& plan, const int8_t* llr, void* out, int32_t* iters_out, uint8_t* synd_out,
                     long long words, long long first_item, int quirk, int out_packed, int variant)
{
    BatchCode* b = reinterpret_cast<BatchCode*>(rec);
    b->synd_out = synd_out;
    b->variant = variant;
    b->plan = plan;
    b->llr = llr;
    b->out = out;
    b->iters_out = iters_out;
    b->words = words;
    b->first_item = first_item;
    b->quirk = quirk;
    b->out_packed = out_packed;
}

}  // namespace ldpc
