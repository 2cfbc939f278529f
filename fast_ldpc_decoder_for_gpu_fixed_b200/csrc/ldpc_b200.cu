// C ABI of the B200 fixed-point LDPC decoding engine (declared in include/ldpc_b200.h).
//
// Host-side responsibilities:
//   * code objects: the H matrix as CSR rows in the reference's layer order
//     (src/matrix/<code>/constantes_decoder.h:3 + constantes_gpu.h:6-16), and
//     the level schedule that lets rows of one level run concurrently while
//     reproducing the reference's serial in-place row order bit for bit;
//   * decoder objects (src/decoder_template/CGPUDecoder.cpp:14-54 and the
//     plugin constructors): device copies of the schedule, the I/O staging
//     buffers the reference keeps in device_V / d_MSG_C_2_V, streams;
//   * decode calls: host buffers (the reference's synchronous decode(),
//     src/decoder_oms/CGPU_Decoder_OMS_SIMD.cu:97-147) with the H2D copy,
//     decoding and D2H copy pipelined over chunks of words; device buffers on a
//     caller stream.
// Errors are status codes plus a per-thread message; nothing exits the
// process (the reference's ERROR_CHECK prints and exit(0)s,
// src/custom_api/custom_cuda.cu:5-17).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ldpc_b200.h"
#include "frame_kernel.cuh"
#include "qc_kernel.cuh"

using namespace ldpc;

static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int ldpc_internal_fail(int code, const char* msg) { return fail(code, "%s", msg); }

// The dynamic shared-memory limit is an attribute of the kernel function, shared by
// every decoder that launches it: only ever raise it, so that a later decoder of a
// smaller code does not lower it under an earlier one.
cudaError_t ldpc_internal_raise_smem(const void* fn, size_t bytes)
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess || (size_t)fa.maxDynamicSharedSizeBytes >= bytes) return e;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

#define CUDA_TRY(x)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess)                                                               \
            return fail(e_ == cudaErrorMemoryAllocation ? LDPC_ERR_NOMEM : LDPC_ERR_CUDA,    \
                        "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

static const int kMaxDegree = 32;

struct ldpc_code {
    int n = 0, m = 0, e = 0, dmax = 0;
    std::vector<int32_t> row_ptr, cols;
    std::vector<uint8_t> row_class;
    // schedule
    std::vector<int32_t> order;   // order[r'] = row in table order
    std::vector<int2> levels;     // (first r', count)
    int widest = 0;
    // quasi-cyclic description, when the code was built from one
    bool qc = false;
    int z = 0, mb = 0, nb = 0;
    std::vector<int32_t> shifts;  // [mb][nb], -1 = zero block
};

struct ldpc_decoder {
    int kind = 0, pack = 0, device = 0;
    bool early = false;  // LDPC_FLAG_EARLY_STOP
    unsigned early_slack = LDPC_EARLY_STOP_DEFAULT_SLACK;
    size_t nb_words = 0;
    int n = 0, m = 0, e = 0;
    Plan plan{};
    uint16_t* d_cols = nullptr;
    uint8_t* d_rowdeg = nullptr;
    uint8_t* d_rowcls = nullptr;
    int2* d_levels = nullptr;
    int32_t* d_edge_orig = nullptr;
    int32_t* d_vptr = nullptr;   // flooding: variable -> message indices (Plan::vptr / vedge)
    int32_t* d_vedge = nullptr;
    int8_t* d_in = nullptr;    // staging for decode_host (reference: d_MSG_C_2_V as input staging)
    uint8_t* d_out = nullptr;  // staging for decode_host (reference: d_MSG_C_2_V as output staging)
    void* d_aux = nullptr;     // staging of iteration counts and syndrome flags for ldpc_decode_host_ex
    cudaStream_t s_comp = nullptr, s_h2d = nullptr, s_d2h = nullptr;
    int threads = 0, smem = 0, ctas_per_sm = 0, regs = 0;
    const void* kfn = nullptr;
    const void* kfn_alt = nullptr;  // the same kernel with the other early-stop setting (paths 1, 3 and 4)
    // path 1, LDPC_LEARNED: the general, the offset-only (every scale 1.0) and the OMS kernel
    // (every scale 1.0 and every offset 1: OMS's arithmetic, without its first-iteration
    // quirk, which the learned kind does not have) with and without the early stop;
    // ldpc_decoder_set_learned picks from them
    const void* kfn_lrn[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};  // [constants][early stop]
    // 0 = level-scheduled kernel, 1 = QC register-message kernel, 2 = level-scheduled, 2 frames per CTA,
    // 3 = one frame per CTA, 4 = QC register-message, 2 frames per CTA, 5 = QC register-message with
    // per-frame early stop and lane refill (persistent CTAs)
    int path = 0;
    bool pf_levels = false;  // path 0 with the per-frame early stop (SIMD4; counts per frame)
    bool frame2 = false;     // path 3 with two frames per CTA (decode_frame2_kernel)
    int sms = 0;  // paths 3 and 5: multiprocessors (grid size)
    // path 3 (frame_kernel.cuh): the stages of one iteration, their records, the message
    // scratch (fslots CTA slots) and the status word the kernel sets when a copy wait gave up
    FrameStages fst{};
    FrameStage* d_fst = nullptr;
    unsigned char* d_frec = nullptr;
    unsigned char* d_fmsg = nullptr;
    int* d_status = nullptr;
    long long fslots = 0;
    int grid_mult = 1;  // CTAs per 4-frame word
    QCParams qcp{};
    uint16_t* d_lut = nullptr;  // LDPC_LEARNED magnitude tables [its][2][128]
    int lut_its = 0;
};

// Row schedule and CTA width of a decoder, for the training kernels (train.cu).
int ldpc_internal_plan(const ldpc_decoder* d, Plan* plan, int* threads)
{
    if (!d || !d->d_cols) return -1;
    *plan = d->plan;
    *threads = std::min(256, std::max(32, (d->threads + 31) / 32 * 32));
    return 0;
}

// ------------------------------------------------------------------------
// codes
// ------------------------------------------------------------------------

static int build_schedule(ldpc_code* c)
{
    std::vector<int> lastlev(c->n, -1), level(c->m, 0);
    int nlev = 0;
    for (int r = 0; r < c->m; r++) {
        int L = 0;
        for (int k = c->row_ptr[r]; k < c->row_ptr[r + 1]; k++) L = std::max(L, lastlev[c->cols[k]] + 1);
        level[r] = L;
        for (int k = c->row_ptr[r]; k < c->row_ptr[r + 1]; k++) lastlev[c->cols[k]] = L;
        nlev = std::max(nlev, L + 1);
    }
    c->order.resize(c->m);
    for (int r = 0; r < c->m; r++) c->order[r] = r;
    // any order inside a level is exact; group equal degrees to keep warps uniform
    std::stable_sort(c->order.begin(), c->order.end(), [&](int a, int b) {
        if (level[a] != level[b]) return level[a] < level[b];
        int da = c->row_ptr[a + 1] - c->row_ptr[a], db = c->row_ptr[b + 1] - c->row_ptr[b];
        return da > db;
    });
    c->levels.assign(nlev, make_int2(0, 0));
    for (int i = 0; i < c->m; i++) {
        int L = level[c->order[i]];
        if (c->levels[L].y == 0) c->levels[L].x = i;
        c->levels[L].y++;
    }
    c->widest = 0;
    for (auto& l : c->levels) c->widest = std::max(c->widest, l.y);
    return LDPC_OK;
}

static int code_init(ldpc_code* c)
{
    c->e = c->row_ptr[c->m];
    c->dmax = 0;
    for (int r = 0; r < c->m; r++) {
        int d = c->row_ptr[r + 1] - c->row_ptr[r];
        if (d < 1) return fail(LDPC_ERR_ARG, "row %d has no edge", r);
        c->dmax = std::max(c->dmax, d);
    }
    for (int k = 0; k < c->e; k++)
        if (c->cols[k] < 0 || c->cols[k] >= c->n)
            return fail(LDPC_ERR_ARG, "edge %d: variable index %d outside [0,%d)", k, c->cols[k], c->n);
    return build_schedule(c);
}

extern "C" int ldpc_code_create(ldpc_code** out, int n_vars, int n_checks, const int32_t* row_ptr,
                                const int32_t* cols, const uint8_t* row_class)
{
    if (!out || !row_ptr || !cols || n_vars <= 0 || n_checks <= 0)
        return fail(LDPC_ERR_ARG, "ldpc_code_create: null pointer or empty code");
    if (n_vars > 65535) return fail(LDPC_ERR_UNSUPPORTED, "ldpc_code_create: n=%d > 65535", n_vars);
    if (row_ptr[0] != 0) return fail(LDPC_ERR_ARG, "row_ptr[0] must be 0");
    for (int r = 0; r < n_checks; r++)
        if (row_ptr[r + 1] < row_ptr[r]) return fail(LDPC_ERR_ARG, "row_ptr not monotone at %d", r);
    ldpc_code* c = new ldpc_code();
    c->n = n_vars;
    c->m = n_checks;
    c->row_ptr.assign(row_ptr, row_ptr + n_checks + 1);
    c->cols.assign(cols, cols + row_ptr[n_checks]);
    c->row_class.assign(n_checks, 0);
    if (row_class)
        for (int r = 0; r < n_checks; r++) c->row_class[r] = row_class[r] ? 1 : 0;
    int rc = code_init(c);
    if (rc) {
        delete c;
        return rc;
    }
    *out = c;
    return LDPC_OK;
}

extern "C" int ldpc_code_create_from_table(ldpc_code** out, int n, int k_checks, int m_edges, int nb_degres,
                                           int deg1, int deg1_rows, int deg2, int deg2_rows,
                                           const uint32_t* pos)
{
    if (!out || !pos) return fail(LDPC_ERR_ARG, "ldpc_code_create_from_table: null pointer");
    if (nb_degres < 1 || nb_degres > 2) return fail(LDPC_ERR_ARG, "nb_degres must be 1 or 2");
    if (nb_degres == 1) deg2_rows = 0;
    if (deg1 < 1 || deg1_rows < 0 || (nb_degres == 2 && (deg2 < 1 || deg2_rows < 0)))
        return fail(LDPC_ERR_ARG, "bad degree groups");
    if (deg1_rows + deg2_rows != k_checks) return fail(LDPC_ERR_ARG, "row groups do not sum to %d checks", k_checks);
    if ((long long)deg1 * deg1_rows + (long long)deg2 * deg2_rows != m_edges)
        return fail(LDPC_ERR_ARG, "row groups do not sum to %d edges", m_edges);
    std::vector<int32_t> rp(k_checks + 1), cols(m_edges);
    std::vector<uint8_t> cls(k_checks);
    rp[0] = 0;
    for (int r = 0; r < k_checks; r++) {
        rp[r + 1] = rp[r] + (r < deg1_rows ? deg1 : deg2);
        cls[r] = r < deg1_rows ? 0 : 1;
    }
    for (int i = 0; i < m_edges; i++) cols[i] = (int32_t)pos[i];
    return ldpc_code_create(out, n, k_checks, rp.data(), cols.data(), cls.data());
}

extern "C" int ldpc_code_create_qc(ldpc_code** out, int z, int mb, int nb, const int32_t* shifts)
{
    if (!out || !shifts || z < 1 || mb < 1 || nb < 1) return fail(LDPC_ERR_ARG, "ldpc_code_create_qc: bad argument");
    if ((long long)z * nb > 65535) return fail(LDPC_ERR_UNSUPPORTED, "ldpc_code_create_qc: n = %d > 65535", z * nb);
    std::vector<int32_t> rp(1, 0), cols;
    for (int i = 0; i < mb; i++) {
        for (int k = 0; k < z; k++) {
            for (int j = 0; j < nb; j++) {
                int s = shifts[i * nb + j];
                if (s < -1 || s >= z) return fail(LDPC_ERR_ARG, "shift %d of block (%d,%d) outside [-1,%d)", s, i, j, z);
                if (s >= 0) cols.push_back(j * z + (k + s) % z);
            }
            rp.push_back((int32_t)cols.size());
        }
    }
    ldpc_code* c = nullptr;
    int rc = ldpc_code_create(&c, z * nb, z * mb, rp.data(), cols.data(), nullptr);
    if (rc) return rc;
    c->qc = true;
    c->z = z;
    c->mb = mb;
    c->nb = nb;
    c->shifts.assign(shifts, shifts + mb * nb);
    *out = c;
    return LDPC_OK;
}

extern "C" int ldpc_code_load(ldpc_code** out, const char* path)
{
    if (!out || !path) return fail(LDPC_ERR_ARG, "ldpc_code_load: null pointer");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(LDPC_ERR_ARG, "cannot open %s", path);
    char magic[8];
    uint32_t hdr[6];
    int rc = LDPC_OK;
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "LDPCH001", 8) || fread(hdr, 4, 6, f) != 6) {
        fclose(f);
        return fail(LDPC_ERR_ARG, "%s: not an .ldpc table", path);
    }
    uint32_t n = hdr[0], k = hdr[1], m = hdr[2], ng = hdr[3], cb = hdr[4];
    if (ng < 1 || ng > 1024 || (cb != 2 && cb != 4) || k == 0 || m == 0) {
        fclose(f);
        return fail(LDPC_ERR_ARG, "%s: bad header", path);
    }
    std::vector<uint32_t> groups(2 * ng);
    std::vector<uint32_t> pos(m);
    if (fread(groups.data(), 4, 2 * ng, f) != 2 * ng) rc = fail(LDPC_ERR_ARG, "%s: truncated", path);
    if (!rc) {
        if (cb == 2) {
            std::vector<uint16_t> p16(m);
            if (fread(p16.data(), 2, m, f) != m) rc = fail(LDPC_ERR_ARG, "%s: truncated", path);
            for (uint32_t i = 0; i < m; i++) pos[i] = p16[i];
        } else if (fread(pos.data(), 4, m, f) != m) {
            rc = fail(LDPC_ERR_ARG, "%s: truncated", path);
        }
    }
    fclose(f);
    if (rc) return rc;
    std::vector<int32_t> rp(1, 0), cols(pos.begin(), pos.end());
    std::vector<uint8_t> cls;
    for (uint32_t gi = 0; gi < ng; gi++)
        for (uint32_t i = 0; i < groups[2 * gi + 1]; i++) {
            rp.push_back(rp.back() + (int32_t)groups[2 * gi]);
            cls.push_back(gi > 0 ? 1 : 0);
        }
    if (rp.size() != k + 1 || (uint32_t)rp.back() != m) return fail(LDPC_ERR_ARG, "%s: inconsistent groups", path);
    return ldpc_code_create(out, (int)n, (int)k, rp.data(), cols.data(), cls.data());
}

extern "C" int ldpc_code_info(const ldpc_code* c, int* info)
{
    if (!c || !info) return fail(LDPC_ERR_ARG, "ldpc_code_info: null pointer");
    info[0] = c->n;
    info[1] = c->m;
    info[2] = c->e;
    info[3] = c->dmax;
    info[4] = (int)c->levels.size();
    info[5] = c->widest;
    info[6] = c->n - c->m;
    info[7] = 0;
    return LDPC_OK;
}

extern "C" void ldpc_code_destroy(ldpc_code* c) { delete c; }

// ------------------------------------------------------------------------
// kernels table
// ------------------------------------------------------------------------

namespace ldpc {
const void* kernel_table_simd4(int kind, int variant);
const void* kernel_table_f16x2(int kind, int variant);
const void* kernel_table_i8(int kind, int variant);
const void* kernel_table_qc(int kind, int dt, bool exact, int layers, bool pow2, int et, int wpt);
const void* kernel_table_qc_refill(int kind, int dt, bool exact, int layers, bool pow2);
const void* kernel_qc_exact_of(const void* f);
const void* kernel_table_qc_split(int kind, int dt, int layers, int split, bool et);
const void* kernel_table_simd4_pf(int kind, int variant);
const void* kernel_table_f16x2h(int kind, int variant);
const void* kernel_table_frame(int kind, int variant, bool et);
const void* kernel_table_frame2(int kind, int variant, bool et);
const void* kernel_table_flood(int kind, int variant);
}

// shared memory of the QC kernel: the APP, 4 bytes per variable per pair of frames
// (wpt = 2: 4 frames, 8 bytes per variable)
static size_t qc_smem(const ldpc_code* c, int wpt) { return (size_t)c->n * 4 * wpt; }

// The QC register-message kernel for the code, or null: 4 frames per CTA (*wpt = 2)
// when an instantiation matches the code's shape, else 2 frames per CTA (*wpt = 1)
// with the smallest instantiated row degree that holds it.  Fills q for that layout.
// refill: the per-frame early-stop kernel with lane refill (4 frames per CTA) instead.
// et: 0 = no early stop, 1 = per CTA (word or, with 2 frames per CTA, frame pair), 2 = per
// frame pair in the 4-frame kernel (LDPC_FLAG_EARLY_STOP_PAIRS)
static const void* qc_kernel_for(const ldpc_code* c, int kind, QCParams& q, int et = 0, int* wpt_out = nullptr,
                                 bool refill = false, bool ofs = false)
{
    if (!c->qc || c->mb > QC_MAX_LAYERS || c->z > 256 || (long long)c->n * 8 > (1 << 20)) return nullptr;
    int deg[QC_MAX_LAYERS], dt = 0;
    bool exact = true;
    for (int i = 0; i < c->mb; i++) {
        int d = 0;
        for (int j = 0; j < c->nb; j++)
            if (c->shifts[i * c->nb + j] >= 0) d++;
        if (d == 0 || d > QC_MAX_DEG) return nullptr;
        for (int k = 1; k < c->z; k++)
            if (c->row_class[i * c->z + k] != c->row_class[i * c->z]) return nullptr;
        deg[i] = d;
        if (i > 0 && d != dt) exact = false;
        dt = std::max(dt, d);
    }
    const bool pow2 = (c->z & (c->z - 1)) == 0;
    // KIND_* values equal LDPC_* values; ofs: the learned kind with every scale 1.0
    const int k = (kind == LDPC_XMS) ? LDPC_OMS : (ofs && kind == LDPC_LEARNED ? KIND_LEARNED_OFS : kind);
    const int e = kind != LDPC_2NMS ? et : 0;
    int wpt = 2;
    const void* f =
        refill ? kernel_table_qc_refill(k, dt, exact, c->mb, pow2) : kernel_table_qc(k, dt, exact, c->mb, pow2, e, 2);
    if (!f && !refill) {
        wpt = 1;
        for (int D : {10, 14, 18, 24})
            if (D >= dt && (f = kernel_table_qc(k, D, false, c->mb, false, e ? 1 : 0, 1))) break;
    }
    if (!f) return nullptr;
    const int vb = 4 * wpt;  // APP bytes per variable
    memset(&q, 0, sizeof q);
    q.z = c->z;
    q.n = c->n;
    q.layers = c->mb;
    q.zb = vb * c->z;
    for (int i = 0; i < c->mb; i++) {
        int d = 0;
        for (int j = 0; j < c->nb; j++) {
            const int sh = c->shifts[i * c->nb + j];
            if (sh < 0) continue;
            q.cz4[i * QC_MAX_DEG + d] = vb * j * c->z;
            q.s[i * QC_MAX_DEG + d] = vb * sh;
            d++;
        }
        q.deg[i] = deg[i];
        q.cls[i] = c->row_class[i * c->z];
    }
    if (wpt_out) *wpt_out = wpt;
    return f;
}

// Path 7: the 2-frame QC kernel with each check row over 4 lanes (Z <= 128, so that a CTA has
// at most 512 threads) for a code that has a 2-frame QC kernel; q as for that kernel.
static const void* qc_split_kernel_for(const ldpc_code* c, int kind, QCParams& q, bool et, int* split_out)
{
    int wpt = 2;
    if (kind == LDPC_2NMS || !qc_kernel_for(c, kind, q, et ? 1 : 0, &wpt) || wpt != 1) return nullptr;
    const int split = c->z * 4 <= 512 ? 4 : 0;
    if (!split) return nullptr;
    int dt = 0;
    for (int i = 0; i < c->mb; i++) dt = std::max(dt, q.deg[i]);
    const int k = kind == LDPC_XMS ? LDPC_OMS : kind;
    for (int D : {10, 14, 18, 24}) {
        if (D < dt) continue;
        if (const void* f = kernel_table_qc_split(k, D, c->mb, split, et)) {
            *split_out = split;
            return f;
        }
    }
    return nullptr;
}

// variant: 0/1 = every row has degree 6/7 (fully unrolled), 2/3/4 = rows of
// degree <= 8/16/32 (unused edge slots predicated off)
static int degree_variant(const ldpc_code* c)
{
    bool uniform = true;
    for (int r = 1; r < c->m && uniform; r++)
        uniform = (c->row_ptr[r + 1] - c->row_ptr[r]) == (c->row_ptr[1] - c->row_ptr[0]);
    if (uniform && c->dmax == 6) return 0;
    if (uniform && c->dmax == 7) return 1;
    if (c->dmax <= 8) return 2;
    if (c->dmax <= 16) return 3;
    return 4;
}

static const void* kernel_for(int pack, int kind, int variant)
{
    // xMS = OMS arithmetic without the first-iteration quirk; LEARNED is row 4 of the tables
    int k = (kind == LDPC_XMS) ? LDPC_OMS : (kind == LDPC_LEARNED ? 4 : kind);
    switch (pack) {
    case LDPC_PACK_SIMD4: return kernel_table_simd4(k, variant);
    case LDPC_PACK_F16X2: return kernel_table_f16x2(k, variant);
    case LDPC_PACK_I8: return kernel_table_i8(k, variant);
    }
    return nullptr;
}

static size_t smem_bytes(int pack, int npad, int dmax, int m)
{
    size_t esz = pack == LDPC_PACK_I8 ? 1 : 4;
    size_t wpc = pack == LDPC_PACK_SIMD4 ? 1 : (pack == LDPC_PACK_F16X2 ? 2 : 4);
    return wpc * esz * ((size_t)npad + (size_t)dmax * m);
}

// ------------------------------------------------------------------------
// decoders
// ------------------------------------------------------------------------

static void decoder_free(ldpc_decoder* d)
{
    if (!d) return;
    cudaFree(d->d_cols);
    cudaFree(d->d_rowdeg);
    cudaFree(d->d_rowcls);
    cudaFree(d->d_levels);
    cudaFree(d->d_edge_orig);
    cudaFree(d->d_vptr);
    cudaFree(d->d_vedge);
    cudaFree(d->d_in);
    cudaFree(d->d_out);
    cudaFree(d->d_aux);
    cudaFree(d->d_fmsg);
    cudaFree(d->d_fst);
    cudaFree(d->d_frec);
    cudaFree(d->d_status);
    cudaFree(d->d_lut);
    if (d->s_comp) cudaStreamDestroy(d->s_comp);
    if (d->s_h2d) cudaStreamDestroy(d->s_h2d);
    if (d->s_d2h) cudaStreamDestroy(d->s_d2h);
    delete d;
}

static int decoder_setup(ldpc_decoder* d, const ldpc_code* c)
{
    const int m = c->m, dmax = c->dmax;
    std::vector<uint16_t> cols((size_t)dmax * m, 0);
    std::vector<int32_t> eorig((size_t)dmax * m, -1);
    std::vector<uint8_t> deg(m), cls(m);
    for (int rp = 0; rp < m; rp++) {
        int r = c->order[rp], b = c->row_ptr[r], dg = c->row_ptr[r + 1] - b;
        deg[rp] = (uint8_t)dg;
        cls[rp] = c->row_class[r];
        for (int j = 0; j < dg; j++) {
            cols[(size_t)j * m + rp] = (uint16_t)c->cols[b + j];
            eorig[(size_t)j * m + rp] = b + j;
        }
    }
    CUDA_TRY(cudaMalloc(&d->d_cols, cols.size() * sizeof(uint16_t)));
    CUDA_TRY(cudaMalloc(&d->d_edge_orig, eorig.size() * sizeof(int32_t)));
    CUDA_TRY(cudaMalloc(&d->d_rowdeg, m));
    CUDA_TRY(cudaMalloc(&d->d_rowcls, m));
    CUDA_TRY(cudaMalloc(&d->d_levels, c->levels.size() * sizeof(int2)));
    CUDA_TRY(cudaMemcpy(d->d_cols, cols.data(), cols.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d->d_edge_orig, eorig.data(), eorig.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d->d_rowdeg, deg.data(), m, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d->d_rowcls, cls.data(), m, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d->d_levels, c->levels.data(), c->levels.size() * sizeof(int2), cudaMemcpyHostToDevice));
    {
        // variable -> message indices j * m + r' (the flooding schedule's APP rebuild)
        std::vector<int32_t> vptr(c->n + 1, 0), vedge(c->e);
        for (int rp = 0; rp < m; rp++)
            for (int j = 0; j < deg[rp]; j++) vptr[cols[(size_t)j * m + rp] + 1]++;
        for (int v = 0; v < c->n; v++) vptr[v + 1] += vptr[v];
        std::vector<int32_t> fill(vptr.begin(), vptr.end() - 1);
        for (int rp = 0; rp < m; rp++)
            for (int j = 0; j < deg[rp]; j++) vedge[fill[cols[(size_t)j * m + rp]]++] = j * m + rp;
        CUDA_TRY(cudaMalloc(&d->d_vptr, vptr.size() * sizeof(int32_t)));
        CUDA_TRY(cudaMalloc(&d->d_vedge, vedge.size() * sizeof(int32_t)));
        CUDA_TRY(cudaMemcpy(d->d_vptr, vptr.data(), vptr.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(d->d_vedge, vedge.data(), vedge.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    }
    Plan& P = d->plan;
    P.n = c->n;
    P.npad = (c->n + 15) / 16 * 16;
    P.m = m;
    P.dmax = dmax;
    P.nlevels = (int)c->levels.size();
    P.cols = d->d_cols;
    P.rowdeg = d->d_rowdeg;
    P.rowcls = d->d_rowcls;
    P.levels = d->d_levels;
    P.edge_orig = d->d_edge_orig;
    P.vptr = d->d_vptr;
    P.vedge = d->d_vedge;
    return LDPC_OK;
}

// Path 3: cuts each level of the schedule into stages (consecutive rows of the level, at most
// d->threads - 32 of them and at most one ring slot of bytes, the slot sized so that two CTAs fit
// on an SM where the frame allows it) and lays out their records and message offsets,
// 16-byte aligned for the bulk copies (FrameStage in frame_kernel.cuh).  base_smem: the
// kernel's shared memory before the ring (the APP and the learned tables).
// two: the layout of decode_frame2_kernel (edge slots of u16 columns, a 64-byte header, one
// CTA per SM with two frames' APP).
static int frame_stages_setup(ldpc_decoder* d, const ldpc_code* c, size_t base_smem, bool two)
{
    const int T = d->threads - 32;  // rows per stage; the last warp is the producer's
    auto pad16 = [](long long x) { return (x + 15) / 16 * 16; };
    int smem_sm = 0, reserved = 0, smem_blk = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, d->device));
    CUDA_TRY(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, d->device));
    CUDA_TRY(cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device));
    // a stage slot holds the header, the row words, the column pairs and the messages of
    // its rows: at least one row of the largest degree
    // entries per row: pairs of edges (one frame), or edges (two frames); 4 bytes of columns
    // per pair entry or 2 per edge entry, 2 bytes of messages per entry either way
    const int hdr = two ? FRAME2_HEADER : FRAME_STAGE_HEADER, cb = two ? 2 : 4;
    auto entries = [&](int dg) { return two ? dg : (dg + 1) / 2; };
    const long long slot_min = hdr + 16 + pad16((long long)cb * entries(c->dmax)) + pad16(2ll * entries(c->dmax));
    const long long static_smem = 512;  // the kernel's static shared memory, rounded up
    long long slot_cap = 0;
    for (int ctas = two ? 1 : 2; ctas >= 1 && slot_cap < slot_min; ctas--) {
        const long long avail = (long long)(ctas == 1 ? smem_blk : smem_sm / ctas - reserved) - static_smem -
                                (long long)base_smem;
        slot_cap = avail / FRAME_RING / 16 * 16;
    }
    if (slot_cap < slot_min)
        return fail(LDPC_ERR_UNSUPPORTED, "LDPC_PACK_FRAME: no room for the stage ring next to the frame");
    std::vector<FrameStage> st;
    std::vector<unsigned char> rec;
    long long moff = 0;
    int slot_max = 0;
    auto slot_bytes = [&](int rows, int pairs) {
        return hdr + pad16(4ll * rows) + pad16((long long)cb * pairs) + pad16(2ll * pairs);
    };
    auto emit = [&](int r0, int rows) {
        // entry slots (pairs, or edges): rows sorted by decreasing degree, so slot p is a
        // prefix of the rows
        int cnt[16] = {0}, poff[16] = {0};
        for (int i = 0; i < rows; i++) {
            const int r = c->order[r0 + i], dg = c->row_ptr[r + 1] - c->row_ptr[r];
            for (int p = 0; p < entries(dg); p++) cnt[p]++;
        }
        int pairs = 0;
        for (int p = 0; p < 16; p++) {
            poff[p] = pairs;
            pairs += cnt[p];
        }
        FrameStage s{};
        const long long cols_off = hdr + pad16(4ll * rows);
        s.rec_bytes = (int)(cols_off + pad16((long long)cb * pairs));
        s.msg_bytes = (int)pad16(2ll * pairs);
        s.rec_off = (int)rec.size();
        s.msg_off = (int)moff;
        rec.resize(rec.size() + s.rec_bytes, 0);
        unsigned char* b = rec.data() + s.rec_off;
        reinterpret_cast<int32_t*>(b)[0] = rows;
        reinterpret_cast<int32_t*>(b)[1] = s.rec_bytes;
        for (int p = 0; p < (two ? 16 : 8); p++) reinterpret_cast<uint16_t*>(b + (two ? 32 : 16))[p] = (uint16_t)poff[p];
        for (int i = 0; i < rows; i++) {
            const int r = c->order[r0 + i], e0 = c->row_ptr[r], dg = c->row_ptr[r + 1] - e0;
            reinterpret_cast<uint32_t*>(b + hdr)[i] = (uint32_t)dg | (uint32_t)c->row_class[r] << 8;
            if (two) {
                for (int j = 0; j < dg; j++) reinterpret_cast<uint16_t*>(b + cols_off)[poff[j] + i] = (uint16_t)c->cols[e0 + j];
                continue;
            }
            for (int p = 0; p < (dg + 1) / 2; p++) {
                const uint32_t lo = (uint32_t)c->cols[e0 + 2 * p];
                const uint32_t hi = 2 * p + 1 < dg ? (uint32_t)c->cols[e0 + 2 * p + 1] : 0u;  // odd degree: dummy
                reinterpret_cast<uint32_t*>(b + cols_off)[poff[p] + i] = lo | hi << 16;
            }
        }
        moff += s.msg_bytes;
        slot_max = std::max(slot_max, s.rec_bytes + s.msg_bytes);
        st.push_back(s);
    };
    for (const int2& lv : c->levels) {
        int r0 = lv.x, rows = 0, pairs = 0;
        for (int i = lv.x; i < lv.x + lv.y; i++) {
            const int r = c->order[i], np = entries(c->row_ptr[r + 1] - c->row_ptr[r]);
            if (rows > 0 && (rows == T || slot_bytes(rows + 1, pairs + np) > slot_cap)) {
                emit(r0, rows);
                r0 = i;
                rows = pairs = 0;
            }
            rows++;
            pairs += np;
        }
        if (rows) emit(r0, rows);
    }
    if (rec.size() > (size_t)INT32_MAX || moff > INT32_MAX)
        return fail(LDPC_ERR_UNSUPPORTED, "LDPC_PACK_FRAME: stage records too large");
    CUDA_TRY(cudaMalloc(&d->d_fst, st.size() * sizeof(FrameStage)));
    CUDA_TRY(cudaMalloc(&d->d_frec, rec.size()));
    CUDA_TRY(cudaMalloc(&d->d_status, sizeof(int)));
    CUDA_TRY(cudaMemcpy(d->d_fst, st.data(), st.size() * sizeof(FrameStage), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d->d_frec, rec.data(), rec.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(d->d_status, 0, sizeof(int)));
    d->fst.st = d->d_fst;
    d->fst.rec = d->d_frec;
    d->fst.slot_bytes = moff;
    d->fst.nst = (int)st.size();
    d->fst.slot_sz = slot_max;
    d->fst.status = d->d_status;
    return LDPC_OK;
}

extern "C" int ldpc_decoder_create(ldpc_decoder** out, const ldpc_code* c, int kind, size_t nb_frames, int pack,
                                   int flags)
{
    if (!out || !c) return fail(LDPC_ERR_ARG, "ldpc_decoder_create: null pointer");
    if (kind < LDPC_MS || kind > LDPC_LEARNED) return fail(LDPC_ERR_ARG, "unknown decoder kind %d", kind);
    if (nb_frames < 1) return fail(LDPC_ERR_SHAPE, "nb_frames must be >= 1");
    if (flags & ~(LDPC_FLAG_EARLY_STOP | LDPC_FLAG_EARLY_STOP_FRAMES | LDPC_FLAG_FLOODING | LDPC_FLAG_EARLY_STOP_PAIRS))
        return fail(LDPC_ERR_ARG, "unknown flags 0x%x", flags);
    const bool per_frame = flags & LDPC_FLAG_EARLY_STOP_FRAMES;
    const bool pairs = flags & LDPC_FLAG_EARLY_STOP_PAIRS;
    const bool flood = flags & LDPC_FLAG_FLOODING;
    if (pairs && per_frame)
        return fail(LDPC_ERR_ARG, "LDPC_FLAG_EARLY_STOP_PAIRS and LDPC_FLAG_EARLY_STOP_FRAMES exclude each other");
    if (flood && (per_frame || pairs || (pack != LDPC_PACK_AUTO && pack != LDPC_PACK_F16X2)))
        return fail(LDPC_ERR_UNSUPPORTED, "LDPC_FLAG_FLOODING: the flooding schedule runs on the 4-frame "
                                          "LDPC_PACK_F16X2 level kernel, per-word early stop only");
    const bool early = (flags & LDPC_FLAG_EARLY_STOP) || per_frame || pairs;
    const int etm = pairs ? 2 : 1;  // the QC kernels' early-stop mode when early
    if (early && kind == LDPC_2NMS)
        return fail(LDPC_ERR_ARG, "LDPC_FLAG_EARLY_STOP: LDPC_2NMS has the reference's own early termination");
    // LDPC_PACK_F16X2_SPLIT: the F16X2 arithmetic on the 2-frame QC kernel with split rows
    const bool split_req = pack == LDPC_PACK_F16X2_SPLIT;
    if (split_req) {
        if (flood) return fail(LDPC_ERR_UNSUPPORTED, "LDPC_FLAG_FLOODING: not on LDPC_PACK_F16X2_SPLIT");
        pack = LDPC_PACK_F16X2;
    }
    const int pack_req = pack;
    // AUTO: the QC register kernel where one fits (below); otherwise fp16x2 with 2 frames per
    // CTA for the fixed-iteration MS / OMS / NMS / xMS decoders (the fastest level kernel where
    // it applies), else SIMD4 (early stop; 2NMS; LEARNED, whose SIMD4 tables take any constants)
    if (pack == LDPC_PACK_AUTO)
        pack = flood || (!early && (kind == LDPC_MS || kind == LDPC_OMS || kind == LDPC_NMS || kind == LDPC_XMS))
                   ? LDPC_PACK_F16X2
                   : LDPC_PACK_SIMD4;
    if (pack < LDPC_PACK_SIMD4 || pack > LDPC_PACK_FRAME) return fail(LDPC_ERR_ARG, "unknown pack %d", pack);
    bool frame = pack == LDPC_PACK_FRAME;
    if (frame) pack = LDPC_PACK_I8;  // the arithmetic of that path
    if (c->dmax > kMaxDegree) return fail(LDPC_ERR_UNSUPPORTED, "row degree %d > %d", c->dmax, kMaxDegree);
    int npad = (c->n + 15) / 16 * 16;
    // fp16x2 without early termination: 2 frames per CTA (half the shared memory)
    const bool half = pack == LDPC_PACK_F16X2 && kind != LDPC_2NMS && !early && !flood;
    size_t smem = half ? 4 * ((size_t)npad + (size_t)c->dmax * c->m) : smem_bytes(pack, npad, c->dmax, c->m);
    if (flood) smem += 8 * (size_t)npad;  // the channel values the flooding APP is rebuilt from
    const size_t lut_smem = kind == LDPC_LEARNED ? 512 : 0;  // the iteration's magnitude tables
    smem += lut_smem;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    int smem_max = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    QCParams probe;
    bool qc_ok = !flood && (pack_req == LDPC_PACK_AUTO || pack == LDPC_PACK_F16X2);
    int probe_wpt = 2;
    qc_ok = qc_ok && qc_kernel_for(c, kind, probe, false, &probe_wpt) && qc_smem(c, probe_wpt) + 512 <= (size_t)smem_max;
    // the 2-frame QC kernel is an explicit LDPC_PACK_F16X2 choice: AUTO keeps the level kernels
    // for those shapes (faster on some, slower on others, and a different early-stop unit)
    qc_ok = qc_ok && (probe_wpt == 2 || pack_req == LDPC_PACK_F16X2);
    if (!frame && smem > (size_t)smem_max && !qc_ok) {
        if (pack_req != LDPC_PACK_AUTO || kind == LDPC_2NMS || flood)
            return fail(LDPC_ERR_UNSUPPORTED, "decoder state of one frame group needs %zu B of shared memory (> %d)",
                        smem, smem_max);
        frame = true;  // one frame per CTA with packed row state
    }
    const size_t frame_smem = (size_t)npad + lut_smem;  // the APP; messages live in the decoder's scratch
    if (frame) {
        if (kind == LDPC_2NMS)
            return fail(LDPC_ERR_UNSUPPORTED, "LDPC_PACK_FRAME: 2NMS terminates per 4-frame word; use another pack");
        if (c->dmax > FRAME_MAX_DEGREE)
            return fail(LDPC_ERR_UNSUPPORTED, "LDPC_PACK_FRAME: row degree %d > %d", c->dmax, FRAME_MAX_DEGREE);
        if (frame_smem > (size_t)smem_max)
            return fail(LDPC_ERR_UNSUPPORTED, "one frame's state needs %zu B of shared memory (> %d)", frame_smem,
                        smem_max);
    }
    ldpc_decoder* d = new ldpc_decoder();
    d->kind = kind;
    d->early = early;
    d->pack = pack;
    d->device = dev;
    d->nb_words = nb_frames;
    d->n = c->n;
    d->m = c->m;
    d->e = c->e;
    int rc = decoder_setup(d, c);
    if (rc) {
        decoder_free(d);
        return rc;
    }
    int qc_wpt = 2;
    const void* qk = !frame && !flood && (pack_req == LDPC_PACK_AUTO || pack_req == LDPC_PACK_F16X2)
                         ? qc_kernel_for(c, kind, d->qcp, early ? etm : 0, &qc_wpt)
                         : nullptr;
    if (qc_wpt == 1 && pack_req != LDPC_PACK_F16X2) qk = nullptr;
    int split = 0;
    const void* qsk = split_req && !frame ? qc_split_kernel_for(c, kind, d->qcp, early, &split) : nullptr;
    if (split_req && (!qsk || per_frame)) {
        decoder_free(d);
        return fail(LDPC_ERR_UNSUPPORTED, "LDPC_PACK_F16X2_SPLIT: needs a QC code with a 2-frame QC kernel "
                                          "(24-column bases), Z <= 128, no per-frame early stop");
    }
    if (qsk) {
        QCParams alt;
        int s2 = 0;
        d->kfn = qsk;
        d->kfn_alt = qc_split_kernel_for(c, kind, alt, !early, &s2);
        d->path = 7;
        d->grid_mult = 2;
        d->pack = LDPC_PACK_F16X2;
        d->smem = (int)(qc_smem(c, 1) + lut_smem);
        d->threads = c->z * split;
    } else if (frame) {
        const int k = kind == LDPC_XMS ? LDPC_OMS : kind;  // KIND_* values equal LDPC_* values
        d->path = 3;
        d->pack = LDPC_PACK_FRAME;
        d->grid_mult = 4;
        // the rows of a stage, then one warp whose last thread issues the bulk copies; two
        // frames per CTA where their APP and a stage ring fit (odd-row counts of a frame below
        // 2^16), else one
        d->threads = std::min(FRAME_MAX_THREADS, std::max(32, (c->widest + 31) / 32 * 32)) + 32;
        d->frame2 = c->m < 65536 &&
                    frame_stages_setup(d, c, frame_smem + (size_t)npad, true) == LDPC_OK;
        if (!d->frame2) {
            cudaFree(d->d_fst);
            cudaFree(d->d_frec);
            cudaFree(d->d_status);
            d->d_fst = nullptr;
            d->d_frec = nullptr;
            d->d_status = nullptr;
            rc = frame_stages_setup(d, c, frame_smem, false);
            if (rc) {
                decoder_free(d);
                return rc;
            }
        }
        d->kfn = (d->frame2 ? kernel_table_frame2 : kernel_table_frame)(k, degree_variant(c), early);
        d->kfn_alt = (d->frame2 ? kernel_table_frame2 : kernel_table_frame)(k, degree_variant(c), !early);
        d->smem = (int)(frame_smem + (d->frame2 ? (size_t)npad : 0) + (size_t)FRAME_RING * d->fst.slot_sz);
        if (d->smem > smem_max) {
            decoder_free(d);
            return fail(LDPC_ERR_UNSUPPORTED, "LDPC_PACK_FRAME: the frame and its stage ring need %d B of shared "
                                              "memory (> %d)", d->smem, smem_max);
        }
    } else if (per_frame && qk && qc_wpt == 2 && qc_smem(c, 2) + QC_STAGE * (size_t)c->n <= (size_t)smem_max &&
               (d->kfn = qc_kernel_for(c, kind, d->qcp, true, nullptr, true))) {
        d->path = 5;
        d->pack = LDPC_PACK_F16X2;
        d->smem = (int)(qc_smem(c, 2) + QC_STAGE * (size_t)c->n);  // the APP and the staged frames
        d->threads = c->z;
    } else if (qk && qc_smem(c, qc_wpt) + lut_smem <= (size_t)smem_max) {
        QCParams alt;
        d->kfn = qk;
        d->kfn_alt = qc_kernel_for(c, kind, alt, early ? 0 : etm);  // for ldpc_decoder_set_early_stop (same layout)
        if (kind == LDPC_LEARNED && qc_wpt == 2)
            for (int e = 0; e < 2; e++) {
                for (int o = 0; o < 2; o++)
                    d->kfn_lrn[o][e] = qc_kernel_for(c, kind, alt, e != 0 ? etm : 0, nullptr, false, o != 0);
                d->kfn_lrn[2][e] = qc_kernel_for(c, LDPC_OMS, alt, e != 0 ? etm : 0);
            }
        d->path = qc_wpt == 2 ? 1 : 4;
        d->grid_mult = qc_wpt == 2 ? 1 : 2;
        d->pack = LDPC_PACK_F16X2;
        d->smem = (int)(qc_smem(c, qc_wpt) + lut_smem);
        d->threads = c->z;
    } else if (flood) {
        // every row per iteration: as many threads as rows, up to 256
        d->kfn = kernel_table_flood(kind == LDPC_XMS ? LDPC_OMS : (kind == LDPC_LEARNED ? 4 : kind), degree_variant(c));
        d->path = 6;
        d->smem = (int)smem;
        d->threads = std::min(256, std::max(32, (c->m + 31) / 32 * 32));
    } else if (half) {
        d->kfn = kernel_table_f16x2h(kind == LDPC_XMS ? LDPC_OMS : (kind == LDPC_LEARNED ? 3 : kind), degree_variant(c));
        d->path = 2;
        d->grid_mult = 2;
        d->smem = (int)smem;
        d->threads = std::min(256, std::max(32, (c->widest + 31) / 32 * 32));
    } else {
        if (per_frame) {
            // the level kernel with the per-frame early stop: SIMD4 only (one frame per byte lane)
            const int k = kind == LDPC_XMS ? LDPC_OMS : (kind == LDPC_LEARNED ? KIND_LEARNED : kind);
            d->kfn = pack == LDPC_PACK_SIMD4 ? kernel_table_simd4_pf(k, degree_variant(c)) : nullptr;
            d->pf_levels = d->kfn != nullptr;
        } else {
            d->kfn = kernel_for(pack, kind, degree_variant(c));
        }
        d->smem = (int)smem;
        d->threads = std::min(256, std::max(32, (c->widest + 31) / 32 * 32));
    }
    if (pairs && d->path != 1 && d->path != 4 && d->path != 7) {
        decoder_free(d);
        return fail(LDPC_ERR_UNSUPPORTED, "LDPC_FLAG_EARLY_STOP_PAIRS: needs a QC register kernel (decoder path 1 or 4)");
    }
    if (per_frame && d->path != 3 && d->path != 5 && !d->pf_levels) {
        decoder_free(d);
        return fail(LDPC_ERR_UNSUPPORTED, "LDPC_FLAG_EARLY_STOP_FRAMES: needs the level kernel with LDPC_PACK_SIMD4 "
                                          "(or AUTO), the QC register kernel with 4 frames per CTA (the regular 8x16 "
                                          "base, Z a power of two) or LDPC_PACK_FRAME");
    }
    if (d->path == 5 || d->path == 3) {
        cudaError_t ec = cudaDeviceGetAttribute(&d->sms, cudaDevAttrMultiProcessorCount, dev);
        if (ec != cudaSuccess) {
            decoder_free(d);
            return fail(LDPC_ERR_CUDA, "decoder setup: %s", cudaGetErrorString(ec));
        }
    }
    cudaError_t e1 = ldpc_internal_raise_smem(d->kfn, d->smem);
    if (e1 == cudaSuccess && d->kfn_alt) e1 = ldpc_internal_raise_smem(d->kfn_alt, d->smem);
    for (int o = 0; o < 3; o++)
        for (int e = 0; e < 2; e++)
            if (e1 == cudaSuccess && d->kfn_lrn[o][e]) e1 = ldpc_internal_raise_smem(d->kfn_lrn[o][e], d->smem);
    cudaFuncAttributes fa;
    cudaError_t e2 = cudaFuncGetAttributes(&fa, d->kfn);
    cudaError_t e3 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d->ctas_per_sm, d->kfn, d->threads, d->smem);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
        cudaError_t e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
        decoder_free(d);
        return fail(LDPC_ERR_CUDA, "kernel setup: %s", cudaGetErrorString(e));
    }
    d->regs = fa.numRegs;
    if (d->ctas_per_sm < 1) {
        decoder_free(d);
        return fail(LDPC_ERR_UNSUPPORTED, "kernel cannot be resident (smem %d B, %d threads)", d->smem, d->threads);
    }
    if (d->path == 3) {
        // one message slot per resident CTA: a byte per edge slot of the stage records
        d->fslots = (long long)d->ctas_per_sm * d->sms;
        const size_t bytes = (size_t)d->fslots * (size_t)d->fst.slot_bytes;
        cudaError_t ea = cudaMalloc(&d->d_fmsg, bytes);
        d->fst.msg = d->d_fmsg;
        if (ea != cudaSuccess) {
            decoder_free(d);
            return fail(ea == cudaErrorMemoryAllocation ? LDPC_ERR_NOMEM : LDPC_ERR_CUDA,
                        "message scratch of %zu B: %s", bytes, cudaGetErrorString(ea));
        }
    }
    cudaError_t es = cudaStreamCreateWithFlags(&d->s_comp, cudaStreamNonBlocking);
    if (es == cudaSuccess) es = cudaStreamCreateWithFlags(&d->s_h2d, cudaStreamNonBlocking);
    if (es == cudaSuccess) es = cudaStreamCreateWithFlags(&d->s_d2h, cudaStreamNonBlocking);
    if (es != cudaSuccess) {
        decoder_free(d);
        return fail(LDPC_ERR_CUDA, "stream creation: %s", cudaGetErrorString(es));
    }
    *out = d;
    return LDPC_OK;
}

extern "C" int ldpc_decoder_set_early_stop(ldpc_decoder* d, int enabled, int slack)
{
    if (!d) return fail(LDPC_ERR_ARG, "ldpc_decoder_set_early_stop: null decoder");
    if (enabled && d->kind == LDPC_2NMS)
        return fail(LDPC_ERR_ARG, "LDPC_FLAG_EARLY_STOP: LDPC_2NMS has the reference's own early termination");
    if (enabled && d->path == 2)
        return fail(LDPC_ERR_ARG, "early stop needs a decoder created with LDPC_FLAG_EARLY_STOP for this packing");
    if (slack < 0) return fail(LDPC_ERR_ARG, "ldpc_decoder_set_early_stop: slack must be >= 0");
    if (!enabled && d->pf_levels)
        return fail(LDPC_ERR_ARG, "the per-frame early stop of this decoder cannot be turned off; create one "
                                  "without LDPC_FLAG_EARLY_STOP_FRAMES");
    if ((d->path == 1 || d->path == 3 || d->path == 4 || d->path == 7) && (enabled != 0) != d->early)
        std::swap(d->kfn, d->kfn_alt);
    d->early = enabled != 0;
    d->early_slack = (unsigned)slack;
    return LDPC_OK;
}

// fp16 bit pattern of x, which must be exactly representable (normal or zero)
static uint16_t half_bits(double x)
{
    if (x == 0.0) return 0;
    const uint16_t sign = x < 0 ? 0x8000 : 0;
    double a = x < 0 ? -x : x;
    int e = 0;
    while (a >= 2.0) { a /= 2.0; e++; }
    while (a < 1.0) { a *= 2.0; e--; }
    return (uint16_t)(sign | ((e + 15) << 10) | ((int)((a - 1.0) * 1024.0 + 0.5) & 0x3ff));
}

// LDPC_LEARNED magnitude tables [n_iters][2][128] for the packing (fp16: (k, b) pairs)
static int build_learned_lut(bool fp16, int n_iters, const int8_t* offsets, const uint8_t* scales,
                             std::vector<uint16_t>& lut)
{
    lut.assign((size_t)n_iters * 256, 0);
    if (fp16) {
        // the fp16 kernels compute floor(min * s / 128) - offset as round(min * k + b) with
        // k = s / 128, b = -offset - 15/32 (packs.cuh, h2::mags): exact when k has at most 4
        // fraction bits (s a multiple of 8) and b is an fp16 (|offset| <= 31)
        for (int i = 0; i < 2 * n_iters; i++)
            if (scales[i] % 8 != 0 || offsets[i] < -31 || offsets[i] > 31)
                return fail(LDPC_ERR_UNSUPPORTED,
                            "LDPC_PACK_F16X2 LDPC_LEARNED decoders need scales that are multiples of 8 and offsets "
                            "in [-31, 31] (got scale %d, offset %d); use LDPC_PACK_SIMD4 or LDPC_PACK_I8 for others",
                            (int)scales[i], (int)offsets[i]);
        for (int t = 0; t < n_iters; t++)
            for (int g = 0; g < 2; g++) {
                const uint16_t k = half_bits(scales[2 * t + g] / 128.0);
                const uint16_t b = half_bits(-offsets[2 * t + g] - 15.0 / 32.0);
                uint16_t* e = &lut[(size_t)t * 256 + g * 128];
                e[0] = e[1] = k;  // (k, k) and (b, b) as f16x2 words
                e[2] = e[3] = b;
            }
    } else {
        for (int t = 0; t < n_iters; t++)
            for (int g = 0; g < 2; g++)
                for (int m = 0; m < 128; m++) {
                    int c = ((m * (int)scales[2 * t + g]) >> 7) - offsets[2 * t + g];
                    lut[(size_t)t * 256 + g * 128 + m] = (uint16_t)(c < 0 ? 0 : (c > 31 ? 31 : c));
                }
    }
    return LDPC_OK;
}

extern "C" int ldpc_decoder_set_learned(ldpc_decoder* d, int n_iters, const int8_t* offsets, const uint8_t* scales)
{
    if (!d || !offsets || !scales) return fail(LDPC_ERR_ARG, "ldpc_decoder_set_learned: null pointer");
    if (d->kind != LDPC_LEARNED) return fail(LDPC_ERR_ARG, "ldpc_decoder_set_learned: decoder kind is not LDPC_LEARNED");
    if (n_iters < 1 || n_iters > LDPC_LEARNED_MAX_ITERS)
        return fail(LDPC_ERR_ARG, "ldpc_decoder_set_learned: n_iters must be in [1, %d]", LDPC_LEARNED_MAX_ITERS);
    std::vector<uint16_t> lut;
    int rc = build_learned_lut(d->pack == LDPC_PACK_F16X2, n_iters, offsets, scales, lut);
    if (rc) return rc;
    if (!d->d_lut) CUDA_TRY(cudaMalloc(&d->d_lut, sizeof(uint16_t) * 256 * LDPC_LEARNED_MAX_ITERS));
    CUDA_TRY(cudaMemcpy(d->d_lut, lut.data(), lut.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    d->lut_its = n_iters;
    if (d->kfn_lrn[0][0]) {
        // the QC register kernel: constants with every scale 1.0 (offsets only) take the kernel
        // whose magnitude is min - offset, without the floor step; with every offset 1 as well
        // that is OMS's magnitude clamp(min - 1, 0, 31) in every iteration, and the OMS kernel
        // (launched without the OMS first-iteration quirk, J.quirk = 0) computes it
        bool ofs = true, oms = true;
        for (int i = 0; i < 2 * n_iters; i++) {
            ofs = ofs && scales[i] == 128;
            oms = oms && scales[i] == 128 && offsets[i] == 1;
        }
        const int sel = oms ? 2 : (ofs ? 1 : 0);
        d->kfn = d->kfn_lrn[sel][d->early];
        d->kfn_alt = d->kfn_lrn[sel][!d->early];
    }
    return LDPC_OK;
}

extern "C" int ldpc_decoder_info(const ldpc_decoder* d, int* info)
{
    if (!d || !info) return fail(LDPC_ERR_ARG, "ldpc_decoder_info: null pointer");
    info[0] = d->kind;
    info[1] = d->pack;
    info[2] = (int)d->nb_words;
    info[3] = d->threads;
    info[4] = d->smem;
    info[5] = d->ctas_per_sm;
    info[6] = d->regs;
    info[7] = d->path;
    return LDPC_OK;
}

extern "C" int ldpc_decoder_destroy(ldpc_decoder* d)
{
    if (!d) return LDPC_OK;
    cudaError_t e = cudaDeviceSynchronize();
    decoder_free(d);
    if (e != cudaSuccess) return fail(LDPC_ERR_CUDA, "ldpc_decoder_destroy: %s", cudaGetErrorString(e));
    return LDPC_OK;
}

static int launch(ldpc_decoder* d, const int8_t* llr, void* out, int out_packed, long long word0, long long words,
                  long long total_words, int iters, int32_t* iters_out, int8_t* app_out, int8_t* msg_out,
                  cudaStream_t st, const Job* sim = nullptr, uint8_t* synd_out = nullptr)
{
    Job J{};
    if (sim) J = *sim;
    if (d->kind == LDPC_LEARNED) {
        if (!d->d_lut) return fail(LDPC_ERR_ARG, "LDPC_LEARNED decoder: set its offsets and scales first");
        J.lut = d->d_lut;
        J.lut_its = d->lut_its;
    }
    J.llr = llr;
    J.out = out;
    J.out_packed = out_packed;
    J.interleaved = d->kind == LDPC_XMS;
    J.total_words = total_words;
    J.word0 = word0;
    J.iters = iters;
    J.quirk = d->kind == LDPC_OMS;
    J.early = d->early ? 1 : 0;
    J.early_slack = d->early_slack;
    J.iters_out = iters_out;
    J.synd_out = synd_out;
    J.app_out = app_out;
    J.msg_out = msg_out;
    if ((d->path == 4 || d->path == 7) && iters_out)  // each 2-frame CTA raises its word's count with atomicMax
        CUDA_TRY(cudaMemsetAsync(iters_out, 0, sizeof(int32_t) * (size_t)words, st));
    if (d->path == 5) {
        // persistent CTAs, at most the resident ones, each decoding a strided share of the frames
        if (iters > 255) return fail(LDPC_ERR_UNSUPPORTED, "LDPC_FLAG_EARLY_STOP_FRAMES: at most 255 iterations");
        long long frames = 4 * words;
        const long long grid = std::min(words, (long long)d->ctas_per_sm * d->sms);
        void* a[] = {(void*)&d->qcp, (void*)&J, (void*)&frames};
        CUDA_TRY(cudaLaunchKernel(d->kfn, dim3((unsigned)grid), dim3(d->threads), a, d->smem, st));
        return LDPC_OK;
    }
    if (d->path == 3) {
        // persistent CTAs, one message-scratch slot each
        long long frames = 4 * words;
        const long long grid = std::min(d->frame2 ? frames / 2 : frames, d->fslots);
        void* a[] = {(void*)&d->plan, (void*)&J, (void*)&d->fst, (void*)&frames};
        CUDA_TRY(cudaLaunchKernel(d->kfn, dim3((unsigned)grid), dim3(d->threads), a, d->smem, st));
        return LDPC_OK;
    }
    const void* kfn = d->kfn;
    if (d->path == 1 && d->early && d->early_slack >= LDPC_EARLY_SLACK_ANY) {
        // every iteration a candidate: the 4-frame QC kernel's exact-gate twin, where it has one
        if (const void* x = kernel_qc_exact_of(kfn)) {
            if (d->smem > 48 * 1024) CUDA_TRY(ldpc_internal_raise_smem(x, d->smem));
            kfn = x;
        }
    }
    void* args[] = {(d->path == 1 || d->path == 4 || d->path == 7) ? (void*)&d->qcp : (void*)&d->plan, (void*)&J};
    CUDA_TRY(cudaLaunchKernel(kfn, dim3((unsigned)(words * d->grid_mult)), dim3(d->threads), args, d->smem, st));
    return LDPC_OK;
}

static int check_decode_args(ldpc_decoder* d, const void* in, const void* out, size_t n_words, int iters)
{
    if (!d || !in || !out) return fail(LDPC_ERR_ARG, "decode: null pointer");
    if (iters < 1) return fail(LDPC_ERR_ARG, "decode: iterations must be >= 1 (got %d)", iters);
    if (n_words < 1 || n_words > d->nb_words)
        return fail(LDPC_ERR_SHAPE, "decode: %zu words requested, decoder holds %zu", n_words, d->nb_words);
    return LDPC_OK;
}

extern "C" int ldpc_decode_device(ldpc_decoder* d, const int8_t* d_llr, void* d_out, size_t n_words, int iters,
                                  int out_format, int32_t* d_iters_out, uint8_t* d_syndrome_ok, void* stream)
{
    int rc = check_decode_args(d, d_llr, d_out, n_words, iters);
    if (rc) return rc;
    if (out_format != LDPC_OUT_BYTES && out_format != LDPC_OUT_PACKED)
        return fail(LDPC_ERR_ARG, "decode: unknown out_format %d", out_format);
    CUDA_TRY(cudaSetDevice(d->device));
    return launch(d, d_llr, d_out, out_format == LDPC_OUT_PACKED, 0, (long long)n_words, (long long)n_words, iters,
                  d_iters_out, nullptr, nullptr, (cudaStream_t)stream, nullptr, d_syndrome_ok);
}

extern "C" int ldpc_decode_device_state(ldpc_decoder* d, const int8_t* d_llr, uint8_t* d_hard, size_t n_words,
                                        int iters, int32_t* d_iters_out, int8_t* d_app, int8_t* d_msg, void* stream)
{
    int rc = check_decode_args(d, d_llr, d_hard, n_words, iters);
    if (rc) return rc;
    if (((d->path >= 3 && d->path != 6) || d->pf_levels) && (d_app || d_msg))  // paths 3, 4, 5, 7, per-frame 0
        return fail(LDPC_ERR_UNSUPPORTED, "this decoder (path %d) has no state dumps", d->path);
    CUDA_TRY(cudaSetDevice(d->device));
    return launch(d, d_llr, d_hard, 0, 0, (long long)n_words, (long long)n_words, iters, d_iters_out, d_app, d_msg,
                  (cudaStream_t)stream);
}

extern "C" int ldpc_simulate(ldpc_decoder* d, size_t n_words, int iters, float sigma, uint64_t seed, uint64_t offset,
                             const uint8_t* d_codewords, size_t n_codewords, int n_vars, int64_t* d_counts,
                             uint8_t* d_hard, void* stream)
{
    if (!d || !d_counts) return fail(LDPC_ERR_ARG, "simulate: null pointer");
    if (d->kind == LDPC_XMS) return fail(LDPC_ERR_UNSUPPORTED, "simulate: xMS reads word-interleaved input; use OMS");
    if (d->path == 5)
        return fail(LDPC_ERR_UNSUPPORTED, "simulate: LDPC_FLAG_EARLY_STOP_FRAMES decoders read LLRs from memory "
                                          "(ldpc_channel_awgn, then ldpc_decode_device)");
    if (iters < 1) return fail(LDPC_ERR_ARG, "simulate: iterations must be >= 1 (got %d)", iters);
    if (n_words < 1 || n_words > d->nb_words)
        return fail(LDPC_ERR_SHAPE, "simulate: %zu words requested, decoder holds %zu", n_words, d->nb_words);
    if (n_vars < 0 || n_vars > d->n || sigma < 0 || (d_codewords && n_codewords == 0))
        return fail(LDPC_ERR_ARG, "simulate: bad n_vars / sigma / codewords");
    CUDA_TRY(cudaSetDevice(d->device));
    Job J{};
    J.gen = 1;
    J.sigma = sigma;
    J.seed = seed;
    J.offset = offset;
    J.cw = d_codewords;
    J.n_cw = (long long)n_codewords;
    J.counts = reinterpret_cast<unsigned long long*>(d_counts);
    J.n_vars = n_vars;
    return launch(d, nullptr, d_hard, 0, 0, (long long)n_words, (long long)n_words, iters, nullptr, nullptr, nullptr,
                  (cudaStream_t)stream, &J);
}

// Host-buffer decode of all nb_words words: the H2D copy of chunk i+1 and the D2H copy of
// chunk i-1 overlap the decoding of chunk i (three streams).  out_format selects 0/1 bytes
// (the reference's) or packed bits; iters_out / synd_out (host, nullable) receive the
// iteration counts (per word, or per frame on paths 3 and 5) and the syndrome flags.
static int decode_host_impl(ldpc_decoder* d, const int8_t* llr, void* out, int iters, int out_format,
                            int32_t* iters_out, uint8_t* synd_out)
{
    int rc = check_decode_args(d, llr, out, d->nb_words, iters);
    if (rc) return rc;
    if (out_format != LDPC_OUT_BYTES && out_format != LDPC_OUT_PACKED)
        return fail(LDPC_ERR_ARG, "decode: unknown out_format %d", out_format);
    CUDA_TRY(cudaSetDevice(d->device));
    const size_t W = d->nb_words, fb = 4 * (size_t)d->n;  // LLR bytes per word-group of frames
    const size_t ob = out_format == LDPC_OUT_PACKED ? 4 * (size_t)((d->n + 7) / 8) : fb;  // output bytes per word
    const size_t ipw = (d->path == 3 || d->path == 5 || d->pf_levels) ? 4 : 1;  // iteration counts per word
    if (!d->d_in) {
        CUDA_TRY(cudaMalloc(&d->d_in, W * fb));
        CUDA_TRY(cudaMalloc(&d->d_out, W * fb));
    }
    if ((iters_out || synd_out) && !d->d_aux) CUDA_TRY(cudaMalloc(&d->d_aux, W * 4 * (sizeof(int32_t) + 1)));
    int32_t* d_its = iters_out ? reinterpret_cast<int32_t*>(d->d_aux) : nullptr;
    uint8_t* d_syn = synd_out ? reinterpret_cast<uint8_t*>(d->d_aux) + W * 4 * sizeof(int32_t) : nullptr;
    // chunks of words: copy-in of chunk i+1 and copy-out of chunk i-1 overlap decoding of chunk i
    size_t chunks = (d->kind == LDPC_XMS) ? 1 : std::min<size_t>(8, std::max<size_t>(1, W / 256));
    size_t per = (W + chunks - 1) / chunks;
    std::vector<cudaEvent_t> ev_in, ev_dec;
    for (size_t c0 = 0, i = 0; c0 < W; c0 += per, i++) {
        size_t words = std::min(per, W - c0);
        cudaEvent_t a, b;
        CUDA_TRY(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
        ev_in.push_back(a);
        ev_dec.push_back(b);
        size_t off = c0 * fb, bytes = words * fb;
        if (d->kind == LDPC_XMS) {
            off = 0;
            bytes = W * fb;
        }
        CUDA_TRY(cudaMemcpyAsync(d->d_in + off, llr + off, bytes, cudaMemcpyHostToDevice, d->s_h2d));
        CUDA_TRY(cudaEventRecord(a, d->s_h2d));
        CUDA_TRY(cudaStreamWaitEvent(d->s_comp, a, 0));
        const int8_t* src = (d->kind == LDPC_XMS) ? d->d_in : d->d_in + c0 * fb;
        rc = launch(d, src, d->d_out + c0 * ob, out_format == LDPC_OUT_PACKED, (long long)c0, (long long)words,
                    (long long)W, iters, d_its ? d_its + c0 * ipw : nullptr, nullptr, nullptr, d->s_comp, nullptr,
                    d_syn ? d_syn + 4 * c0 : nullptr);
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(b, d->s_comp));
        CUDA_TRY(cudaStreamWaitEvent(d->s_d2h, b, 0));
        CUDA_TRY(cudaMemcpyAsync(static_cast<uint8_t*>(out) + c0 * ob, d->d_out + c0 * ob, words * ob,
                                 cudaMemcpyDeviceToHost, d->s_d2h));
        if (d_its)
            CUDA_TRY(cudaMemcpyAsync(iters_out + c0 * ipw, d_its + c0 * ipw, words * ipw * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, d->s_d2h));
        if (d_syn)
            CUDA_TRY(cudaMemcpyAsync(synd_out + 4 * c0, d_syn + 4 * c0, words * 4, cudaMemcpyDeviceToHost, d->s_d2h));
    }
    cudaError_t e = cudaStreamSynchronize(d->s_d2h);
    for (auto ev : ev_in) cudaEventDestroy(ev);
    for (auto ev : ev_dec) cudaEventDestroy(ev);
    if (e != cudaSuccess) return fail(LDPC_ERR_CUDA, "decode_host: %s", cudaGetErrorString(e));
    int status = 0;
    rc = ldpc_decoder_status(d, &status);
    if (rc) return rc;
    if (status) return fail(LDPC_ERR_CUDA, "decode_host: a wait on the copy engine gave up (results invalid)");
    return LDPC_OK;
}

extern "C" int ldpc_decoder_status(ldpc_decoder* d, int* status)
{
    if (!d || !status) return fail(LDPC_ERR_ARG, "ldpc_decoder_status: null pointer");
    *status = 0;
    if (!d->d_status) return LDPC_OK;
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaMemcpy(status, d->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (*status) CUDA_TRY(cudaMemset(d->d_status, 0, sizeof(int)));
    return LDPC_OK;
}

extern "C" int ldpc_decode_host(ldpc_decoder* d, const int8_t* llr, uint8_t* hard, int iters)
{
    if (!d) return fail(LDPC_ERR_ARG, "decode: null decoder");
    return decode_host_impl(d, llr, hard, iters, LDPC_OUT_BYTES, nullptr, nullptr);
}

extern "C" int ldpc_decode_host_ex(ldpc_decoder* d, const int8_t* llr, void* out, int iters, int out_format,
                                   int32_t* iters_out, uint8_t* syndrome_ok)
{
    if (!d) return fail(LDPC_ERR_ARG, "decode: null decoder");
    return decode_host_impl(d, llr, out, iters, out_format, iters_out, syndrome_ok);
}

// ------------------------------------------------------------------------
// misc
// ------------------------------------------------------------------------

extern "C" const char* ldpc_last_error_string(void) { return g_err.c_str(); }
extern "C" int ldpc_version(void) { return 1; }

__global__ void simd_selftest_kernel(int op, const uint32_t* a, const uint32_t* b, uint32_t* o, size_t n)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t x = a[i], y = b[i], r = 0;
    switch (op) {
    case 0: r = __vsubss4(x, y); break;
    case 1: r = __vaddss4(x, y); break;
    case 2: r = __vabs4(x); break;
    case 3: r = __vminu4(x, y); break;
    case 4: r = __vmaxu4(x, y); break;
    case 5: r = __vsubus4(x, y); break;
    case 6: r = __vcmpgts4(x, y); break;
    case 7: r = __vcmpeq4(x, y); break;
    case 8: r = __vneg4(x); break;
    case 9: r = __vsetgts4(x, y); break;
    }
    o[i] = r;
}

extern "C" int ldpc_simd_selftest(int op, const uint32_t* a, const uint32_t* b, uint32_t* o, size_t n, void* stream)
{
    if (!a || !b || !o || op < 0 || op > 9) return fail(LDPC_ERR_ARG, "ldpc_simd_selftest: bad argument");
    if (n == 0) return LDPC_OK;
    simd_selftest_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(op, a, b, o, n);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

// ------------------------------------------------------------------------
// INT32 issue-rate probe (roofline denominator of the integer decode kernels)
// ------------------------------------------------------------------------

// 8 independent chains per thread; MIX selects LOP3-only (0), IADD3-only (1) or alternating (2).
template <int MIX>
__global__ void __launch_bounds__(256) int_peak_kernel(uint32_t* out, uint32_t seed, int iters)
{
    uint32_t v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = seed * (i + 3) + threadIdx.x;
    const uint32_t k = seed ^ 0x9e3779b9u;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            // chains read their neighbour so that no closed form exists
            if (MIX == 0 || (MIX == 2 && (i & 1)))
                v[i] = (v[i] ^ v[(i + 1) & 7]) & (v[i] | k);  // one LOP3
            else
                v[i] = v[i] + v[(i + 1) & 7] + k;             // one IADD3
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) x ^= v[i];
    if (x == 0x12345678u) out[blockIdx.x] = x;  // keeps the chains live
}

extern "C" int ldpc_probe_int_peak(double* lane_ops_per_s, void* stream)
{
    if (!lane_ops_per_s) return fail(LDPC_ERR_ARG, "ldpc_probe_int_peak: null pointer");
    int dev = 0, sms = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint32_t* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(uint32_t) * sms * 8));
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    double best = 0;
    for (int mix = 0; mix < 3; mix++) {
        for (int rep = 0; rep < 3; rep++) {
            CUDA_TRY(cudaEventRecord(a, st));
            if (mix == 0) int_peak_kernel<0><<<blocks, threads, 0, st>>>(d, 7u + rep, iters);
            if (mix == 1) int_peak_kernel<1><<<blocks, threads, 0, st>>>(d, 7u + rep, iters);
            if (mix == 2) int_peak_kernel<2><<<blocks, threads, 0, st>>>(d, 7u + rep, iters);
            CUDA_TRY(cudaEventRecord(b, st));
            CUDA_TRY(cudaEventSynchronize(b));
            float ms = 0;
            CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
            double ops = (double)blocks * threads * iters * 8;
            if (ms > 0 && rep > 0) best = std::max(best, ops / (ms * 1e-3));
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    *lane_ops_per_s = best;
    return LDPC_OK;
}

// ------------------------------------------------------------------------
// batches of several codes: one persistent kernel (batch_kernel.cu)
// ------------------------------------------------------------------------

namespace ldpc {
const void* kernel_table_batch(int pack, int kind, int variant);
const void* kernel_table_batch_pf(int kind, int variant);
size_t batch_code_bytes();
void batch_code_fill(void* rec, const Plan& plan, const int8_t* llr, void* out, int32_t* iters_out, uint8_t* synd_out,
                     long long words, long long first_item, int quirk, int out_packed, int variant);
}  // namespace ldpc

struct ldpc_batch {
    int kind = 0, device = 0, pack = LDPC_PACK_SIMD4, variant = 0;
    bool early = false, use_graph = false;
    bool per_frame = false;  // LDPC_FLAG_EARLY_STOP_FRAMES: iteration counts per frame
    unsigned slack = LDPC_EARLY_STOP_DEFAULT_SLACK;
    std::vector<ldpc_decoder*> plans;  // each code's tables and schedule (decoder_setup)
    std::vector<int> cls;              // degree class of each code: 0 <= 8, 1 <= 16, 2 <= 32
    std::vector<int> dvar;             // its variant of the per-code kernels (degree_variant)
    std::vector<int> widest;           // its widest level
    // per-code strategy: one launch per code of that code's own decoder, chosen per code
    // among the candidate kernels (BatchCand) by ldpc_batch_autotune or set uniformly by
    // ldpc_batch_configure
    bool per_code = false;
    std::vector<ldpc_code> codes;                      // copies (the caller may destroy its codes)
    std::vector<std::vector<ldpc_decoder*>> pc_dec;    // [code][candidate], created on first use
    std::vector<int> pc_choice;                        // [code] candidate
    void* d_codes = nullptr;           // BatchCode[n]
    void* h_codes = nullptr;           // pinned staging of the same
    unsigned long long* d_counter = nullptr;
    const void* kfn = nullptr;
    int threads = 128, smem = 0, ctas_per_sm = 0, grid = 0, sms = 0;
    uint16_t* d_lut = nullptr;
    int lut_its = 0;
    std::vector<int8_t> off;
    std::vector<uint8_t> sc;
    cudaGraphExec_t exec = nullptr;
    std::vector<uintptr_t> key;     // what the captured graph was made for
    std::vector<uintptr_t> staged;  // what the staged records describe
    cudaEvent_t done = nullptr;  // the last launch (h_codes may be rewritten after it)
    // per-code strategy: the codes' launches run side by side, forked from and joined back to
    // the caller's stream (inside a graph capture too), so one code's early-stop tail overlaps
    // the others' work
    std::vector<cudaStream_t> side;  // one per code after the first
    std::vector<cudaEvent_t> fork;   // [0]: the fork point, [i]: code i's end
};

// Kernels the per-code strategy can give a code: the layered level kernels of the three
// packings, the QC register kernel (QC codes only: 4 frames per CTA on the regular base,
// path 1, else 2 frames per CTA with early stop per frame pair, path 4) and the flooding
// schedule (path 6)
enum BatchCand { CAND_SIMD4 = 0, CAND_F16X2 = 1, CAND_I8 = 2, CAND_QC = 3, CAND_FLOOD = 4, CAND_QC_SPLIT = 5, CAND_COUNT = 6 };

static void batch_free(ldpc_batch* b)
{
    if (!b) return;
    for (auto* d : b->plans) decoder_free(d);
    for (auto& v : b->pc_dec)
        for (auto* d : v)
            if (d) decoder_free(d);
    cudaFree(b->d_codes);
    cudaFreeHost(b->h_codes);
    cudaFree(b->d_counter);
    cudaFree(b->d_lut);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->done) cudaEventDestroy(b->done);
    for (auto x : b->side) cudaStreamDestroy(x);
    for (auto x : b->fork) cudaEventDestroy(x);
    delete b;
}

static size_t batch_smem(const ldpc_batch* b, int pack)
{
    size_t s = 0;
    for (auto* d : b->plans)
        s = std::max(s, smem_bytes(pack, d->plan.npad, d->plan.dmax, d->plan.m));
    return s + (b->kind == LDPC_LEARNED ? 512 : 0);
}

// LDPC_LEARNED tables of the batch for a packing
static int batch_lut(ldpc_batch* b, int pack)
{
    if (b->kind != LDPC_LEARNED || b->off.empty()) return LDPC_OK;
    std::vector<uint16_t> lut;
    int rc = build_learned_lut(pack == LDPC_PACK_F16X2, b->lut_its, b->off.data(), b->sc.data(), lut);
    if (rc) return rc;
    if (!b->d_lut) CUDA_TRY(cudaMalloc(&b->d_lut, sizeof(uint16_t) * 256 * LDPC_LEARNED_MAX_ITERS));
    CUDA_TRY(cudaMemcpy(b->d_lut, lut.data(), lut.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    return LDPC_OK;
}

// Frees the per-code decoders (they are re-created on use); a captured graph that refers
// to their tables is dropped with them
static void batch_drop_decoders(ldpc_batch* b)
{
    cudaDeviceSynchronize();
    for (auto& v : b->pc_dec)
        for (auto*& d : v)
            if (d) {
                decoder_free(d);
                d = nullptr;
            }
    b->key.clear();
}

// The decoder of candidate `cand` for code i (created on first use, then kept), with the
// batch's kind, early stop and learned constants.  Fails when the candidate cannot serve the
// code (shared memory, row degree, not a QC code, constants off the fp16 grid).
static int batch_code_decoder(ldpc_batch* b, int i, int cand, ldpc_decoder** out)
{
    ldpc_decoder*& d = b->pc_dec[i][cand];
    if (!d) {
        ldpc_code c = b->codes[i];
        int pack = cand == CAND_SIMD4 ? LDPC_PACK_SIMD4
                   : cand == CAND_I8  ? LDPC_PACK_I8
                   : cand == CAND_QC_SPLIT ? LDPC_PACK_F16X2_SPLIT
                                           : LDPC_PACK_F16X2;
        const bool qc_cand = cand == CAND_QC || cand == CAND_QC_SPLIT;
        if (!qc_cand) c.qc = false;  // the level kernels, also for a QC code
        else if (!c.qc) return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d is not quasi-cyclic", i);
        const int flags = (b->per_frame ? LDPC_FLAG_EARLY_STOP_FRAMES : (b->early ? LDPC_FLAG_EARLY_STOP : 0)) |
                          (cand == CAND_FLOOD ? LDPC_FLAG_FLOODING : 0);
        // nb_frames only bounds the words of a call; the batch passes its own counts
        int rc = ldpc_decoder_create(&d, &c, b->kind, (size_t)1 << 40, pack, flags);
        if (rc) return rc;
        if (cand == CAND_QC && d->path != 1 && d->path != 4) {
            decoder_free(d);
            d = nullptr;
            return fail(LDPC_ERR_UNSUPPORTED, "batch: code %d has no QC register kernel", i);
        }
        if (b->kind == LDPC_LEARNED && !b->off.empty()) {
            rc = ldpc_decoder_set_learned(d, b->lut_its, b->off.data(), b->sc.data());
            if (rc) {
                decoder_free(d);
                d = nullptr;
                return rc;
            }
        }
    }
    d->early_slack = b->slack;
    if (out) *out = d;
    return LDPC_OK;
}

// selects the strategy: one persistent kernel with this packing, CTA width and
// resident CTAs per SM (0 = as many as fit), or (per_code) one launch of each
// code's own level kernel with this packing
static int batch_configure(ldpc_batch* b, int pack, int threads, int ctas_per_sm, bool per_code = false)
{
    int smem_max = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device));
    const size_t lut = b->kind == LDPC_LEARNED ? 512 : 0;
    if (per_code) {
        (void)lut;
        for (size_t i = 0; i < b->codes.size(); i++) {
            int rc = batch_code_decoder(b, (int)i, pack, nullptr);
            if (rc) return fail(rc, "batch: code %zu does not fit pack %d: %s", i, pack, ldpc_last_error_string());
        }
        for (size_t i = 0; i < b->codes.size(); i++) b->pc_choice[i] = pack;
        b->per_code = true;
        b->pack = pack;
        b->kfn = nullptr;
        b->grid = 0;
        b->threads = 0;
        b->smem = 0;
        b->ctas_per_sm = 0;
        b->key.clear();
        return LDPC_OK;
    }
    const int k = b->kind == LDPC_LEARNED ? 4 : b->kind;
    const void* kfn = b->per_frame ? (pack == LDPC_PACK_SIMD4 ? kernel_table_batch_pf(b->kind, b->variant) : nullptr)
                                   : kernel_table_batch(pack, k, b->variant);
    if (!kfn)
        return fail(LDPC_ERR_UNSUPPORTED, "batch: no kernel for pack %d%s", pack,
                    b->per_frame ? " with the per-frame early stop (SIMD4 only)" : "");
    const size_t smem = batch_smem(b, pack);
    if (smem > (size_t)smem_max)
        return fail(LDPC_ERR_UNSUPPORTED, "batch: the largest code needs %zu B of shared memory with pack %d", smem, pack);
    int rc = batch_lut(b, pack);
    if (rc) return rc;
    CUDA_TRY(ldpc_internal_raise_smem(kfn, smem));
    int occ = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, threads, smem));
    if (occ < 1) return fail(LDPC_ERR_UNSUPPORTED, "batch: kernel cannot be resident (%zu B, %d threads)", smem, threads);
    b->per_code = false;
    b->pack = pack;
    b->kfn = kfn;
    b->threads = threads;
    b->smem = (int)smem;
    b->ctas_per_sm = ctas_per_sm > 0 ? std::min(ctas_per_sm, occ) : occ;
    b->grid = b->ctas_per_sm * b->sms;
    b->key.clear();  // a captured graph no longer matches
    return LDPC_OK;
}

extern "C" int ldpc_batch_create(ldpc_batch** out, const ldpc_code* const* codes, int n_codes, int kind, int pack,
                                 int flags)
{
    if (!out || !codes || n_codes < 1) return fail(LDPC_ERR_ARG, "ldpc_batch_create: no codes");
    if (kind < LDPC_MS || kind > LDPC_LEARNED || kind == LDPC_XMS)
        return fail(LDPC_ERR_ARG, "ldpc_batch_create: kind %d (xMS reads interleaved input; use OMS)", kind);
    if (flags & ~(LDPC_FLAG_EARLY_STOP | LDPC_FLAG_EARLY_STOP_FRAMES | LDPC_BATCH_GRAPH))
        return fail(LDPC_ERR_ARG, "unknown flags 0x%x", flags);
    if ((flags & (LDPC_FLAG_EARLY_STOP | LDPC_FLAG_EARLY_STOP_FRAMES)) && kind == LDPC_2NMS)
        return fail(LDPC_ERR_ARG, "LDPC_FLAG_EARLY_STOP: LDPC_2NMS has the reference's own early termination");
    if (pack != LDPC_PACK_AUTO && (pack < LDPC_PACK_SIMD4 || pack > LDPC_PACK_I8))
        return fail(LDPC_ERR_ARG, "ldpc_batch_create: pack %d (SIMD4, F16X2, I8 or AUTO)", pack);
    int dmax = 0;
    for (int i = 0; i < n_codes; i++) {
        if (!codes[i]) return fail(LDPC_ERR_ARG, "ldpc_batch_create: null code %d", i);
        dmax = std::max(dmax, codes[i]->dmax);
    }
    if (dmax > kMaxDegree) return fail(LDPC_ERR_UNSUPPORTED, "row degree %d > %d", dmax, kMaxDegree);
    ldpc_batch* b = new ldpc_batch();
    b->kind = kind;
    b->per_frame = flags & LDPC_FLAG_EARLY_STOP_FRAMES;
    b->early = (flags & LDPC_FLAG_EARLY_STOP) || b->per_frame;
    b->use_graph = flags & LDPC_BATCH_GRAPH;
    b->variant = dmax <= 8 ? 0 : (dmax <= 16 ? 1 : 2);
    cudaError_t e = cudaGetDevice(&b->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_codes, batch_code_bytes() * n_codes);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_codes, batch_code_bytes() * n_codes);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    for (int i = 0; i < n_codes && e == cudaSuccess; i++) {
        cudaEvent_t ev = nullptr;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) b->fork.push_back(ev);
        if (e == cudaSuccess && i > 0) {
            cudaStream_t sx = nullptr;
            e = cudaStreamCreateWithFlags(&sx, cudaStreamNonBlocking);
            if (e == cudaSuccess) b->side.push_back(sx);
        }
    }
    if (e != cudaSuccess) {
        batch_free(b);
        return fail(LDPC_ERR_CUDA, "ldpc_batch_create: %s", cudaGetErrorString(e));
    }
    for (int i = 0; i < n_codes; i++) {
        b->codes.push_back(*codes[i]);
        b->pc_dec.push_back(std::vector<ldpc_decoder*>(CAND_COUNT, nullptr));
        b->pc_choice.push_back(CAND_SIMD4);
        const int dm = codes[i]->dmax;
        b->cls.push_back(dm <= 8 ? 0 : (dm <= 16 ? 1 : 2));
        b->dvar.push_back(degree_variant(codes[i]));
        b->widest.push_back(codes[i]->widest);
        ldpc_decoder* d = new ldpc_decoder();
        b->plans.push_back(d);
        int rc = decoder_setup(d, codes[i]);
        if (rc) {
            batch_free(b);
            return rc;
        }
    }
    int rc = LDPC_ERR_UNSUPPORTED;
    const int order[3] = {LDPC_PACK_SIMD4, LDPC_PACK_I8, LDPC_PACK_F16X2};
    for (int i = 0; i < 3 && rc; i++) {
        const int p = pack == LDPC_PACK_AUTO ? order[i] : pack;
        rc = batch_configure(b, p, 128, 0);
        if (pack != LDPC_PACK_AUTO) break;
    }
    if (rc) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return LDPC_OK;
}

extern "C" int ldpc_batch_set_learned(ldpc_batch* b, int n_iters, const int8_t* offsets, const uint8_t* scales)
{
    if (!b || !offsets || !scales) return fail(LDPC_ERR_ARG, "ldpc_batch_set_learned: null pointer");
    if (b->kind != LDPC_LEARNED) return fail(LDPC_ERR_ARG, "ldpc_batch_set_learned: batch kind is not LDPC_LEARNED");
    if (n_iters < 1 || n_iters > LDPC_LEARNED_MAX_ITERS)
        return fail(LDPC_ERR_ARG, "ldpc_batch_set_learned: n_iters must be in [1, %d]", LDPC_LEARNED_MAX_ITERS);
    b->off.assign(offsets, offsets + 2 * n_iters);
    b->sc.assign(scales, scales + 2 * n_iters);
    b->lut_its = n_iters;
    batch_drop_decoders(b);  // re-created with the new constants
    int rc = LDPC_OK;
    if (b->per_code) {
        for (size_t i = 0; i < b->codes.size() && !rc; i++) rc = batch_code_decoder(b, (int)i, b->pc_choice[i], nullptr);
    } else {
        rc = batch_configure(b, b->pack, b->threads, b->ctas_per_sm, false);
    }
    if (rc) {
        b->off.clear();
        b->sc.clear();
        b->lut_its = 0;
    }
    return rc;
}

extern "C" int ldpc_batch_set_early_stop(ldpc_batch* b, int enabled, int slack)
{
    if (!b) return fail(LDPC_ERR_ARG, "ldpc_batch_set_early_stop: null batch");
    if (enabled && b->kind == LDPC_2NMS)
        return fail(LDPC_ERR_ARG, "LDPC_FLAG_EARLY_STOP: LDPC_2NMS has the reference's own early termination");
    if (slack < 0) return fail(LDPC_ERR_ARG, "ldpc_batch_set_early_stop: slack must be >= 0");
    if (!enabled && b->per_frame)
        return fail(LDPC_ERR_ARG, "the per-frame early stop of this batch cannot be turned off; create one without "
                                  "LDPC_FLAG_EARLY_STOP_FRAMES");
    if (b->early != (enabled != 0)) batch_drop_decoders(b);  // per-code decoders: re-created with the flag
    b->early = enabled != 0;
    b->slack = (unsigned)slack;
    b->key.clear();
    return LDPC_OK;
}

extern "C" int ldpc_batch_decode(ldpc_batch* b, const int8_t* const* d_llr, void* const* d_out, const size_t* n_words,
                                 int iters, int out_format, int32_t* const* d_iters_out,
                                 uint8_t* const* d_syndrome_ok, void* stream)
{
    if (!b || !d_llr || !d_out || !n_words) return fail(LDPC_ERR_ARG, "ldpc_batch_decode: null pointer");
    if (iters < 1) return fail(LDPC_ERR_ARG, "ldpc_batch_decode: iterations must be >= 1 (got %d)", iters);
    if (out_format != LDPC_OUT_BYTES && out_format != LDPC_OUT_PACKED)
        return fail(LDPC_ERR_ARG, "ldpc_batch_decode: unknown output format %d", out_format);
    if (b->kind == LDPC_LEARNED && b->off.empty())
        return fail(LDPC_ERR_ARG, "LDPC_LEARNED batch: set its offsets and scales first");
    if (b->use_graph && !stream)
        return fail(LDPC_ERR_ARG, "LDPC_BATCH_GRAPH: pass a stream (the legacy default stream cannot be captured)");
    const int n = (int)b->plans.size();
    long long total = 0;
    std::vector<uintptr_t> recs = {(uintptr_t)out_format};
    for (int i = 0; i < n; i++) {
        if (n_words[i] > 0 && (!d_llr[i] || !d_out[i]))
            return fail(LDPC_ERR_ARG, "ldpc_batch_decode: null buffer for code %d", i);
        total += (long long)n_words[i];
        recs.push_back((uintptr_t)d_llr[i]);
        recs.push_back((uintptr_t)d_out[i]);
        recs.push_back((uintptr_t)n_words[i]);
        recs.push_back((uintptr_t)(d_iters_out ? d_iters_out[i] : nullptr));
        recs.push_back((uintptr_t)(d_syndrome_ok ? d_syndrome_ok[i] : nullptr));
    }
    if (total == 0) return LDPC_OK;
    std::vector<uintptr_t> key = recs;
    for (uintptr_t x : {(uintptr_t)b->kfn, (uintptr_t)b->grid, (uintptr_t)b->threads, (uintptr_t)iters,
                        (uintptr_t)b->early, (uintptr_t)b->slack, (uintptr_t)stream, (uintptr_t)b->d_lut,
                        (uintptr_t)b->per_code, (uintptr_t)b->pack})
        key.push_back(x);
    CUDA_TRY(cudaSetDevice(b->device));
    cudaStream_t st = (cudaStream_t)stream;
    if (recs != b->staged) {
        // the staging buffer may still feed the previous launch's copy
        CUDA_TRY(cudaEventSynchronize(b->done));
        b->staged = recs;
        long long first = 0;
        for (int i = 0; i < n; i++) {
            batch_code_fill(static_cast<char*>(b->h_codes) + i * batch_code_bytes(), b->plans[i]->plan, d_llr[i],
                            d_out[i], d_iters_out ? d_iters_out[i] : nullptr,
                            d_syndrome_ok ? d_syndrome_ok[i] : nullptr, (long long)n_words[i], first,
                            b->kind == LDPC_OMS, out_format == LDPC_OUT_PACKED, b->cls[i]);
            first += (long long)n_words[i];
        }
    }
    Job J{};
    J.iters = iters;
    J.quirk = b->kind == LDPC_OMS;
    J.early = b->early ? 1 : 0;
    J.early_slack = b->slack;
    J.lut = b->d_lut;
    J.lut_its = b->lut_its;
    void* codes = b->d_codes;
    unsigned long long* counter = b->d_counter;
    void* args[] = {(void*)&codes, (void*)&n, (void*)&counter, (void*)&total, (void*)&J};
    if (b->per_code)
        for (int i = 0; i < n; i++) {
            ldpc_decoder* dc = nullptr;
            int rc = batch_code_decoder(b, i, b->pc_choice[i], &dc);
            if (rc) return rc;
            key.push_back((uintptr_t)dc->kfn);
        }
    // the launches; per code: each code's own decoder (launch()), the codes forked onto the
    // batch's side streams from `st` and joined back to it
    auto enqueue = [&]() -> cudaError_t {
        if (b->per_code) {
            cudaError_t e = cudaEventRecord(b->fork[0], st);
            for (int i = 0; i < n && e == cudaSuccess; i++) {
                if (n_words[i] == 0) continue;
                cudaStream_t si = i == 0 ? st : b->side[i - 1];
                if (i > 0) e = cudaStreamWaitEvent(si, b->fork[0], 0);
                if (e != cudaSuccess) break;
                ldpc_decoder* dc = b->pc_dec[i][b->pc_choice[i]];
                if (launch(dc, d_llr[i], d_out[i], out_format == LDPC_OUT_PACKED, 0, (long long)n_words[i],
                           (long long)n_words[i], iters, d_iters_out ? d_iters_out[i] : nullptr, nullptr, nullptr, si,
                           nullptr, d_syndrome_ok ? d_syndrome_ok[i] : nullptr))
                    return cudaErrorLaunchFailure;
                if (i > 0) e = cudaEventRecord(b->fork[i], si);
                if (e == cudaSuccess && i > 0) e = cudaStreamWaitEvent(st, b->fork[i], 0);
            }
            return e;
        }
        cudaError_t e = cudaMemcpyAsync(b->d_codes, b->h_codes, batch_code_bytes() * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), st);
        if (e == cudaSuccess)
            e = cudaLaunchKernel(b->kfn, dim3((unsigned)b->grid), dim3(b->threads), args, b->smem, st);
        return e;
    };
    if (b->use_graph) {
        if (!b->exec || key != b->key) {
            if (b->exec) {
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
            cudaGraph_t g = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = enqueue();
            cudaError_t e2 = cudaStreamEndCapture(st, &g);
            if (e == cudaSuccess) e = e2;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(LDPC_ERR_CUDA, "ldpc_batch_decode: graph capture: %s", cudaGetErrorString(e));
            b->key = key;
        }
        CUDA_TRY(cudaGraphLaunch(b->exec, st));
    } else {
        CUDA_TRY(enqueue());
    }
    CUDA_TRY(cudaEventRecord(b->done, st));
    return LDPC_OK;
}

// the per-code strategy with the per-code choices as they stand
static void batch_use_per_code(ldpc_batch* b)
{
    b->per_code = true;
    b->kfn = nullptr;
    b->grid = b->threads = b->smem = b->ctas_per_sm = 0;
    b->key.clear();
}

// Per-code choice: for each code, every candidate kernel (BatchCand) is timed alone on that
// code's inputs and its frames whose decisions fail the syndrome are counted (the
// d_syndrome_ok flags).  The fastest candidate wins among those that leave no more failing
// frames than the reference's layered schedule (SIMD4) does, within 2 % and 2 frames: the
// flooding schedule and the 2-frame QC kernel's per-pair early stop may converge differently.
static int batch_tune_codes(ldpc_batch* b, const int8_t* const* d_llr, void* const* d_out, const size_t* n_words,
                            int iters, int32_t* const* d_iters_out, cudaStream_t st)
{
    size_t fmax = 0;
    for (size_t i = 0; i < b->codes.size(); i++) fmax = std::max(fmax, 4 * n_words[i]);
    if (fmax == 0) return LDPC_OK;
    uint8_t* d_syn = nullptr;
    CUDA_TRY(cudaMalloc(&d_syn, fmax));
    std::vector<uint8_t> h_syn(fmax);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (size_t i = 0; i < b->codes.size(); i++) {
        if (n_words[i] == 0) continue;
        const long long w = (long long)n_words[i];
        long long base_fail = -1;
        double best = 1e30;
        int best_c = b->pc_choice[i];
        for (int c = 0; c < CAND_COUNT; c++) {
            ldpc_decoder* dc = nullptr;
            if (batch_code_decoder(b, (int)i, c, &dc)) continue;
            int32_t* its = d_iters_out ? d_iters_out[i] : nullptr;
            if (launch(dc, d_llr[i], d_out[i], 0, 0, w, w, iters, its, nullptr, nullptr, st, nullptr, d_syn)) continue;
            if (cudaMemcpyAsync(h_syn.data(), d_syn, 4 * w, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                continue;
            long long fail_c = 0;
            for (long long f = 0; f < 4 * w; f++) fail_c += h_syn[f] == 0;
            cudaEventRecord(e0, st);
            bool ok = true;
            for (int r = 0; r < 3 && ok; r++)
                ok = !launch(dc, d_llr[i], d_out[i], 0, 0, w, w, iters, its, nullptr, nullptr, st, nullptr, nullptr);
            cudaEventRecord(e1, st);
            float ms = 0.f;
            if (!ok || cudaEventSynchronize(e1) != cudaSuccess) continue;
            cudaEventElapsedTime(&ms, e0, e1);
            if (c == CAND_SIMD4) base_fail = fail_c;
            const bool equal_fer = base_fail < 0 || fail_c <= base_fail + std::max(2LL, base_fail / 50);
            if (equal_fer && ms / 3 < best) {
                best = ms / 3;
                best_c = c;
            }
        }
        b->pc_choice[i] = best_c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_syn);
    b->key.clear();
    return LDPC_OK;
}

extern "C" int ldpc_batch_autotune(ldpc_batch* b, const int8_t* const* d_llr, void* const* d_out,
                                   const size_t* n_words, int iters, int32_t* const* d_iters_out, double* best_ms,
                                   void* stream)
{
    if (!b) return fail(LDPC_ERR_ARG, "ldpc_batch_autotune: null batch");
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaSetDevice(b->device));
    // the kernel of each code for the per-code strategy (schedule, packing, frames per CTA)
    int rc = batch_tune_codes(b, d_llr, d_out, n_words, iters, d_iters_out, st);
    if (rc) return rc;
    const std::vector<int> choice = b->pc_choice;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    const int packs[3] = {LDPC_PACK_SIMD4, LDPC_PACK_F16X2, LDPC_PACK_I8};
    const int widths[4] = {0, 64, 128, 256};  // 0: the per-code strategy (once, with the tuned choices)
    double best = 1e30;
    int bp = b->pack, bt = b->threads, bc = 0;
    bool bpc = false;
    const bool graph = b->use_graph;
    b->use_graph = false;  // time the launches themselves
    for (int p : packs) {
        for (int t : widths) {
            for (int half = 0; half < 2; half++) {
                if (t == 0) {
                    if (half || p != LDPC_PACK_SIMD4) continue;
                    b->pc_choice = choice;
                    batch_use_per_code(b);
                } else {
                    if (batch_configure(b, p, t, 0)) continue;
                    const int ctas = half ? std::max(1, b->ctas_per_sm / 2) : b->ctas_per_sm;
                    if (half && ctas == b->ctas_per_sm) continue;
                    if (batch_configure(b, p, t, ctas)) continue;
                }
                rc = ldpc_batch_decode(b, d_llr, d_out, n_words, iters, LDPC_OUT_BYTES, d_iters_out, nullptr, stream);
                if (rc) continue;
                float ms = 0.f;
                cudaEventRecord(e0, st);
                for (int r = 0; r < 3 && !rc; r++)
                    rc = ldpc_batch_decode(b, d_llr, d_out, n_words, iters, LDPC_OUT_BYTES, d_iters_out, nullptr, stream);
                cudaEventRecord(e1, st);
                if (rc || cudaEventSynchronize(e1) != cudaSuccess) continue;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms / 3 < best) {
                    best = ms / 3;
                    bp = p;
                    bt = t;
                    bc = b->ctas_per_sm;
                    bpc = b->per_code;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->use_graph = graph;
    b->pc_choice = choice;
    if (bpc) {
        batch_use_per_code(b);
    } else {
        rc = batch_configure(b, bp, bt, bc, false);
        if (rc) return rc;
    }
    if (best_ms) *best_ms = best;
    return best < 1e30 ? LDPC_OK : fail(LDPC_ERR_UNSUPPORTED, "ldpc_batch_autotune: no configuration ran");
}

extern "C" int ldpc_batch_set_code_kernel(ldpc_batch* b, int code, int candidate)
{
    if (!b || code < 0 || code >= (int)b->codes.size() || candidate < 0 || candidate >= CAND_COUNT)
        return fail(LDPC_ERR_ARG, "ldpc_batch_set_code_kernel: bad argument");
    CUDA_TRY(cudaSetDevice(b->device));
    int rc = batch_code_decoder(b, code, candidate, nullptr);
    if (rc) return rc;
    if (!b->per_code) {
        // the other codes keep the persistent kernel's packing as their level kernel
        for (size_t i = 0; i < b->codes.size(); i++)
            if ((int)i != code) b->pc_choice[i] = b->pack;
    }
    b->pc_choice[code] = candidate;
    batch_use_per_code(b);
    return LDPC_OK;
}

extern "C" int ldpc_batch_code_info(const ldpc_batch* b, int code, int* info)
{
    if (!b || !info || code < 0 || code >= (int)b->codes.size())
        return fail(LDPC_ERR_ARG, "ldpc_batch_code_info: bad argument");
    const int c = b->pc_choice[code];
    const ldpc_decoder* d = b->pc_dec[code][c];
    info[0] = c;
    info[1] = d ? d->path : -1;
    info[2] = d ? d->threads : 0;
    info[3] = d ? d->smem : 0;
    info[4] = d ? d->ctas_per_sm : 0;
    return LDPC_OK;
}

extern "C" int ldpc_batch_configure(ldpc_batch* b, int per_code, int pack, int threads, int ctas_per_sm)
{
    if (!b) return fail(LDPC_ERR_ARG, "ldpc_batch_configure: null batch");
    if (pack < LDPC_PACK_SIMD4 || pack > LDPC_PACK_I8) return fail(LDPC_ERR_ARG, "ldpc_batch_configure: pack %d", pack);
    if (!per_code && (threads < 32 || threads > 256 || threads % 32 || ctas_per_sm < 0))
        return fail(LDPC_ERR_ARG, "ldpc_batch_configure: threads must be 32..256 in steps of 32, ctas_per_sm >= 0");
    return batch_configure(b, pack, threads, ctas_per_sm, per_code != 0);
}

extern "C" int ldpc_batch_info(const ldpc_batch* b, int* info)
{
    if (!b || !info) return fail(LDPC_ERR_ARG, "ldpc_batch_info: null pointer");
    info[0] = b->kind;
    info[1] = b->pack;
    info[2] = b->threads;
    info[3] = b->smem;
    info[4] = b->ctas_per_sm;
    info[5] = b->grid;
    info[6] = b->use_graph;
    info[7] = (int)b->plans.size();
    info[8] = b->per_code;
    return LDPC_OK;
}

extern "C" int ldpc_batch_destroy(ldpc_batch* b)
{
    if (!b) return LDPC_OK;
    cudaError_t e = cudaDeviceSynchronize();
    batch_free(b);
    if (e != cudaSuccess) return fail(LDPC_ERR_CUDA, "ldpc_batch_destroy: %s", cudaGetErrorString(e));
    return LDPC_OK;
}

// ------------------------------------------------------------------------
// Decoding without any allocation
// ------------------------------------------------------------------------
//
// Some callers may not allocate device memory once they are running: real-time
// receive chains and plugin hosts that reserve all GPU memory at start-up, where
// cudaMalloc can stall for milliseconds, cudaFree synchronises the whole device,
// and a framework-owned memory pool may refuse the request outright.  For them,
// ldpc_decode_noalloc decodes with the level-scheduled kernel and no allocation:
// the per-code tables that ldpc_decoder_create puts in its own device buffers
// (column table, row degrees, row groups, level list) go instead into the fixed
// array below, which every GPU that loads this library holds until exit.
//
// The tables reach that array as kernel parameters (chunks of kNoallocChunk bytes
// copied by noalloc_upload_kernel), not by a copy from host memory: a launch takes
// its parameters by value when it is issued, so nothing refers to a host buffer after
// the call returns, and the host never waits for earlier work in the stream.

#define LDPC_NOALLOC_SCRATCH_BYTES (256 * 1024)

static __device__ __align__(256) unsigned char g_noalloc_scratch[LDPC_NOALLOC_SCRATCH_BYTES];

// 30 KiB per launch: kernel parameters may hold up to 32764 bytes (CUDA 12.1 and later)
static const unsigned kNoallocChunk = 30 * 1024;

struct NoallocChunk {
    unsigned offset;  // byte offset in g_noalloc_scratch (a multiple of 4)
    unsigned words;   // 32-bit words in data
    uint32_t data[kNoallocChunk / 4];
};

__global__ void noalloc_upload_kernel(const __grid_constant__ NoallocChunk c)
{
    uint32_t* dst = reinterpret_cast<uint32_t*>(g_noalloc_scratch + c.offset);
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < c.words; i += gridDim.x * blockDim.x)
        dst[i] = c.data[i];
}

// host image of the tables and the parameter block, filled per call under the mutex
static unsigned char g_noalloc_host[LDPC_NOALLOC_SCRATCH_BYTES];
static NoallocChunk g_noalloc_chunk;
static std::mutex g_noalloc_mutex;
static const int kNoallocMaxDevices = 64;
// device address of g_noalloc_scratch, looked up once per device by the first call there
static void* g_noalloc_dev_ptr[kNoallocMaxDevices];

extern "C" int ldpc_decode_noalloc(const ldpc_code* c, int kind, int pack, const int8_t* d_llr, uint8_t* d_hard,
                                   size_t n_words, int iters, void* stream)
{
    if (!c || !d_llr || !d_hard) return fail(LDPC_ERR_ARG, "ldpc_decode_noalloc: null pointer");
    if (kind < LDPC_MS || kind > LDPC_XMS) return fail(LDPC_ERR_ARG, "ldpc_decode_noalloc: unknown kind %d", kind);
    if (pack == LDPC_PACK_AUTO) pack = LDPC_PACK_SIMD4;
    if (pack < LDPC_PACK_SIMD4 || pack > LDPC_PACK_I8) return fail(LDPC_ERR_ARG, "ldpc_decode_noalloc: unknown pack");
    if (iters < 1) return fail(LDPC_ERR_ARG, "ldpc_decode_noalloc: iterations must be >= 1 (got %d)", iters);
    if (n_words < 1) return fail(LDPC_ERR_SHAPE, "ldpc_decode_noalloc: n_words must be >= 1");
    if (c->dmax > kMaxDegree) return fail(LDPC_ERR_UNSUPPORTED, "row degree %d > %d", c->dmax, kMaxDegree);
    const int m = c->m, dmax = c->dmax, nlev = (int)c->levels.size();
    // layout: cols u16 [dmax][m] | rowdeg u8 [m] | rowcls u8 [m] | pad to 8 | levels int2 [nlev]
    const size_t off_deg = (size_t)dmax * m * 2, off_cls = off_deg + m, off_lev = (off_cls + m + 7) / 8 * 8;
    const size_t bytes = off_lev + (size_t)nlev * sizeof(int2);
    if (bytes > LDPC_NOALLOC_SCRATCH_BYTES)
        return fail(LDPC_ERR_UNSUPPORTED,
                    "ldpc_decode_noalloc: the code's tables need %zu bytes, more than the %d-byte static array",
                    bytes, LDPC_NOALLOC_SCRATCH_BYTES);
    const int npad = (c->n + 15) / 16 * 16;
    const size_t smem = smem_bytes(pack, npad, dmax, m);
    int dev = 0, smem_max = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoallocMaxDevices) return fail(LDPC_ERR_UNSUPPORTED, "device %d out of range", dev);
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (smem > (size_t)smem_max)
        return fail(LDPC_ERR_UNSUPPORTED, "decoder state of one frame group needs %zu B of shared memory (> %d)", smem,
                    smem_max);
    const void* kfn = kernel_for(pack, kind, degree_variant(c));
    if (!kfn) return fail(LDPC_ERR_UNSUPPORTED, "ldpc_decode_noalloc: no kernel for this pack/kind");

    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    // set-up, once per device with that device current: the device address of the array
    // (in host code the array's name is only a host-side stand-in)
    if (!g_noalloc_dev_ptr[dev]) {
        void* p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_dev_ptr[dev] = p;
    }
    unsigned char* base = static_cast<unsigned char*>(g_noalloc_dev_ptr[dev]);
    // every byte the kernel reads is rewritten for this call
    uint16_t* hcols = reinterpret_cast<uint16_t*>(g_noalloc_host);
    uint8_t* hdeg = g_noalloc_host + off_deg;
    uint8_t* hcls = g_noalloc_host + off_cls;
    int2* hlev = reinterpret_cast<int2*>(g_noalloc_host + off_lev);
    const size_t padded = (bytes + 3) / 4 * 4;
    memset(g_noalloc_host, 0, padded);
    for (int rp = 0; rp < m; rp++) {
        const int r = c->order[rp], b = c->row_ptr[r], dg = c->row_ptr[r + 1] - b;
        hdeg[rp] = (uint8_t)dg;
        hcls[rp] = c->row_class[r];
        for (int j = 0; j < dg; j++) hcols[(size_t)j * m + rp] = (uint16_t)c->cols[b + j];
    }
    for (int l = 0; l < nlev; l++) hlev[l] = c->levels[l];
    cudaStream_t st = (cudaStream_t)stream;
    for (size_t off = 0; off < padded; off += kNoallocChunk) {
        const size_t len = std::min<size_t>(kNoallocChunk, padded - off);
        g_noalloc_chunk.offset = (unsigned)off;
        g_noalloc_chunk.words = (unsigned)(len / 4);
        memcpy(g_noalloc_chunk.data, g_noalloc_host + off, len);
        void* ua[] = {(void*)&g_noalloc_chunk};
        const unsigned blocks = (unsigned)std::min<size_t>(32, (len / 4 + 255) / 256);
        CUDA_TRY(cudaLaunchKernel((const void*)noalloc_upload_kernel, dim3(blocks), dim3(256), ua, 0, st));
    }

    Plan P{};
    P.n = c->n;
    P.npad = npad;
    P.m = m;
    P.dmax = dmax;
    P.nlevels = nlev;
    P.cols = reinterpret_cast<const uint16_t*>(base);
    P.rowdeg = base + off_deg;
    P.rowcls = base + off_cls;
    P.levels = reinterpret_cast<const int2*>(base + off_lev);
    P.edge_orig = nullptr;
    Job J{};
    J.llr = d_llr;
    J.out = d_hard;
    J.interleaved = kind == LDPC_XMS;
    J.total_words = (long long)n_words;
    J.iters = iters;
    J.quirk = kind == LDPC_OMS;
    const int threads = std::min(256, std::max(32, (c->widest + 31) / 32 * 32));
    CUDA_TRY(ldpc_internal_raise_smem(kfn, smem));
    void* args[] = {(void*)&P, (void*)&J};
    CUDA_TRY(cudaLaunchKernel(kfn, dim3((unsigned)n_words), dim3(threads), args, smem, st));
    return LDPC_OK;
}
