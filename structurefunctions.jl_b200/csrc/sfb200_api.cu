// sfb200_api.cu -- the C ABI (include/sfb200.h): contexts, plans, device workspace, runs.
//
// A run is: [H2D copy of the caller's arrays] -> pack kernel (SoA + FP32 images + bounds) ->
// [FP32 window table] -> [joint value windows] -> pair kernel -> [copy-out kernel | D2H copy].
// Everything is queued on one stream; host outputs are returned after a stream synchronize.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "../../include/sfb200.h"
#include "sfb200_internal.h"
#include "sfb200_kernels.cuh"
#include "sfb200_prep.cuh"

using namespace sfb;

struct sfb200_ctx {
    int device = 0;
    int nsm = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // batched rounds, double-buffered so that the next round can be enqueued while one runs: per
    // buffer the work items (pinned host staging + device copy), launch counters, the graph and the
    // event recorded after the round (the buffer is free again once it has fired)
    static constexpr int kRoundBufs = 2;
    struct RoundBuf {
        void* h_items = nullptr;
        void* d_items = nullptr;
        size_t items_cap = 0;   // WorkItem capacity of both copies
        unsigned* d_counters = nullptr;
        int counters_cap = 0;
        cudaGraphExec_t exec = nullptr;
        cudaEvent_t done = nullptr;
        bool pending = false;
        unsigned long long seq = 0;  // round number of the last round enqueued from this buffer
    } rb[kRoundBufs];
    unsigned long long rounds_enqueued = 0;
    bool batch_graph = true;    // capture rounds as a graph (cleared if capture is refused)
    // slice memory: a stream-ordered pool owned by the context (freed blocks stay reserved for the
    // next slices instead of going back to the driver)
    cudaMemPool_t pool = nullptr;
    // the kernels of one round run concurrently on these streams (fork / join through events)
    static constexpr int kLanes = 8;
    cudaStream_t lane[kLanes] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kLanes] = {};
    cudaStream_t prep_stream = nullptr;  // slice preparation, overlapping the running round
    cudaStream_t side_stream = nullptr;  // reads and frees of finished slices (not behind later rounds)
    void* noalloc_ptr = nullptr;  // device address of the no-allocation scratch (looked up on first use)
};

// Device buffers of one run over n <= cap points: raw inputs, the packed SoA layout, the point
// order, and the accumulated histogram. A plan owns one (for sfb200_run); every slice its own.
struct Workspace {
    long long cap = 0;
    void* d_rawx = nullptr;
    void* d_rawu = nullptr;
    double* d_X64 = nullptr;
    double* d_U64 = nullptr;
    float* d_XF = nullptr;
    float* d_UF = nullptr;
    double* d_XM = nullptr;       // mixed sphere: FP64 p(3), U(3), W(3)[, up] per point (SoA)
    // spatial order: Morton keys and the permutation (double-buffered for the radix sort)
    unsigned* d_keys = nullptr;   // 2 * cap
    int* d_perm = nullptr;        // 2 * cap
    unsigned* d_box = nullptr;    // 6
    void* d_sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    double* d_sums = nullptr;
    unsigned long long* d_counts = nullptr;
    unsigned long long* d_aux = nullptr;  // [0] rechecked pairs, [1] |x| bound, [2] |u| bound
    size_t bytes = 0;                     // device bytes held
    void* block = nullptr;                // slices: every buffer above lies in this one pooled block
};

struct sfb200_plan {
    sfb200_ctx* ctx = nullptr;
    sfb200_plan_desc desc{};
    bool sphere = false, joint = false;
    bool fp32 = false;   // precision FP32: FP32-bulk kernels with the FP64 recheck
    bool mixed = false;  // precision MIXED: FP64 differences / numerators, FP32 normalisation + accumulation
    bool promoted = false;  // precision MIXED requested, the FP64 kernels run (flat single-pass 2D rows)
    int sp2d_rows = 0;      // >= 2: a joint plan of that many consecutive flat single-pass 2D rows
    bool df = false;  // FP32 records carry (hi, lo) pairs (an input is FP64, or the sphere basis)
    bool l_only = false;  // the joint value depends on du_L only (compensated in FP32)
    int D = 0, W = 0, nb = 0, nv = 0, nops = 0, nops_pad = 0, opl = 0, vorder = 1;
    GenOps gen{};
    // exact key tables (flat: squared edges; sphere: edges with -0.0 moved just below +0.0)
    std::vector<double> exact_tab;
    double* d_exact = nullptr;
    std::vector<double> vedges;
    double* d_vedges = nullptr;
    LinearParams dlin{}, vlin{};
    // FP64 table
    LutGeom lg64{};
    LutEntry64* d_lut64 = nullptr;
    int lut64_bytes = 0;
    // flat byte table (FP64 and mixed 1D kernels): kByteCells bytes + kByteEdges padded edges
    unsigned char* d_lut8 = nullptr;
    // FP32 table (mixed): edge keys, geometry, window parameters
    std::vector<double> ck;
    double* d_ck = nullptr;
    LutGeom lg32{};
    LutEntry32* d_lut32 = nullptr;
    WindowParams wp{};
    double* d_rowlo = nullptr;
    float* d_vwin = nullptr;
    Workspace ws;  // the workspace of sfb200_run
    long long n_sums = 0, n_counts = 0;
    std::vector<double> h_sums;
    std::vector<unsigned long long> h_counts;
    sfb200_stats stats{};
    bool stats_pending = false;
    int tile_ovr = 0, priv_ovr = -1, bps_ovr = 0;
    double vq = 1.0, vq_inv = 1.0;  // joint mixed: fixed-point scale of the value offsets
    double vqc = 1.0, vqc_inv = 1.0;  // mixed joint: coarse scale of the packed cells
    int vfine_lo = 1, nfine = 0;      // mixed joint: value bins with exact offsets
    int order_ovr = -1;   // -1 auto, 0 caller order, 1 Morton order
    int shard_index = 0, shard_count = 1;  // sfb200_run covers shard shard_index of shard_count
    int cols_ovr = 0;     // run-length histogram columns (0 auto)
    int sort_ovr = -1;    // J-tile order of the flat 1D kernels: -1 auto (sorted), 0 storage order, 1 sorted
    unsigned long long* d_range = nullptr;  // sfb200_distance_range: min / max key bits
    // FP64 sphere (1D): the chord formulation (default) or the reference formulation (the pair frame
    // for every pair); -1 automatic, 1 reference, 2 chord
    int form_ovr = -1;
    LutGeom lgc{};                    // chord-key table of the FP64 chord kernel
    LutEntry64* d_lutc = nullptr;
    int lutc_bytes = 0;
    bool fp64_sphere_1d() const { return sphere && !joint && !fp32 && !mixed; }
    bool chord64() const { return fp64_sphere_1d() && form_ovr != 1; }

};

// ------------------------------------------------------------------------------- errors

// The message of the calling thread's last failed call and the context it was made on: per thread,
// so that threads sharing a context (slice preparation beside the round loop) never race on it.
static thread_local std::string t_err;
static thread_local const sfb200_ctx* t_err_ctx = nullptr;

static int set_err(sfb200_ctx* ctx, int code, const char* fmt, ...);

// Raises a kernel's dynamic shared-memory limit to at least `bytes` (per device; never lowers it).
// The limit is process-wide per function, and threads may configure and launch the same kernel at
// once (slice preparation beside the round loop): lowering it could fail another thread's launch
// between its own raise and its launch.
static int raise_smem_limit(sfb200_ctx* ctx, const void* fn, size_t bytes)
{
    static std::mutex mu;
    static std::unordered_map<const void*, size_t> limit[64];
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = limit[ctx->device & 63][fn];
    if (bytes <= cur) return 0;
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return set_err(ctx, SFB200_ERR_CUDA, "shared memory limit: %s", cudaGetErrorString(e));
    cur = bytes;
    return 0;
}

static int set_err(sfb200_ctx* ctx, int code, const char* fmt, ...)
{
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        t_err = buf;
        t_err_ctx = ctx;
    }
    return code;
}

static int cuda_fail(sfb200_ctx* ctx, cudaError_t e, const char* what)
{
    return set_err(ctx, SFB200_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define CK(call)                                                       \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);       \
    } while (0)

extern "C" int sfb200_abi_version(void) { return SFB200_ABI_VERSION; }

// Tile-pair shards balanced by pairs. The tile pairs of n points in tiles of T are numbered row by
// row (ti <= tj); a diagonal tile pair holds s(s - 1) / 2 pairs and an off-diagonal one s_i s_j, with
// s = T except for the last, partial tile. Shard k of c starts at the first tile pair p whose
// preceding pairs reach k / c of all N(N - 1) / 2, so every shard is within one tile pair of an equal
// share (equal tile-pair counts would leave the shard holding the most diagonal tiles short).
static void shard_range(long long n, int T, long long index, long long count, long long* lo, long long* hi)
{
    const long long nt = (n + T - 1) / T;
    const unsigned __int128 total = (unsigned __int128)n * (unsigned __int128)(n > 0 ? n - 1 : 0) / 2;
    auto first_at = [&](long long k) -> long long {
        if (k <= 0) return 0;
        if (k >= count) return nt * (nt + 1) / 2;
        const unsigned __int128 target = (total * (unsigned __int128)k + (unsigned __int128)(count - 1)) /
                                         (unsigned __int128)count;  // ceil(total k / count)
        unsigned __int128 cum = 0;
        long long p = 0;
        for (long long ti = 0; ti < nt; ++ti) {
            const long long si = std::min<long long>(T, n - ti * T);
            const long long sl = n - (nt - 1) * T;  // the last tile's size
            const unsigned __int128 diag = (unsigned __int128)(si * (si - 1) / 2);
            const unsigned __int128 full = (unsigned __int128)si * (unsigned __int128)T;
            const long long noff = nt - 1 - ti;  // off-diagonal tile pairs of the row
            const unsigned __int128 row = diag + (noff > 0 ? full * (unsigned __int128)(noff - 1) + (unsigned __int128)si * sl : 0);
            if (cum + row < target) {
                cum += row;
                p += 1 + noff;
                continue;
            }
            if (cum >= target) return p;
            cum += diag;
            ++p;
            if (cum >= target) return p;
            // off-diagonal tile pairs of `full` pairs each (the row's last one may be partial)
            const unsigned __int128 need = target - cum;
            long long k2 = (long long)((need + full - 1) / full);
            if (k2 > noff) k2 = noff;
            return p + k2;
        }
        return p;
    };
    *lo = first_at(index);
    *hi = first_at(index + 1);
}

extern "C" int sfb200_shard_bounds(int64_t n, int32_t tile, int32_t index, int32_t count, int64_t* tp_lo,
                                   int64_t* tp_hi)
{
    if (n < 0 || tile < 1 || count < 1 || index < 0 || index >= count || !tp_lo || !tp_hi) return SFB200_ERR_INVALID_ARG;
    long long lo, hi;
    shard_range(n, tile, index, count, &lo, &hi);
    *tp_lo = lo;
    *tp_hi = hi;
    return SFB200_OK;
}

extern "C" const char* sfb200_last_error(const sfb200_ctx* ctx)
{
    if (!ctx) return "null context";
    return t_err_ctx == ctx ? t_err.c_str() : "";
}

// ------------------------------------------------------------------------------- context

extern "C" int sfb200_ctx_create(int device, sfb200_ctx** out)
{
    if (!out) return SFB200_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return SFB200_ERR_CUDA;
    if (device < 0 || device >= ndev) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = new (std::nothrow) sfb200_ctx();
    if (!ctx) return SFB200_ERR_OOM;
    ctx->device = device;
    if ((e = cudaSetDevice(device)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&ctx->ev0)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev1)) != cudaSuccess) {
        delete ctx;
        return SFB200_ERR_CUDA;
    }
    *out = ctx;
    return SFB200_OK;
}

extern "C" int sfb200_ctx_destroy(sfb200_ctx* ctx)
{
    if (!ctx) return SFB200_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->prep_stream) cudaStreamSynchronize(ctx->prep_stream);
    for (auto& b : ctx->rb) {
        if (b.done) cudaEventSynchronize(b.done);
        if (b.exec) cudaGraphExecDestroy(b.exec);
        if (b.done) cudaEventDestroy(b.done);
        if (b.h_items) cudaFreeHost(b.h_items);
        cudaFree(b.d_items);
        cudaFree(b.d_counters);
    }
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    for (int k = 0; k < sfb200_ctx::kLanes; ++k) {
        if (ctx->lane[k]) cudaStreamSynchronize(ctx->lane[k]);
        if (ctx->join[k]) cudaEventDestroy(ctx->join[k]);
        if (ctx->lane[k]) cudaStreamDestroy(ctx->lane[k]);
    }
    if (ctx->prep_stream) cudaStreamDestroy(ctx->prep_stream);
    if (ctx->side_stream) {
        cudaStreamSynchronize(ctx->side_stream);
        cudaStreamDestroy(ctx->side_stream);
    }
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SFB200_OK;
}

extern "C" void* sfb200_ctx_stream(sfb200_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

// ------------------------------------------------------------------------------- plan building

static int op_code(const sfb200_operator& o)
{
    switch (o.kind) {
    case SFB200_OP_PROJECTED:
        if (o.nl == 1 && o.nt == 0) return OC_L1;
        if (o.nl == 2 && o.nt == 0) return OC_L2;
        if (o.nl == 0 && o.nt == 2) return OC_T2;
        if (o.nl == 3 && o.nt == 0) return OC_L3;
        if (o.nl == 0 && o.nt == 3) return OC_T3;
        if (o.nl == 1 && o.nt == 2) return OC_L1T2;
        if (o.nl == 2 && o.nt == 1) return OC_L2T1;
        return OC_GEN;
    case SFB200_OP_S2: return OC_S2;
    case SFB200_OP_S3: return OC_S3;
    case SFB200_OP_FULLVEC: return o.nf == 2 ? OC_S2 : OC_GEN;
    case SFB200_OP_T2C: return OC_T2C;
    case SFB200_OP_L1T2C: return OC_L1T2C;
    }
    return OC_GEN;
}

static int op_order(const sfb200_operator& o)
{
    switch (o.kind) {
    case SFB200_OP_PROJECTED: return o.nl + o.nt;
    case SFB200_OP_S2: case SFB200_OP_T2C: return 2;
    case SFB200_OP_S3: case SFB200_OP_L1T2C: return 3;
    case SFB200_OP_FULLVEC: return o.nf;
    case SFB200_OP_SP2D: return o.nl < 3 ? 2 : 3;
    }
    return 1;
}

static double bits_to_double(unsigned long long b)
{
    double d;
    std::memcpy(&d, &b, 8);
    return d;
}

// Relative half-width of the mixed sphere kernel's ambiguity band around an edge's chord key:
// far above the FP64 error of the chord and of the edge images (~1e-15), far below a cell.
static const double kChordWrel = 0x1p-40;

// Cell geometry over FP64 keys for the exact table. With wrel > 0, a cell is also marked SLOW when
// the band [e (1 - wrel), e (1 + wrel)] of one of its edges reaches into a neighbouring cell, so the
// kernel's in-cell band test (|key - e| <= wrel e) sees every key of the band.
static void build_lut64(const std::vector<double>& tab, LutGeom& g, std::vector<LutEntry64>& out, double wrel = 0.0)
{
    double mn = INFINITY, mx = 0.0;
    for (double v : tab) {
        if (v > 0.0 && std::isfinite(v)) { mn = std::min(mn, v); mx = std::max(mx, v); }
    }
    int e_lo = 0, e_hi = 0;
    if (mx > 0.0) {
        e_lo = std::max(std::ilogb(mn) - 1, -1022);
        e_hi = std::min(std::ilogb(mx) + 1, 1023);
    }
    int m = 3;
    for (;; ++m) {
        const long long nc = (long long)(e_hi - e_lo + 1) << m;
        const int shift = 52 - m;
        const long long base = (long long)(e_lo + 1023) << m;
        bool multi = false;
        // a cell with two distinct edge values needs a finer m
        for (size_t k = 1; k < tab.size() && !multi; ++k) {
            if (!(tab[k] > 0.0) || !std::isfinite(tab[k]) || tab[k] == tab[k - 1] || !(tab[k - 1] > 0.0)) continue;
            unsigned long long ba, bb;
            std::memcpy(&ba, &tab[k - 1], 8);
            std::memcpy(&bb, &tab[k], 8);
            long long ca = std::min(std::max((long long)(ba >> shift) - base, 0ll), nc - 1);
            long long cb = std::min(std::max((long long)(bb >> shift) - base, 0ll), nc - 1);
            if (ca == cb) multi = true;
        }
        if (!multi || m >= 10 || ((long long)(e_hi - e_lo + 1) << (m + 1)) > 4096) break;
    }
    g.shift = 52 - m;
    g.ncell = (e_hi - e_lo + 1) << m;
    g.base = (long long)(e_lo + 1023) << m;
    out.assign(g.ncell, LutEntry64{});
    for (int c = 0; c < g.ncell; ++c) {
        const double klo = (c == 0) ? 0.0 : bits_to_double((unsigned long long)(g.base + c) << g.shift);
        const double khi = (c == g.ncell - 1) ? INFINITY : bits_to_double((unsigned long long)(g.base + c + 1) << g.shift);
        int below = 0, cnt = 0, distinct = 0;
        double val = NAN;
        for (double v : tab) {
            if (v < klo) { ++below; continue; }
            const bool inside = (c == g.ncell - 1) ? (v >= klo) : (v >= klo && v < khi);
            if (inside) {
                if (cnt == 0 || v != val) ++distinct;
                val = v;
                ++cnt;
            }
        }
        LutEntry64 e;
        e.base = below;
        e.mult = cnt;
        e.e = cnt ? val : NAN;
        if (distinct > 1) e.mult = LUT_FLAG_SLOW;
        out[c] = e;
    }
    if (wrel > 0.0) {
        auto cell_of = [&](double key) -> long long {
            unsigned long long b;
            std::memcpy(&b, &key, 8);
            b &= 0x7fffffffffffffffull;
            long long c = (long long)(b >> g.shift) - g.base;
            return std::min(std::max(c, 0ll), (long long)g.ncell - 1);
        };
        for (double v : tab) {
            if (!(v > 0.0) || !std::isfinite(v)) continue;
            const long long c0 = cell_of(v * (1.0 - 2.0 * wrel)), c1 = cell_of(v * (1.0 + 2.0 * wrel));
            if (c0 != c1)
                for (long long c = c0; c <= c1; ++c) out[c].mult = LUT_FLAG_SLOW;
        }
    }
}

// Byte table of the flat FP64 / mixed 1D kernels over the squared-edge table `tab` (sorted): cell c
// covers the keys whose high word, sign bit cleared, shifted right by 18 equals c, i.e. [lo_c, hi_c)
// with lo_c = bits(c << 50). The cell's byte is the number of edges strictly below lo_c when the
// cell holds at most one distinct edge, no repeated edge and only keys the FP32 arithmetic takes
// (within [2^-100, 2^100]); otherwise kByteSlow. `out` receives the bytes followed by the edges padded
// with +inf to kByteEdges doubles. Returns false when the table cannot hold the edges (> 254).
static bool build_byte_table(const std::vector<double>& tab, std::vector<unsigned char>& out)
{
    const int ne = (int)tab.size();
    if (ne > kByteEdges - 2) return false;
    out.assign((size_t)kByteCells + sizeof(double) * kByteEdges, 0);
    double* sqx = reinterpret_cast<double*>(out.data() + kByteCells);
    for (int k = 0; k < kByteEdges; ++k) sqx[k] = k < ne ? tab[k] : INFINITY;
    for (int c = 0; c < kByteCells; ++c) {
        const double lo = bits_to_double((unsigned long long)c << 50);
        const double hi = bits_to_double((unsigned long long)(c + 1) << 50);  // NaN/inf for the top cells
        int below = 0, inside = 0;
        bool repeat = false;
        for (int k = 0; k < ne; ++k) {
            if (tab[k] < lo) ++below;
            else if (tab[k] < hi || !(hi == hi)) {
                ++inside;
                if (k > 0 && tab[k] == tab[k - 1]) repeat = true;
            }
        }
        const bool fp32_ok = lo >= 0x1p-100 && hi <= 0x1p100;
        out[c] = (inside > 1 || repeat || !fp32_ok) ? (unsigned char)kByteSlow : (unsigned char)below;
    }
    return true;
}

// Cell geometry over FP32 keys for the window table; fails if the edge keys leave FP32's range.
static bool geom_lut32(const std::vector<double>& keys, LutGeom& g)
{
    double mn = INFINITY, mx = 0.0;
    for (double v : keys) {
        if (v > 0.0 && std::isfinite(v)) { mn = std::min(mn, v); mx = std::max(mx, v); }
    }
    int e_lo = 0, e_hi = 0;
    if (mx > 0.0) {
        e_lo = std::ilogb(mn) - 2;
        e_hi = std::ilogb(mx) + 1;
        if (e_lo < -100 || e_hi > 100) return false;
    }
    int m = 3;
    for (;; ++m) {
        const long long nc = (long long)(e_hi - e_lo + 1) << m;
        const int shift = 23 - m;
        const long long base = (long long)(e_lo + 127) << m;
        bool multi = false;
        for (size_t k = 1; k < keys.size() && !multi; ++k) {
            if (!(keys[k] > 0.0) || keys[k] == keys[k - 1] || !(keys[k - 1] > 0.0)) continue;
            const float fa = (float)keys[k - 1], fb = (float)keys[k];
            unsigned ba, bb;
            std::memcpy(&ba, &fa, 4);
            std::memcpy(&bb, &fb, 4);
            long long ca = std::min(std::max((long long)(ba >> shift) - base, 0ll), nc - 1);
            long long cb = std::min(std::max((long long)(bb >> shift) - base, 0ll), nc - 1);
            if (ca == cb) multi = true;
        }
        if (!multi || m >= 10 || ((long long)(e_hi - e_lo + 1) << (m + 1)) > 2048) break;
    }
    g.shift = 23 - m;
    g.ncell = (e_hi - e_lo + 1) << m;
    g.base = (long long)(e_lo + 127) << m;
    return true;
}

static double chord2_of(double r, double radius)
{
    if (r < 0.0 || (r == 0.0 && std::signbit(r))) return -1.0;
    if (r == 0.0) return 0.0;
    const double half = r / (2.0 * radius);
    if (half >= 0.5 * M_PI) return 5.0;
    const double s = 2.0 * std::sin(half);
    return s * s;
}

static int validate_bins(sfb200_ctx* ctx, const sfb200_bins& b, const char* what, bool allow_sq)
{
    if (b.n_edges < 2) return set_err(ctx, SFB200_ERR_INVALID_ARG, "%s: need at least 2 edges", what);
    if (b.n_edges > 65536) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "%s: more than 65536 edges", what);
    if (b.kind == SFB200_BINS_LINEAR) {
        if (!(std::isfinite(b.first) && std::isfinite(b.last) && std::isfinite(b.inv_step) &&
              std::isfinite(b.step) && b.step > 0.0 && b.last > b.first))
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "%s: LinearBinEdges needs finite first < last and step > 0", what);
        return SFB200_OK;
    }
    if (b.kind == SFB200_BINS_SQTABLE && !allow_sq)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "%s: a squared-edge table is only meaningful for Euclidean distances", what);
    if (b.kind != SFB200_BINS_TABLE && b.kind != SFB200_BINS_SQTABLE)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "%s: unknown bin kind %d", what, b.kind);
    if (!b.edges) return set_err(ctx, SFB200_ERR_INVALID_ARG, "%s: edges pointer is NULL", what);
    for (int k = 0; k < b.n_edges; ++k) {
        if (std::isnan(b.edges[k])) return set_err(ctx, SFB200_ERR_INVALID_ARG, "%s: NaN edge", what);
        if (k && b.edges[k] < b.edges[k - 1])
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "%s: edges must be sorted (non-decreasing)", what);
    }
    return SFB200_OK;
}

static LinearParams linear_of(const sfb200_bins& b)
{
    LinearParams p;
    p.first = b.first;
    p.last = b.last;
    p.inv_step = b.inv_step;
    p.step = b.step;
    p.neg_f_inv = -b.first * b.inv_step;
    p.n = b.n_edges;
    return p;
}

// Frees the input / layout buffers of a workspace (its histogram buffers with `outputs`).
// Releases the buffers of w (with `outputs`, the histogram too). A pooled slice block is freed in
// order on stream s, after the work already enqueued there.
static void free_workspace(Workspace& w, bool outputs, cudaStream_t s = nullptr)
{
    if (w.block) {
        cudaFreeAsync(w.block, s);
        w = Workspace{};
        return;
    }
    cudaFree(w.d_rawx); cudaFree(w.d_rawu);
    cudaFree(w.d_X64); cudaFree(w.d_U64); cudaFree(w.d_XF); cudaFree(w.d_UF); cudaFree(w.d_XM);
    cudaFree(w.d_keys); cudaFree(w.d_perm); cudaFree(w.d_box); cudaFree(w.d_sort_tmp);
    w.d_rawx = w.d_rawu = nullptr;
    w.d_X64 = w.d_U64 = nullptr;
    w.d_XF = w.d_UF = nullptr;
    w.d_XM = nullptr;
    w.d_keys = nullptr;
    w.d_perm = nullptr;
    w.d_box = nullptr;
    w.d_sort_tmp = nullptr;
    w.sort_tmp_bytes = 0;
    w.cap = 0;
    if (outputs) {
        cudaFree(w.d_sums); cudaFree(w.d_counts); cudaFree(w.d_aux);
        w.d_sums = nullptr;
        w.d_counts = nullptr;
        w.d_aux = nullptr;
    }
}

static void free_plan_device(sfb200_plan* p)
{
    free_workspace(p->ws, true);
    cudaFree(p->d_exact); cudaFree(p->d_vedges); cudaFree(p->d_lut64); cudaFree(p->d_ck);
    cudaFree(p->d_lut32); cudaFree(p->d_rowlo); cudaFree(p->d_vwin); cudaFree(p->d_lut8); cudaFree(p->d_range);
    cudaFree(p->d_lutc);
}

extern "C" int sfb200_plan_destroy(sfb200_plan* p)
{
    if (!p) return SFB200_ERR_INVALID_ARG;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    free_plan_device(p);
    delete p;
    return SFB200_OK;
}

template <typename T>
static cudaError_t upload(T** dst, const T* src, size_t count)
{
    cudaError_t e = cudaMalloc((void**)dst, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    if (count) e = cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

static int plan_build(sfb200_ctx* ctx, sfb200_plan* p)
{
    const sfb200_plan_desc& d = p->desc;
    if (d.geometry != SFB200_GEOM_FLAT && d.geometry != SFB200_GEOM_SPHERE)
        return set_err(ctx, SFB200_ERR_UNSUPPORTED, "unknown geometry %d", d.geometry);
    if (d.dim != 2 && d.dim != 3)
        return set_err(ctx, SFB200_ERR_DIMENSION, "expected spatial/velocity dimension D=2 or D=3 on axis 1; got D=%d", d.dim);
    p->sphere = d.geometry == SFB200_GEOM_SPHERE;
    p->D = d.dim;
    p->W = p->sphere ? 2 : d.dim;
    if (p->sphere) {
        if (d.angle_unit != SFB200_ANGLE_DEG && d.angle_unit != SFB200_ANGLE_RAD)
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "unknown angle unit %d", d.angle_unit);
        if (!(std::isfinite(d.radius) && d.radius > 0.0))
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "sphere radius must be finite and positive");
    }
    if (d.precision != SFB200_PREC_FP64 && d.precision != SFB200_PREC_MIXED && d.precision != SFB200_PREC_FP32)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "unknown precision %d", d.precision);
    if ((d.x_dtype != SFB200_F64 && d.x_dtype != SFB200_F32) || (d.u_dtype != SFB200_F64 && d.u_dtype != SFB200_F32))
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "x_dtype/u_dtype must be F64 or F32");
    p->fp32 = d.precision == SFB200_PREC_FP32;
    p->mixed = d.precision == SFB200_PREC_MIXED;
    p->joint = d.joint != 0;
    p->df = p->fp32 && (p->sphere || d.x_dtype == SFB200_F64 || d.u_dtype == SFB200_F64);
    if (d.n_ops < 1 || d.n_ops > SFB200_MAX_OPS)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "n_ops must be in 1..%d", SFB200_MAX_OPS);
    // consecutive rows of the flat two-dimensional single pass share one joint plan (one launch)
    bool rows = p->joint && !p->sphere && d.n_ops >= 2 && d.n_ops <= 6 && d.ops[0].nl >= 0 &&
                d.ops[0].nl + d.n_ops <= 6;
    for (int k = 0; rows && k < d.n_ops; ++k)
        rows = d.ops[k].kind == SFB200_OP_SP2D && d.ops[k].nl == d.ops[0].nl + k;
    if (p->joint && d.n_ops != 1 && !rows)
        return set_err(ctx, SFB200_ERR_INVALID_ARG,
                       "a joint histogram takes exactly one operator (or consecutive flat single-pass 2D rows)");
    p->sp2d_rows = rows ? d.n_ops : 0;
    for (int k = 0; k < d.n_ops; ++k) {
        const sfb200_operator& o = d.ops[k];
        if (o.kind < SFB200_OP_PROJECTED || o.kind > SFB200_OP_SP2D)
            return set_err(ctx, SFB200_ERR_UNSUPPORTED, "unknown operator kind %d", o.kind);
        if (o.kind == SFB200_OP_SP2D && o.nl > 5)
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "single-pass row must be in 0..5");
        if (o.nl < 0 || o.nt < 0 || o.nf < 0 || o.nl > 16 || o.nt > 16 || o.nf > 16)
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "operator powers must be in 0..16");
    }
    // Flat rows of the two-dimensional single pass requested at precision MIXED (and plans of several
    // rows at any precision) run the FP64 joint kernels, whose results meet those tolerances too. Their cubic rows put many values within 2^-8
    // of a half bin width of zero, which the mixed kernel recomputes pair by pair in FP64, and their
    // small tables let the FP64 kernel run several blocks per SM. Measured on B200 (20000 points,
    // 50 x 50 bins, six rows): 22.9 ms mixed (one row 1.8 ms, the cubic rows 4.0-5.2 ms) against
    // 10.0 ms in FP64 (1.6-1.7 ms per row).
    p->promoted = p->joint && !p->sphere && d.ops[0].kind == SFB200_OP_SP2D && (p->mixed || (p->fp32 && p->sp2d_rows));
    if (p->promoted) p->mixed = p->fp32 = p->df = false;
    int rc = validate_bins(ctx, d.distance, "distance_bins", !p->sphere);
    if (rc) return rc;
    if (p->joint && (rc = validate_bins(ctx, d.value, "value_bins", false))) return rc;

    p->nb = d.distance.n_edges - 1;
    p->nv = p->joint ? d.value.n_edges - 1 : 0;
    p->nops = d.n_ops;
    if (p->joint && (long long)p->nb * p->nv > (1ll << 24))
        return set_err(ctx, SFB200_ERR_UNSUPPORTED, "joint histogram larger than 2^24 cells");
    if (!p->joint && p->nb > 4096)
        return set_err(ctx, SFB200_ERR_UNSUPPORTED, "more than 4096 distance bins");

    // operator list -> kernel
    int codes[SFB200_MAX_OPS];
    for (int k = 0; k < d.n_ops; ++k) codes[k] = op_code(d.ops[k]);
    p->opl = -1;
    if (d.n_ops == 1 && codes[0] == OC_L2) p->opl = OPL_L2;
    else if (d.n_ops == 1 && codes[0] == OC_L3) p->opl = OPL_L3;
    else if (d.n_ops == 1 && codes[0] == OC_L1) p->opl = OPL_L1;
    else if (d.n_ops == 4 && codes[0] == OC_L2 && codes[1] == OC_T2 && codes[2] == OC_L3 && codes[3] == OC_T3)
        p->opl = OPL_QUAD;
    else if (d.n_ops == 4 && codes[0] == OC_S2 && codes[1] == OC_L2 && codes[2] == OC_S3 && codes[3] == OC_L3)
        p->opl = OPL_SP;
    p->nops_pad = d.n_ops;
    if (p->opl < 0) {
        if (d.n_ops == 1) p->opl = OPL_GEN1;
        else if (d.n_ops == 2) p->opl = OPL_GEN2;
        else if (d.n_ops <= 4) { p->opl = OPL_GEN4; p->nops_pad = 4; }
        else { p->opl = OPL_GEN8; p->nops_pad = 8; }
    }
    for (int k = 0; k < SFB200_MAX_OPS; ++k) {
        if (k < d.n_ops) p->gen.op[k] = d.ops[k];
        else p->gen.op[k] = sfb200_operator{SFB200_OP_PROJECTED, 0, 0, 0};
    }
    p->vorder = op_order(d.ops[0]);
    p->l_only = d.ops[0].kind == SFB200_OP_PROJECTED && d.ops[0].nt == 0;

    // distance tables
    const sfb200_bins& db = d.distance;
    const bool dlinear = db.kind == SFB200_BINS_LINEAR;
    if (dlinear) p->dlin = linear_of(db);
    if (!dlinear) {
        p->exact_tab.resize(db.n_edges);
        for (int k = 0; k < db.n_edges; ++k) {
            const double e = db.edges[k];
            if (p->sphere) p->exact_tab[k] = (e == 0.0 && std::signbit(e)) ? -4.9406564584124654e-324 : e;
            else p->exact_tab[k] = (db.kind == SFB200_BINS_SQTABLE) ? e : e * e;
        }
        for (int k = 1; k < db.n_edges; ++k)
            if (p->exact_tab[k] < p->exact_tab[k - 1])
                return set_err(ctx, SFB200_ERR_INVALID_ARG,
                               "distance_bins: Euclidean edges must be non-negative (their squares must stay sorted)");
    }
    // edge keys of the FP32 path (and the chord keys of the mixed and FP64 chord sphere paths)
    if (p->fp32 || (p->mixed && p->sphere) || p->fp64_sphere_1d()) {
        p->ck.resize(db.n_edges);
        for (int k = 0; k < db.n_edges; ++k) {
            double r = dlinear ? std::fma((double)k, db.step, db.first) : db.edges[k];
            if (p->sphere) {
                p->ck[k] = chord2_of(r, d.radius);
            } else if (dlinear) {
                p->ck[k] = r < 0.0 ? -1.0 : r * r;
            } else {
                p->ck[k] = p->exact_tab[k];
            }
        }
        if (p->fp32 && !geom_lut32(p->ck, p->lg32))
            return set_err(ctx, SFB200_ERR_UNSUPPORTED,
                           "distance edges outside the FP32 range of the fp32 kernel; use precision=mixed or fp64");
        const double u32 = 0x1p-24, u64 = 0x1p-53;
        if (p->sphere) {
            // (hi, lo) records: the chord carries ~2u per component plus the FMA chain; the FP64
            // arc length differs from the chord image of the edges by ~1e-15 relative.
            p->wp.A = 9.0 * u32 * 1.1 + 1e-14;
            p->wp.Bm = 4.0 * std::sqrt(3.0) * u32 * u32 * 1.1;
            p->wp.Cm = 0.0;
            p->wp.use_bound = 0;
            p->wp.short_rel = 0.0;
            p->wp.short_key = 0x1p-40;                 // (near-)coincident: frame degenerate
            p->wp.anti_key = 4.0 - 0x1p-40;            // (near-)antipodal: frame degenerate
        } else {
            // FP32 inputs are exact floats: differences carry u. FP64 inputs come as (hi, lo)
            // pairs: differences carry 2u plus the u^2 |x| residual of the split.
            p->wp.A = (p->D + (p->df ? 5 : 3)) * u32 * 1.1 + 8.0 * p->D * u64 + (dlinear ? 1e-14 : 0.0);
            p->wp.Bm = p->df ? 4.0 * std::sqrt((double)p->D) * u32 * u32 * 1.1 : 0.0;
            p->wp.Cm = 0.0;
            p->wp.use_bound = 1;
            p->wp.short_rel = p->df ? 0x1p-20 : 0.0;
            p->wp.short_key = 0.0;
            p->wp.anti_key = INFINITY;
        }
    }
    if (p->joint) {
        if (d.value.kind == SFB200_BINS_LINEAR) p->vlin = linear_of(d.value);
        else p->vedges.assign(d.value.edges, d.value.edges + d.value.n_edges);
    }
    if (p->joint && (p->fp32 || p->mixed)) {
        // fixed-point scale of the value offsets from the bin centres: 2^k with (half width) 2^k < 2^30
        double hw = 0.0;
        if (d.value.kind == SFB200_BINS_LINEAR) {
            hw = 0.5 * d.value.step;
        } else {
            for (size_t k = 0; k < p->vedges.size(); ++k)
                if (!std::isfinite(p->vedges[k]))
                    return set_err(ctx, SFB200_ERR_UNSUPPORTED,
                                   "value_bins: infinite edges need precision=fp64 for a joint histogram");
            for (size_t k = 0; k + 1 < p->vedges.size(); ++k) hw = std::max(hw, 0.5 * (p->vedges[k + 1] - p->vedges[k]));
        }
        int ex = 0;
        if (hw > 0.0 && std::isfinite(hw)) std::frexp(hw, &ex);  // hw < 2^ex
        p->vq = std::ldexp(1.0, 30 - ex);
        p->vq_inv = std::ldexp(1.0, ex - 30);
        p->vqc = std::ldexp(1.0, 22 - ex);
        p->vqc_inv = std::ldexp(1.0, ex - 22);
        // value bins whose values come closer to zero than the half width keep exact offsets
        p->vfine_lo = 1;
        p->nfine = 0;
        int lo = 0, hi = -1;
        for (int k = 1; k <= p->nv; ++k) {
            double a0, a1;
            if (d.value.kind == SFB200_BINS_LINEAR) {
                a0 = std::fma((double)(k - 1), d.value.step, d.value.first);
                a1 = std::fma((double)k, d.value.step, d.value.first);
            } else {
                a0 = p->vedges[k - 1];
                a1 = p->vedges[k];
            }
            const double mn = (a0 < 0.0 && a1 > 0.0) ? 0.0 : std::min(std::fabs(a0), std::fabs(a1));
            if (mn < 2.0 * hw) {
                if (hi < 0) lo = k;
                hi = k;
            }
        }
        if (hi >= lo && hi > 0) {
            p->vfine_lo = lo;
            p->nfine = hi - lo + 1;
        }
    }

    // device allocations
    cudaError_t e;
    if (!p->exact_tab.empty() && (e = upload(&p->d_exact, p->exact_tab.data(), p->exact_tab.size())) != cudaSuccess)
        return cuda_fail(ctx, e, "upload distance table");
    if (p->mixed && p->sphere) {
        std::vector<LutEntry64> lut;
        build_lut64(p->ck, p->lg64, lut, kChordWrel);
        p->lut64_bytes = (int)(lut.size() * sizeof(LutEntry64));
        if ((e = upload(&p->d_lut64, lut.data(), lut.size())) != cudaSuccess) return cuda_fail(ctx, e, "upload table");
    } else if (!dlinear && !p->fp32) {
        std::vector<LutEntry64> lut;
        build_lut64(p->exact_tab, p->lg64, lut);
        p->lut64_bytes = (int)(lut.size() * sizeof(LutEntry64));
        if ((e = upload(&p->d_lut64, lut.data(), lut.size())) != cudaSuccess) return cuda_fail(ctx, e, "upload table");
    }
    if (!p->sphere && !dlinear && !p->fp32 && (!p->joint || p->mixed)) {
        std::vector<unsigned char> bt;
        if (build_byte_table(p->exact_tab, bt) && (e = upload(&p->d_lut8, bt.data(), bt.size())) != cudaSuccess)
            return cuda_fail(ctx, e, "upload byte table");
    }
    if (p->fp64_sphere_1d()) {  // the chord kernel's table (the r-edge table above stays for the other)
        std::vector<LutEntry64> lut;
        build_lut64(p->ck, p->lgc, lut, kChordWrel);
        p->lutc_bytes = (int)(lut.size() * sizeof(LutEntry64));
        if ((e = upload(&p->d_lutc, lut.data(), lut.size())) != cudaSuccess) return cuda_fail(ctx, e, "upload table");
    }
    if (p->fp32) {
        if ((e = upload(&p->d_ck, p->ck.data(), p->ck.size())) != cudaSuccess) return cuda_fail(ctx, e, "upload keys");
        if ((e = cudaMalloc(&p->d_lut32, sizeof(LutEntry32) * p->lg32.ncell)) != cudaSuccess)
            return cuda_fail(ctx, e, "alloc table");
    }
    if (!p->vedges.empty() && (e = upload(&p->d_vedges, p->vedges.data(), p->vedges.size())) != cudaSuccess)
        return cuda_fail(ctx, e, "upload value edges");
    if (p->joint && p->fp32) {
        std::vector<double> rowlo(p->nb + 2, 0.0);
        for (int b = 1; b <= p->nb; ++b) rowlo[b] = std::max(p->ck[b - 1], 0.0);
        if ((e = upload(&p->d_rowlo, rowlo.data(), rowlo.size())) != cudaSuccess) return cuda_fail(ctx, e, "upload rows");
        if ((e = cudaMalloc(&p->d_vwin, sizeof(float) * (p->nb + 2))) != cudaSuccess) return cuda_fail(ctx, e, "alloc windows");
    }
    const long long jrows = std::max(1, p->sp2d_rows);  // joint matrices (single-pass rows)
    p->n_sums = p->joint ? (long long)p->nb * p->nv * jrows : (long long)p->nb * p->nops;
    p->n_counts = p->joint ? (long long)p->nb * p->nv * jrows : (long long)p->nb;
    if ((e = cudaMalloc(&p->ws.d_sums, sizeof(double) * p->n_sums)) != cudaSuccess) return cuda_fail(ctx, e, "alloc sums");
    if ((e = cudaMalloc(&p->ws.d_counts, sizeof(unsigned long long) * p->n_counts)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc counts");
    if ((e = cudaMalloc(&p->ws.d_aux, sizeof(unsigned long long) * 4)) != cudaSuccess) return cuda_fail(ctx, e, "alloc aux");
    p->h_sums.resize(p->n_sums);
    p->h_counts.resize(p->n_counts);

    // the kernel exists for this combination
    KernelChoice kc;
    if (p->mixed)
        kc = p->joint ? pick_joint_mx(p->sphere, p->D, p->opl)
                      : (p->sphere ? pick_sphere1d_mx(p->D, p->opl, 0) : pick_flat1d_mx(p->D, p->opl, 0));
    else
        kc = p->joint ? (p->sp2d_rows ? pick_sp2d(p->D, true, 2) : pick_joint(p->sphere, p->D, p->fp32, true, p->df, p->opl))
                      : (p->sphere ? pick_sphere1d(p->D, p->fp32, p->opl, 0)
                                   : pick_flat1d(p->D, p->fp32, p->df, p->opl, 0));
    if (!kc.fn) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "no kernel for this operator on the joint mixed path");
    return SFB200_OK;
}

extern "C" int sfb200_plan_create(sfb200_ctx* ctx, const sfb200_plan_desc* desc, sfb200_plan** out)
{
    if (!ctx || !desc || !out) return set_err(ctx, SFB200_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    sfb200_plan* p = new (std::nothrow) sfb200_plan();
    if (!p) return set_err(ctx, SFB200_ERR_OOM, "out of host memory");
    p->ctx = ctx;
    p->desc = *desc;
    const int rc = plan_build(ctx, p);
    if (rc != SFB200_OK) {
        free_plan_device(p);
        delete p;
        return rc;
    }
    p->desc.distance.edges = nullptr;  // tables were copied
    p->desc.value.edges = nullptr;
    *out = p;
    return SFB200_OK;
}

extern "C" int sfb200_plan_output_sizes(const sfb200_plan* p, int64_t* n_sums, int64_t* n_counts)
{
    if (!p) return SFB200_ERR_INVALID_ARG;
    if (n_sums) *n_sums = p->n_sums;
    if (n_counts) *n_counts = p->n_counts;
    return SFB200_OK;
}

extern "C" int sfb200_plan_set_launch(sfb200_plan* p, int tile, int privatization, int blocks_per_sm)
{
    if (!p) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = p->ctx;
    if (tile != 0 && tile != 32 && tile != 64 && tile != 128 && tile != 256 && tile != 512 && tile != 768)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "tile must be 0, 32, 64, 128, 256, 512 or 768");
    if (tile > 512 && !(p->joint && p->mixed))
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "tiles of 768 points exist for the mixed joint kernel only");
    if (privatization != -1 && privatization != 0 && privatization != 1 && privatization != 2 &&
        privatization != 3 && privatization != 4 && privatization != 6 && privatization != 8 &&
        privatization != 32)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "privatization must be -1 (auto), 0, 1, 2, 3, 4, 6, 8 or 32");
    if (blocks_per_sm < 0 || blocks_per_sm > 32)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "blocks_per_sm must be in 0..32");
    p->tile_ovr = tile;
    p->priv_ovr = privatization;
    p->bps_ovr = blocks_per_sm;
    return SFB200_OK;
}

extern "C" int sfb200_plan_set_option(sfb200_plan* p, int option, int64_t value)
{
    if (!p) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = p->ctx;
    switch (option) {
    case SFB200_OPT_POINT_ORDER:
        if (value < -1 || value > 2) return set_err(ctx, SFB200_ERR_INVALID_ARG, "point order must be -1, 0, 1 or 2");
        p->order_ovr = (int)value;
        return SFB200_OK;
    case SFB200_OPT_SHARD:
        if (value < 0 || (value & 0xffffffffll) >= (value >> 32) || (value >> 32) > 65536)
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "shard: index (low 32 bits) must be below the count (high 32 bits)");
        p->shard_index = (int)(value & 0xffffffffll);
        p->shard_count = (int)(value >> 32);
        return SFB200_OK;
    case SFB200_OPT_FORMULATION:
        if (value != -1 && value != 1 && value != 2)
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "formulation must be -1 (auto), 1 (reference) or 2 (chord)");
        p->form_ovr = (int)value;
        return SFB200_OK;
    case SFB200_OPT_TILE_SORT:
        if (value < -1 || value > 1) return set_err(ctx, SFB200_ERR_INVALID_ARG, "tile sort must be -1, 0 or 1");
        p->sort_ovr = (int)value;
        return SFB200_OK;
    case SFB200_OPT_HIST_COLUMNS:
        if (value < 0 || value > 32 || (value & (value - 1)))
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "histogram columns must be 0 (auto) or a power of two <= 32");
        p->cols_ovr = (int)value;
        return SFB200_OK;
    }
    return set_err(ctx, SFB200_ERR_INVALID_ARG, "unknown plan option %d", option);
}

// ------------------------------------------------------------------------------- run

// Grows the input / layout buffers of `w` to n points (its histogram buffers are sized by the plan).
// The buffers of a workspace over `cap` points (and, with `outputs`, the histogram), in order,
// through alloc(&ptr, bytes). Shared by the per-buffer allocation of plans and the one pooled block
// of a slice.
template <class Alloc>
static int workspace_layout(sfb200_plan* p, Workspace& w, long long cap, bool outputs, Alloc&& alloc)
{
    sfb200_ctx* ctx = p->ctx;
    const int nx64 = p->sphere ? 8 : p->D;
    const int nxf = p->sphere ? (p->D == 3 ? 20 : 18) : (p->df ? 2 * p->D : p->D);
    CK(alloc(&w.d_rawx, sizeof(double) * p->W * cap));
    CK(alloc(&w.d_rawu, sizeof(double) * p->D * cap));
    CK(alloc((void**)&w.d_X64, sizeof(double) * nx64 * cap));
    CK(alloc((void**)&w.d_U64, sizeof(double) * p->D * cap));
    if (p->fp32) {
        CK(alloc((void**)&w.d_XF, sizeof(float) * nxf * cap));
        if (!p->sphere) CK(alloc((void**)&w.d_UF, sizeof(float) * (p->df ? 2 : 1) * p->D * cap));
    }
    if ((p->mixed && p->sphere) || p->fp64_sphere_1d()) CK(alloc((void**)&w.d_XM, sizeof(double) * 10 * cap));
    CK(alloc((void**)&w.d_keys, sizeof(unsigned) * 2 * cap));
    CK(alloc((void**)&w.d_perm, sizeof(int) * 2 * cap));
    CK(alloc((void**)&w.d_box, sizeof(unsigned) * 6));
    size_t tmp = 0;  // size query only: launches nothing
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, w.d_keys, w.d_keys + cap, w.d_perm, w.d_perm + cap,
                                       (int)cap, 0, 32, ctx->stream));
    CK(alloc(&w.d_sort_tmp, std::max<size_t>(tmp, 16)));
    w.sort_tmp_bytes = tmp;
    if (outputs) {
        CK(alloc((void**)&w.d_sums, sizeof(double) * std::max<long long>(p->n_sums, 1)));
        CK(alloc((void**)&w.d_counts, sizeof(unsigned long long) * std::max<long long>(p->n_counts, 1)));
        CK(alloc((void**)&w.d_aux, sizeof(unsigned long long) * 4));
    }
    return SFB200_OK;
}

// Grows the buffers of `w` (a plan's) to at least n points (contents are not kept).
static int ensure_workspace(sfb200_plan* p, Workspace& w, long long n)
{
    sfb200_ctx* ctx = p->ctx;
    if (n <= w.cap) return SFB200_OK;
    if (w.cap) CK(cudaStreamSynchronize(ctx->stream));  // old buffers may still be in use
    free_workspace(w, false);
    const long long cap = std::max<long long>(n, 1024);
    size_t bytes = 0;
    const int rc = workspace_layout(p, w, cap, false, [&](void** ptr, size_t b) {
        bytes += b;
        return cudaMalloc(ptr, b);
    });
    if (rc) return rc;
    w.cap = cap;
    w.bytes = bytes + (size_t)(p->n_sums + p->n_counts + 4) * 8;
    return SFB200_OK;
}

// All buffers of a slice over n points as one block from the context's pool, allocated in order on
// stream s (it may be used by work enqueued on s, or on streams that wait for s, from here on).
static int slice_workspace(sfb200_plan* p, Workspace& w, long long n, cudaStream_t s)
{
    sfb200_ctx* ctx = p->ctx;
    if (!ctx->pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        CK(cudaMemPoolCreate(&ctx->pool, &props));
        unsigned long long keep = ~0ull;  // keep freed blocks for the next slices
        CK(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    const long long cap = std::max<long long>(n, 2);
    // first pass: offsets from 0 (256-byte aligned); second pass: the same offsets in the block
    size_t off = 0;
    Workspace probe;
    int rc = workspace_layout(p, probe, cap, true, [&](void** ptr, size_t b) {
        *ptr = reinterpret_cast<void*>(off + 256);  // non-null stand-in, never dereferenced
        off += (b + 255) & ~(size_t)255;
        return cudaSuccess;
    });
    if (rc) return rc;
    CK(cudaMallocFromPoolAsync(&w.block, off, ctx->pool, s));
    off = 0;
    rc = workspace_layout(p, w, cap, true, [&](void** ptr, size_t b) {
        *ptr = static_cast<char*>(w.block) + off;
        off += (b + 255) & ~(size_t)255;
        return cudaSuccess;
    });
    if (rc) return rc;
    w.cap = cap;
    w.bytes = off;
    return SFB200_OK;
}

template <typename TX, typename TU>
static void launch_pack(sfb200_plan* p, Workspace& w, const void* x, const void* u, int n, const int* perm,
                        cudaStream_t s)
{
    const int tb = 256, nblk = (n + tb - 1) / tb;
    if (p->sphere)
        k_pack_sphere<TX, TU><<<nblk, tb, 0, s>>>((const TX*)x, (const TU*)u, n, p->D, p->desc.angle_unit, perm,
                                                  w.d_X64, w.d_U64, p->fp32 ? w.d_XF : nullptr,
                                                  w.d_XM, w.d_aux + 1);
    else
        k_pack_flat<TX, TU><<<nblk, tb, 0, s>>>((const TX*)x, (const TU*)u, n, p->D, p->df, perm, w.d_X64,
                                                w.d_U64, p->fp32 ? w.d_XF : nullptr,
                                                p->fp32 ? w.d_UF : nullptr, w.d_aux + 1);
}

// Points below this count keep the caller's order: the sort costs more than the runs it lengthens.
static const long long kOrderMinPoints = 16384;

// Storage order of a run of n points: 0 the caller's, 1 Morton, 2 scattered. The joint sphere path
// keeps the caller's order: its FP64 value binning uses the reference's pair frame, whose rounding
// is not symmetric in the two points, so the pair orientation (i < j in caller order) must be kept.
// The flat joint path scatters by default (its cells are hit by value, and neighbouring lanes with
// neighbouring points would collide on cells); 1D paths use Morton order from kOrderMinPoints.
static int point_order(const sfb200_plan* p, long long n)
{
    if (p->joint && p->sphere) return 0;
    if (p->order_ovr >= 0) return p->order_ovr;
    if (p->joint) return n >= kOrderMinPoints ? 2 : 0;
    return n >= kOrderMinPoints ? 1 : 0;
}

static unsigned long long gcd_u64(unsigned long long a, unsigned long long b)
{
    while (b) {
        const unsigned long long t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Scattered permutation: slot i -> (i * mult) mod n with mult coprime to n.
static int launch_scatter(sfb200_plan* p, Workspace& w, int n, cudaStream_t s, const int** perm)
{
    sfb200_ctx* ctx = p->ctx;
    unsigned long long mult = 2654435761ull % (unsigned long long)n;
    if (mult < 2) mult = 2;
    while (gcd_u64(mult, (unsigned long long)n) != 1ull) ++mult;
    k_scatter_perm<<<(n + 255) / 256, 256, 0, s>>>(n, mult, w.d_perm + w.cap);
    CK(cudaGetLastError());
    *perm = w.d_perm + w.cap;
    return SFB200_OK;
}

// Morton keys of the caller's points, radix-sorted with their indices; returns the permutation
// (slot -> caller index) in device memory.
template <typename TX>
static int launch_order(sfb200_plan* p, Workspace& w, const void* x, int n, cudaStream_t s, const int** perm)
{
    sfb200_ctx* ctx = p->ctx;
    const int tb = 256, nblk = (n + tb - 1) / tb;
    CK(cudaMemsetAsync(w.d_box, 0xff, sizeof(unsigned) * 3, s));
    CK(cudaMemsetAsync(w.d_box + 3, 0, sizeof(unsigned) * 3, s));
    k_morton_box<TX><<<nblk, tb, 0, s>>>((const TX*)x, n, p->W, p->sphere, p->desc.angle_unit, w.d_box);
    k_morton_keys<TX><<<nblk, tb, 0, s>>>((const TX*)x, n, p->W, p->sphere, p->desc.angle_unit, w.d_box,
                                          w.d_keys, w.d_perm);
    CK(cudaGetLastError());
    size_t tmp = w.sort_tmp_bytes;
    CK(cub::DeviceRadixSort::SortPairs(w.d_sort_tmp, tmp, w.d_keys, w.d_keys + w.cap, w.d_perm, w.d_perm + w.cap,
                                       n, 0, 32, s));
    *perm = w.d_perm + w.cap;
    return SFB200_OK;
}

// Host mirror of BlockHist<R, NV, PRIV>::bytes (sfb200_acc.cuh); `lc`: run-length table columns.
static size_t hist_bytes(bool fp32, int NV, int priv, int NW, int NBP, int lc)
{
    const size_t rs = fp32 ? 4 : 8;
    size_t b;
    if (priv == 0) {
        b = (size_t)NW * NV * NBP * rs * (fp32 ? 2 : 1) + (size_t)NW * NBP * (fp32 ? 4 : 8);
    } else if (priv == 3 || priv == 6) {
        b = (size_t)NV * NBP * 8 + (size_t)NBP * 8 + (size_t)NV * NBP * lc * rs + (size_t)NBP * lc * 4;
    } else {
        const int C = priv == 2 ? 1 : priv;  // 2: warp-aggregated with leader atomics, one copy
        b = (size_t)NV * NBP * 8 + (size_t)NBP * 8 + (size_t)NW * NV * NBP * C * rs + (size_t)NW * NBP * C * 4;
    }
    return (b + 15) & ~(size_t)15;
}

// Whether a launch of this plan with tiles of T points sorts its J tiles (sfb200_plan_set_option
// SFB200_OPT_TILE_SORT): flat 1D kernels of precision FP64 / MIXED, single runs, 256-point tiles.
static bool sorts_tiles(const sfb200_plan* p, int T, bool batch)
{
    return !p->joint && !p->sphere && !p->fp32 && T == 256 && p->sort_ovr != 0 && !batch;
}

static size_t smem_bytes(const sfb200_plan* p, int T, int lut_bytes, bool smem_hist, int priv, int lc = 32,
                         bool batch = false)
{
    const int NW = T / 32, NBP = p->nb + 2, NV = p->nops_pad;
    lut_bytes += sorts_tiles(p, T, batch) ? kSortScratchBytes : 0;  // the sort's counters beside the records
    if (p->mixed) {
        const int rec = p->sphere ? 10 : 2 * p->D;  // doubles per j record
        if (p->joint) {
            const size_t ndp = (size_t)((p->nb + 31) & ~31);  // slots per value bin (swizzled rows)
            // cells (split words), fine words (split) and FP64 cells of the bins near zero, centres
            return (size_t)lut_bytes + (size_t)rec * T * 8 + (ndp * p->nv + 2 * ndp * p->nfine) * 8 +
                   (size_t)p->nv * 12;  // + value-bin centres (FP64 and FP32)
        }
        return (size_t)lut_bytes + (size_t)rec * T * 8 + hist_bytes(true, NV, priv, NW, NBP, lc);
    }
    if (p->joint) {
        const long long ncell = (long long)p->nb * p->nv * std::max(1, p->sp2d_rows);
        if (!p->fp32) {
            const int nx = p->sphere ? 8 : p->D;
            return (size_t)(nx + p->D) * T * 8 + (smem_hist ? (size_t)ncell * 12 : 0);
        }
        const int nx = p->sphere ? (p->D == 3 ? 20 : 18) : (p->df ? 4 : 2) * p->D;
        return (size_t)lut_bytes + (size_t)nx * T * 4 + (size_t)ncell * 12 + (size_t)(p->nb + 2) * 4;
    }
    if (p->chord64())  // FP64 chord records p(3), U(3), W(3), up/pad
        return (size_t)lut_bytes + (size_t)10 * T * 8 + hist_bytes(false, NV, priv, NW, NBP, lc);
    if (!p->fp32) {
        const int nx = p->sphere ? 8 : p->D;
        return (size_t)lut_bytes + (size_t)(nx + p->D) * T * 8 + hist_bytes(false, NV, priv, NW, NBP, lc);
    }
    // sphere: NF floats per point; flat: one record of (hi[, lo]) x and u padded to 4 floats
    const int nx = p->sphere ? (p->D == 3 ? 20 : 18) : ((((p->df ? 4 : 2) * p->D) + 3) & ~3);
    return (size_t)lut_bytes + (((size_t)nx * T * 4 + 15) & ~(size_t)15) + hist_bytes(true, NV, priv, NW, NBP, lc);
}

static long long tile_pairs(long long n, int T)
{
    const long long nt = (n + T - 1) / T;
    return nt * (nt + 1) / 2;
}

// Default histogram mode (overridable per plan): two open runs per lane (6) for the flat FP64 and
// MIXED kernels of single runs with 256-point tiles from 32768 points and a specialised operator list
// (the generic lists of two and eight operators spill registers in that mode), the run-length table
// (3) otherwise. Measured on B200 (c1 shape, 3D, four operators, 64 bins): two open runs 9.63 / 11.71 ms
// (mixed / FP64) against 10.21 / 13.33 ms at 65536 points, 2.55 / 3.11 against 2.66 / 3.55 ms at
// 32768, but 0.89 against 0.84 ms (mixed) at 16384 and 20-28 % slower with 64-point tiles (c0), where
// rows are short and the second run's registers cost more than the flushes they save.
static int default_privatization(const sfb200_plan* p, long long n, int T)
{
    const bool generic = p->opl == OPL_GEN1 || p->opl == OPL_GEN2 || p->opl == OPL_GEN4 || p->opl == OPL_GEN8;
    if (!p->sphere && !p->fp32 && !generic && T == 256 && n >= 32768) return 6;
    return 3;
}

// Copies (if on the host), orders and packs the points of one run into `w`, zeroes its histogram,
// and builds the data-dependent tables of the FP32-bulk kernels. Everything is queued on stream s.
static int prepare_inputs(sfb200_plan* p, Workspace& w, const void* x, const void* u, long long n, uint32_t flags,
                          cudaStream_t s, int* launches)
{
    sfb200_ctx* ctx = p->ctx;
    const bool dev_in = flags & SFB200_RUN_DEVICE_INPUT;
    CK(cudaMemsetAsync(w.d_sums, 0, sizeof(double) * p->n_sums, s));
    CK(cudaMemsetAsync(w.d_counts, 0, sizeof(unsigned long long) * p->n_counts, s));
    CK(cudaMemsetAsync(w.d_aux, 0, sizeof(unsigned long long) * 4, s));
    if (n < 2) return SFB200_OK;
    int rc = ensure_workspace(p, w, n);
    if (rc) return rc;
    const size_t xs = p->desc.x_dtype == SFB200_F64 ? 8 : 4;
    const size_t us = p->desc.u_dtype == SFB200_F64 ? 8 : 4;
    const void* xin = x;
    const void* uin = u;
    if (!dev_in) {
        CK(cudaMemcpyAsync(w.d_rawx, x, xs * p->W * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(w.d_rawu, u, us * p->D * n, cudaMemcpyHostToDevice, s));
        xin = w.d_rawx;
        uin = w.d_rawu;
    }
    const bool x64 = xs == 8, u64 = us == 8;
    const int* perm = nullptr;
    const int order = point_order(p, n);
    if (order == 1) {
        rc = x64 ? launch_order<double>(p, w, xin, (int)n, s, &perm) : launch_order<float>(p, w, xin, (int)n, s, &perm);
        if (rc) return rc;
        *launches += 2;  // box + keys (the radix sort's own launches are not counted)
    } else if (order == 2) {
        rc = launch_scatter(p, w, (int)n, s, &perm);
        if (rc) return rc;
        *launches += 1;
    }
    if (x64 && u64) launch_pack<double, double>(p, w, xin, uin, (int)n, perm, s);
    else if (x64) launch_pack<double, float>(p, w, xin, uin, (int)n, perm, s);
    else if (u64) launch_pack<float, double>(p, w, xin, uin, (int)n, perm, s);
    else launch_pack<float, float>(p, w, xin, uin, (int)n, perm, s);
    ++*launches;
    CK(cudaGetLastError());
    if (p->fp32) {
        k_build_lut32<<<(p->lg32.ncell + 127) / 128, 128, 0, s>>>(p->d_ck, (int)p->ck.size(), p->wp, p->lg32,
                                                                w.d_aux + 1, p->d_lut32);
        ++*launches;
        CK(cudaGetLastError());
        if (p->joint) {
            ValueWindowParams vw;
            vw.nd = p->nb;
            vw.D = p->D;
            vw.order = p->vorder;
            vw.sphere = p->sphere;
            vw.x_f64 = x64;
            vw.u_f64 = u64;
            vw.df = p->df;
            vw.l_only = p->l_only;
            vw.inv_step = p->desc.value.kind == SFB200_BINS_LINEAR ? p->vlin.inv_step : 0.0;
            vw.neg_f_inv = p->desc.value.kind == SFB200_BINS_LINEAR ? p->vlin.neg_f_inv : 0.0;
            k_value_windows<<<1, 128, 0, s>>>(p->d_rowlo, vw, w.d_aux + 1, p->d_vwin);
            ++*launches;
            CK(cudaGetLastError());
        }
    }

    return SFB200_OK;
}

// Tiles of the batched kernels (one per launch, shared by every slice of the launch): 256 points for
// the 1D histograms; for the joint histogram, whose large shared table leaves room for one block per
// SM, 768 (flat) or 512 (sphere) points, so that each block carries many warps.
static const int kBatchTile1D = 256;
static int batch_tile(const sfb200_plan* p) { return p->joint ? (p->sphere ? 512 : 768) : kBatchTile1D; }

static long long tile_pairs(long long n, int T);

// Default tile of a single joint run over n points. The mixed flat kernel runs one block per SM (its
// cell table fills shared memory), so it takes the largest tile (768, 512, 256 points) that still gives
// every SM a tile pair; the other joint kernels 512 points from 32768, 256 from 4096, else 64.
static int joint_tile(const sfb200_plan* p, long long n, int nsm)
{
    if (p->sp2d_rows) {  // one block per SM (the rows' cells fill shared memory): the widest tile that
                         // still gives every SM a tile pair
        for (int T : {512, 256})
            if (tile_pairs(n, T) >= nsm) return T;
        return n >= 1024 ? 256 : 64;
    }
    if (p->mixed && !p->sphere) {
        for (int T : {768, 512, 256})
            if (tile_pairs(n, T) >= nsm) return T;
        return n >= 1024 ? 256 : 64;
    }
    if (n >= 32768) return 512;
    return n >= 4096 ? 256 : 64;
}

// Launch configuration of one run over n points: kernel, tile, block size, shared memory, grid and
// the kernel arguments. `batch`: the batched (serving) form of the mixed kernels, with a fixed tile
// so that slices of one variant share a launch.
struct LaunchCfg {
    KernelChoice kc{};
    int T = 0, threads = 0;
    size_t smem = 0;
    long long ntp = 0, grid = 0;
    PairArgs a{};
};

static int configure(sfb200_plan* p, Workspace& w, long long n, bool batch, LaunchCfg* out)
{
    sfb200_ctx* ctx = p->ctx;
    const bool dlinear = p->desc.distance.kind == SFB200_BINS_LINEAR;
    int lut_bytes = 0;
    // flat kernels of precision FP64 / MIXED (1D) and MIXED (joint) bin with the byte table when the
    // plan has one and a block has enough pairs to repay copying its 10 KB into shared memory (about
    // four 256 x 256 tile pairs; never in batched rounds, whose blocks set up per work item); the
    // cell table of a few hundred bytes otherwise
    const long long pairs_per_block = n * (n - 1) / 2 / std::max(1, ctx->nsm * 4);
    const bool byte_lut = p->d_lut8 && !p->sphere && !p->fp32 && (!p->joint || p->mixed) && !batch &&
                          pairs_per_block >= (1ll << 18);
    if (byte_lut) lut_bytes = kByteCells + (int)sizeof(double) * kByteEdges;
    else if (p->fp32) lut_bytes = p->lg32.ncell * (int)sizeof(LutEntry32);
    else if (p->mixed) lut_bytes = p->lut64_bytes;  // exact table (flat) or chord table (sphere); 0 if linear
    else if (p->chord64()) lut_bytes = p->lutc_bytes;
    else if (!dlinear && !p->joint) lut_bytes = p->lut64_bytes;
    int T;
    bool smem_hist = true;
    KernelChoice kc;
    size_t smem;
    int dev_smem_max = 0;
    CK(cudaDeviceGetAttribute(&dev_smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    int flush_every = 0;
    int hist_cols = 32;
    // threads per point of the tile: the single-pass row groups run one block per SM (their cells fill
    // shared memory), with two threads per point for twice the warps
    const int split = p->sp2d_rows ? 2 : 1;
    if (p->joint) {
        T = p->tile_ovr ? p->tile_ovr : joint_tile(p, n, ctx->nsm);
        if (batch) T = batch_tile(p);
        smem = smem_bytes(p, T, lut_bytes, true, 0);
        while ((p->mixed || p->sp2d_rows) && smem > (size_t)dev_smem_max && T > 64 && !p->tile_ovr && !batch) {
            T = T > 512 ? 512 : T / 2;
            smem = smem_bytes(p, T, lut_bytes, true, 0);
        }
        if (smem > (size_t)dev_smem_max) {
            if (p->fp32 || p->mixed)
                return set_err(ctx, SFB200_ERR_UNSUPPORTED,
                               "joint histogram of %d x %d cells does not fit shared memory on the mixed path; use fp64",
                               p->nb, p->nv);
            smem_hist = false;
            smem = smem_bytes(p, T, lut_bytes, false, 0);
        }
        kc = p->mixed ? (batch ? pick_joint_mx_batch(p->sphere, p->D, p->opl) : pick_joint_mx(p->sphere, p->D, p->opl, T))
                   : p->sp2d_rows ? pick_sp2d(p->D, smem_hist, split)
                                  : pick_joint(p->sphere, p->D, p->fp32, smem_hist, p->df, p->opl);
        // block cells hold at most 2^31 pairs between flushes (T^2 pairs per tile pair); the mixed
        // kernel's packed cells fewer than 2^20
        flush_every = (int)std::max<long long>(1, (p->mixed ? (1ll << 20) - 1 : (1ll << 31)) / ((long long)T * T));
    } else {
        if (batch) {
            T = batch_tile(p);
        } else if (p->tile_ovr) {
            T = p->tile_ovr;
        } else {
            T = 64;
            for (int cand : {256, 128}) {
                if (tile_pairs(n, cand) >= 4ll * ctx->nsm) { T = cand; break; }
            }
        }
        int want = p->priv_ovr >= 0 ? p->priv_ovr : default_privatization(p, n, T);
        if (want == 6 && (p->sphere || p->fp32)) want = 3;  // two open runs: flat FP64 / MIXED kernels only
        if (p->mixed && batch)
            kc = p->sphere ? pick_sphere1d_mx_batch(p->D, p->opl) : pick_flat1d_mx_batch(p->D, p->opl);
        else if (p->mixed)
            kc = p->sphere ? pick_sphere1d_mx(p->D, p->opl, want) : pick_flat1d_mx(p->D, p->opl, want, dlinear);
        else if (p->chord64())
            kc = pick_sphere1d_chord64(p->D, p->opl, want);
        else
            kc = p->sphere ? pick_sphere1d(p->D, p->fp32, p->opl, want)
                           : pick_flat1d(p->D, p->fp32, p->df, p->opl, want);
        if (T > kc.max_threads) T = kc.max_threads;
        if (kc.priv == 3 || kc.priv == 6) {
            // run-length table: the most columns (<= 32) that leave room for 3 blocks per SM,
            // at least one column
            hist_cols = p->cols_ovr ? p->cols_ovr : 32;
            if (!p->cols_ovr) {
                int smem_sm = 0;
                CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
                while (hist_cols > 1 && smem_bytes(p, T, lut_bytes, true, kc.priv, hist_cols, batch) + 1024 > (size_t)smem_sm / 3)
                    hist_cols /= 2;
            }
        }
        smem = smem_bytes(p, T, lut_bytes, true, kc.priv, hist_cols, batch);
        while (smem > (size_t)dev_smem_max && T > 32) {
            T /= 2;
            smem = smem_bytes(p, T, lut_bytes, true, kc.priv, hist_cols, batch);
        }
        if (smem > (size_t)dev_smem_max)
            return set_err(ctx, SFB200_ERR_UNSUPPORTED, "%d bins x %d operators do not fit shared memory",
                           p->nb, p->nops);
        if (kc.priv == 3 || kc.priv == 6) {
            // FP32 table cells are folded into FP64 before any of them holds more than ~4096
            // pair terms (NW warps x T steps per tile pair add into one column)
            flush_every = (p->fp32 || p->mixed) ? std::max(1, 4096 / ((T / 32) * T)) : 64;
        } else if (kc.priv > 0) {
            // FP32 copies are folded into FP64 before any lane-bin cell can hold more than ~512 terms
            const int copies = kc.priv == 2 ? 1 : kc.priv;
            flush_every = (p->fp32 || p->mixed) ? std::max(1, 512 * copies / (32 * T)) : 64;
        }
    }
    if (!kc.fn) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "no kernel for this plan");
    if (batch && T != batch_tile(p))
        return set_err(ctx, SFB200_ERR_UNSUPPORTED, "histogram too large for the batched kernels' fixed tiles");
    {
        const int rc = raise_smem_limit(ctx, kc.fn, smem);
        if (rc) return rc;
    }
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kc.fn, T * split, smem));
    if (occ < 1) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "kernel does not fit on an SM (%zu bytes shared)", smem);
    if (p->bps_ovr) occ = std::min(occ, p->bps_ovr);
    const long long ntp = tile_pairs(n, T);
    const long long grid = std::min<long long>(ntp, (long long)ctx->nsm * occ);
    // the warp-aggregated FP32 histogram counts in 32 bits per warp and bin without folding
    if (!p->joint && kc.priv == 0 && (p->fp32 || p->mixed) && ((ntp + grid - 1) / grid) * 32ll * T >= (1ll << 32))
        return set_err(ctx, SFB200_ERR_UNSUPPORTED,
                       "privatization 0 would overflow its 32-bit counters at %lld points; use another", n);

    PairArgs a{};
    a.n = (int)n;
    a.ntiles = (int)((n + T - 1) / T);
    a.ntp = ntp;
    a.X64 = w.d_X64;
    a.U64 = w.d_U64;
    a.XF = w.d_XF;
    a.UF = w.d_UF;
    a.XM = w.d_XM;
    a.lut = p->fp32 ? (const void*)p->d_lut32 : (p->chord64() ? (const void*)p->d_lutc : (const void*)p->d_lut64);
    a.lg = p->fp32 ? p->lg32 : (p->chord64() ? p->lgc : p->lg64);
    a.chord_wrel = kChordWrel;
    a.chord_short = 0x1p-40;         // (near-)coincident: the reference frame is degenerate
    a.chord_anti = 4.0 - 0x1p-40;    // (near-)antipodal: likewise
    a.lut_bytes = lut_bytes;
    a.lut8 = p->d_lut8;
    a.byte_lut = byte_lut ? 1 : 0;
    // flat 1D kernels (FP64 / MIXED) with 256-point tiles stage off-diagonal J tiles sorted by distance
    // (single runs; the batched rounds keep the storage order, their slices are mostly small)
    a.sort_j = sorts_tiles(p, T, batch) ? 1 : 0;
    a.edges = p->d_exact;
    a.n_edges = p->desc.distance.n_edges;
    a.dist_linear = dlinear;
    a.dlin = p->dlin;
    a.radius = p->desc.radius;
    a.nb = p->nb;
    a.nops = p->nops;
    a.nv = p->nv;
    a.val_linear = p->joint && p->desc.value.kind == SFB200_BINS_LINEAR;
    a.vlin = p->vlin;
    a.vedges = p->d_vedges;
    a.n_vedges = p->joint ? p->desc.value.n_edges : 0;
    a.vwin = p->d_vwin;
    a.flush_every = flush_every;
    a.hist_cols = hist_cols;
    // per-pair relative value error: compensated du_L carries ~(6 order + 6) u; otherwise only
    // the rounding of t itself (the rest is in the per-row absolute window)
    a.vrel = (float)((p->l_only ? (6.0 * p->vorder + 6.0) * 1.25 : 4.0) * 0x1p-24);
    // mixed: the FP32 value carries ~5 ulps per order of L / T (conversion, rsqrtf, scaling)
    if (p->mixed) a.vrel = (float)((5.0 * p->vorder + 3.0) * 1.25 * 0x1p-24);
    a.vq = p->vq;
    a.vq_inv = p->vq_inv;
    a.vqc = p->vqc;
    a.vqc_inv = p->vqc_inv;
    a.vfine_lo = p->vfine_lo;
    a.nfine = p->nfine;
    a.gen = p->gen;
    a.g_sums = w.d_sums;
    a.g_counts = w.d_counts;
    a.g_stats = w.d_aux;
    out->kc = kc;
    out->T = T;
    out->threads = T * split;
    out->smem = smem;
    out->ntp = ntp;
    out->grid = (long long)ctx->nsm * occ;  // resident blocks; a single run launches min(grid, ntp)
    out->a = a;
    // this plan's shard of the tile pairs (contiguous ranges of equal pair counts; the batched form
    // walks explicit item ranges instead)
    if (batch) {
        out->a.tp_lo = 0;
        out->a.tp_hi = ntp;
    } else {
        long long lo, hi;
        shard_range(n, T, p->shard_index, p->shard_count, &lo, &hi);
        out->a.tp_lo = lo;
        out->a.tp_hi = hi;
    }
    return SFB200_OK;
}

extern "C" int sfb200_run(sfb200_plan* p, const void* x, const void* u, int64_t n, uint32_t flags,
                          double* sums, uint64_t* counts, void* stream)
{
    if (!p) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = p->ctx;
    if (n < 0) return set_err(ctx, SFB200_ERR_INVALID_ARG, "negative point count");
    if (n > (1ll << 31) - 1024) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "more than 2^31 points");
    if (!sums || !counts) return set_err(ctx, SFB200_ERR_INVALID_ARG, "sums/counts pointer is NULL");
    if (n > 0 && (!x || !u)) return set_err(ctx, SFB200_ERR_INVALID_ARG, "x/u pointer is NULL");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    const bool dev_out = flags & SFB200_RUN_DEVICE_OUTPUT;
    const bool accumulate = flags & SFB200_RUN_ACCUMULATE;
    int launches = 0;
    p->stats = sfb200_stats{};
    p->stats.pairs = n * (n - 1) / 2;
    p->stats_pending = false;
    int rc = prepare_inputs(p, p->ws, x, u, n, flags, s, &launches);
    if (rc) return rc;
    if (n >= 2) {
        LaunchCfg cfg;
        rc = configure(p, p->ws, n, false, &cfg);
        if (rc) return rc;
        const long long grid = std::min(cfg.grid, cfg.a.tp_hi - cfg.a.tp_lo);
        void* args[] = {&cfg.a};
        CK(cudaEventRecord(ctx->ev0, s));
        if (grid > 0) {
            CK(cudaLaunchKernel(cfg.kc.fn, dim3((unsigned)grid), dim3(cfg.threads), args, cfg.smem, s));
            ++launches;
        }
        CK(cudaEventRecord(ctx->ev1, s));
        CK(cudaGetLastError());
        p->stats.tile = cfg.T;
        p->stats.threads = cfg.threads;
        p->stats.privatization = p->joint ? -1 : cfg.kc.priv;
        p->stats.blocks = (int)grid;
        p->stats_pending = true;
    }

    if (dev_out) {
        const long long m = std::max(p->n_sums, p->n_counts);
        if (m > 0) {
            k_finalize<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(p->ws.d_sums, p->ws.d_counts, p->n_sums, p->n_counts,
                                                                 sums, (unsigned long long*)counts, accumulate);
            ++launches;
            CK(cudaGetLastError());
        }
        p->stats.kernel_launches = launches;
        return SFB200_OK;
    }
    CK(cudaMemcpyAsync(p->h_sums.data(), p->ws.d_sums, sizeof(double) * p->n_sums, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(p->h_counts.data(), p->ws.d_counts, sizeof(unsigned long long) * p->n_counts,
                       cudaMemcpyDeviceToHost, s));
    unsigned long long aux0 = 0;
    CK(cudaMemcpyAsync(&aux0, p->ws.d_aux, sizeof(aux0), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (long long k = 0; k < p->n_sums; ++k) sums[k] = (accumulate ? sums[k] : 0.0) + p->h_sums[k];
    for (long long k = 0; k < p->n_counts; ++k) counts[k] = (accumulate ? counts[k] : 0ull) + p->h_counts[k];
    p->stats.rechecked = (int64_t)aux0;
    p->stats.kernel_launches = launches;
    if (p->stats_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) p->stats.kernel_ms = ms;
        p->stats_pending = false;
    }
    return SFB200_OK;
}

// Smallest and largest pair distance over all pairs i < j (the reference's auto-binning scan,
// _minmax_matrix_for_autobins / minmax_i, src/Calculations/dispatch.jl:205-298), on the device.
extern "C" int sfb200_distance_range(sfb200_plan* p, const void* x, const void* u, int64_t n, uint32_t flags,
                                     double* dmin, double* dmax, void* stream)
{
    if (!p) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = p->ctx;
    if (!dmin || !dmax) return set_err(ctx, SFB200_ERR_INVALID_ARG, "dmin/dmax pointer is NULL");
    if (n < 2) return set_err(ctx, SFB200_ERR_INVALID_ARG, "a distance range needs at least 2 points");
    if (n > (1ll << 31) - 1024) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "more than 2^31 points");
    if (!x || !u) return set_err(ctx, SFB200_ERR_INVALID_ARG, "x/u pointer is NULL");
    if (flags & ~SFB200_RUN_DEVICE_INPUT)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "sfb200_distance_range takes only SFB200_RUN_DEVICE_INPUT");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    int launches = 0;
    int rc = prepare_inputs(p, p->ws, x, u, n, flags, s, &launches);
    if (rc) return rc;
    if (!p->d_range) CK(cudaMalloc((void**)&p->d_range, 2 * sizeof(unsigned long long)));
    static const unsigned long long init[2] = {0x7ff0000000000000ull, 0ull};  // +inf, +0
    CK(cudaMemcpyAsync(p->d_range, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int ntiles = (int)((n + 255) / 256);
    const long long ntp = (long long)ntiles * (ntiles + 1) / 2;
    const unsigned grid = (unsigned)std::min<long long>(ntp, (long long)ctx->nsm * 4);
    if (p->sphere) k_key_range<3, true><<<grid, 256, 0, s>>>(p->ws.d_X64, (int)n, ntiles, ntp, p->d_range);
    else if (p->D == 2) k_key_range<2, false><<<grid, 256, 0, s>>>(p->ws.d_X64, (int)n, ntiles, ntp, p->d_range);
    else k_key_range<3, false><<<grid, 256, 0, s>>>(p->ws.d_X64, (int)n, ntiles, ntp, p->d_range);
    CK(cudaGetLastError());
    unsigned long long h[2];
    CK(cudaMemcpyAsync(h, p->d_range, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const double kmin = bits_to_double(h[0]), kmax = bits_to_double(h[1]);
    if (!p->sphere) {
        *dmin = std::sqrt(kmin);  // sqrt is monotone and correctly rounded: min of the distances
        *dmax = std::sqrt(kmax);
    } else {
        // arc length R sigma, sigma = 2 atan(|d|, |s|) with |s|^2 = 4 - |d|^2 (the pair frame's angle)
        auto arc = [&](double c2) {
            return p->desc.radius * 2.0 * std::atan2(std::sqrt(c2), std::sqrt(std::max(4.0 - c2, 0.0)));
        };
        *dmin = arc(kmin);
        *dmax = arc(kmax);
    }
    return SFB200_OK;
}

extern "C" int sfb200_plan_last_stats(const sfb200_plan* pc, sfb200_stats* out)
{
    if (!pc || !out) return SFB200_ERR_INVALID_ARG;
    sfb200_plan* p = const_cast<sfb200_plan*>(pc);
    sfb200_ctx* ctx = p->ctx;
    if (p->stats_pending) {
        CK(cudaEventSynchronize(ctx->ev1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        p->stats.kernel_ms = ms;
        unsigned long long aux0 = 0;
        CK(cudaMemcpy(&aux0, p->ws.d_aux, sizeof(aux0), cudaMemcpyDeviceToHost));
        p->stats.rechecked = (int64_t)aux0;
        p->stats_pending = false;
    }
    *out = p->stats;
    return SFB200_OK;
}

// ------------------------------------------------------------------------------- serving

struct sfb200_slice {
    sfb200_plan* plan = nullptr;
    Workspace w;
    LaunchCfg cfg;
    long long n = 0;
    cudaEvent_t ready = nullptr;  // preparation finished (recorded on the preparation stream)
    cudaEvent_t used = nullptr;   // recorded after the last read (on the reader's stream)
    unsigned long long last_round = 0;  // number of the last round that listed this slice (0: none)
};

// Orders stream s after the last round that listed slice sl, if that round may still be running.
// Only that round is waited for, not the rounds queued after it. (A round buffer's event is only
// re-recorded once the round that used it before has completed, so a buffer that has moved on to a
// later round, or is no longer pending, means the slice's round is done.)
static int wait_slice_round(sfb200_ctx* ctx, const sfb200_slice* sl, cudaStream_t s)
{
    if (!sl->last_round) return SFB200_OK;
    const auto& b = ctx->rb[(sl->last_round - 1) % sfb200_ctx::kRoundBufs];
    if (b.pending && b.seq == sl->last_round) CK(cudaStreamWaitEvent(s, b.done, 0));
    return SFB200_OK;
}

static int side_stream(sfb200_ctx* ctx, cudaStream_t* out)
{
    if (!ctx->side_stream) CK(cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking));
    *out = ctx->side_stream;
    return SFB200_OK;
}

extern "C" int sfb200_slice_create(sfb200_plan* p, const void* x, const void* u, int64_t n, uint32_t flags,
                                   void* stream, sfb200_slice** out)
{
    if (!p || !out) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = p->ctx;
    *out = nullptr;
    if (p->promoted)
        return set_err(ctx, SFB200_ERR_UNSUPPORTED,
                       "flat single-pass 2D rows run the FP64 joint kernel: run them with sfb200_run, not as batched slices");
    if (!p->mixed) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "batched slices need a plan of precision MIXED");
    if (n < 0) return set_err(ctx, SFB200_ERR_INVALID_ARG, "negative point count");
    if (n > (1ll << 31) - 1024) return set_err(ctx, SFB200_ERR_UNSUPPORTED, "more than 2^31 points");
    if (n > 0 && (!x || !u)) return set_err(ctx, SFB200_ERR_INVALID_ARG, "x/u pointer is NULL");
    if (flags & ~SFB200_RUN_DEVICE_INPUT) return set_err(ctx, SFB200_ERR_INVALID_ARG, "slice flags: DEVICE_INPUT only");
    CK(cudaSetDevice(ctx->device));
    if (!ctx->prep_stream) CK(cudaStreamCreateWithFlags(&ctx->prep_stream, cudaStreamNonBlocking));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->prep_stream;
    sfb200_slice* sl = new (std::nothrow) sfb200_slice();
    if (!sl) return SFB200_ERR_OOM;
    sl->plan = p;
    sl->n = n;
    int rc = slice_workspace(p, sl->w, n, s);
    int launches = 0;
    if (!rc) rc = prepare_inputs(p, sl->w, x, u, n, flags, s, &launches);
    if (!rc && n >= 2) rc = configure(p, sl->w, n, true, &sl->cfg);
    cudaError_t e = cudaSuccess;
    if (!rc) {
        e = cudaEventCreateWithFlags(&sl->ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(sl->ready, s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "slice event");
    }
    if (rc) {
        cudaStreamSynchronize(s);
        if (sl->ready) cudaEventDestroy(sl->ready);
        free_workspace(sl->w, true, s);
        delete sl;
        return rc;
    }
    if (n < 2) sl->cfg.ntp = 0;
    *out = sl;
    return SFB200_OK;
}

extern "C" int sfb200_slice_get_info(const sfb200_slice* sl, sfb200_slice_info* out)
{
    if (!sl || !out) return SFB200_ERR_INVALID_ARG;
    out->n_points = sl->n;
    out->pairs = sl->n * (sl->n - 1) / 2;
    out->tile_pairs = sl->cfg.ntp;
    out->device_bytes = (int64_t)sl->w.bytes;
    return SFB200_OK;
}

extern "C" int sfb200_slice_destroy(sfb200_slice* sl)
{
    if (!sl) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = sl->plan->ctx;
    CK(cudaSetDevice(ctx->device));
    // free in stream order after the preparation, the slice's last round and its last read; the host
    // does not wait
    cudaStream_t s = nullptr;
    int rc = side_stream(ctx, &s);
    if (rc) return rc;
    if (sl->ready) CK(cudaStreamWaitEvent(s, sl->ready, 0));
    if ((rc = wait_slice_round(ctx, sl, s))) return rc;
    if (sl->used) CK(cudaStreamWaitEvent(s, sl->used, 0));
    free_workspace(sl->w, true, s);
    if (sl->ready) cudaEventDestroy(sl->ready);
    if (sl->used) cudaEventDestroy(sl->used);
    delete sl;
    return SFB200_OK;
}

extern "C" int sfb200_device_memory(sfb200_ctx* ctx, int64_t* free_bytes, int64_t* total_bytes)
{
    if (!ctx || !free_bytes || !total_bytes) return SFB200_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    size_t f = 0, t = 0;
    CK(cudaMemGetInfo(&f, &t));
    if (ctx->pool) {  // blocks the context's pool holds but no slice uses are free for slices
        unsigned long long reserved = 0, used = 0;
        CK(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
        CK(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used));
        if (reserved > used) f += (size_t)(reserved - used);
    }
    *free_bytes = (int64_t)f;
    *total_bytes = (int64_t)t;
    return SFB200_OK;
}

extern "C" int sfb200_slice_read(sfb200_slice* sl, double* sums, uint64_t* counts, uint32_t flags, void* stream)
{
    if (!sl || !sums || !counts) return SFB200_ERR_INVALID_ARG;
    sfb200_plan* p = sl->plan;
    sfb200_ctx* ctx = p->ctx;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (!s) {
        const int rc = side_stream(ctx, &s);
        if (rc) return rc;
    }
    const bool accumulate = flags & SFB200_RUN_ACCUMULATE;
    CK(cudaStreamWaitEvent(s, sl->ready, 0));  // a slice with no tile pairs is read without a round
    {
        const int rc = wait_slice_round(ctx, sl, s);
        if (rc) return rc;
    }
    if (!sl->used) CK(cudaEventCreateWithFlags(&sl->used, cudaEventDisableTiming));
    if (flags & SFB200_RUN_DEVICE_OUTPUT) {
        const long long m = std::max(p->n_sums, p->n_counts);
        k_finalize<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(sl->w.d_sums, sl->w.d_counts, p->n_sums, p->n_counts,
                                                             sums, (unsigned long long*)counts, accumulate);
        CK(cudaGetLastError());
        CK(cudaEventRecord(sl->used, s));
        return SFB200_OK;
    }
    std::vector<double> hs(p->n_sums);
    std::vector<unsigned long long> hc(p->n_counts);
    CK(cudaMemcpyAsync(hs.data(), sl->w.d_sums, sizeof(double) * p->n_sums, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hc.data(), sl->w.d_counts, sizeof(unsigned long long) * p->n_counts, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(sl->used, s));
    CK(cudaStreamSynchronize(s));
    for (long long k = 0; k < p->n_sums; ++k) sums[k] = (accumulate ? sums[k] : 0.0) + hs[k];
    for (long long k = 0; k < p->n_counts; ++k) counts[k] = (accumulate ? counts[k] : 0ull) + hc[k];
    return SFB200_OK;
}

// Tile pairs per work item: small enough to balance the end of a round across SMs, large enough
// that the per-item setup (table copy, histogram clear and merge) stays a few percent.
static long long item_tile_pairs(const sfb200_plan* p) { return p->joint ? 1 : 4; }

extern "C" int sfb200_batch_run(sfb200_ctx* ctx, int32_t n, sfb200_slice* const* slices, const int64_t* tp_begin,
                                const int64_t* tp_end, void* stream)
{
    if (!ctx || n < 0 || (n > 0 && (!slices || !tp_begin || !tp_end))) return SFB200_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    // group the listed ranges by kernel; chunks of at most kBatchSlices slices per launch
    struct Launch {
        const void* fn;
        int threads;
        size_t smem;
        int nslices;
        BatchArgs args;
        size_t item0, nitems;
    };
    std::vector<Launch> launches;
    std::vector<WorkItem> items;
    std::vector<int> order(n);
    for (int k = 0; k < n; ++k) {
        order[k] = k;
        const sfb200_slice* sl = slices[k];
        if (!sl || sl->plan->ctx != ctx) return set_err(ctx, SFB200_ERR_INVALID_ARG, "slice %d is NULL or of another context", k);
        if (tp_begin[k] < 0 || tp_end[k] > sl->cfg.ntp || tp_begin[k] > tp_end[k])
            return set_err(ctx, SFB200_ERR_INVALID_ARG, "slice %d: tile-pair range [%lld, %lld) outside [0, %lld)", k,
                           (long long)tp_begin[k], (long long)tp_end[k], sl->cfg.ntp);
        for (int j = 0; j < k; ++j)
            if (slices[j] == sl) return set_err(ctx, SFB200_ERR_INVALID_ARG, "slice %d listed twice in one round", k);
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return reinterpret_cast<uintptr_t>(slices[a]->cfg.kc.fn) < reinterpret_cast<uintptr_t>(slices[b]->cfg.kc.fn);
    });
    for (int oi = 0; oi < n; ++oi) {
        const int k = order[oi];
        const sfb200_slice* sl = slices[k];
        if (tp_end[k] <= tp_begin[k]) continue;
        if (launches.empty() || launches.back().fn != sl->cfg.kc.fn || launches.back().nslices == kBatchSlices) {
            Launch L{};
            L.fn = sl->cfg.kc.fn;
            L.threads = sl->cfg.threads;
            L.item0 = items.size();
            launches.push_back(L);
        }
        Launch& L = launches.back();
        const int j = L.nslices++;
        L.args.s[j] = sl->cfg.a;
        L.smem = std::max(L.smem, sl->cfg.smem);
        const long long step = item_tile_pairs(sl->plan);
        for (long long q = tp_begin[k]; q < tp_end[k]; q += step)
            items.push_back(WorkItem{j, 0, q, std::min<long long>(q + step, tp_end[k])});
        L.nitems = items.size() - L.item0;
    }
    if (launches.empty()) return SFB200_OK;
    // lanes and events on first use; this round's buffer must have been consumed by the round that
    // used it before (two rounds back); the slices must be prepared
    if (!ctx->fork) {
        CK(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
        for (int k = 0; k < sfb200_ctx::kLanes; ++k) {
            CK(cudaStreamCreateWithFlags(&ctx->lane[k], cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&ctx->join[k], cudaEventDisableTiming));
        }
        for (auto& b : ctx->rb) CK(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    }
    sfb200_ctx::RoundBuf& B = ctx->rb[ctx->rounds_enqueued % sfb200_ctx::kRoundBufs];
    if (B.pending) CK(cudaEventSynchronize(B.done));
    B.pending = false;
    for (int k = 0; k < n; ++k) CK(cudaStreamWaitEvent(s, slices[k]->ready, 0));
    // buffers (before any capture)
    if (items.size() > B.items_cap) {
        if (B.h_items) cudaFreeHost(B.h_items);
        cudaFree(B.d_items);
        B.h_items = nullptr;
        B.d_items = nullptr;
        B.items_cap = 0;
        const size_t cap = std::max<size_t>(items.size() * 2, 4096);
        CK(cudaMallocHost(&B.h_items, cap * sizeof(WorkItem)));
        CK(cudaMalloc(&B.d_items, cap * sizeof(WorkItem)));
        B.items_cap = cap;
    }
    if ((int)launches.size() > B.counters_cap) {
        cudaFree(B.d_counters);
        B.d_counters = nullptr;
        const int cap = std::max<int>((int)launches.size() * 2, 64);
        CK(cudaMalloc(&B.d_counters, cap * sizeof(unsigned)));
        B.counters_cap = cap;
    }
    std::memcpy(B.h_items, items.data(), items.size() * sizeof(WorkItem));
    const WorkItem* d_items = static_cast<const WorkItem*>(B.d_items);
    for (size_t l = 0; l < launches.size(); ++l) {
        Launch& L = launches[l];
        const int rc = raise_smem_limit(ctx, L.fn, L.smem);
        if (rc) return rc;
        L.args.items = d_items + L.item0;
        L.args.n_items = (int)L.nitems;
        L.args.counter = B.d_counters + l;
    }
    // grids (before any capture): at most the resident blocks, at most one block per item
    std::vector<long long> grids(launches.size());
    for (size_t l = 0; l < launches.size(); ++l) {
        int occ = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, launches[l].fn, launches[l].threads, launches[l].smem));
        grids[l] = std::min<long long>((long long)launches[l].nitems, (long long)ctx->nsm * std::max(occ, 1));
    }
    // item copy and counter reset on s, then the kernels forked over the lanes (they run
    // concurrently and share the SMs), joined back into s
    const int nlanes = (int)std::min<size_t>(launches.size(), sfb200_ctx::kLanes);
    auto enqueue = [&]() -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(B.d_items, B.h_items, items.size() * sizeof(WorkItem),
                                        cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(B.d_counters, 0, launches.size() * sizeof(unsigned), s);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->fork, s);
        for (int k = 0; k < nlanes && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(ctx->lane[k], ctx->fork, 0);
        for (size_t l = 0; l < launches.size() && e == cudaSuccess; ++l) {
            Launch& L = launches[l];
            void* args[] = {&L.args};
            e = cudaLaunchKernel(L.fn, dim3((unsigned)grids[l]), dim3(L.threads), args, L.smem,
                                 ctx->lane[l % sfb200_ctx::kLanes]);
        }
        for (int k = 0; k < nlanes && e == cudaSuccess; ++k) {
            e = cudaEventRecord(ctx->join[k], ctx->lane[k]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->join[k], 0);
        }
        return e;
    };
    auto finish = [&]() -> int {
        CK(cudaEventRecord(B.done, s));
        B.pending = true;
        B.seq = ++ctx->rounds_enqueued;
        for (int k = 0; k < n; ++k)
            if (tp_end[k] > tp_begin[k]) slices[k]->last_round = B.seq;
        return SFB200_OK;
    };
    if (ctx->batch_graph) {
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t e1 = enqueue();
            e = cudaStreamEndCapture(s, &graph);
            if (e1 != cudaSuccess) e = e1;
        }
        if (e == cudaSuccess && B.exec) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(B.exec, graph, &info) != cudaSuccess) {
                cudaGetLastError();
                cudaGraphExecDestroy(B.exec);
                B.exec = nullptr;
            }
        }
        if (e == cudaSuccess && !B.exec) e = cudaGraphInstantiate(&B.exec, graph, 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(B.exec, s);
        if (graph) cudaGraphDestroy(graph);
        if (e == cudaSuccess) return finish();
        // capture or replay refused: run this and later rounds with plain launches
        cudaGetLastError();
        ctx->batch_graph = false;
        for (auto& b : ctx->rb)
            if (b.exec && &b != &B) CK(cudaEventSynchronize(b.done));
        for (auto& b : ctx->rb) {
            if (b.exec) cudaGraphExecDestroy(b.exec);
            b.exec = nullptr;
        }
    }
    CK(enqueue());
    return finish();
}

extern "C" int sfb200_batch_wait(sfb200_ctx* ctx)
{
    if (!ctx) return SFB200_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    for (auto& b : ctx->rb) {
        if (b.pending) CK(cudaEventSynchronize(b.done));
        b.pending = false;
    }
    return SFB200_OK;
}

extern "C" int sfb200_batch_wait_oldest(sfb200_ctx* ctx, int64_t* round)
{
    if (!ctx) return SFB200_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    sfb200_ctx::RoundBuf* oldest = nullptr;
    for (auto& b : ctx->rb)
        if (b.pending && (!oldest || b.seq < oldest->seq)) oldest = &b;
    if (round) *round = oldest ? (int64_t)oldest->seq : 0;
    if (!oldest) return SFB200_OK;
    CK(cudaEventSynchronize(oldest->done));
    oldest->pending = false;
    return SFB200_OK;
}

extern "C" int sfb200_batch_query(sfb200_ctx* ctx, int32_t* done)
{
    if (!ctx || !done) return SFB200_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    *done = 1;
    for (auto& b : ctx->rb) {
        if (!b.pending) continue;
        const cudaError_t e = cudaEventQuery(b.done);
        if (e == cudaErrorNotReady) {
            *done = 0;
            continue;
        }
        CK(e);
        b.pending = false;
    }
    return SFB200_OK;
}

// ------------------------------------------------------------------------------- no allocation
//
// sfb200_run_noalloc: the mixed / FP64 flat 1D run without any device allocation, for callers that
// must not allocate device memory while they run -- a loop that reserved its whole device budget up
// front, or a process sharing the device where an allocation could fail under memory pressure or
// make the device wait (cudaMalloc / cudaFree may synchronise it). Its scratch (packed points and the
// accumulators) is one file-scope device array of fixed size, so at most kNoAllocMaxPoints points and
// kNoAllocMaxSums / kNoAllocMaxCounts histogram entries fit. Every call zeroes the accumulators it
// uses; the packed points are overwritten. All calls on a device share the one array: calls whose work
// overlaps on the GPU (different streams or host threads) race on it, so callers serialise them.

static constexpr long long kNoAllocMaxPoints = 1ll << 16;          // points per call
static constexpr long long kNoAllocMaxSums = 32768;                // nb x n_ops doubles
static constexpr long long kNoAllocMaxCounts = 4096;               // nb counts
static constexpr long long kNoAllocWords =                         // 8-byte words of scratch
    2 * 3 * kNoAllocMaxPoints + kNoAllocMaxSums + kNoAllocMaxCounts + 8;

// 3.4 MiB, held by every device that loads the library: X64 (D x N), U64 (D x N), sums, counts, aux
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

// Device address of the scratch array on ctx's device (which the caller has made current). The
// first call on a context looks it up and the context keeps it: a context lives on one device, and a
// device reset, which would move the array, invalidates the context with it. Host code only ever
// passes this address to kernels: the array's name on the host is a host-side stand-in, not a device
// address.
static std::mutex g_noalloc_mutex;  // threads sharing a context look the address up once

static int noalloc_scratch(sfb200_ctx* ctx, void** out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!ctx->noalloc_ptr) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return cuda_fail(ctx, e, "scratch address");
        ctx->noalloc_ptr = ptr;
    }
    *out = ctx->noalloc_ptr;
    return SFB200_OK;
}

extern "C" int sfb200_run_noalloc(sfb200_plan* p, const void* x, const void* u, int64_t n, uint32_t flags,
                                  double* sums, uint64_t* counts, void* stream)
{
    if (!p) return SFB200_ERR_INVALID_ARG;
    sfb200_ctx* ctx = p->ctx;
    if (p->sphere || p->joint || p->fp32)
        return set_err(ctx, SFB200_ERR_UNSUPPORTED, "sfb200_run_noalloc takes flat 1D plans of precision MIXED or FP64");
    if (flags & ~SFB200_RUN_ACCUMULATE)
        return set_err(ctx, SFB200_ERR_INVALID_ARG, "sfb200_run_noalloc: inputs and outputs are device pointers; "
                                                    "only SFB200_RUN_ACCUMULATE may be set");
    if (n < 0) return set_err(ctx, SFB200_ERR_INVALID_ARG, "negative point count");
    if (n > kNoAllocMaxPoints)
        return set_err(ctx, SFB200_ERR_UNSUPPORTED, "sfb200_run_noalloc: %lld points exceed its fixed scratch of %lld",
                       (long long)n, kNoAllocMaxPoints);
    if (p->n_sums > kNoAllocMaxSums || p->n_counts > kNoAllocMaxCounts)
        return set_err(ctx, SFB200_ERR_UNSUPPORTED,
                       "sfb200_run_noalloc: %lld sums / %lld counts exceed its fixed scratch of %lld / %lld",
                       p->n_sums, p->n_counts, kNoAllocMaxSums, kNoAllocMaxCounts);
    if (!sums || !counts) return set_err(ctx, SFB200_ERR_INVALID_ARG, "sums/counts pointer is NULL");
    if (n > 0 && (!x || !u)) return set_err(ctx, SFB200_ERR_INVALID_ARG, "x/u pointer is NULL");
    CK(cudaSetDevice(ctx->device));
    void* base = nullptr;
    int rc = noalloc_scratch(ctx, &base);
    if (rc) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    // a workspace view of the scratch: X64 | U64 | sums | counts | aux
    unsigned long long* words = static_cast<unsigned long long*>(base);
    const long long D = p->D;
    Workspace w;
    w.cap = n;
    w.d_X64 = reinterpret_cast<double*>(words);
    w.d_U64 = reinterpret_cast<double*>(words + D * std::max<long long>(n, 1));
    w.d_sums = reinterpret_cast<double*>(words + 2 * 3 * kNoAllocMaxPoints);
    w.d_counts = words + 2 * 3 * kNoAllocMaxPoints + kNoAllocMaxSums;
    w.d_aux = words + 2 * 3 * kNoAllocMaxPoints + kNoAllocMaxSums + kNoAllocMaxCounts;
    // the array keeps the previous call's contents: the accumulators must start at zero
    CK(cudaMemsetAsync(w.d_sums, 0, sizeof(double) * p->n_sums, s));
    CK(cudaMemsetAsync(w.d_counts, 0, sizeof(unsigned long long) * p->n_counts, s));
    CK(cudaMemsetAsync(w.d_aux, 0, sizeof(unsigned long long) * 4, s));
    if (n >= 2) {
        // caller's point order (no sort buffers); inputs read from the caller's device arrays
        const bool x64 = p->desc.x_dtype == SFB200_F64, u64 = p->desc.u_dtype == SFB200_F64;
        if (x64 && u64) launch_pack<double, double>(p, w, x, u, (int)n, nullptr, s);
        else if (x64) launch_pack<double, float>(p, w, x, u, (int)n, nullptr, s);
        else if (u64) launch_pack<float, double>(p, w, x, u, (int)n, nullptr, s);
        else launch_pack<float, float>(p, w, x, u, (int)n, nullptr, s);
        CK(cudaGetLastError());
        LaunchCfg cfg;
        rc = configure(p, w, n, false, &cfg);
        if (rc) return rc;
        const long long grid = std::min(cfg.grid, cfg.a.tp_hi - cfg.a.tp_lo);
        void* args[] = {&cfg.a};
        if (grid > 0) CK(cudaLaunchKernel(cfg.kc.fn, dim3((unsigned)grid), dim3(cfg.threads), args, cfg.smem, s));
    }
    const long long m = std::max(p->n_sums, p->n_counts);
    k_finalize<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(w.d_sums, w.d_counts, p->n_sums, p->n_counts, sums,
                                                         (unsigned long long*)counts, flags & SFB200_RUN_ACCUMULATE);
    CK(cudaGetLastError());
    return SFB200_OK;
}
