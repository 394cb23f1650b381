// sfb200_kernels.cuh -- the pair kernels.
//
// Layout in HBM (per run, built by the pack kernels from the caller's column-major arrays):
//   FP64 SoA  X64[c * n + i]: flat: D coordinates; sphere: p(3), E(2), N(3) of the local basis.
//             U64[c * n + i]: D velocity components.
//   FP32 SoA  XF[c * n + i]:  flat: D coordinates; sphere: p(3), U(3), W(3)[, up] (ambient tangent
//             velocity U = u_e E + u_n N and its quarter turn W = u_n E - u_e N).
//             UF[c * n + i]:  flat: D velocity components.
// Every point set is tiny next to HBM (N = 200k sphere points: 8.8 MB FP64 + 8 MB FP32) and stays
// L2-resident; the kernels are FP32/FP64 issue-bound, not bandwidth-bound.
//
// Schedule: the N points are cut into tiles of T = blockDim.x points. A block owns an upper-
// triangle tile pair (ti <= tj) at a time (persistent grid, stride gridDim.x): thread t holds point
// ti*T + t in registers, the J tile is staged in shared memory and broadcast, so each thread walks
// the T pairs of its row. Diagonal tiles keep j > i only.
//
// Accumulation (sfb200_acc.cuh): per-warp private histograms in shared memory at a selectable
// privatization depth -- warp-aggregated (__match_any_sync + shuffle tree, leader update, FP32
// two-sum cells) or C copies per warp up to one column per lane -- merged per block in FP64 and
// added to the global FP64 sums / uint64 counts with one atomic per bin.
#pragma once

#include "sfb200_common.cuh"
#include "sfb200_exact.cuh"
#include "sfb200_ops.cuh"
#include "sfb200_acc.cuh"

namespace sfb {

struct PairArgs {
    int n;             // points
    int ntiles;        // ceil(n / T)
    long long ntp;     // ntiles (ntiles + 1) / 2
    long long tp_lo;   // this launch walks tile pairs [tp_lo, tp_hi) (a shard of [0, ntp))
    long long tp_hi;
    const double* X64; // FP64 SoA positions / sphere basis
    const double* U64; // FP64 SoA velocities
    const float* XF;   // FP32 SoA (mixed)
    const float* UF;
    const double* XM;  // FP64 sphere records for the mixed kernels: p(3), U(3), W(3)[, up] (SoA)
    const void* lut;   // LutEntry64 (FP64 kernels) or LutEntry32 (mixed)
    LutGeom lg;
    int lut_bytes;     // bytes of the table copied to shared memory (0: no table)
    const double* edges; // exact edge table in key space: flat squared edges, sphere raw edges
    int n_edges;
    int dist_linear;   // 1: LinearBinEdges search on r (flat: sqrt(r^2))
    const unsigned char* lut8;  // flat byte table (kByteCells bytes) + padded edges (kByteEdges doubles)
    int byte_lut;      // 1: the flat kernels bin with the byte table (it replaces `lut` in shared memory)
    int sort_j;        // 1: off-diagonal J tiles of 256 points are staged sorted by distance (flat 1D)
    LinearParams dlin;
    double radius;     // sphere
    double chord_wrel; // mixed sphere: relative half-width of the chord ambiguity band at an edge
    double chord_short;// mixed sphere: chord^2 below this is recomputed (near-coincident)
    double chord_anti; // mixed sphere: chord^2 above this is recomputed (near-antipodal)
    int nb;            // distance bins
    int nops;          // operators (1D)
    // joint
    int nv;            // value bins
    int val_linear;
    LinearParams vlin;
    const double* vedges;
    int n_vedges;
    const float* vwin; // per distance row: absolute half-width of the value ambiguity window in
                       // value-bin index units (mixed)
    float vrel;        // relative half-width: window += (|t| + |first/step|) * vrel
    double vq;         // fixed-point scale of the value offsets (power of two), and its inverse
    double vq_inv;
    double vqc;        // mixed joint: coarse scale of the packed cells (power of two), and its inverse
    double vqc_inv;
    int vfine_lo;      // mixed joint: value bins [vfine_lo, vfine_lo + nfine) keep exact offsets
    int nfine;
    int flush_every;   // privatized histograms: fold copies into FP64 every this many tile pairs
    int hist_cols;     // run-length histogram: table columns (power of two <= 32)
    GenOps gen;
    double* g_sums;
    unsigned long long* g_counts;
    unsigned long long* g_stats; // [0] rechecked pairs
};

// ---------------------------------------------------------------------------- batched launches
// One launch serves many independent point sets ("slices"): the arguments of up to kBatchSlices
// slices travel in the kernel parameter block (constant bank, uniform per block), and the blocks of a
// persistent grid pull work items -- a slice and a range of its tile pairs -- from a device counter.
struct WorkItem {
    int slice;
    int pad;
    long long p0, p1;  // tile pairs [p0, p1) of the slice
};

constexpr int kBatchSlices = 48;  // 48 x sizeof(PairArgs) stays below the 32 KB parameter limit

struct BatchArgs {
    const WorkItem* items;
    int n_items;
    unsigned* counter;  // zeroed before the launch
    PairArgs s[kBatchSlices];
};
static_assert(sizeof(BatchArgs) <= 32000, "batch arguments must fit the kernel parameter block");

template <class RUN>
__device__ __forceinline__ void batch_items(const BatchArgs& b, RUN run)
{
    __shared__ int s_item;
    for (;;) {
        __syncthreads();  // the previous item (and its use of shared memory) is finished
        if (threadIdx.x == 0) s_item = (int)atomicAdd(b.counter, 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= b.n_items) break;
        const WorkItem w = b.items[it];
        run(b.s[w.slice], w.p0, w.p1);
    }
}

// ---------------------------------------------------------------------------- J-tile staging
// Stages the J tile in shared memory, in the order of each record's squared distance from a
// reference point of the I tile. Every pair of the tile pair is still formed exactly once (a tile
// pair is a full T x T block of pairs when ti != tj), so the result does not depend on the order;
// what changes is the sequence of bins a lane walks: sorted by distance, a lane's bins rise almost
// monotonically across the tile, and its run-length histogram runs last for tens to hundreds of
// pairs instead of a few (each run ends in shared-memory atomics).
//
// Counting sort over 256 buckets taken from the float bits of the FP32 key (two octaves of the
// squared distance at 128 buckets per octave, cyclically): a tile whose keys span less than two
// octaves -- every tile far from the reference point -- comes out sorted up to one rotation and to
// the order inside a bucket (0.5 % of the key); closer tiles come out partly sorted. Must be called
// by all 256 threads of the block (it holds barriers); thread t < jn passes point j0 + t's record.
template <int R>
__device__ __forceinline__ void stage_sorted(const double (&rec)[R], bool has, float key, double* srec,
                                             unsigned* s_cnt, unsigned* s_wtot)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    s_cnt[t] = 0u;
    const unsigned bucket = (__float_as_uint(key) >> 16) & 255u;
    __syncthreads();
    unsigned rank = 0u;
    if (has) rank = atomicAdd(&s_cnt[bucket], 1u);
    __syncthreads();
    const unsigned v = s_cnt[t];
    unsigned incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_wtot[warp] = incl;
    __syncthreads();
    unsigned off = 0u;
    for (int w = 0; w < warp; ++w) off += s_wtot[w];
    s_cnt[t] = off + incl - v;  // first slot of bucket t
    __syncthreads();
    if (has) {
        double2* dst = reinterpret_cast<double2*>(srec + (size_t)(s_cnt[bucket] + rank) * R);
#pragma unroll
        for (int q = 0; q < R / 2; ++q) dst[q] = make_double2(rec[2 * q], rec[2 * q + 1]);
    }
}

// Shared-memory scratch of the tile sort: 256 bucket counters and 8 warp totals (a multiple of 16
// bytes, so that what follows stays aligned). Reserved only in launches that sort.
constexpr int kSortScratchBytes = (256 + 8) * 4;

// Flat J tile: record [x(D), u(D) us] of point j0 + t in slot t (storage order) or in distance order
// from I-tile point `iref` (`sorted`, block-uniform; needs blockDim.x == 256).
template <int D>
__device__ __forceinline__ void stage_flat_j(const PairArgs& a, int j0, int jn, double us, bool sorted, int iref,
                                             double* srec, unsigned* s_cnt, unsigned* s_wtot)
{
    const int t = threadIdx.x;
    const int n = a.n;
    const bool has = t < jn;
    double rec[2 * D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        rec[d] = has ? a.X64[(size_t)d * n + j0 + t] : 0.0;
        rec[D + d] = has ? a.U64[(size_t)d * n + j0 + t] * us : 0.0;
    }
    if (!sorted) {
        if (has) {
            double2* dst = reinterpret_cast<double2*>(srec + (size_t)t * 2 * D);
#pragma unroll
            for (int q = 0; q < D; ++q) dst[q] = make_double2(rec[2 * q], rec[2 * q + 1]);
        }
        return;
    }
    float key = 0.f;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const float c = (float)(rec[d] - a.X64[(size_t)d * n + iref]);
        key = fmaf(c, c, key);
    }
    stage_sorted<2 * D>(rec, has, key, srec, s_cnt, s_wtot);
}

// Copies the kernel's bin table into shared memory (the byte table and its padded edges, or the
// cell table of `lut`), 16 bytes per thread and step.
__device__ __forceinline__ void load_bin_table(const PairArgs& a, unsigned char* dst)
{
    const int4* src = static_cast<const int4*>(a.byte_lut ? (const void*)a.lut8 : a.lut);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int k = threadIdx.x; k < a.lut_bytes / 16; k += blockDim.x) d4[k] = src[k];
}

// Exact FP64 bin of a flat pair from r^2 (src/BinEdges.jl:515-517).
__device__ __forceinline__ int flat_exact_bin(const PairArgs& a, double r2)
{
    if (r2 != r2) return a.n_edges;
    if (a.dist_linear) return linear_bin(a.dlin, SFB_SQRT(r2));
    return count_below(a.edges, a.n_edges, r2);
}

// Exact FP64 bin of a sphere pair from r (digitize(r, edges), src/Calculations/serial.jl:258).
__device__ __forceinline__ int sphere_exact_bin(const PairArgs& a, double r)
{
    if (r != r) return a.n_edges;
    if (a.dist_linear) return linear_bin(a.dlin, r);
    return count_below(a.edges, a.n_edges, r);
}

__device__ __forceinline__ int lut64_bin(const LutEntry64* lut, const PairArgs& a, double key)
{
    const LutEntry64 e = lut[lut_cell64(key, a.lg)];
    if (e.mult & LUT_FLAG_SLOW) return count_below_ool(a.edges, a.n_edges, key);
    return e.base + (key > e.e ? e.mult : 0);
}

// Value bin of the joint histogram (digitize(val, value_bins)), exact FP64.
__device__ __forceinline__ int value_exact_bin(const PairArgs& a, double v)
{
    if (a.val_linear) return linear_bin(a.vlin, v);
    // searchsortedfirst with isless: NaN sorts above every edge.
    if (v != v) return a.n_vedges;
    int lo = 0, hi = a.n_vedges;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const double e = a.vedges[mid];
        const bool less = e < v || (e == v && e == 0.0 && signbit(e) && !signbit(v));
        if (less) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// ================================================================================================
// Flat (Euclidean) 1D, FP64
// ================================================================================================
template <int D, class OPS, int PRIV>
__global__ void __launch_bounds__(256) k_flat1d_fp64(const PairArgs a)
{
    constexpr int NV = OPS::n;
    using Needs = ListNeeds<OPS>;
    using Hist = BlockHist<double, NV, PRIV>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x, NW = T >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.n;
    const LutEntry64* lut = reinterpret_cast<const LutEntry64*>(smem);
    const unsigned char* lut8 = smem;
    const double* sqx = reinterpret_cast<const double*>(smem + kByteCells);
    double* srec = reinterpret_cast<double*>(smem + a.lut_bytes);  // T records x(D) u(D)
    // the tile sort's counters (only when this launch sorts), then the histogram
    unsigned* s_cnt = reinterpret_cast<unsigned*>(srec + (size_t)2 * D * T);
    unsigned* s_wtot = s_cnt + 256;
    Hist hist;
    hist.init(reinterpret_cast<unsigned char*>(s_cnt) + (a.sort_j ? kSortScratchBytes : 0), NW, a.nb + 2, a.hist_cols);
    load_bin_table(a, smem);

    int iter = 0;
    for (long long p = a.tp_lo + blockIdx.x; p < a.tp_hi; p += gridDim.x, ++iter) {
        hist.close_runs(lane);
        if (PRIV && iter && a.flush_every && iter % a.flush_every == 0) hist.fold();
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        double xi[D], ui[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            xi[d] = iv ? a.X64[(size_t)d * n + i] : 0.0;
            ui[d] = iv ? a.U64[(size_t)d * n + i] : 0.0;
        }
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        const bool diag = ti == tj;
        stage_flat_j<D>(a, j0, jn, 1.0, a.sort_j && !diag && T == 256, ti * T + min(T / 2, n - 1 - ti * T), srec,
                        s_cnt, s_wtot);
        __syncthreads();
        auto pair = [&](int jj, int& key, double (&v)[NV]) {
            double dx[D], du[D];
#pragma unroll
            for (int q = 0; q < D; ++q) {  // D double2 per record
                const double2 t = reinterpret_cast<const double2*>(srec + jj * 2 * D)[q];
                const int c0 = 2 * q, c1 = 2 * q + 1;
                if (c0 < D) dx[c0] = SFB_SUB(t.x, xi[c0]); else du[c0 - D] = t.x - ui[c0 - D];
                if (c1 < D) dx[c1] = SFB_SUB(t.y, xi[c1]); else du[c1 - D] = t.y - ui[c1 - D];
            }
            // r^2 exactly as the reference: left-to-right, no contraction (decides the bin)
            const double h2 = SFB_ADD(SFB_MUL(dx[0], dx[0]), SFB_MUL(dx[1], dx[1]));
            double r2 = h2;
            if constexpr (D == 3) r2 = SFB_ADD(h2, SFB_MUL(dx[2], dx[2]));
            if (a.byte_lut) {
                bool slow;
                key = byte_bin(lut8, sqx, r2, slow);
                if (slow) key = count_below_ool(a.edges, a.n_edges, r2);
            } else if (a.dist_linear) {
                key = (r2 != r2) ? a.n_edges : linear_bin(a.dlin, SFB_SQRT(r2));
            } else {
                key = (r2 != r2) ? a.n_edges : lut64_bin(lut, a, r2);
            }

            double L = 0.0, Tt = 0.0, Q = 0.0;
            const double rs = rsqrt(r2);
            if constexpr (Needs::L) {
                double pp = dx[0] * du[0];
#pragma unroll
                for (int d = 1; d < D; ++d) pp = fma(dx[d], du[d], pp);
                L = pp * rs;
            }
            if constexpr (Needs::T) {
                const double t = fma(du[1], dx[0], -du[0] * dx[1]);
                Tt = (D == 2) ? t * rs : t * rsqrt(h2);
            }
            if constexpr (Needs::Q) {
                Q = du[0] * du[0];
#pragma unroll
                for (int d = 1; d < D; ++d) Q = fma(du[d], du[d], Q);
            }
            eval_ops(OPS{}, L, Tt, Q - L * L, Q, D, a.gen, v);
        };
        if constexpr (Hist::RUN) {
            if (iv) {
                constexpr int UNR = PRIV == 6 ? 1 : 2;  // two open runs: one pair per iteration
#pragma unroll (UNR)
                for (int jj = diag ? (int)threadIdx.x + 1 : 0; jj < jn; ++jj) {
                    int key;
                    double v[NV];
                    pair(jj, key, v);
                    hist.add(key, v, lane, warp);
                }
            }
        } else {
            for (int jj = 0; jj < jn; ++jj) {
                const bool valid = iv && (!diag || jj > (int)threadIdx.x);
                int key;
                double v[NV];
                pair(jj, key, v);
                hist.add(valid ? key : a.nb + 1, v, lane, warp);
            }
        }
    }
    hist.merge(a.g_sums, a.g_counts, a.nops, a.nb);
}

// ================================================================================================
// Flat (Euclidean) 1D, FP32 bulk + FP64 recheck
//
// FP64 inputs are carried as FP32 (hi, lo) pairs with hi + lo equal to the FP64 value to ~2^-48
// relative, and differences are formed as (b_hi - a_hi) + (b_lo - a_lo): the difference of two
// nearby coordinates (or velocities) then keeps full FP32 relative accuracy instead of inheriting
// the rounding error of the coordinates themselves. FP32 inputs are exact in one float.
// ================================================================================================
template <bool DF>
__device__ __forceinline__ float df_diff(const float* s, int c, int D, int T, int jj, const float* a)
{
    if constexpr (DF) return __fadd_rn(__fsub_rn(s[c * T + jj], a[c]), __fsub_rn(s[(D + c) * T + jj], a[D + c]));
    else return __fsub_rn(s[c * T + jj], a[c]);
}

// The J tile is staged as one record per point, [x_hi(D) u_hi(D) | x_lo(D) u_lo(D)] padded to a
// multiple of 4 floats, and read with 128-bit broadcast loads: one shared-memory transaction per
// 4 floats instead of one per component.
template <int D, bool DF>
struct FlatRec {
    static constexpr int NRAW = (DF ? 4 : 2) * D;
    static constexpr int NR = (NRAW + 3) & ~3;
};

template <int NR>
__device__ __forceinline__ void load_rec4(const float* base, float (&r)[NR])
{
#pragma unroll
    for (int q = 0; q < NR / 4; ++q) {
        const float4 t = reinterpret_cast<const float4*>(base)[q];
        r[4 * q] = t.x;
        r[4 * q + 1] = t.y;
        r[4 * q + 2] = t.z;
        r[4 * q + 3] = t.w;
    }
}

template <int D, bool DFX, bool DFU, class OPS, int PRIV>
__global__ void __launch_bounds__(256) k_flat1d_mixed(const PairArgs a)
{
    static_assert(DFX == DFU, "records carry (hi, lo) for both or neither");
    constexpr int NV = OPS::n;
    constexpr int NXF = DFX ? 2 * D : D;
    constexpr int NUF = DFU ? 2 * D : D;
    constexpr int NR = FlatRec<D, DFX>::NR;
    using Needs = ListNeeds<OPS>;
    using Hist = BlockHist<float, NV, PRIV>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x, NW = T >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.n;
    LutEntry32* lut = reinterpret_cast<LutEntry32*>(smem);
    float* srec = reinterpret_cast<float*>(smem + a.lut_bytes);  // T records of NR floats
    __shared__ unsigned long long s_recheck;
    Hist hist;
    hist.init(smem + a.lut_bytes + (size_t)NR * T * 4, NW, a.nb + 2, a.hist_cols);
    for (int k = threadIdx.x; k < a.lut_bytes / (int)sizeof(LutEntry32); k += T)
        lut[k] = static_cast<const LutEntry32*>(a.lut)[k];
    if (threadIdx.x == 0) s_recheck = 0ull;
    unsigned long long my_recheck = 0;

    int iter = 0;
    for (long long p = a.tp_lo + blockIdx.x; p < a.tp_hi; p += gridDim.x, ++iter) {
        hist.close_runs(lane);
        if (PRIV && iter && a.flush_every && iter % a.flush_every == 0) hist.fold();
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        float xi[NXF], ui[NUF];
#pragma unroll
        for (int c = 0; c < NXF; ++c) xi[c] = iv ? a.XF[(size_t)c * n + i] : 0.f;
#pragma unroll
        for (int c = 0; c < NUF; ++c) ui[c] = iv ? a.UF[(size_t)c * n + i] : 0.f;
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        if ((int)threadIdx.x < jn) {
            float* rec = srec + (size_t)threadIdx.x * NR;
            const int jg = j0 + threadIdx.x;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                rec[d] = a.XF[(size_t)d * n + jg];
                rec[D + d] = a.UF[(size_t)d * n + jg];
                if constexpr (DFX) {
                    rec[2 * D + d] = a.XF[(size_t)(D + d) * n + jg];
                    rec[3 * D + d] = a.UF[(size_t)(D + d) * n + jg];
                }
            }
#pragma unroll
            for (int c = FlatRec<D, DFX>::NRAW; c < NR; ++c) rec[c] = 0.f;
        }
        __syncthreads();
        const bool diag = ti == tj;
        for (int jj = 0; jj < jn; ++jj) {
            const bool valid = iv && (!diag || jj > (int)threadIdx.x);
            float rj[NR];
            load_rec4<NR>(srec + (size_t)jj * NR, rj);
            float dx[D], du[D];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                if constexpr (DFX) {
                    dx[d] = __fadd_rn(__fsub_rn(rj[d], xi[d]), __fsub_rn(rj[2 * D + d], xi[D + d]));
                    du[d] = __fadd_rn(__fsub_rn(rj[D + d], ui[d]), __fsub_rn(rj[3 * D + d], ui[D + d]));
                } else {
                    dx[d] = __fsub_rn(rj[d], xi[d]);
                    du[d] = __fsub_rn(rj[D + d], ui[d]);
                }
            }
            const float h2 = fmaf(dx[1], dx[1], dx[0] * dx[0]);
            float r2 = h2;
            if constexpr (D == 3) r2 = fmaf(dx[2], dx[2], h2);
            const LutEntry32 e = lut[lut_cell32(r2, a.lg)];
            int bin = e.base + (r2 > e.hi ? (e.mult & 0xffff) : 0);
            bool slow = (e.mult & LUT_FLAG_SLOW) || (r2 >= e.lo && r2 <= e.hi);

            float L = 0.f, Tt = 0.f, Q = 0.f;
            const float rs = rsqrtf(r2);
            if constexpr (Needs::L) {
                float pp = dx[0] * du[0];
#pragma unroll
                for (int d = 1; d < D; ++d) pp = fmaf(dx[d], du[d], pp);
                L = pp * rs;
            }
            if constexpr (Needs::T) {
                const float t = fmaf(du[1], dx[0], -du[0] * dx[1]);
                Tt = (D == 2) ? t * rs : t * rsqrtf(h2);
            }
            if constexpr (Needs::Q) {
                Q = du[0] * du[0];
#pragma unroll
                for (int d = 1; d < D; ++d) Q = fmaf(du[d], du[d], Q);
            }
            float v[NV];
            eval_ops(OPS{}, L, Tt, Q - L * L, Q, D, a.gen, v);

            slow = slow && valid;
            if (__any_sync(FULL, slow)) {
                if (slow) {
                    // FP64 recheck from the original inputs (reference arithmetic for the bin).
                    const int j = j0 + jj;
                    double dx64[D], du64[D];
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        dx64[d] = SFB_SUB(a.X64[(size_t)d * n + j], a.X64[(size_t)d * n + i]);
                        du64[d] = a.U64[(size_t)d * n + j] - a.U64[(size_t)d * n + i];
                    }
                    const double h264 = SFB_ADD(SFB_MUL(dx64[0], dx64[0]), SFB_MUL(dx64[1], dx64[1]));
                    double r264 = h264;
                    if constexpr (D == 3) r264 = SFB_ADD(h264, SFB_MUL(dx64[2], dx64[2]));
                    bin = flat_exact_bin(a, r264);
                    const double rs64 = rsqrt(r264);
                    double L64 = 0.0, T64 = 0.0, Q64 = 0.0;
                    if constexpr (Needs::L) {
                        double pp = dx64[0] * du64[0];
#pragma unroll
                        for (int d = 1; d < D; ++d) pp = fma(dx64[d], du64[d], pp);
                        L64 = pp * rs64;
                    }
                    if constexpr (Needs::T) {
                        const double t = fma(du64[1], dx64[0], -du64[0] * dx64[1]);
                        T64 = (D == 2) ? t * rs64 : t * rsqrt(h264);
                    }
                    if constexpr (Needs::Q) {
                        Q64 = du64[0] * du64[0];
#pragma unroll
                        for (int d = 1; d < D; ++d) Q64 = fma(du64[d], du64[d], Q64);
                    }
                    double v64[NV];
                    eval_ops(OPS{}, L64, T64, Q64 - L64 * L64, Q64, D, a.gen, v64);
#pragma unroll
                    for (int o = 0; o < NV; ++o) v[o] = (float)v64[o];
                }
                const unsigned sb = __ballot_sync(FULL, slow);
                if (lane == 0) my_recheck += __popc(sb);
            }
            const int key = valid ? bin : a.nb + 1;
            hist.add(key, v, lane, warp);
        }
    }
    if (lane == 0 && my_recheck) atomicAdd(&s_recheck, my_recheck);
    hist.merge(a.g_sums, a.g_counts, a.nops, a.nb);
    if (threadIdx.x == 0 && s_recheck) atomicAdd(&a.g_stats[0], s_recheck);
}

// ================================================================================================
// Sphere 1D, FP64 (reference geodesic frame per pair)
// ================================================================================================
__device__ __forceinline__ void load_sph64(const double* X, int n, int i, SphPoint& P)
{
    P.p[0] = X[(size_t)0 * n + i]; P.p[1] = X[(size_t)1 * n + i]; P.p[2] = X[(size_t)2 * n + i];
    P.E[0] = X[(size_t)3 * n + i]; P.E[1] = X[(size_t)4 * n + i];
    P.N[0] = X[(size_t)5 * n + i]; P.N[1] = X[(size_t)6 * n + i]; P.N[2] = X[(size_t)7 * n + i];
}

template <int D, class OPS, int PRIV>
__global__ void __launch_bounds__(256) k_sphere1d_fp64(const PairArgs a)
{
    constexpr int NV = OPS::n;
    constexpr int NX = 8;  // p(3), E(2), N(3)
    using Hist = BlockHist<double, NV, PRIV>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x, NW = T >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.n;
    LutEntry64* lut = reinterpret_cast<LutEntry64*>(smem);
    double* sx = reinterpret_cast<double*>(smem + a.lut_bytes);  // NX * T
    double* su = sx + NX * T;                                     // D * T
    Hist hist;
    hist.init(reinterpret_cast<unsigned char*>(su + D * T), NW, a.nb + 2, a.hist_cols);
    for (int k = threadIdx.x; k < a.lut_bytes / (int)sizeof(LutEntry64); k += T)
        lut[k] = static_cast<const LutEntry64*>(a.lut)[k];

    int iter = 0;
    for (long long p = a.tp_lo + blockIdx.x; p < a.tp_hi; p += gridDim.x, ++iter) {
        hist.close_runs(lane);
        if (PRIV && iter && a.flush_every && iter % a.flush_every == 0) hist.fold();
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        SphPoint A;
        double uA[D];
        if (iv) load_sph64(a.X64, n, i, A);
        else { for (int k = 0; k < 3; ++k) { A.p[k] = 0.0; A.N[k] = 0.0; } A.E[0] = A.E[1] = 0.0; }
#pragma unroll
        for (int d = 0; d < D; ++d) uA[d] = iv ? a.U64[(size_t)d * n + i] : 0.0;
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        if ((int)threadIdx.x < jn) {
#pragma unroll
            for (int c = 0; c < NX; ++c) sx[c * T + threadIdx.x] = a.X64[(size_t)c * n + j0 + threadIdx.x];
#pragma unroll
            for (int d = 0; d < D; ++d) su[d * T + threadIdx.x] = a.U64[(size_t)d * n + j0 + threadIdx.x];
        }
        __syncthreads();
        const bool diag = ti == tj;
        auto pair = [&](int jj, int& key, double (&v)[NV]) {
            SphPoint B;
            B.p[0] = sx[0 * T + jj]; B.p[1] = sx[1 * T + jj]; B.p[2] = sx[2 * T + jj];
            B.E[0] = sx[3 * T + jj]; B.E[1] = sx[4 * T + jj];
            B.N[0] = sx[5 * T + jj]; B.N[1] = sx[6 * T + jj]; B.N[2] = sx[7 * T + jj];
            double r, tA[2], tB[2];
            const bool ok = x_sphere_frame(A, B, a.radius, r, tA, tB);
            int bin;
            if (a.dist_linear) bin = linear_bin(a.dlin, r);
            else bin = (r != r) ? a.n_edges : lut64_bin(lut, a, r);
            key = ok ? bin : a.nb + 1;
            double uB[D], du[D];
#pragma unroll
            for (int d = 0; d < D; ++d) uB[d] = su[d * T + jj];
            x_sphere_delta<D>(tA, tB, uA, uB, du);
            const double L = du[0], Tt = du[1];
            double Q = du[0] * du[0] + du[1] * du[1];
            if constexpr (D == 3) Q = fma(du[2], du[2], Q);
            eval_ops(OPS{}, L, Tt, Q - L * L, Q, D, a.gen, v);
        };
        if constexpr (Hist::RUN) {
            if (iv) {
                for (int jj = diag ? (int)threadIdx.x + 1 : 0; jj < jn; ++jj) {
                    int key;
                    double v[NV];
                    pair(jj, key, v);
                    hist.add(key, v, lane, warp);
                }
            }
        } else {
            for (int jj = 0; jj < jn; ++jj) {
                const bool valid = iv && (!diag || jj > (int)threadIdx.x);
                int key;
                double v[NV];
                pair(jj, key, v);
                hist.add(valid ? key : a.nb + 1, v, lane, warp);
            }
        }
    }
    hist.merge(a.g_sums, a.g_counts, a.nops, a.nb);
}

// ================================================================================================
// Sphere 1D, FP32 bulk + FP64 recheck.
//
// With d = q - p (chord vector) and s = p + q, the reference's transported increments reduce to
//   du_L = d . (U_B - U_A) / sin(sigma),  du_T = d . (W_B - W_A) / sin(sigma),
//   sin^2(sigma) = |d|^2 |s|^2 / 4,
// because t_A = d - (d.p) p and t_B = (d.p) q + d differ from d only along p and q, which are
// orthogonal to the tangent vectors U, W at their own point. The bin is decided on the chord
// |d|^2, which is monotone in the arc length, against the chord images of the edges. Per-point
// records are FP32 (hi, lo) pairs of the FP64 basis and velocities (p, U, W[, up]), so d, s and the
// velocity differences keep FP32 relative accuracy at every separation, including the antipode
// (|s| -> 0). Coincident, antipodal and near-edge pairs are recomputed with the reference frame in
// FP64.
// ================================================================================================
template <int D, class OPS, int PRIV>
__global__ void __launch_bounds__(256) k_sphere1d_mixed(const PairArgs a)
{
    constexpr int NV = OPS::n;
    using Needs = ListNeeds<OPS>;
    using Hist = BlockHist<float, NV, PRIV>;
    constexpr int NF = (D == 3) ? 20 : 18;  // (hi, lo) of p(3), U(3), W(3)[, up]
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x, NW = T >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.n;
    LutEntry32* lut = reinterpret_cast<LutEntry32*>(smem);
    float* sx = reinterpret_cast<float*>(smem + a.lut_bytes);  // NF * T
    __shared__ unsigned long long s_recheck;
    Hist hist;
    hist.init(smem + a.lut_bytes + (((size_t)NF * T * 4 + 15) & ~(size_t)15), NW, a.nb + 2, a.hist_cols);
    for (int k = threadIdx.x; k < a.lut_bytes / (int)sizeof(LutEntry32); k += T)
        lut[k] = static_cast<const LutEntry32*>(a.lut)[k];
    if (threadIdx.x == 0) s_recheck = 0ull;
    unsigned long long my_recheck = 0;

    int iter = 0;
    for (long long p = a.tp_lo + blockIdx.x; p < a.tp_hi; p += gridDim.x, ++iter) {
        hist.close_runs(lane);
        if (PRIV && iter && a.flush_every && iter % a.flush_every == 0) hist.fold();
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        float fa[NF];
#pragma unroll
        for (int c = 0; c < NF; ++c) fa[c] = iv ? a.XF[(size_t)c * n + i] : 0.f;
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        if ((int)threadIdx.x < jn) {
#pragma unroll
            for (int c = 0; c < NF; ++c) sx[c * T + threadIdx.x] = a.XF[(size_t)c * n + j0 + threadIdx.x];
        }
        __syncthreads();
        const bool diag = ti == tj;
        for (int jj = 0; jj < jn; ++jj) {
            const bool valid = iv && (!diag || jj > (int)threadIdx.x);
            float d[3], sv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                d[c] = df_diff<true>(sx, c, 3, T, jj, fa);
                sv[c] = __fadd_rn(__fadd_rn(sx[c * T + jj], fa[c]), __fadd_rn(sx[(3 + c) * T + jj], fa[3 + c]));
            }
            const float ch2 = fmaf(d[2], d[2], fmaf(d[1], d[1], d[0] * d[0]));
            const LutEntry32 e = lut[lut_cell32(ch2, a.lg)];
            int bin = e.base + (ch2 > e.hi ? (e.mult & 0xffff) : 0);
            bool slow = (e.mult & LUT_FLAG_SLOW) || (ch2 >= e.lo && ch2 <= e.hi);
            const float ss = fmaf(sv[2], sv[2], fmaf(sv[1], sv[1], sv[0] * sv[0]));
            const float inv_s = rsqrtf(0.25f * ch2 * ss);
            float L = 0.f, Tt = 0.f, Q = 0.f;
            {
                float dU[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) dU[c] = df_diff<true>(sx + 6 * T, c, 3, T, jj, fa + 6);
                L = fmaf(d[2], dU[2], fmaf(d[1], dU[1], d[0] * dU[0])) * inv_s;
            }
            if constexpr (Needs::T || Needs::Q) {
                float dW[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) dW[c] = df_diff<true>(sx + 12 * T, c, 3, T, jj, fa + 12);
                Tt = fmaf(d[2], dW[2], fmaf(d[1], dW[1], d[0] * dW[0])) * inv_s;
                Q = fmaf(Tt, Tt, L * L);
                if constexpr (D == 3) {
                    const float dw = df_diff<true>(sx + 18 * T, 0, 1, T, jj, fa + 18);
                    Q = fmaf(dw, dw, Q);
                }
            }
            float v[NV];
            eval_ops(OPS{}, L, Tt, Q - L * L, Q, D, a.gen, v);

            slow = slow && valid;
            bool ok = true;
            if (__any_sync(FULL, slow)) {
                if (slow) {
                    const int j = j0 + jj;
                    SphPoint A, B;
                    load_sph64(a.X64, n, i, A);
                    load_sph64(a.X64, n, j, B);
                    double r, tA[2], tB[2], uA[D], uB[D], du[D];
                    ok = x_sphere_frame(A, B, a.radius, r, tA, tB);
                    bin = sphere_exact_bin(a, r);
#pragma unroll
                    for (int dd = 0; dd < D; ++dd) {
                        uA[dd] = a.U64[(size_t)dd * n + i];
                        uB[dd] = a.U64[(size_t)dd * n + j];
                    }
                    x_sphere_delta<D>(tA, tB, uA, uB, du);
                    double Q64 = du[0] * du[0] + du[1] * du[1];
                    if constexpr (D == 3) Q64 = fma(du[2], du[2], Q64);
                    double v64[NV];
                    eval_ops(OPS{}, du[0], du[1], Q64 - du[0] * du[0], Q64, D, a.gen, v64);
#pragma unroll
                    for (int o = 0; o < NV; ++o) v[o] = (float)v64[o];
                }
                const unsigned sb = __ballot_sync(FULL, slow);
                if (lane == 0) my_recheck += __popc(sb);
            }
            const int key = (valid && ok) ? bin : a.nb + 1;
            hist.add(key, v, lane, warp);
        }
    }
    if (lane == 0 && my_recheck) atomicAdd(&s_recheck, my_recheck);
    hist.merge(a.g_sums, a.g_counts, a.nops, a.nb);
    if (threadIdx.x == 0 && s_recheck) atomicAdd(&a.g_stats[0], s_recheck);
}

}  // namespace sfb
