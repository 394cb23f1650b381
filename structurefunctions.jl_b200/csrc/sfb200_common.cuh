// sfb200_common.cuh -- device helpers shared by every pair kernel.
//
//  * bin lookup tables (LUTs) over the bit pattern of a non-negative key (r^2, r or chord^2);
//  * warp aggregation of per-pair contributions with __match_any_sync + a peer tree reduction,
//    so each histogram cell is updated once per warp step by one leader lane;
//  * upper-triangle tile-pair decoding.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/sfb200.h"

namespace sfb {

constexpr unsigned FULL = 0xffffffffu;

// ----------------------------------------------------------------------------------------------
// Bin lookup tables.
//
// A table covers keys by cells of equal width in log2 space: cell = (bits(key) >> shift) - base,
// clamped to [0, ncell - 1], where `shift` keeps `m` mantissa bits. Cell 0 also covers every key
// below its upper end (down to +0) and the last cell every key above its lower end (up to +inf and
// NaN). Edge keys are compared strictly: bin(key) = #{k : edge_k < key}, which is the reference's
// `searchsortedfirst(edges, key) - 1` for sorted edges (src/BinEdges.jl:517, 56).
//
// Exact table (FP64 kernels): each cell holds the number of edges below the cell, plus at most one
// distinct edge value `e` inside the cell with its multiplicity: bin = base + (key > e ? mult : 0).
// A cell with two or more distinct edge values is flagged and resolved by binary search.
//
// Window table (FP32 kernels): each edge k is widened to an interval [lo_k, hi_k] in FP32 that
// contains every FP32 key whose FP64 counterpart could fall on the other side of edge_k. A cell
// holds the number of intervals certainly below it and at most one interval inside it; a key inside
// that interval (or in a flagged cell) is recomputed in FP64.
// ----------------------------------------------------------------------------------------------

constexpr int LUT_SLOW = 1;  // resolve this cell by an exact FP64 recheck

struct LutEntry64 {   // 16 bytes
    int32_t base;     // edges strictly below the cell
    int32_t mult;     // multiplicity of `e` (0: no edge in the cell); LUT_SLOW flag in bit 30
    double e;         // the one distinct edge value inside the cell
};

struct LutEntry32 {   // 16 bytes
    int32_t base;     // intervals certainly below the cell
    int32_t mult;     // edges in the interval inside the cell; bit 30: slow cell
    float lo, hi;     // the interval inside the cell (NaN: none)
};

constexpr int32_t LUT_FLAG_SLOW = 1 << 30;

struct LutGeom {
    int32_t shift;    // 52 - m (FP64 keys) or 23 - m (FP32 keys)
    int32_t ncell;
    int64_t base;     // bits >> shift of the first cell's lower end
};

// FP64 key -> cell. shift = 52 - m >= 42, so the cell index lives in the high word of the key:
// (bits >> shift) == (hi >> (shift - 32)), and base < 2^22 fits 32-bit arithmetic.
__device__ __forceinline__ int lut_cell64(double key, const LutGeom& g)
{
    const int hi = __double2hiint(key) & 0x7fffffff;
    int c = (hi >> (g.shift - 32)) - (int)g.base;
    c = max(c, 0);
    c = min(c, g.ncell - 1);
    return c;
}

__device__ __forceinline__ int lut_cell32(float key, const LutGeom& g)
{
    const uint32_t bits = __float_as_uint(key) & 0x7fffffffu;
    int c = (int)(bits >> g.shift) - (int)g.base;
    c = max(c, 0);
    c = min(c, g.ncell - 1);
    return c;
}

// Byte table (flat FP64 kernels): one byte per quarter octave of the key over the whole FP64
// range, indexed by the key's high word with no clamping: cell = (hi & 0x7fffffff) >> 18 (11
// exponent bits and the top 2 mantissa bits; 8192 cells). A cell holds b = the number of edges
// strictly below the cell's lower end, and the cell contains at most one edge, sqx[b] (the padded
// edge table: sqx[k] = edge k for k < n_edges, +inf above), so that
//     bin(key) = #{k : edge_k < key} = b + (key > sqx[b]).
// Cells with two or more edges, a repeated edge, or keys the FP32 arithmetic of the mixed kernels
// must not see (outside [2^-100, 2^100], NaN, infinity) hold kByteSlow: the pair takes the exact
// out-of-line route. The table lives in shared memory beside the 256-entry padded edge array.
constexpr int kByteCells = 8192;
constexpr int kByteEdges = 256;     // padded edge array entries (n_edges <= 254)
constexpr unsigned kByteSlow = 255u;

__device__ __forceinline__ int byte_bin(const unsigned char* lut8, const double* sqx, double key, bool& slow)
{
    const unsigned c = ((unsigned)__double2hiint(key) & 0x7fffffffu) >> 18;
    const unsigned b = lut8[c];
    slow = b == kByteSlow;
    return (int)b + (key > sqx[b] ? 1 : 0);
}

// Exact count of table entries strictly below key (binary search; `tab` sorted, n entries).
__device__ __forceinline__ int count_below(const double* __restrict__ tab, int n, double key)
{
    int lo = 0, hi = n;  // answer in [lo, hi]
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (tab[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// count_below kept out of line, for the rare table cells that hold more than one edge: the pair
// loops only branch to it.
static __device__ __noinline__ int count_below_ool(const double* __restrict__ tab, int n, double key)
{
    return count_below(tab, n, key);
}

// LinearBinEdges search, src/BinEdges.jl:114-131, returning the bin (searchsortedfirst - 1).
// NaN keys return n (out of range); the reference throws there.
struct LinearParams {
    double first, last, inv_step, step, neg_f_inv;
    int32_t n;  // number of edges
};

__device__ __forceinline__ int linear_bin(const LinearParams& p, double x)
{
    if (x <= p.first) return 0;
    if (x > p.last) return p.n;
    if (x != x) return p.n;
    const double t = __fma_rn(x, p.inv_step, p.neg_f_inv);
    long long idx = (long long)floor(t) + 1;
    idx = idx < 1 ? 1 : idx;
    idx = idx > p.n ? p.n : idx;
    const double u = __fma_rn((double)(idx - 1), p.step, p.first);
    return (int)(u < x ? idx : idx - 1);
}

// ----------------------------------------------------------------------------------------------
// Warp aggregation.
//
// `peers` is the set of lanes holding the same histogram cell (from __match_any_sync). After the
// call the lowest lane of each peer group holds the group's sum of every value in v[]. Tree
// reduction over the peers in lane order: in round k the lanes whose rank among their peers is a
// multiple of 2^k add the partial of the next surviving peer; at most ceil(log2(group)) rounds.
// All 32 lanes must call it (full-warp shuffles).
// ----------------------------------------------------------------------------------------------
template <int NV, typename T>
__device__ __forceinline__ void reduce_peers(unsigned peers, int lane, T (&v)[NV])
{
    const unsigned below = (1u << lane) - 1u;
    int rank = __popc(peers & below);
    unsigned pending = peers & ~below & ~(1u << lane);  // higher peers still holding a partial
    while (__any_sync(FULL, pending != 0u)) {
        const int next = __ffs(pending);
        const int src = next ? next - 1 : lane;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const T t = __shfl_sync(FULL, v[k], src);
            if (next) v[k] += t;
        }
        const unsigned done = __ballot_sync(FULL, rank & 1);
        pending &= ~done;
        rank >>= 1;
    }
}

// Knuth two-sum accumulation into a (hi, lo) FP32 pair: hi + lo tracks the exact running sum to
// about 2^-48 relative.
__device__ __forceinline__ void two_sum_acc(float& hi, float& lo, float v)
{
    const float s = __fadd_rn(hi, v);
    const float bp = __fsub_rn(s, hi);
    const float ap = __fsub_rn(s, bp);
    const float e = __fadd_rn(__fsub_rn(hi, ap), __fsub_rn(v, bp));
    hi = s;
    lo = __fadd_rn(lo, e);
}

// ----------------------------------------------------------------------------------------------
// Upper-triangle tile pairs: p in [0, nt(nt+1)/2) -> (ti <= tj), row-major by ti.
// ----------------------------------------------------------------------------------------------
__device__ __forceinline__ void decode_tile_pair(long long p, int nt, int& ti, int& tj)
{
    const double b = 2.0 * nt + 1.0;
    long long r = (long long)((b - sqrt(b * b - 8.0 * (double)p)) * 0.5);
    auto row_start = [nt](long long i) { return i * (long long)nt - (i * (i - 1)) / 2; };
    if (r < 0) r = 0;
    if (r > nt - 1) r = nt - 1;
    while (r > 0 && row_start(r) > p) --r;
    while (r < nt - 1 && row_start(r + 1) <= p) ++r;
    ti = (int)r;
    tj = (int)(r + (p - row_start(r)));
}

}  // namespace sfb
