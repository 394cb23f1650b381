// sfb200_prep.cuh -- per-run preparation kernels: input packing (column-major caller arrays ->
// SoA, FP32 images, spherical bases), the coordinate bound, the FP32 window table, and the copy of
// the accumulated histogram into caller device buffers.
#pragma once

#include "sfb200_common.cuh"
#include "sfb200_sphmath.h"

namespace sfb {

// Block maxima of two non-negative doubles, folded into bound[0], bound[1] with integer atomicMax
// (non-negative IEEE doubles order like their bit patterns). Call once per block, all threads.
__device__ __forceinline__ void block_max2_to(double vx, double vu, unsigned long long* bound)
{
    __shared__ double red[2][32];
    for (int o = 16; o > 0; o >>= 1) {
        vx = fmax(vx, __shfl_xor_sync(FULL, vx, o));
        vu = fmax(vu, __shfl_xor_sync(FULL, vu, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[0][warp] = vx; red[1][warp] = vu; }
    __syncthreads();
    if (warp == 0) {
        const bool in = lane < (int)(blockDim.x >> 5);
        vx = in ? red[0][lane] : 0.0;
        vu = in ? red[1][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            vx = fmax(vx, __shfl_xor_sync(FULL, vx, o));
            vu = fmax(vu, __shfl_xor_sync(FULL, vu, o));
        }
        if (lane == 0 && vx > 0.0) atomicMax(&bound[0], (unsigned long long)__double_as_longlong(vx));
        if (lane == 0 && vu > 0.0) atomicMax(&bound[1], (unsigned long long)__double_as_longlong(vu));
    }
}

// ---------------------------------------------------------------- spatial order of the points
//
// The pair kernels visit the j of a tile in storage order. Storing the points along a Morton
// (Z-order) curve makes consecutive j spatial neighbours, so the distance from a fixed i changes
// slowly along the loop and the run-length histogram mostly extends runs. The order never changes
// which pairs are formed (each unordered pair is still visited once) and every pair quantity used
// for binning is symmetric in the two points, so counts are unchanged; only the summation order of
// the sums differs.

// Unsigned image of a float that orders like the float (for integer atomicMin / atomicMax).
__device__ __forceinline__ unsigned float_order_key(float f)
{
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float float_from_order_key(unsigned k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Per-dimension bounding box of the Morton coordinates, as order keys: box[0..2] minima (start at
// 0xffffffff), box[3..5] maxima (start at 0). Flat: the D coordinates; sphere: the unit vector.
template <typename TX>
__device__ __forceinline__ int morton_coords(const TX* __restrict__ x, int i, int W, bool sphere, int unit, float* c)
{
    if (!sphere) {
        for (int d = 0; d < W; ++d) c[d] = (float)x[(size_t)W * i + d];
        return W;
    }
    float lon = (float)x[(size_t)2 * i], lat = (float)x[(size_t)2 * i + 1];
    if (unit == SFB200_ANGLE_DEG) {
        lon *= 0.017453292519943295f;
        lat *= 0.017453292519943295f;
    }
    float sl, cl, sp, cp;
    sincosf(lon, &sl, &cl);
    sincosf(lat, &sp, &cp);
    c[0] = cp * cl;
    c[1] = cp * sl;
    c[2] = sp;
    return 3;
}

template <typename TX>
__global__ void k_morton_box(const TX* __restrict__ x, int n, int W, int sphere, int unit, unsigned* box)
{
    __shared__ unsigned smin[3], smax[3];
    if (threadIdx.x < 3) { smin[threadIdx.x] = 0xffffffffu; smax[threadIdx.x] = 0u; }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        float c[3];
        const int nd = morton_coords(x, i, W, sphere != 0, unit, c);
        for (int d = 0; d < nd; ++d) {
            if (c[d] != c[d]) continue;  // NaN coordinates do not widen the box
            const unsigned k = float_order_key(c[d]);
            atomicMin(&smin[d], k);
            atomicMax(&smax[d], k);
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&box[threadIdx.x], smin[threadIdx.x]);
        atomicMax(&box[3 + threadIdx.x], smax[threadIdx.x]);
    }
}

// Spread the low 16 bits of v to the even bit positions / the low 10 bits to every third position.
__device__ __forceinline__ unsigned spread2(unsigned v)
{
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
__device__ __forceinline__ unsigned spread3(unsigned v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Morton key and identity index of every point (points with a NaN coordinate sort last).
template <typename TX>
__global__ void k_morton_keys(const TX* __restrict__ x, int n, int W, int sphere, int unit, const unsigned* box,
                              unsigned* keys, int* idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float c[3];
    const int nd = morton_coords(x, i, W, sphere != 0, unit, c);
    const int bits = nd == 2 ? 16 : 10;
    const float top = (float)((1 << bits) - 1);
    unsigned q[3] = {0u, 0u, 0u};
    bool nan = false;
    for (int d = 0; d < nd; ++d) {
        const float lo = float_from_order_key(box[d]), hi = float_from_order_key(box[3 + d]);
        const float ext = hi - lo;
        if (c[d] != c[d]) { nan = true; continue; }
        const float t = ext > 0.f ? (c[d] - lo) / ext * top : 0.f;
        q[d] = (unsigned)fminf(fmaxf(t, 0.f), top);
    }
    unsigned key;
    if (nan) key = 0xffffffffu;
    else if (nd == 2) key = spread2(q[0]) | (spread2(q[1]) << 1);
    else key = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
    keys[i] = key;
    idx[i] = i;
}

// Scattered order: slot i holds point (i * mult) mod n, mult coprime to n (a bijection). Used by the
// joint histograms, whose threads should hit unrelated cells: with neighbouring points in
// neighbouring lanes (gridded input, or the Morton order) a warp's lanes often update the same cell
// at once, and shared-memory atomics to one address serialise.
__global__ void k_scatter_perm(int n, unsigned long long mult, int* perm)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = (int)(((unsigned long long)i * mult) % (unsigned long long)n);
}

// FP32 image of an FP64 value as (hi, lo): hi = fl32(v), lo = fl32(v - hi); hi + lo equals v to
// about 2^-48 relative.
__device__ __forceinline__ void split_df(double v, float& hi, float& lo)
{
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

template <typename TX, typename TU>
__global__ void k_pack_flat(const TX* __restrict__ x, const TU* __restrict__ u, int n, int D, int df,
                            const int* __restrict__ perm, double* X64, double* U64, float* XF, float* UF,
                            unsigned long long* bound)
{
    // with df, every FP32 value is stored as (hi, lo) (lo = 0 for FP32 inputs); slot i holds caller
    // point perm[i] (the identity without a permutation)
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mx = 0.0, mu = 0.0;
    if (i < n) {
        const size_t src = perm ? (size_t)perm[i] : (size_t)i;
        for (int d = 0; d < D; ++d) {
            const double xv = (double)x[(size_t)D * src + d];
            const double uv = (double)u[(size_t)D * src + d];
            X64[(size_t)d * n + i] = xv;
            U64[(size_t)d * n + i] = uv;
            if (XF) {
                float h, l;
                split_df(xv, h, l);
                XF[(size_t)d * n + i] = h;
                if (df) XF[(size_t)(D + d) * n + i] = l;
                split_df(uv, h, l);
                UF[(size_t)d * n + i] = h;
                if (df) UF[(size_t)(D + d) * n + i] = l;
            }
            mx = fmax(mx, fabs(xv));  // fmax ignores NaN coordinates
            mu = fmax(mu, fabs(uv));
        }
    }
    block_max2_to(mx, mu, bound);
}

// Sphere: lon/lat -> p, E, N in FP64 with the shared degree-exact sincos (identical to the CPU
// check), velocities as given; FP32 images p, U = u_e E + u_n N, W = u_n E - u_e N, [up].
template <typename TX, typename TU>
__global__ void k_pack_sphere(const TX* __restrict__ x, const TU* __restrict__ u, int n, int D,
                              int unit, const int* __restrict__ perm, double* X64, double* U64, float* XF,
                              double* XM, unsigned long long* bound)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t src = (i < n && perm) ? (size_t)perm[i] : (size_t)i;
    double mu = 0.0;
    if (i < n) {
        for (int d = 0; d < D; ++d) mu = fmax(mu, fabs((double)u[(size_t)D * src + d]));
    }
    block_max2_to(1.0, mu, bound);
    if (i >= n) return;
    const double lon = (double)x[(size_t)2 * src], lat = (double)x[(size_t)2 * src + 1];
    double sl, cl, sp, cp;
    if (unit == SFB200_ANGLE_DEG) {
        sfb_sincosd(lon, &sl, &cl);
        sfb_sincosd(lat, &sp, &cp);
    } else {
        sfb_sincos(lon, &sl, &cl);
        sfb_sincos(lat, &sp, &cp);
    }
    const double p0 = SFB_MUL(cp, cl), p1 = SFB_MUL(cp, sl), p2 = sp;
    const double E0 = -sl, E1 = cl;
    const double N0 = SFB_MUL(-sp, cl), N1 = SFB_MUL(-sp, sl), N2 = cp;
    const double c[8] = {p0, p1, p2, E0, E1, N0, N1, N2};
    for (int k = 0; k < 8; ++k) X64[(size_t)k * n + i] = c[k];
    double uv[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < D; ++d) {
        uv[d] = (double)u[(size_t)D * src + d];
        U64[(size_t)d * n + i] = uv[d];
    }
    if (XM) {
        // FP64 records: p at 0..2, U at 3..5, W at 6..8, up at 9
        const double ue = uv[0], un = uv[1];
        const double m[10] = {p0, p1, p2, ue * E0 + un * N0, ue * E1 + un * N1, un * N2,
                              un * E0 - ue * N0, un * E1 - ue * N1, -ue * N2, uv[2]};
        for (int k = 0; k < 9 + (D == 3); ++k) XM[(size_t)k * n + i] = m[k];
    }
    if (XF) {
        // records of (hi, lo) pairs: p at 0..5, U at 6..11, W at 12..17, up at 18..19
        const double ue = uv[0], un = uv[1];
        const double P[3] = {p0, p1, p2};
        const double U[3] = {ue * E0 + un * N0, ue * E1 + un * N1, un * N2};
        const double W[3] = {un * E0 - ue * N0, un * E1 - ue * N1, -ue * N2};
        for (int k = 0; k < 3; ++k) {
            float h, l;
            split_df(P[k], h, l);
            XF[(size_t)k * n + i] = h;
            XF[(size_t)(3 + k) * n + i] = l;
            split_df(U[k], h, l);
            XF[(size_t)(6 + k) * n + i] = h;
            XF[(size_t)(9 + k) * n + i] = l;
            split_df(W[k], h, l);
            XF[(size_t)(12 + k) * n + i] = h;
            XF[(size_t)(15 + k) * n + i] = l;
        }
        if (D == 3) {
            float h, l;
            split_df(uv[2], h, l);
            XF[(size_t)18 * n + i] = h;
            XF[(size_t)19 * n + i] = l;
        }
    }
}

// Window parameters of the FP32 key: |key32 - key64| <= A |c| + B sqrt|c| + C near an edge key c.
// B and C carry the rounding of FP64 coordinates to FP32 and scale with the coordinate bound M
// (from the pack kernel) as B = Bm * M, C = Cm * M^2; `short_rel` marks keys below (short_rel*M)^2
// (flat) or below `short_key` (sphere) for FP64 recomputation; keys above `anti_key` likewise.
struct WindowParams {
    double A, Bm, Cm;
    int use_bound;       // 1: M from the pack kernel; 0: M = 1
    double short_rel;    // flat: short pairs have r < short_rel * M (0: none)
    double short_key;    // sphere: absolute key threshold
    double anti_key;     // keys above this are recomputed (sphere near-antipodal); +inf: none
};

// One thread per cell: certain-below count, the single overlapping edge interval, slow flags.
__global__ void k_build_lut32(const double* __restrict__ ck, int nk, WindowParams wp, LutGeom g,
                              const unsigned long long* bound_bits, LutEntry32* out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.ncell) return;
    const double M = wp.use_bound ? __longlong_as_double((long long)*bound_bits) : 1.0;
    const double B = wp.Bm * M, C = wp.Cm * M * M;
    auto lo_of = [&](int k) {
        const double v = ck[k];
        const double w = 2.0 * (wp.A * fabs(v) + B * sqrt(fabs(v)) + C);
        return v - w;
    };
    auto hi_of = [&](int k) {
        const double v = ck[k];
        const double w = 2.0 * (wp.A * fabs(v) + B * sqrt(fabs(v)) + C);
        return v + w;
    };
    const int sh = g.shift;
    const double Klo = (c == 0) ? 0.0
        : (double)__uint_as_float((unsigned)((g.base + c) << sh));
    const double Khi = (c == g.ncell - 1) ? __longlong_as_double(0x7ff0000000000000ll)
        : (double)__uint_as_float((unsigned)((g.base + c + 1) << sh));
    // first k with hi_k >= Klo  (intervals before it are certainly below the cell)
    int lo = 0, hi = nk;
    while (lo < hi) { const int m = (lo + hi) >> 1; if (hi_of(m) < Klo) lo = m + 1; else hi = m; }
    const int k0 = lo;
    // first k with lo_k >= Khi (intervals from it on are certainly above the cell)
    lo = k0; hi = nk;
    while (lo < hi) { const int m = (lo + hi) >> 1; if (lo_of(m) < Khi) lo = m + 1; else hi = m; }
    const int k1 = lo;
    LutEntry32 e;
    e.base = k0;
    e.mult = 0;
    e.lo = __int_as_float(0x7fc00000);
    e.hi = __int_as_float(0x7fc00000);
    if (k1 > k0) {
        if (ck[k0] == ck[k1 - 1]) {
            e.mult = k1 - k0;
            e.lo = __double2float_rd(lo_of(k0));
            e.hi = __double2float_ru(hi_of(k0));
        } else {
            e.mult = LUT_FLAG_SLOW;
        }
    }
    double short_key = wp.short_key;
    if (wp.short_rel > 0.0) short_key = (wp.short_rel * M) * (wp.short_rel * M);
    if (Klo < short_key || Khi > wp.anti_key) e.mult |= LUT_FLAG_SLOW;
    out[c] = e;
}

// Joint FP32 kernels: half-width, in value-bin index units, of the band around a value edge inside
// which the FP32 value may sit on the other side of the FP64 value. Per distance row b the pair
// separation is at least sqrt(row_key_lo[b]) (r for flat, chord for sphere), which bounds the
// direction error; |du| is bounded by 2 sqrt(3) max|u|. For an operator of order k the value error
// is k |du|_max^(k-1) times the increment error. Rows 0 and nd+1 are out of range.
struct ValueWindowParams {
    int nd;
    int D;
    int order;
    int sphere;
    int x_f64;
    int u_f64;
    int df;           // (hi, lo) records: input rounding is u^2, not u
    int l_only;       // value depends on du_L only, computed with a compensated dot product
    double inv_step;  // value bins: 1/step
    double neg_f_inv; // -first/step
};

__global__ void k_value_windows(const double* __restrict__ row_key_lo, ValueWindowParams p,
                                const unsigned long long* bound, float* out)
{
    const double u32 = 0x1p-24;
    const double M = p.sphere ? 1.0 : __longlong_as_double((long long)bound[0]);
    const double U = __longlong_as_double((long long)bound[1]);
    for (int b = threadIdx.x; b < p.nd + 2; b += blockDim.x) {
        if (b == 0 || b == p.nd + 1) { out[b] = 3.0e38f; continue; }
        const double rlo = sqrt(fmax(row_key_lo[b], 0.0));
        const double rin = p.df ? u32 * u32 : u32;  // rounding of the stored inputs
        const double pos_err = (p.x_f64 || p.sphere) ? 2.0 * sqrt((double)p.D) * M * rin : 0.0;
        const double arith = p.l_only ? 0.0 : (p.D + 8) * u32;  // relative part handled per pair when l_only
        const double eps_dir = (rlo > 0.0 ? pos_err / rlo : (pos_err > 0.0 ? 1e30 : 0.0)) + arith;
        const double U2 = 2.0 * sqrt(3.0) * U;
        const double eps_L = U2 * eps_dir + (p.u_f64 ? 2.0 * sqrt(3.0) * U * rin : 0.0) + (p.l_only ? 0.0 : U2 * 8.0 * u32);
        double scale = 1.0;
        for (int k = 1; k < p.order; ++k) scale *= U2;
        const double wv = 4.0 * (p.order > 0 ? p.order : 1) * scale * eps_L;
        const double wt = wv * fabs(p.inv_step) + 4.0 * fabs(p.neg_f_inv) * u32 + 1e-6;
        out[b] = (float)fmin(wt, 3.0e38);
    }
}

// Smallest and largest pair key over all pairs i < j of the packed points: r^2 (flat; the reference's
// left-to-right sum of squared differences) or the squared chord |q - p|^2 of the unit position
// vectors (sphere). Tile pairs of 256 points as the pair kernels; each thread keeps its row's range,
// each warp reduces, and lane 0 folds it into out[0] (min) / out[1] (max) with 64-bit integer
// atomics on the keys' bit patterns (keys are >= 0, whose IEEE bits order like the values). NaN keys
// are skipped (fmin / fmax), as the reference's `<` comparisons skip them. out must hold +inf / 0.
template <int NC, bool SPHERE>
__global__ void __launch_bounds__(256) k_key_range(const double* __restrict__ X64, int n, int ntiles, long long ntp,
                                                   unsigned long long* out)
{
    __shared__ double sx[NC * 256];
    const int t = threadIdx.x;
    double mn = INFINITY, mx = 0.0;
    for (long long p = blockIdx.x; p < ntp; p += gridDim.x) {
        int ti, tj;
        decode_tile_pair(p, ntiles, ti, tj);
        const int i = ti * 256 + t;
        const bool iv = i < n;
        double xi[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) xi[c] = iv ? X64[(size_t)c * n + i] : 0.0;
        __syncthreads();
        const int j0 = tj * 256;
        const int jn = min(256, n - j0);
        if (t < jn) {
#pragma unroll
            for (int c = 0; c < NC; ++c) sx[c * 256 + t] = X64[(size_t)c * n + j0 + t];
        }
        __syncthreads();
        if (iv) {
            for (int jj = (ti == tj) ? t + 1 : 0; jj < jn; ++jj) {
                double k = 0.0;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const double d = __dsub_rn(sx[c * 256 + jj], xi[c]);
                    k = (c == 0) ? __dmul_rn(d, d) : __dadd_rn(k, __dmul_rn(d, d));
                }
                mn = fmin(mn, k);
                mx = fmax(mx, k);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((t & 31) == 0) {
        atomicMin(&out[0], (unsigned long long)__double_as_longlong(mn));
        atomicMax(&out[1], (unsigned long long)__double_as_longlong(mx));
    }
}


// Device outputs: out = (accumulate ? out : 0) + accumulated histogram.
__global__ void k_finalize(const double* __restrict__ s, const unsigned long long* __restrict__ c,
                           long long ns, long long nc, double* out_s, unsigned long long* out_c,
                           int accumulate)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ns) out_s[k] = (accumulate ? out_s[k] : 0.0) + s[k];
    if (k < nc) out_c[k] = (accumulate ? out_c[k] : 0ull) + c[k];
}

}  // namespace sfb
