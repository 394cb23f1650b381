// sfb200_mixed.cuh -- the mixed-precision pair kernels (precision SFB200_PREC_MIXED).
//
// Split of the arithmetic:
//   FP64  every difference of two points (dx, du; the sphere's chord d = q - p, s = p + q and the
//         tangent-velocity differences), the squared distance that decides the bin, and the dot /
//         cross-product numerators of the projections (p = dx . du, the cross product dx x du).
//         The differences are then exact to a rounding, so the numerators keep full relative
//         accuracy even when the projection cancels (du nearly perpendicular to r): a pair's value
//         is accurate to a few FP32 ulps relative to itself, which keeps every bin within the
//         1e-6 per-bin tolerance down to bins holding a single pair.
//   FP32  the normalisation by 1/r (rsqrtf), every operator power, and the accumulation (per-lane
//         run sums folded into the block FP64 histogram, see sfb200_acc.cuh).
// The flat squared distance is computed exactly as the reference (left to right, no contraction),
// so the bin comes from the exact FP64 table and no pair is rechecked. The sphere bins on the FP64
// chord |q - p|^2 against the chord images of the edges and recomputes with the reference frame
// in FP64 the pairs within 2^-40 (relative) of an edge image, near-coincident and near-antipodal
// pairs. Transverse quantities avoid Q - L^2: T2 is |dx x du|^2 / r^2 (3D) or T^2 (2D), and Q is
// L^2 + T2.
#pragma once

#include "sfb200_joint.cuh"

namespace sfb {

// FP32 image of an FP64 value (round to nearest).
__device__ __forceinline__ float f32(double v) { return __double2float_rn(v); }

// Loads `NP` double2 from shared memory into r[2 * NP].
template <int NP>
__device__ __forceinline__ void load_rec2(const double* base, double (&r)[2 * NP])
{
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        const double2 t = reinterpret_cast<const double2*>(base)[q];
        r[2 * q] = t.x;
        r[2 * q + 1] = t.y;
    }
}

// Velocity scale: velocities are multiplied by us = 2^-ku (exact) when they are loaded, with
// |u| us <= 1 from the pack kernel's bound, so every FP32 value is of order one: an operator of order
// k then carries us^k, removed exactly at the merge. Coordinates are not scaled (the squared distance
// decides the bin and stays the reference's); pairs whose squared distance leaves [2^-100, 2^100]
// (and, for the 3D transverse direction, whose horizontal part does) are evaluated in FP64.
__device__ __forceinline__ int pow2_exponent_above(unsigned long long bound_bits)
{
    // smallest k with bound <= 2^k (0 for a zero or non-finite bound)
    const double b = __longlong_as_double((long long)bound_bits);
    if (!(b > 0.0) || !(b < 1e300)) return 0;
    int e;
    const double m = frexp(b, &e);  // b = m 2^e, m in [0.5, 1)
    return m == 0.5 ? e - 1 : e;
}

// Order of operator K (its sums scale as us^order).
template <int K>
__device__ __forceinline__ int op_order_of(const sfb200_operator& g)
{
    if constexpr (K == OC_L1) return 1;
    else if constexpr (K == OC_L2 || K == OC_T2 || K == OC_S2 || K == OC_T2C) return 2;
    else if constexpr (K == OC_L3 || K == OC_T3 || K == OC_S3 || K == OC_L1T2 || K == OC_L2T1 || K == OC_L1T2C) return 3;
    else {
        switch (g.kind) {
        case SFB200_OP_PROJECTED: return g.nl + g.nt;
        case SFB200_OP_S2: case SFB200_OP_T2C: return 2;
        case SFB200_OP_S3: case SFB200_OP_L1T2C: return 3;
        case SFB200_OP_FULLVEC: return g.nf;
        case SFB200_OP_SP2D: return g.nl < 3 ? 2 : 3;
        }
        return 0;
    }
}

template <int... K>
__device__ __forceinline__ void op_unscale(OpList<K...>, const GenOps& g, int ku, double (&sc)[sizeof...(K)])
{
    int k = 0;
    ((sc[k] = ldexp(1.0, ku * op_order_of<K>(g.op[k])), ++k), ...);
}

__device__ __forceinline__ bool f32_range_ok(float v) { return v >= 0x1p-100f && v <= 0x1p100f; }

// A finite FP32 number that is zero or normal (not subnormal, infinite or NaN). Written out with
// comparisons: the C library's isnormal has no device implementation.
__device__ __forceinline__ bool f32_zero_or_normal(float v)
{
    const float m = fabsf(v);
    return m == 0.f || (m >= 0x1p-126f && m <= 0x1.fffffep127f);
}

// Approximate reciprocal square root (rsqrt.approx) for arguments known to be normal: no
// denormal handling is needed around it.
__device__ __forceinline__ float rsqrt_normal(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Per-pair FP32 primitives of a flat pair from FP64 differences (du already scaled by us).
// Returns false when the pair must be evaluated in FP64 because its horizontal squared distance (the
// 3D transverse direction) leaves FP32's range; the caller checks r^2 itself (the byte table routes
// such keys out of line already).
template <int D, class OPS>
__device__ __forceinline__ bool flat_primitives_mx(const double (&dx)[D], const double (&du)[D], double r2, double h2,
                                                   float& L, float& Tt, float& T2, float& Q)
{
    using N = ListNeeds2<OPS>;
    const float r2f = f32(r2);
    bool fine = true;
    const float rs = rsqrt_normal(r2f);
    L = 0.f;
    Tt = 0.f;
    T2 = 0.f;
    Q = 0.f;
    double p = 0.0;
    if constexpr (N::L || N::T2 || N::Q) {
        p = dx[0] * du[0];
#pragma unroll
        for (int d = 1; d < D; ++d) p = fma(dx[d], du[d], p);
        L = f32(p) * rs;
    }
    // cz = (dx x du)_z: the signed transverse numerator in 2D and 3D (n_hat = z_hat x r_hat)
    double cz = 0.0;
    if constexpr (N::T || (D == 2 && (N::T2 || N::Q))) cz = fma(dx[0], du[1], -(dx[1] * du[0]));
    if constexpr (D == 2) {
        if constexpr (N::T || N::T2 || N::Q) {
            Tt = f32(cz) * rs;
            T2 = Tt * Tt;
        }
    } else {
        if constexpr (N::T) {
            const float h2f = f32(h2);
            fine = fine && f32_range_ok(h2f);
            Tt = f32(cz) * rsqrt_normal(h2f);
        }
        if constexpr (N::T2 || N::Q) {
            // |dx x du|^2 = |dx|^2 |du|^2 - (dx . du)^2 (Lagrange), in FP64
            double q = du[0] * du[0];
#pragma unroll
            for (int d = 1; d < D; ++d) q = fma(du[d], du[d], q);
            const double c2 = fma(q, r2, -(p * p));
            T2 = f32(c2) * (rs * rs);
        }
    }
    if constexpr (N::Q) Q = fmaf(L, L, T2);
    return fine;
}

// FP64 values of a flat pair (the FP64 kernel's formulas) rounded to FP32; du already scaled.
template <int D, class OPS>
__device__ __forceinline__ void flat_values_fp64(const double (&dx)[D], const double (&du)[D], double r2, double h2,
                                                 const GenOps& g, float (&v)[OPS::n])
{
    constexpr int NV = OPS::n;
    const double rs = rsqrt(r2);
    double pp = dx[0] * du[0];
#pragma unroll
    for (int d = 1; d < D; ++d) pp = fma(dx[d], du[d], pp);
    const double L = pp * rs;
    const double t = fma(du[1], dx[0], -du[0] * dx[1]);
    const double Tt = (D == 2) ? t * rs : t * rsqrt(h2);
    double Q = du[0] * du[0];
#pragma unroll
    for (int d = 1; d < D; ++d) Q = fma(du[d], du[d], Q);
    double v64[NV];
    eval_ops(OPS{}, L, Tt, Q - L * L, Q, D, g, v64);
#pragma unroll
    for (int o = 0; o < NV; ++o) v[o] = f32(v64[o]);
}

// flat_values_fp64 out of line (pairs with r^2 outside the FP32 range are rare): scalar arguments,
// the operator descriptors read in place from the kernel parameters (grid constants).
template <int D, class OPS>
struct FlatValues {
    float v[OPS::n];
};

template <int D, class OPS>
__device__ __noinline__ FlatValues<D, OPS> flat_values_fp64_ool(double dx0, double dx1, double dx2, double du0,
                                                                double du1, double du2, double r2, double h2,
                                                                const GenOps* g)
{
    double dx[D], du[D];
    dx[0] = dx0;
    dx[1] = dx1;
    du[0] = du0;
    du[1] = du1;
    if constexpr (D == 3) {
        dx[2] = dx2;
        du[2] = du2;
    }
    FlatValues<D, OPS> r;
    flat_values_fp64<D, OPS>(dx, du, r2, h2, *g, r.v);
    return r;
}

// The LinearBinEdges search of a flat pair on its correctly rounded distance sqrt(r2), kept out of line
// (the mixed kernels take it only for pairs near an edge); NaN keys fall out of range.
static __device__ __noinline__ int linear_bin_sqrt_ool(const LinearParams* p, double r2)
{
    return (r2 != r2) ? p->n : linear_bin(*p, SFB_SQRT(r2));
}

// ================================================================================================
// Flat (Euclidean) 1D
//
// The run-length histogram (PRIV 3) needs no warp-synchronous step, so each lane walks its own
// range of j (j > i on a diagonal tile) and no pair is masked; the other histogram modes step the
// warp in lockstep with out-of-range pairs sent to the dropped row.
// ================================================================================================
// SINGLE: the single-run kernel (J-tile sorting and the byte table compiled in); the batched kernel
// leaves both out, so that its tighter register budget (four blocks per SM) holds without spills.
// LIN: compiled for a LinearBinEdges distance axis (the bin from the FP32 distance, the FP64 search
// near an edge); the other forms take the FP64 search for every pair of such an axis.
template <int D, class OPS, int PRIV, bool SINGLE = true, bool LIN = false>
__device__ __forceinline__ void flat1d_mx_run(const PairArgs& a, long long p0, long long p1, long long ps)
{
    constexpr int NV = OPS::n;
    constexpr int NP = D;  // double2 per j record: x(D) u(D)
    using Hist = BlockHist<float, NV, PRIV>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x, NW = T >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.n;
    const LutEntry64* lut = reinterpret_cast<const LutEntry64*>(smem);
    const unsigned char* lut8 = smem;
    const double* sqx = reinterpret_cast<const double*>(smem + kByteCells);
    double* srec = reinterpret_cast<double*>(smem + a.lut_bytes);  // T records of 2D doubles
    // the tile sort's counters (only when this launch sorts), then the histogram
    unsigned* s_cnt = reinterpret_cast<unsigned*>(srec + (size_t)2 * NP * T);
    unsigned* s_wtot = s_cnt + 256;
    Hist hist;
    hist.init(reinterpret_cast<unsigned char*>(s_cnt) + (a.sort_j ? kSortScratchBytes : 0), NW, a.nb + 2, a.hist_cols);
    load_bin_table(a, smem);
    const int ku = pow2_exponent_above(a.g_stats[2]);
    const double us = ldexp(1.0, -ku);
    // LinearBinEdges distance axis: FP32 images of the search's scale and offset, and the last index
    const float linv = (float)a.dlin.inv_step, lnegf = (float)a.dlin.neg_f_inv;
    const float ltop = (float)(a.dlin.n - 1);

    int iter = 0;
    for (long long p = p0; p < p1; p += ps, ++iter) {
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
            ui[d] = iv ? a.U64[(size_t)d * n + i] * us : 0.0;
        }
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        const bool diag = ti == tj;
        stage_flat_j<D>(a, j0, jn, us, SINGLE && a.sort_j && !diag && T == 256, ti * T + min(T / 2, n - 1 - ti * T),
                        srec, s_cnt, s_wtot);
        __syncthreads();
        // one pair: key (bin) and values
        auto pair = [&](int jj, int& key, float (&v)[NV]) {
            double rj[2 * NP];
            load_rec2<NP>(srec + jj * 2 * NP, rj);
            double dx[D], du[D];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                dx[d] = SFB_SUB(rj[d], xi[d]);
                du[d] = rj[D + d] - ui[d];
            }
            // r^2 exactly as the reference: left-to-right, no contraction (decides the bin)
            const double h2 = SFB_ADD(SFB_MUL(dx[0], dx[0]), SFB_MUL(dx[1], dx[1]));
            double r2 = h2;
            if constexpr (D == 3) r2 = SFB_ADD(h2, SFB_MUL(dx[2], dx[2]));
            bool slow;
            if (SINGLE && a.byte_lut) {
                key = byte_bin(lut8, sqx, r2, slow);  // slow: several edges in the cell or r^2 outside FP32
            } else if (LIN) {
                // the FMA search's bin from the FP32 distance r2f rsqrt(r2f) (relative error below
                // 2^-22): t = (r - first) / step, bin = floor(t) + 1 in range; within 2^-19 of the
                // index scale from an integer (an edge), or r^2 outside FP32, the FP64 search decides
                const float r2f = f32(r2);
                slow = !f32_range_ok(r2f);
                const float t = fmaf(r2f * rsqrt_normal(r2f), linv, lnegf);
                const float fl = floorf(t);
                const float fr = t - fl;
                const float wt = (fabsf(t) + fabsf(lnegf)) * 0x1p-19f;
                if (slow || !(fr > wt && fr < 1.f - wt)) key = linear_bin_sqrt_ool(&a.dlin, r2);
                else key = t < 0.f ? 0 : (fl >= ltop ? a.dlin.n : (int)fl + 1);
            } else {
                if (a.dist_linear) key = (r2 != r2) ? a.n_edges : linear_bin(a.dlin, SFB_SQRT(r2));
                else key = (r2 != r2) ? a.n_edges : lut64_bin(lut, a, r2);
                slow = !f32_range_ok(f32(r2));
            }
            float L, Tt, T2, Q;
            const bool fine = flat_primitives_mx<D, OPS>(dx, du, r2, h2, L, Tt, T2, Q);
            eval_ops(OPS{}, L, Tt, T2, Q, D, a.gen, v);
            if (slow || !fine) {
                if (SINGLE && slow && a.byte_lut) key = count_below_ool(a.edges, a.n_edges, r2);
                const FlatValues<D, OPS> f = flat_values_fp64_ool<D, OPS>(
                    dx[0], dx[1], D == 3 ? dx[D - 1] : 0.0, du[0], du[1], D == 3 ? du[D - 1] : 0.0, r2, h2, &a.gen);
#pragma unroll
                for (int o = 0; o < NV; ++o) v[o] = f.v[o];
            }
        };
        if constexpr (Hist::RUN) {
            if (iv) {
                // two open runs (PRIV 6): one pair per iteration, so that their extra registers fit
                // the three-block bound without spills
                constexpr int UNR = PRIV == 6 ? 1 : 2;
#pragma unroll (UNR)
                for (int jj = diag ? (int)threadIdx.x + 1 : 0; jj < jn; ++jj) {
                    int key;
                    float v[NV];
                    pair(jj, key, v);
                    hist.add(key, v, lane, warp);
                }
            }
        } else {
            for (int jj = 0; jj < jn; ++jj) {
                const bool valid = iv && (!diag || jj > (int)threadIdx.x);
                int key;
                float v[NV];
                pair(jj, key, v);
                hist.add(valid ? key : a.nb + 1, v, lane, warp);
            }
        }
    }
    double unscale[NV];  // formed after the pair loop: no registers held across it
    op_unscale(OPS{}, a.gen, pow2_exponent_above(a.g_stats[2]), unscale);
    hist.merge(a.g_sums, a.g_counts, a.nops, a.nb, unscale);
}

template <int D, class OPS, int PRIV, bool LIN = false>
__global__ void __launch_bounds__(256, OPS::n >= 4 ? 3 : 4) k_flat1d_mx(const __grid_constant__ PairArgs a)
{
    flat1d_mx_run<D, OPS, PRIV, true, LIN>(a, a.tp_lo + blockIdx.x, a.tp_hi, gridDim.x);
}

// Batched form: work items (slice, tile-pair range) pulled from a device counter.
template <int D, class OPS, int PRIV>
__global__ void __launch_bounds__(256, OPS::n >= 4 ? 3 : 4) k_flat1d_mx_batch(const __grid_constant__ BatchArgs b)
{
    batch_items(b, [&](const PairArgs& a, long long q0, long long q1) { flat1d_mx_run<D, OPS, PRIV, false>(a, q0, q1, 1); });
}

// ================================================================================================
// Sphere 1D
//
// Per point (FP64, built by the pack kernel): p (unit position), U = u_e E + u_n N (ambient tangent
// velocity), W = u_n E - u_e N (U turned by a quarter), [u_up]. With d = q - p and s = p + q the
// reference's transported increments are du_L = d . (U_B - U_A) / sin(sigma) and
// du_T = d . (W_B - W_A) / sin(sigma), with sin^2(sigma) = |d|^2 |s|^2 / 4.
// ================================================================================================
// Chord-key bin from the FP64 table with its ambiguity test.
__device__ __forceinline__ int sphere_chord_bin(const LutEntry64* lut, const PairArgs& a, double ch2, bool& slow)
{
    const LutEntry64 e = lut[lut_cell64(ch2, a.lg)];
    slow = (e.mult & LUT_FLAG_SLOW) || fabs(ch2 - e.e) <= a.chord_wrel * e.e || ch2 < a.chord_short ||
           ch2 > a.chord_anti || ch2 != ch2;
    return e.base + (ch2 > e.e ? e.mult : 0);
}

// FP64 reference recomputation of a sphere pair: bin (nb + 1 when the frame is degenerate) and the
// values scaled by us^order, in the kernel's value type R. Kept out of line (it is rare and large);
// inputs and the result travel by value so that the caller's arrays stay in registers.
template <int NV, typename R = float>
struct ExactPair {
    R v[NV];
    int bin;
};

template <int D, class OPS, typename R = float>
__device__ __forceinline__ ExactPair<OPS::n, R> sphere_pair_exact(const PairArgs& a, int i, int j, int ku)
{
    constexpr int NV = OPS::n;
    ExactPair<NV, R> res;
    double unscale[NV];
    op_unscale(OPS{}, a.gen, ku, unscale);
    SphPoint A, B;
    load_sph64(a.X64, a.n, i, A);
    load_sph64(a.X64, a.n, j, B);
    double r, tA[2], tB[2], uA[D], uB[D], du[D];
    const bool ok = x_sphere_frame(A, B, a.radius, r, tA, tB);
    res.bin = ok ? sphere_exact_bin(a, r) : a.nb + 1;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        uA[d] = a.U64[(size_t)d * a.n + i];
        uB[d] = a.U64[(size_t)d * a.n + j];
    }
    x_sphere_delta<D>(tA, tB, uA, uB, du);
    double Q64 = du[0] * du[0] + du[1] * du[1];
    if constexpr (D == 3) Q64 = fma(du[2], du[2], Q64);
    double v64[NV];
    eval_ops(OPS{}, du[0], du[1], Q64 - du[0] * du[0], Q64, D, a.gen, v64);
#pragma unroll
    for (int o = 0; o < NV; ++o) res.v[o] = R(v64[o] / unscale[o]);
    return res;
}

// Per-pair primitives of a sphere pair from the FP64 records (fields: p 0-2, U 3-5, W 6-8, up 9;
// velocities already scaled by us), in FP32 (the mixed kernel) or FP64 (the FP64 chord kernel, R =
// double: the same formulas with the normalisation and powers kept in FP64). Returns the chord^2.
template <int D, class OPS>
__device__ __forceinline__ double sphere_primitives_mx(const double* ra, const double* rb, double& L, double& Tt,
                                                       double& T2, double& Q)
{
    using N = ListNeeds2<OPS>;
    double d[3], sv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        d[c] = rb[c] - ra[c];
        sv[c] = rb[c] + ra[c];
    }
    const double ch2 = fma(d[2], d[2], fma(d[1], d[1], d[0] * d[0]));
    const double ss = fma(sv[2], sv[2], fma(sv[1], sv[1], sv[0] * sv[0]));
    // sin(sigma) = |d| |s| / 2; degenerate (coincident / antipodal) pairs are recomputed anyway
    const double inv_s = rsqrt(0.25 * ch2 * ss);
    L = 0.0;
    Tt = 0.0;
    T2 = 0.0;
    Q = 0.0;
    if constexpr (N::L || N::Q) {
        double pl = d[0] * (rb[3] - ra[3]);
        pl = fma(d[1], rb[4] - ra[4], pl);
        pl = fma(d[2], rb[5] - ra[5], pl);
        L = pl * inv_s;
    }
    if constexpr (N::T || N::T2 || N::Q) {
        double pt = d[0] * (rb[6] - ra[6]);
        pt = fma(d[1], rb[7] - ra[7], pt);
        pt = fma(d[2], rb[8] - ra[8], pt);
        Tt = pt * inv_s;
        T2 = Tt * Tt;
        if constexpr (D == 3) {
            const double dw = rb[9] - ra[9];
            T2 = fma(dw, dw, T2);
        }
    }
    if constexpr (N::Q) Q = fma(L, L, T2);
    return ch2;
}

template <int D, class OPS>
__device__ __forceinline__ double sphere_primitives_mx(const double* ra, const double* rb, float& L, float& Tt,
                                                       float& T2, float& Q)
{
    using N = ListNeeds2<OPS>;
    double d[3], sv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        d[c] = rb[c] - ra[c];
        sv[c] = rb[c] + ra[c];
    }
    const double ch2 = fma(d[2], d[2], fma(d[1], d[1], d[0] * d[0]));
    const double ss = fma(sv[2], sv[2], fma(sv[1], sv[1], sv[0] * sv[0]));
    // chord^2 and |s|^2 lie in [0, 4]; out-of-range products only occur for the near-coincident or
    // near-antipodal pairs that are recomputed anyway
    const float inv_s = rsqrt_normal(0.25f * f32(ch2) * f32(ss));
    L = 0.f;
    Tt = 0.f;
    T2 = 0.f;
    Q = 0.f;
    if constexpr (N::L || N::Q) {
        double pl = d[0] * (rb[3] - ra[3]);
        pl = fma(d[1], rb[4] - ra[4], pl);
        pl = fma(d[2], rb[5] - ra[5], pl);
        L = f32(pl) * inv_s;
    }
    if constexpr (N::T || N::T2 || N::Q) {
        double pt = d[0] * (rb[6] - ra[6]);
        pt = fma(d[1], rb[7] - ra[7], pt);
        pt = fma(d[2], rb[8] - ra[8], pt);
        Tt = f32(pt) * inv_s;
        T2 = Tt * Tt;
        if constexpr (D == 3) {
            const float dw = f32(rb[9] - ra[9]);
            T2 = fmaf(dw, dw, T2);
        }
    }
    if constexpr (N::Q) Q = fmaf(L, L, T2);
    return ch2;
}

// sphere_pair_exact out of line (the pairs of the chord ambiguity band, near-coincident and
// near-antipodal pairs are rare): the pair loop only branches to it, and the kernel parameters are read
// in place (grid constants), so the FP64 frame's registers are not held across the loop.
template <int D, class OPS, typename R>
__device__ __noinline__ ExactPair<OPS::n, R> sphere_pair_exact_ool(const PairArgs* a, int i, int j, int ku)
{
    return sphere_pair_exact<D, OPS, R>(*a, i, j, ku);
}

template <int D, class OPS, int PRIV, typename R = float>
__device__ __forceinline__ void sphere1d_mx_run(const PairArgs& a, long long p0, long long p1, long long ps)
{
    constexpr int NV = OPS::n;
    constexpr int NP = 5;  // double2 per record: p(3) U(3) W(3) up/pad(1)
    using Hist = BlockHist<R, NV, PRIV>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x, NW = T >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.n;
    LutEntry64* lut = reinterpret_cast<LutEntry64*>(smem);
    double* srec = reinterpret_cast<double*>(smem + a.lut_bytes);
    __shared__ unsigned long long s_recheck;
    Hist hist;
    hist.init(reinterpret_cast<unsigned char*>(srec + (size_t)2 * NP * T), NW, a.nb + 2, a.hist_cols);
    for (int k = threadIdx.x; k < a.lut_bytes / (int)sizeof(LutEntry64); k += T)
        lut[k] = static_cast<const LutEntry64*>(a.lut)[k];
    if (threadIdx.x == 0) s_recheck = 0ull;
    unsigned my_recheck = 0;
    // FP32 values carry velocities scaled into FP32 range; the FP64 chord kernel needs no scaling
    const int ku = sizeof(R) == 4 ? pow2_exponent_above(a.g_stats[2]) : 0;
    const double us = ldexp(1.0, -ku);
    constexpr int NF = 9 + (D == 3);  // stored fields

    int iter = 0;
    for (long long p = p0; p < p1; p += ps, ++iter) {
        hist.close_runs(lane);
        if (PRIV && iter && a.flush_every && iter % a.flush_every == 0) hist.fold();
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        double ra[2 * NP];
#pragma unroll
        for (int c = 0; c < 2 * NP; ++c)
            ra[c] = (iv && c < NF) ? a.XM[(size_t)c * n + i] * (c < 3 ? 1.0 : us) : 0.0;
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        if ((int)threadIdx.x < jn) {
            double* rec = srec + threadIdx.x * 2 * NP;
            const int jg = j0 + threadIdx.x;
#pragma unroll
            for (int c = 0; c < 2 * NP; ++c) rec[c] = (c < NF) ? a.XM[(size_t)c * n + jg] * (c < 3 ? 1.0 : us) : 0.0;
        }
        __syncthreads();
        const bool diag = ti == tj;
        auto pair = [&](int jj, int& key, R (&v)[NV]) {
            double rb[2 * NP];
            load_rec2<NP>(srec + jj * 2 * NP, rb);
            R L, Tt, T2, Q;
            const double ch2 = sphere_primitives_mx<D, OPS>(ra, rb, L, Tt, T2, Q);
            bool slow;
            key = sphere_chord_bin(lut, a, ch2, slow);
            eval_ops(OPS{}, L, Tt, T2, Q, D, a.gen, v);
            if (slow) {
                const ExactPair<NV, R> ex = sphere_pair_exact_ool<D, OPS, R>(&a, i, j0 + jj, ku);
                key = ex.bin;
#pragma unroll
                for (int o = 0; o < NV; ++o) v[o] = ex.v[o];
                ++my_recheck;
            }
        };
        if constexpr (Hist::RUN) {
            if (iv) {
#pragma unroll 2
                for (int jj = diag ? (int)threadIdx.x + 1 : 0; jj < jn; ++jj) {
                    int key;
                    R v[NV];
                    pair(jj, key, v);
                    hist.add(key, v, lane, warp);
                }
            }
        } else {
            for (int jj = 0; jj < jn; ++jj) {
                const bool valid = iv && (!diag || jj > (int)threadIdx.x);
                int key;
                R v[NV];
                if (valid) pair(jj, key, v);
                else {
                    key = a.nb + 1;
#pragma unroll
                    for (int o = 0; o < NV; ++o) v[o] = R(0);
                }
                hist.add(key, v, lane, warp);
            }
        }
    }
    if (my_recheck) atomicAdd(&s_recheck, (unsigned long long)my_recheck);
    double unscale[NV];  // formed after the pair loop: no registers held across it
    op_unscale(OPS{}, a.gen, ku, unscale);
    hist.merge(a.g_sums, a.g_counts, a.nops, a.nb, unscale);
    if (threadIdx.x == 0 && s_recheck) atomicAdd(&a.g_stats[0], s_recheck);
}

template <int D, class OPS, int PRIV>
__global__ void __launch_bounds__(256, 3) k_sphere1d_mx(const __grid_constant__ PairArgs a)
{
    sphere1d_mx_run<D, OPS, PRIV>(a, a.tp_lo + blockIdx.x, a.tp_hi, gridDim.x);
}

// The plain FP64 form of the same chord formulation (precision FP64, the default formulation on the
// sphere): FP64 chord bin with the same ambiguity band, FP64 normalisation, powers and accumulation.
// It differs from the mixed kernel only in precision, so the two time the same algorithm; the
// reference-formulation FP64 kernel (k_sphere1d_fp64: the reference's frame for every pair)
// remains selectable with SFB200_OPT_FORMULATION.
template <int D, class OPS, int PRIV>
__global__ void __launch_bounds__(256, 2) k_sphere1d_chord64(const __grid_constant__ PairArgs a)
{
    sphere1d_mx_run<D, OPS, PRIV, double>(a, a.tp_lo + blockIdx.x, a.tp_hi, gridDim.x);
}

// Batched form: work items (slice, tile-pair range) pulled from a device counter.
template <int D, class OPS, int PRIV>
__global__ void __launch_bounds__(256, 3) k_sphere1d_mx_batch(const __grid_constant__ BatchArgs b)
{
    batch_items(b, [&](const PairArgs& a, long long q0, long long q1) { sphere1d_mx_run<D, OPS, PRIV>(a, q0, q1, 1); });
}

// ================================================================================================
// Joint (distance x value) histogram
//
// The value comes from the FP64 numerators, so its FP32 error is relative to itself (a few ulps):
// the value-bin index t = (v - first) / step is trusted when it lies more than
// (|t| + |first / step|) * vrel from an integer; closer pairs, sphere pairs in the chord ambiguity
// band and every pair of a vector value axis are recomputed in FP64 with the reference formula.
//
// Cells are one 64-bit word each (two native 32-bit atomics per pair, see SplitWords): the count in the
// top 20 bits and, below, the sum of the pair offsets from the value-bin centre in fixed point
// (quantum 2^-21 of the largest half bin width or finer; the packed word decodes exactly while the
// cell holds fewer than 2^20 pairs and the offset sum stays below 2^43 in magnitude, so blocks flush
// at least every 2^20 - 1 pairs). That quantum is far below the 1e-6 tolerance for every value bin
// whose values stay at least a half width away from zero; the bins closer to zero keep their offsets
// in a separate 64-bit word at 2^-30 of the largest half width. There a value can still be tiny next
// to that quantum (S2 or L3 of close pairs on a linear axis around zero, the low bins of a log axis):
// a pair whose |value| is below 2^-8 of the largest half width takes the exact FP64 route and adds its
// FP64 offset into a third, FP64 cell (a shared 64-bit compare-and-swap add, for those pairs only), so
// that every fixed-point offset carries at most 2^-23 of its own value.
//
// Offsets are taken from C_b, the value-bin centre rounded to FP32 in the scaled units of the FP32
// value (per block in shared memory, with its exact FP64 image for the flush). In every coarse bin
// the values lie within a half width of a centre at least three half widths from zero, so the FP32
// subtraction v - C_b is exact (Sterbenz) and its fixed-point image is one FP32 multiply by a power
// of two and one conversion. In the bins near zero the difference is taken exactly as the FP32 sum
// s + e (TwoSum) and both parts are converted; the FP64 route remains for rechecked pairs only.
// ================================================================================================
// A 64-bit shared word kept as two 32-bit halves (lo[k], hi[k]) in separate arrays, so that every
// update is a native 32-bit shared atomic (a 64-bit shared atomic add is a compare-and-swap loop on
// this architecture) and neighbouring cells fall in different banks. The low add returns the old
// half, so the carry it produced is known exactly and goes into the high add with the value's own
// high half: the pair (hi, lo) always holds the exact 64-bit modular sum once the adds are done.
struct SplitWords {
    unsigned* lo;
    unsigned* hi;
    // adds HI * 2^32 + q (q sign-extended to 64 bits); with HI != 0 the high add always happens
    template <unsigned HI>
    __device__ __forceinline__ void add(int k, int q) const
    {
        const unsigned l = (unsigned)q;
        const unsigned old = atomicAdd(&lo[k], l);
        const unsigned h = HI + (q < 0 ? 0xffffffffu : 0u) + (old + l < old ? 1u : 0u);
        if (HI != 0u || h != 0u) atomicAdd(&hi[k], h);
    }
    __device__ __forceinline__ unsigned long long take(int k) const  // read and clear (no other writer)
    {
        const unsigned long long w = ((unsigned long long)hi[k] << 32) | lo[k];
        lo[k] = 0u;
        hi[k] = 0u;
        return w;
    }
};

// Shared-memory slot of joint cell (distance bin d0, value bin v0), both 0-based, in rows of ndp
// slots (nd rounded up to a multiple of 32) per value bin. The distance index is XOR-ed with the low 5
// bits of the value bin: without it a slot's bank (slot mod 32) would be the distance bin's alone, and
// the lanes of a warp, whose pairs crowd into the few most populated distance bins, would queue on the
// same banks; with it, lanes of equal distance bin but different value bins take different banks. The
// XOR permutes each row's aligned groups of 32 slots, so it is a bijection on [0, ndp).
__device__ __forceinline__ int joint_slot(int d0, int v0, int ndp) { return v0 * ndp + (d0 ^ (v0 & 31)); }

__device__ __forceinline__ void joint_flush_packed(const PairArgs& a, const SplitWords& hcell,
                                                   const SplitWords& hfine, double* htiny, int ndp,
                                                   const double* vcen)
{
    const int nd = a.nb;
    const int nslot = ndp * a.nv;
    for (int k = threadIdx.x; k < nslot; k += blockDim.x) {
        if (!(hcell.lo[k] | hcell.hi[k])) continue;
        const unsigned long long w = hcell.take(k);
        const unsigned long long cnt = (w + (1ull << 43)) >> 44;
        const long long off = (long long)(w - (cnt << 44));
        const int v0 = k / ndp;
        const int d0 = (k - v0 * ndp) ^ (v0 & 31);  // slots of distance bins >= nd are never written
        double s = (double)cnt * vcen[v0] + (double)off * a.vqc_inv;
        const int f = v0 + 1 - a.vfine_lo;
        if ((unsigned)f < (unsigned)a.nfine) {
            const int fs = joint_slot(d0, f, ndp);
            s += (double)(long long)hfine.take(fs) * a.vq_inv + htiny[fs];
            htiny[fs] = 0.0;
        }
        const int cell = d0 + nd * v0;
        atomicAdd(&a.g_sums[cell], s);
        atomicAdd(&a.g_counts[cell], cnt);
    }
    __syncthreads();
}

// Exact FP64 route of one joint pair (i, j) (the reference formula for the distance bin, the value
// and the value bin), kept out of line: the pair loop only branches to it for the rare pairs that
// need it. `a` points to the kernel's parameters in place (grid constants); q, fq are the coarse and
// fine fixed-point offsets from the value-bin centre, fo the offset in FP64 and v the value.
struct JointExact {
    int db, vb, q, fq;
    double fo, v;
    bool ok;
};

template <bool SPHERE, int D>
__device__ __noinline__ JointExact joint_exact_pair(const PairArgs* ap, int i, int j, const double* vcen)
{
    const PairArgs& a = *ap;
    const int n = a.n;
    JointExact r{0, 0, 0, 0, 0.0, 0.0, true};
    double du64[D], v64;
    if constexpr (!SPHERE) {
        double dx64[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            dx64[d] = SFB_SUB(a.X64[(size_t)d * n + j], a.X64[(size_t)d * n + i]);
            du64[d] = SFB_SUB(a.U64[(size_t)d * n + j], a.U64[(size_t)d * n + i]);
        }
        const double r264 = x_dot<D>(dx64, dx64);
        r.db = flat_exact_bin(a, r264);
        v64 = x_sf_raw<D>(a.gen.op[0], du64, dx64, r264);
    } else {
        SphPoint A, B;
        load_sph64(a.X64, n, i, A);
        load_sph64(a.X64, n, j, B);
        double rr, tA[2], tB[2], uA[D], uB[D];
        r.ok = x_sphere_frame(A, B, a.radius, rr, tA, tB);
        r.db = sphere_exact_bin(a, rr);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            uA[d] = a.U64[(size_t)d * n + i];
            uB[d] = a.U64[(size_t)d * n + j];
        }
        x_sphere_delta<D>(tA, tB, uA, uB, du64);
        v64 = x_sphere_value<D>(a.gen.op[0], du64);
    }
    r.vb = value_exact_bin(a, v64);
    if (r.vb >= 1 && r.vb <= a.nv) {
        const double off = v64 - vcen[r.vb - 1];  // exact: both within a bin of each other
        r.q = __double2int_rn(off * a.vqc);
        r.fq = __double2int_rn(off * a.vq);
        r.fo = off;
        r.v = v64;
    }
    return r;
}

template <bool SPHERE, int D, class OPS>
__device__ __forceinline__ void joint_mx_run(const PairArgs& a, long long p0, long long p1, long long ps)
{
    constexpr int NP = SPHERE ? 5 : D;
    constexpr int NF = SPHERE ? 9 + (D == 3) : 2 * D;  // stored fields per record
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x;
    const int n = a.n;
    const int nd = a.nb, nv = a.nv;
    const int ndp = (nd + 31) & ~31;  // slots per value bin (joint_slot)
    const int ncell = ndp * nv;
    const LutEntry64* lut = reinterpret_cast<const LutEntry64*>(smem);
    const unsigned char* lut8 = smem;
    const double* sqx = reinterpret_cast<const double*>(smem + kByteCells);
    double* srec = reinterpret_cast<double*>(smem + a.lut_bytes);                                 // T * 2NP
    unsigned* words = reinterpret_cast<unsigned*>(srec + (size_t)2 * NP * T);
    const int nfw = ndp * a.nfine;
    const SplitWords hcell{words, words + ncell};                                  // 2 x ncell
    const SplitWords hfine{words + 2 * ncell, words + 2 * ncell + nfw};            // 2 x ndp * nfine
    double* htiny = reinterpret_cast<double*>(words + 2 * (ncell + nfw));          // ndp * nfine (FP64)
    double* vcen = htiny + nfw;                                                    // nv
    float* vc32 = reinterpret_cast<float*>(vcen + nv);                             // nv
    __shared__ unsigned long long s_recheck;

    load_bin_table(a, smem);
    for (int k = threadIdx.x; k < 2 * ncell + 4 * nfw; k += T) words[k] = 0u;
    if (threadIdx.x == 0) s_recheck = 0ull;
    unsigned my_recheck = 0;
    const int ku = pow2_exponent_above(a.g_stats[2]);
    const double us = ldexp(1.0, -ku);
    double unscale[1];
    op_unscale(OPS{}, a.gen, ku, unscale);
    // the FP32 value is v us^k: fold us^-k into the index scale (every pair exact if that overflows)
    const float vinv = (float)(a.vlin.inv_step * unscale[0]);
    const bool vfast = a.val_linear && isfinite(vinv) && vinv != 0.f;
    const float vnegf = (float)a.vlin.neg_f_inv;
    const float tmax = (float)(a.vlin.n - 1);
    // centres C_b in the FP32 value's units and their exact FP64 images; FP32 offsets need every
    // centre and the fixed-point scale to be normal FP32 numbers
    const float vqcs = (float)(a.vqc * unscale[0]);
    const float vqfs = (float)(a.vq * unscale[0]);
    // below this |value| (2^-8 of the largest half width) a pair of a bin near zero takes the FP64 route
    const double tiny64 = ldexp(a.vq_inv, 22);
    const float tiny32 = (float)(tiny64 / unscale[0]);
    // LinearBinEdges distance axis: FP32 images of the search's scale and offset, and the last index
    const float linv = (float)a.dlin.inv_step, lnegf = (float)a.dlin.neg_f_inv;
    const float ltop = (float)(a.dlin.n - 1);
    bool cok = vfast && vqcs != 0.f && f32_zero_or_normal(vqcs) && vqfs != 0.f && f32_zero_or_normal(vqfs);
    for (int k = threadIdx.x; k < nv; k += T) {
        const double c64 = value_center(a, k + 1);
        const float c = (float)(c64 / unscale[0]);
        const bool normal = f32_zero_or_normal(c);
        vc32[k] = c;
        vcen[k] = normal ? (double)c * unscale[0] : c64;  // any finite reference centre is exact
        cok = cok && normal;
    }
    const bool qfast = __syncthreads_and(cok) != 0;

    // field c of point k as staged: sphere XM (velocity fields scaled), flat x then u (u scaled)
    auto field = [&](int c, int k) -> double {
        if constexpr (SPHERE) return a.XM[(size_t)c * n + k] * (c < 3 ? 1.0 : us);
        else return c < D ? a.X64[(size_t)c * n + k] : a.U64[(size_t)(c - D) * n + k] * us;
    };

    int iter = 0;
    for (long long p = p0; p < p1; p += ps, ++iter) {
        if (iter && iter % a.flush_every == 0) {
            __syncthreads();
            joint_flush_packed(a, hcell, hfine, htiny, ndp, vcen);
        }
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        double ra[2 * NP];
#pragma unroll
        for (int c = 0; c < 2 * NP; ++c) ra[c] = (iv && c < NF) ? field(c, i) : 0.0;
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        if ((int)threadIdx.x < jn) {
            double* rec = srec + threadIdx.x * 2 * NP;
#pragma unroll
            for (int c = 0; c < 2 * NP; ++c) rec[c] = c < NF ? field(c, j0 + threadIdx.x) : 0.0;
        }
        __syncthreads();
        if (!iv) continue;
        const bool diag = ti == tj;
        // one pair (i, j0 + jj): its cell and packed increment (cell < 0: nothing to add) and, in a
        // bin near zero, its fine offset
        struct JointAdd {
            int cell, fidx, q, fq;
        };
        auto eval_pair = [&](int jj) -> JointAdd {
            JointAdd r{-1, -1, 0, 0};
            double rb[2 * NP];
            load_rec2<NP>(srec + jj * 2 * NP, rb);
            float L, Tt, T2, Q;
            int db;
            bool slow = false, fine = true;
            if constexpr (SPHERE) {
                const double ch2 = sphere_primitives_mx<D, OPS>(ra, rb, L, Tt, T2, Q);
                db = sphere_chord_bin(lut, a, ch2, slow);
            } else {
                double dx[D], du[D];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    dx[d] = SFB_SUB(rb[d], ra[d]);
                    du[d] = rb[D + d] - ra[D + d];
                }
                const double h2 = SFB_ADD(SFB_MUL(dx[0], dx[0]), SFB_MUL(dx[1], dx[1]));
                double r2 = h2;
                if constexpr (D == 3) r2 = SFB_ADD(h2, SFB_MUL(dx[2], dx[2]));
                if (a.byte_lut) {
                    db = byte_bin(lut8, sqx, r2, slow);  // slow: the exact route decides the bin
                } else if (a.dist_linear) {
                    // as the flat 1D kernel: the search's bin from the FP32 distance, the FP64 search
                    // within 2^-19 of the index scale from an edge or for r^2 outside FP32
                    const float r2f = f32(r2);
                    slow = !f32_range_ok(r2f);
                    const float t = fmaf(r2f * rsqrt_normal(r2f), linv, lnegf);
                    const float fl = floorf(t);
                    const float fr = t - fl;
                    const float wt = (fabsf(t) + fabsf(lnegf)) * 0x1p-19f;
                    if (slow || !(fr > wt && fr < 1.f - wt)) db = linear_bin_sqrt_ool(&a.dlin, r2);
                    else db = t < 0.f ? 0 : (fl >= ltop ? a.dlin.n : (int)fl + 1);
                } else {
                    db = (r2 != r2) ? a.n_edges : lut64_bin(lut, a, r2);
                    slow = !f32_range_ok(f32(r2));
                }
                // flat bins are exact: a pair outside the distance range needs no value
                if (!slow && (db < 1 || db > nd)) return r;
                fine = flat_primitives_mx<D, OPS>(dx, du, r2, h2, L, Tt, T2, Q);
            }
            float v[1];
            eval_ops(OPS{}, L, Tt, T2, Q, D, a.gen, v);
            const float val = v[0];
            int vb = 0, q = 0, fq = 0;
            if (qfast) {
                // t within wt of an integer (an edge; the range ends are edges too) or NaN: exact route
                const float t = fmaf(val, vinv, vnegf);
                const float fl = floorf(t);
                const float fr = t - fl;
                const float wt = (fabsf(t) + fabsf(vnegf)) * a.vrel;
                vb = (int)fminf(fmaxf(fl, -1.f), tmax) + 1;  // 0 below the range, nv + 1 above
                const bool tiny = (unsigned)(vb - a.vfine_lo) < (unsigned)a.nfine && fabsf(val) < tiny32;
                slow = slow || !fine || tiny || !(fr > wt && fr < 1.f - wt);
                // offset from the bin centre as the exact FP32 sum s + e (TwoSum; e = 0 in the coarse
                // bins, where the subtraction is exact), then both fixed-point images
                const float c = vc32[min(max(vb, 1), nv) - 1];
                const float sd = val - c;
                const float bv = sd - val;
                const float e = (val - (sd - bv)) + (-c - bv);
                q = __float2int_rn(sd * vqcs);
                fq = __float2int_rn(sd * vqfs) + __float2int_rn(e * vqfs);
            } else {
                slow = true;  // vector value edges (or an unrepresentable FP32 scale): exact FP64 route
            }
            bool ok = true;
            if (slow) {
                const JointExact x = joint_exact_pair<SPHERE, D>(&a, i, j0 + jj, vcen);
                db = x.db;
                vb = x.vb;
                q = x.q;
                fq = x.fq;
                ok = x.ok;
                ++my_recheck;
                const int f = vb - a.vfine_lo;
                if (ok && db >= 1 && db <= nd && (unsigned)f < (unsigned)a.nfine && fabs(x.v) < tiny64) {
                    // a tiny value near zero: its exact FP64 offset now, only the count in the cell
                    atomicAdd(&htiny[joint_slot(db - 1, f, ndp)], x.fo);
                    r.cell = joint_slot(db - 1, vb - 1, ndp);
                    return r;
                }
            }
            if (ok && db >= 1 && db <= nd && vb >= 1 && vb <= nv) {
                r.cell = joint_slot(db - 1, vb - 1, ndp);
                const int f = vb - a.vfine_lo;
                if ((unsigned)f < (unsigned)a.nfine) {  // near zero: the offset goes to the fine word
                    r.fidx = joint_slot(db - 1, f, ndp);
                    r.fq = fq;
                } else {
                    r.q = q;
                }
            }
            return r;
        };
        auto commit = [&](const JointAdd& r) {
            if (r.cell < 0) return;
            if (r.fidx >= 0) hfine.add<0u>(r.fidx, r.fq);
            hcell.add<1u << 12>(r.cell, r.q);  // count (bit 44 of the word) and coarse offset
        };
        int jj = diag ? (int)threadIdx.x + 1 : 0;
        if constexpr (!SPHERE) {  // two independent pairs in flight per thread (latency hiding)
            for (; jj + 1 < jn; jj += 2) {
                const JointAdd r0 = eval_pair(jj);
                const JointAdd r1 = eval_pair(jj + 1);
                commit(r0);
                commit(r1);
            }
        }
        for (; jj < jn; ++jj) commit(eval_pair(jj));
    }
    if (my_recheck) atomicAdd(&s_recheck, (unsigned long long)my_recheck);
    __syncthreads();
    joint_flush_packed(a, hcell, hfine, htiny, ndp, vcen);
    if (threadIdx.x == 0 && s_recheck) atomicAdd(&a.g_stats[0], s_recheck);
}

// NT: the block size the launch bound is compiled for. One block per SM either way (the cell table
// fills shared memory); 768 threads (24 warps, 80 registers) hide more of the pair loop's latency than
// 512 (16 warps): c3, 131072 points, 55.9 -> 44.2 ms on B200 (896 threads 43.7 ms, 992 44.6 ms).
template <bool SPHERE, int D, class OPS, int NT = 512>
__global__ void __launch_bounds__(NT, 1) k_joint_mx(const __grid_constant__ PairArgs a)
{
    joint_mx_run<SPHERE, D, OPS>(a, a.tp_lo + blockIdx.x, a.tp_hi, gridDim.x);
}

// Batched form: work items (slice, tile-pair range) pulled from a device counter.
template <bool SPHERE, int D, class OPS, int NT = 512>
__global__ void __launch_bounds__(NT, 1) k_joint_mx_batch(const __grid_constant__ BatchArgs b)
{
    batch_items(b, [&](const PairArgs& a, long long q0, long long q1) { joint_mx_run<SPHERE, D, OPS>(a, q0, q1, 1); });
}

}  // namespace sfb
