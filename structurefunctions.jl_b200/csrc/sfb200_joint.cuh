// sfb200_joint.cuh -- joint (distance x value) histogram kernels, the StructureFunction2DSumsAndCounts
// path (src/Calculations/serial_2d.jl:49-85 Euclidean, 260-303 non-Euclidean).
//
// A pair contributes to cell (dbin, vbin) when both bins are in range; the operator value decides
// vbin, so in FP64 it is computed in the reference's exact operation order (sfb200_exact.cuh).
// The histogram (n_dist x n_val cells, column-major like the reference's matrices) lives in shared
// memory per block when it fits and is updated with shared-memory atomics (cells are many and
// sparsely hit, so warp aggregation buys little); otherwise the kernel adds straight into the global
// FP64 / uint64 accumulators.
//
// The FP32 kernel accumulates each cell as its count and the sum of (v - c_vbin), the value's
// offset from its value-bin centre, in 64-bit fixed point: a cell's values lie within half a bin
// width h of c_vbin, so with the power-of-two scale S = 2^k, h S < 2^30, every offset is one integer
// of at most 2^30 and a block's cell sum stays exact (the quantum 1/S is below 2^-30 h). The merge
// rebuilds sum = count * c_vbin + residual / S in FP64. In the value bins near zero (within two half
// widths), where a value can be tiny next to that quantum, the same 64-bit word holds an FP64 sum of
// the offsets instead (shared FP64 atomic add). Pairs whose value (or distance) lies within
// the FP32 error bound of an edge are recomputed in FP64 with the reference arithmetic.
//
// Both kernels move their block histogram to the global one every `flush_every` tile pairs, so a
// 32-bit cell count never exceeds 2^31 pairs.
#pragma once

#include "sfb200_kernels.cuh"

namespace sfb {

// ------------------------------------------------------------------------------------ FP64
// Add the block's cells into the global histogram and clear them (all threads, after a barrier).
__device__ __forceinline__ void joint_flush_fp64(const PairArgs& a, double* hs, unsigned* hc, int ncell)
{
    for (int k = threadIdx.x; k < ncell; k += blockDim.x) {
        if (hc[k]) {
            atomicAdd(&a.g_sums[k], hs[k]);
            atomicAdd(&a.g_counts[k], (unsigned long long)hc[k]);
            hs[k] = 0.0;
            hc[k] = 0u;
        }
    }
    __syncthreads();
}

template <bool SPHERE, int D, bool SMEM>
__global__ void __launch_bounds__(512) k_joint_fp64(const PairArgs a)
{
    constexpr int NX = SPHERE ? 8 : D;
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x;
    const int n = a.n;
    const int nd = a.nb, nv = a.nv;
    const int ncell = nd * nv;
    double* sx = reinterpret_cast<double*>(smem);  // NX * T
    double* su = sx + NX * T;                       // D * T
    double* hs = su + D * T;                        // ncell (SMEM)
    unsigned* hc = reinterpret_cast<unsigned*>(hs + (SMEM ? ncell : 0));
    const LutEntry64* lut = static_cast<const LutEntry64*>(a.lut);
    const sfb200_operator op = a.gen.op[0];

    if constexpr (SMEM) {
        for (int k = threadIdx.x; k < ncell; k += T) { hs[k] = 0.0; hc[k] = 0u; }
    }
    int iter = 0;
    for (long long p = a.tp_lo + blockIdx.x; p < a.tp_hi; p += gridDim.x, ++iter) {
        if constexpr (SMEM) {
            if (iter && iter % a.flush_every == 0) {
                __syncthreads();
                joint_flush_fp64(a, hs, hc, ncell);
            }
        }
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        double xa[NX], ua[D];
#pragma unroll
        for (int c = 0; c < NX; ++c) xa[c] = iv ? a.X64[(size_t)c * n + i] : 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) ua[d] = iv ? a.U64[(size_t)d * n + i] : 0.0;
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
        if (!iv) continue;
        const int jbeg = (ti == tj) ? (int)threadIdx.x + 1 : 0;
        for (int jj = jbeg; jj < jn; ++jj) {
            double ub[D], du[D];
#pragma unroll
            for (int d = 0; d < D; ++d) ub[d] = su[d * T + jj];
            int db;
            double v;
            if constexpr (!SPHERE) {
                double dx[D];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    dx[d] = SFB_SUB(sx[d * T + jj], xa[d]);
                    du[d] = SFB_SUB(ub[d], ua[d]);
                }
                const double r2 = x_dot<D>(dx, dx);
                if (a.dist_linear) db = (r2 != r2) ? a.n_edges : linear_bin(a.dlin, SFB_SQRT(r2));
                else db = (r2 != r2) ? a.n_edges : lut64_bin(lut, a, r2);
                if (db < 1 || db > nd) continue;
                v = x_sf_raw<D>(op, du, dx, r2);
            } else {
                SphPoint A, B;
                A.p[0] = xa[0]; A.p[1] = xa[1]; A.p[2] = xa[2]; A.E[0] = xa[3]; A.E[1] = xa[4];
                A.N[0] = xa[5]; A.N[1] = xa[6]; A.N[2] = xa[7];
                B.p[0] = sx[0 * T + jj]; B.p[1] = sx[1 * T + jj]; B.p[2] = sx[2 * T + jj];
                B.E[0] = sx[3 * T + jj]; B.E[1] = sx[4 * T + jj];
                B.N[0] = sx[5 * T + jj]; B.N[1] = sx[6 * T + jj]; B.N[2] = sx[7 * T + jj];
                double r, tA[2], tB[2];
                const bool ok = x_sphere_frame(A, B, a.radius, r, tA, tB);
                if (a.dist_linear) db = linear_bin(a.dlin, r);
                else db = (r != r) ? a.n_edges : lut64_bin(lut, a, r);
                if (!ok || db < 1 || db > nd) continue;
                x_sphere_delta<D>(tA, tB, ua, ub, du);
                v = x_sphere_value<D>(op, du);
            }
            const int vb = value_exact_bin(a, v);
            if (vb < 1 || vb > nv) continue;
            const int cell = (db - 1) + nd * (vb - 1);
            if constexpr (SMEM) {
                atomicAdd(&hs[cell], v);
                atomicAdd(&hc[cell], 1u);
            } else {
                atomicAdd(&a.g_sums[cell], v);
                atomicAdd(&a.g_counts[cell], 1ull);
            }
        }
    }
    if constexpr (SMEM) {
        __syncthreads();
        joint_flush_fp64(a, hs, hc, ncell);
    }
}

// ------------------------------------------------------------------------------------ single pass
// Consecutive rows r0 .. r0 + nr - 1 (nr >= 2) of the flat two-dimensional single pass in one launch,
// on one value axis shared by the rows (src/Calculations/serial_single_pass.jl:876-909, the scatter
// :852-864): a pair's distance bin, r^2, inv(sqrt(r2)), du_L = (du . dx) inv_r and |du|^2 are formed
// once, then each row's invariant, its value bin and its cell update (the reference's pass does the
// same; one launch per row would repeat the pair arithmetic for every row). Every quantity is the
// per-row FP64 kernel's (k_joint_fp64 with x_sf_raw), so the result is that of nr single-row runs.
// Row t's cells follow row t - 1's: sums and counts are nr consecutive (n_dist x n_val) matrices.
// SPLIT threads share each point i of the tile (T = blockDim.x / SPLIT points), thread h of them taking
// the j with jj = h mod SPLIT: the cells fill shared memory, so one block runs per SM, and this raises
// its warps without narrowing the tile.
template <int D, bool SMEM, int SPLIT>
__global__ void __launch_bounds__(512 * SPLIT) k_sp2d_fp64(const PairArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x / SPLIT;
    const int tid = threadIdx.x % T, half = threadIdx.x / T;
    const int n = a.n;
    const int nd = a.nb, nv = a.nv;
    const int ncell = nd * nv;  // cells per row
    const int r0 = a.gen.op[0].nl, r1 = r0 + a.nops;
    double* sx = reinterpret_cast<double*>(smem);  // D * T
    double* su = sx + D * T;                        // D * T
    double* hs = su + D * T;                        // nops * ncell (SMEM)
    unsigned* hc = reinterpret_cast<unsigned*>(hs + (SMEM ? (size_t)a.nops * ncell : 0));
    const LutEntry64* lut = static_cast<const LutEntry64*>(a.lut);
    const int nall = a.nops * ncell;

    if constexpr (SMEM) {
        for (int k = threadIdx.x; k < nall; k += blockDim.x) { hs[k] = 0.0; hc[k] = 0u; }
    }
    int iter = 0;
    for (long long p = a.tp_lo + blockIdx.x; p < a.tp_hi; p += gridDim.x, ++iter) {
        if constexpr (SMEM) {
            if (iter && iter % a.flush_every == 0) {
                __syncthreads();
                joint_flush_fp64(a, hs, hc, nall);
            }
        }
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + tid;
        const bool iv = i < n;
        double xa[D], ua[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            xa[d] = iv ? a.X64[(size_t)d * n + i] : 0.0;
            ua[d] = iv ? a.U64[(size_t)d * n + i] : 0.0;
        }
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        if ((int)threadIdx.x < jn) {
#pragma unroll
            for (int d = 0; d < D; ++d) {
                sx[d * T + threadIdx.x] = a.X64[(size_t)d * n + j0 + threadIdx.x];
                su[d * T + threadIdx.x] = a.U64[(size_t)d * n + j0 + threadIdx.x];
            }
        }
        __syncthreads();
        if (!iv) continue;
        const int jbeg = ((ti == tj) ? tid + 1 : 0) + half;
        for (int jj = jbeg; jj < jn; jj += SPLIT) {
            double dx[D], du[D];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                dx[d] = SFB_SUB(sx[d * T + jj], xa[d]);
                du[d] = SFB_SUB(su[d * T + jj], ua[d]);
            }
            const double r2 = x_dot<D>(dx, dx);
            int db;
            if (a.dist_linear) db = (r2 != r2) ? a.n_edges : linear_bin(a.dlin, SFB_SQRT(r2));
            else db = (r2 != r2) ? a.n_edges : lut64_bin(lut, a, r2);
            if (db < 1 || db > nd) continue;
            const double inv_r = SFB_DIV(1.0, SFB_SQRT(r2));
            const double duL = SFB_MUL(x_dot<D>(du, dx), inv_r);
            const double dn2 = x_dot<D>(du, du);
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                if (t < r0 || t >= r1) continue;
                const double v = x_sp2d_row(t, duL, dn2);
                const int vb = value_exact_bin(a, v);
                if (vb < 1 || vb > nv) continue;
                const int cell = (t - r0) * ncell + (db - 1) + nd * (vb - 1);
                if constexpr (SMEM) {
                    atomicAdd(&hs[cell], v);
                    atomicAdd(&hc[cell], 1u);
                } else {
                    atomicAdd(&a.g_sums[cell], v);
                    atomicAdd(&a.g_counts[cell], 1ull);
                }
            }
        }
    }
    if constexpr (SMEM) {
        __syncthreads();
        joint_flush_fp64(a, hs, hc, nall);
    }
}

// ------------------------------------------------------------------------------------ mixed
// Value-bin centre of value bin vb in [1, nv] (FP64: the offsets from it stay within half a bin
// width even where the bin is narrow next to its centre).
__device__ __forceinline__ double value_center(const PairArgs& a, int vb)
{
    if (a.val_linear) return a.vlin.first + ((double)vb - 0.5) * a.vlin.step;
    return 0.5 * a.vedges[vb - 1] + 0.5 * a.vedges[vb];
}

// Compensated dot product (Ogita-Rump-Oishi Dot2): the exact product errors come from fma and the
// sum errors from a two-sum, so the result is as accurate as if computed in twice the precision.
// Used for the joint value axis, where cells near du_L = 0 hold values that a plain FP32 dot product
// (with cancellation) would get wrong in the leading digits.
template <int K>
__device__ __forceinline__ float dot2(const float* x, const float* y)
{
    float p = __fmul_rn(x[0], y[0]);
    float e = __fmaf_rn(x[0], y[0], -p);
#pragma unroll
    for (int k = 1; k < K; ++k) {
        const float q = __fmul_rn(x[k], y[k]);
        const float eq = __fmaf_rn(x[k], y[k], -q);
        const float s = __fadd_rn(p, q);
        const float bp = __fsub_rn(s, p);
        const float es = __fadd_rn(__fsub_rn(p, __fsub_rn(s, bp)), __fsub_rn(q, bp));
        p = s;
        e = __fadd_rn(e, __fadd_rn(eq, es));
    }
    return __fadd_rn(p, e);
}

// Whether value bin vb (1-based) keeps its offsets as an FP64 sum (the bins near zero, where a value
// can be tiny next to a quantum tied to the bin width) rather than in fixed point.
__device__ __forceinline__ bool fine_value_bin(const PairArgs& a, int vb)
{
    return (unsigned)(vb - a.vfine_lo) < (unsigned)a.nfine;
}

// Add the block's cells (count, offset sum: fixed point, or FP64 in the fine bins) into the global FP64
// histogram and clear them (all threads, after a barrier).
__device__ __forceinline__ void joint_flush_mixed(const PairArgs& a, unsigned long long* hres, unsigned* hc,
                                                  int ncell)
{
    for (int k = threadIdx.x; k < ncell; k += blockDim.x) {
        if (hc[k]) {
            const int vb = k / a.nb + 1;
            const double off = fine_value_bin(a, vb) ? __longlong_as_double((long long)hres[k])
                                                     : (double)(long long)hres[k] * a.vq_inv;
            const double s = (double)hc[k] * value_center(a, vb) + off;
            atomicAdd(&a.g_sums[k], s);
            atomicAdd(&a.g_counts[k], (unsigned long long)hc[k]);
            hres[k] = 0ull;
            hc[k] = 0u;
        }
    }
    __syncthreads();
}

template <bool SPHERE, int D, bool DFX, bool DFU, class OPS>
__global__ void __launch_bounds__(512) k_joint_mixed(const PairArgs a)
{
    constexpr int NXF = SPHERE ? ((D == 3) ? 20 : 18) : (DFX ? 2 * D : D);
    constexpr int NUF = SPHERE ? 0 : (DFU ? 2 * D : D);
    constexpr int NV = 1;
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x;
    const int lane = threadIdx.x & 31;
    const int n = a.n;
    const int nd = a.nb, nv = a.nv;
    const int ncell = nd * nv;
    LutEntry32* lut = reinterpret_cast<LutEntry32*>(smem);
    float* sx = reinterpret_cast<float*>(smem + a.lut_bytes);  // NXF * T
    float* su = sx + NXF * T;                                   // NUF * T (flat)
    unsigned long long* hres = reinterpret_cast<unsigned long long*>(su + NUF * T);  // ncell
    unsigned* hc = reinterpret_cast<unsigned*>(hres + ncell);                        // ncell
    float* swin = reinterpret_cast<float*>(hc + ncell);                              // nd + 2
    __shared__ unsigned long long s_recheck;

    for (int k = threadIdx.x; k < a.lut_bytes / (int)sizeof(LutEntry32); k += T)
        lut[k] = static_cast<const LutEntry32*>(a.lut)[k];
    for (int k = threadIdx.x; k < ncell; k += T) { hres[k] = 0ull; hc[k] = 0u; }
    for (int k = threadIdx.x; k < nd + 2; k += T) swin[k] = a.vwin[k];
    if (threadIdx.x == 0) s_recheck = 0ull;
    unsigned long long my_recheck = 0;
    const float vinv = (float)a.vlin.inv_step;
    const float vnegf = (float)a.vlin.neg_f_inv;
    const float tmax = (float)(a.vlin.n - 1);

    int iter = 0;
    for (long long p = a.tp_lo + blockIdx.x; p < a.tp_hi; p += gridDim.x, ++iter) {
        if (iter && iter % a.flush_every == 0) {
            __syncthreads();
            joint_flush_mixed(a, hres, hc, ncell);
        }
        int ti, tj;
        decode_tile_pair(p, a.ntiles, ti, tj);
        const int i = ti * T + threadIdx.x;
        const bool iv = i < n;
        float xa[NXF], ua[NUF > 0 ? NUF : 1];
#pragma unroll
        for (int c = 0; c < NXF; ++c) xa[c] = iv ? a.XF[(size_t)c * n + i] : 0.f;
#pragma unroll
        for (int c = 0; c < NUF; ++c) ua[c] = iv ? a.UF[(size_t)c * n + i] : 0.f;
        __syncthreads();
        const int j0 = tj * T;
        const int jn = min(T, n - j0);
        if ((int)threadIdx.x < jn) {
#pragma unroll
            for (int c = 0; c < NXF; ++c) sx[c * T + threadIdx.x] = a.XF[(size_t)c * n + j0 + threadIdx.x];
#pragma unroll
            for (int c = 0; c < NUF; ++c) su[c * T + threadIdx.x] = a.UF[(size_t)c * n + j0 + threadIdx.x];
        }
        __syncthreads();
        const bool diag = ti == tj;
        for (int jj = 0; jj < jn; ++jj) {
            const bool valid = iv && (!diag || jj > (int)threadIdx.x);
            float key, L, Tt, Q;
            if constexpr (!SPHERE) {
                float dx[D], du[D];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    dx[d] = df_diff<DFX>(sx, d, D, T, jj, xa);
                    du[d] = df_diff<DFU>(su, d, D, T, jj, ua);
                }
                const float h2 = fmaf(dx[1], dx[1], dx[0] * dx[0]);
                float r2 = h2;
                if constexpr (D == 3) r2 = fmaf(dx[2], dx[2], h2);
                key = r2;
                const float rs = rsqrtf(r2);
                L = dot2<D>(dx, du) * rs;
                const float t = fmaf(du[1], dx[0], -du[0] * dx[1]);
                Tt = (D == 2) ? t * rs : t * rsqrtf(h2);
                Q = du[0] * du[0];
#pragma unroll
                for (int d = 1; d < D; ++d) Q = fmaf(du[d], du[d], Q);
            } else {
                float d[3], sv[3], dU[3], dW[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    d[c] = df_diff<true>(sx, c, 3, T, jj, xa);
                    sv[c] = __fadd_rn(__fadd_rn(sx[c * T + jj], xa[c]), __fadd_rn(sx[(3 + c) * T + jj], xa[3 + c]));
                    dU[c] = df_diff<true>(sx + 6 * T, c, 3, T, jj, xa + 6);
                    dW[c] = df_diff<true>(sx + 12 * T, c, 3, T, jj, xa + 12);
                }
                const float ch2 = fmaf(d[2], d[2], fmaf(d[1], d[1], d[0] * d[0]));
                key = ch2;
                const float ss = fmaf(sv[2], sv[2], fmaf(sv[1], sv[1], sv[0] * sv[0]));
                const float inv_s = rsqrtf(0.25f * ch2 * ss);
                L = dot2<3>(d, dU) * inv_s;
                Tt = fmaf(d[2], dW[2], fmaf(d[1], dW[1], d[0] * dW[0])) * inv_s;
                Q = fmaf(Tt, Tt, L * L);
                if constexpr (D == 3) {
                    const float dw = df_diff<true>(sx + 18 * T, 0, 1, T, jj, xa + 18);
                    Q = fmaf(dw, dw, Q);
                }
            }
            const LutEntry32 e = lut[lut_cell32(key, a.lg)];
            int db = e.base + (key > e.hi ? (e.mult & 0xffff) : 0);
            bool slow = (e.mult & LUT_FLAG_SLOW) || (key >= e.lo && key <= e.hi);
            float v[NV];
            eval_ops(OPS{}, L, Tt, Q - L * L, Q, D, a.gen, v);
            float val = v[0];
            int vb;
            {
                float t;
                if (a.val_linear) {
                    t = fmaf(val, vinv, vnegf);
                } else {
                    t = 0.f;
                }
                if (a.val_linear) {
                    const float fl = floorf(t);
                    const float fr = t - fl;
                    // absolute part per distance row + relative part (|t| + |first/step|) * vrel
                    const float wt = swin[min(max(db, 0), nd + 1)] + (fabsf(t) + fabsf(vnegf)) * a.vrel;
                    vb = (t <= 0.f) ? 0 : ((t > tmax) ? a.vlin.n : (int)fl + 1);
                    slow = slow || fr < wt || fr > 1.f - wt || fabsf(t) < wt || fabsf(t - tmax) < wt || !(t == t);
                } else {
                    slow = true;  // vector value edges: exact FP64 search
                    vb = 0;
                }
            }
            slow = slow && valid;
            bool ok = true;
            double v64 = 0.0;
            if (__any_sync(FULL, slow)) {
                if (slow) {
                    const int j = j0 + jj;
                    double du64[D];
                    if constexpr (!SPHERE) {
                        double dx64[D];
#pragma unroll
                        for (int d = 0; d < D; ++d) {
                            dx64[d] = SFB_SUB(a.X64[(size_t)d * n + j], a.X64[(size_t)d * n + i]);
                            du64[d] = SFB_SUB(a.U64[(size_t)d * n + j], a.U64[(size_t)d * n + i]);
                        }
                        const double r264 = x_dot<D>(dx64, dx64);
                        db = flat_exact_bin(a, r264);
                        v64 = x_sf_raw<D>(a.gen.op[0], du64, dx64, r264);
                    } else {
                        SphPoint A, B;
                        load_sph64(a.X64, n, i, A);
                        load_sph64(a.X64, n, j, B);
                        double r, tA[2], tB[2], uA[D], uB[D];
                        ok = x_sphere_frame(A, B, a.radius, r, tA, tB);
                        db = sphere_exact_bin(a, r);
#pragma unroll
                        for (int d = 0; d < D; ++d) {
                            uA[d] = a.U64[(size_t)d * n + i];
                            uB[d] = a.U64[(size_t)d * n + j];
                        }
                        x_sphere_delta<D>(tA, tB, uA, uB, du64);
                        v64 = x_sphere_value<D>(a.gen.op[0], du64);
                    }
                    vb = value_exact_bin(a, v64);
                }
                const unsigned sb = __ballot_sync(FULL, slow);
                if (lane == 0) my_recheck += __popc(sb);
            }
            if (valid && ok && db >= 1 && db <= nd && vb >= 1 && vb <= nv) {
                const int cell = (db - 1) + nd * (vb - 1);
                const double c = value_center(a, vb);
                const double off = (slow ? v64 : (double)val) - c;
                if (fine_value_bin(a, vb)) atomicAdd(reinterpret_cast<double*>(&hres[cell]), off);
                else atomicAdd(&hres[cell], (unsigned long long)__double2ll_rn(off * a.vq));
                atomicAdd(&hc[cell], 1u);
            }
        }
    }
    if (lane == 0 && my_recheck) atomicAdd(&s_recheck, my_recheck);
    __syncthreads();
    joint_flush_mixed(a, hres, hc, ncell);
    if (threadIdx.x == 0 && s_recheck) atomicAdd(&a.g_stats[0], s_recheck);
}

}  // namespace sfb
