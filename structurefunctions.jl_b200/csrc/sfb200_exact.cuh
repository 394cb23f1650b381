// sfb200_exact.cuh -- FP64 pair arithmetic in the reference's exact operation order.
//
// Used wherever a result must equal the FP64 reference bit for bit: the distance of every pair in
// the FP64 kernels (it decides the bin), the operator value in joint histograms (it decides the
// value bin), and every pair the FP32 kernels send back for an FP64 recheck. All arithmetic goes
// through __d*_rn intrinsics (SFB_* macros), so no multiply-add is contracted.
//
//   r^2 = dot(dx, dx), left to right          src/Calculations/serial.jl:83-84
//   _sf_raw and the functors                   src/StructureFunctionTypes.jl:58-151, 227-245
//   n_hat, projections                         src/HelperFunctions.jl:450-468, 624-683
//   geodesic_frame, pair_frame, pair_delta     src/HelperFunctions.jl:186-200, 265-276, 324-348
#pragma once

#include "sfb200_common.cuh"
#include "sfb200_sphmath.h"

namespace sfb {

template <int D>
__device__ __forceinline__ double x_dot(const double* a, const double* b)
{
    double s = SFB_MUL(a[0], b[0]);
#pragma unroll
    for (int k = 1; k < D; ++k) s = SFB_ADD(s, SFB_MUL(a[k], b[k]));
    return s;
}

template <int D>
__device__ __forceinline__ double x_norm2(const double* a)
{
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) s = SFB_ADD(s, SFB_MUL(a[k], a[k]));
    return s;
}

__device__ __forceinline__ double x_lit_pow(double x, int p)
{
    if (p == 0) return 1.0;
    double r = x;
    for (int k = 1; k < p; ++k) r = SFB_MUL(r, x);
    return r;
}

template <int D>
__device__ __forceinline__ void x_nhat(const double* r, double* n)
{
    if constexpr (D == 2) {
        n[0] = -r[1];
        n[1] = r[0];
    } else {
        const double v0 = SFB_SUB(SFB_MUL(0.0, r[2]), SFB_MUL(1.0, r[1]));
        const double v1 = SFB_SUB(SFB_MUL(1.0, r[0]), SFB_MUL(0.0, r[2]));
        const double v2 = SFB_SUB(SFB_MUL(0.0, r[1]), SFB_MUL(0.0, r[0]));
        const double nr = SFB_SQRT(SFB_ADD(SFB_ADD(SFB_MUL(v0, v0), SFB_MUL(v1, v1)), SFB_MUL(v2, v2)));
        n[0] = SFB_DIV(v0, nr);
        n[1] = SFB_DIV(v1, nr);
        n[2] = SFB_DIV(v2, nr);
    }
}

template <int D>
__device__ __forceinline__ double x_transverse_norm2(const double* du, const double* r)
{
    const double dl = x_dot<D>(du, r);
    return SFB_SUB(x_norm2<D>(du), SFB_MUL(dl, dl));
}

// Row t of the two-dimensional single pass from du_L and |du|^2, in the reference's order
// (src/Calculations/serial_single_pass.jl:840-843, 901-905).
__device__ __forceinline__ double x_sp2d_row(int t, double duL, double dn2)
{
    const double duL2 = SFB_MUL(duL, duL);
    switch (t) {
    case 0: return dn2;
    case 1: return duL2;
    case 2: return SFB_SUB(dn2, duL2);
    case 3: return SFB_MUL(duL, dn2);
    case 4: return SFB_MUL(duL, duL2);
    case 5: return SFB_MUL(duL, SFB_SUB(dn2, duL2));
    }
    return __longlong_as_double(0x7ff8000000000000ll);
}

// sf(du, r_hat), src/StructureFunctionTypes.jl:58-151; for the single-pass rows du_L = du . r_hat and
// |du|^2 = du . du (src/Calculations/serial_single_pass.jl:839-841, the path of every metric but the
// flat one).
template <int D>
__device__ double x_functor(const sfb200_operator& op, const double* du, const double* r)
{
    switch (op.kind) {
    case SFB200_OP_SP2D: return x_sp2d_row(op.nl, x_dot<D>(du, r), x_dot<D>(du, du));
    case SFB200_OP_PROJECTED: {
        double ex = 1.0;
        if (op.nl != 0) ex = SFB_MUL(ex, x_lit_pow(x_dot<D>(du, r), op.nl));
        if (op.nt != 0) {
            if (op.nt == 2) {
                ex = SFB_MUL(ex, x_transverse_norm2<D>(du, r));
            } else {
                double n[D];
                x_nhat<D>(r, n);
                ex = SFB_MUL(ex, x_lit_pow(x_dot<D>(du, n), op.nt));
            }
        }
        return ex;
    }
    case SFB200_OP_S2: return x_norm2<D>(du);
    case SFB200_OP_S3: return SFB_MUL(x_dot<D>(du, r), x_norm2<D>(du));
    case SFB200_OP_FULLVEC:
        if (op.nf == 2) return x_norm2<D>(du);
        return x_lit_pow(SFB_SQRT(x_norm2<D>(du)), op.nf);
    case SFB200_OP_T2C: return SFB_DIV(x_transverse_norm2<D>(du, r), (double)(D - 1));
    case SFB200_OP_L1T2C:
        return SFB_MUL(x_dot<D>(du, r), SFB_DIV(x_transverse_norm2<D>(du, r), (double)(D - 1)));
    }
    return __longlong_as_double(0x7ff8000000000000ll);
}

// _sf_raw(sf, du, dx, r2), src/StructureFunctionTypes.jl:227-245.
template <int D>
__device__ double x_sf_raw(const sfb200_operator& op, const double* du, const double* dx, double r2)
{
    if (op.kind == SFB200_OP_SP2D) {  // flat single pass: du_L = (du . dx) * inv(sqrt(r2)) (:889-893)
        const double inv_r = SFB_DIV(1.0, SFB_SQRT(r2));
        return x_sp2d_row(op.nl, SFB_MUL(x_dot<D>(du, dx), inv_r), x_dot<D>(du, du));
    }
    if (op.kind == SFB200_OP_S2) return x_norm2<D>(du);
    if (op.kind == SFB200_OP_PROJECTED && op.nl == 2 && op.nt == 0) {
        const double p = x_dot<D>(du, dx);
        return SFB_DIV(SFB_MUL(p, p), r2);
    }
    if (op.kind == SFB200_OP_PROJECTED && op.nl == 0 && op.nt == 2) {
        const double p = x_dot<D>(du, dx);
        return SFB_SUB(x_norm2<D>(du), SFB_DIV(SFB_MUL(p, p), r2));
    }
    if (op.kind == SFB200_OP_T2C) {
        const double p = x_dot<D>(du, dx);
        return SFB_DIV(SFB_SUB(x_norm2<D>(du), SFB_DIV(SFB_MUL(p, p), r2)), (double)(D - 1));
    }
    const double s = SFB_SQRT(r2);
    double r[D];
#pragma unroll
    for (int k = 0; k < D; ++k) r[k] = SFB_DIV(dx[k], s);
    return x_functor<D>(op, du, r);
}

// ---------------------------------------------------------------------------------- sphere

// Per-point FP64 basis: p (unit position), E (local east; its z component is 0), N (local north).
struct SphPoint {
    double p[3];
    double E[2];
    double N[3];
};

__device__ __forceinline__ double x_dot3(const double* a, const double* b)
{
    return SFB_ADD(SFB_ADD(SFB_MUL(a[0], b[0]), SFB_MUL(a[1], b[1])), SFB_MUL(a[2], b[2]));
}

// geodesic_frame + pair_frame. Returns ok; writes r and the local tangents tA, tB.
__device__ __forceinline__ bool x_sphere_frame(const SphPoint& A, const SphPoint& B, double radius,
                                               double& r, double* tA, double* tB)
{
    const double* p = A.p;
    const double* q = B.p;
    double d[3], s[3], ta[3], tb[3], w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = SFB_SUB(q[k], p[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = SFB_ADD(p[k], q[k]);
    const double dp = x_dot3(d, p);
#pragma unroll
    for (int k = 0; k < 3; ++k) ta[k] = SFB_SUB(d[k], SFB_MUL(dp, p[k]));
#pragma unroll
    for (int k = 0; k < 3; ++k) tb[k] = SFB_ADD(SFB_MUL(dp, q[k]), d[k]);
    w[0] = SFB_SUB(SFB_MUL(p[1], d[2]), SFB_MUL(p[2], d[1]));
    w[1] = SFB_SUB(SFB_MUL(p[2], d[0]), SFB_MUL(p[0], d[2]));
    w[2] = SFB_SUB(SFB_MUL(p[0], d[1]), SFB_MUL(p[1], d[0]));
    const double s2 = x_dot3(w, w);
    const double sigma = SFB_MUL(2.0, sfb_atan2_pos(SFB_SQRT(x_dot3(d, d)), SFB_SQRT(x_dot3(s, s))));
    const bool ok = s2 > 2.2250738585072014e-308;
    const double inv_s = ok ? SFB_DIV(1.0, SFB_SQRT(s2)) : 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ta[k] = SFB_MUL(ta[k], inv_s);
        tb[k] = SFB_MUL(tb[k], inv_s);
    }
    const double EA[3] = {A.E[0], A.E[1], 0.0};
    const double EB[3] = {B.E[0], B.E[1], 0.0};
    tA[0] = x_dot3(ta, EA);
    tA[1] = x_dot3(ta, A.N);
    tB[0] = x_dot3(tb, EB);
    tB[1] = x_dot3(tb, B.N);
    r = SFB_MUL(radius, sigma);
    return ok;
}

// pair_delta(::SphericalGeometry{D}) (src/HelperFunctions.jl:324-348).
template <int D>
__device__ __forceinline__ void x_sphere_delta(const double* tA, const double* tB, const double* uA,
                                               const double* uB, double* du)
{
    const double nA0 = -tA[1], nA1 = tA[0];
    const double nB0 = -tB[1], nB1 = tB[0];
    du[0] = SFB_SUB(SFB_ADD(SFB_MUL(uB[0], tB[0]), SFB_MUL(uB[1], tB[1])),
                    SFB_ADD(SFB_MUL(uA[0], tA[0]), SFB_MUL(uA[1], tA[1])));
    du[1] = SFB_SUB(SFB_ADD(SFB_MUL(uB[0], nB0), SFB_MUL(uB[1], nB1)),
                    SFB_ADD(SFB_MUL(uA[0], nA0), SFB_MUL(uA[1], nA1)));
    if constexpr (D == 3) du[2] = SFB_SUB(uB[2], uA[2]);
}

// sf(du, e1) on the sphere: the pair frame's longitudinal direction is e1 by construction.
template <int D>
__device__ __forceinline__ double x_sphere_value(const sfb200_operator& op, const double* du)
{
    double rh[D];
    rh[0] = 1.0;
#pragma unroll
    for (int k = 1; k < D; ++k) rh[k] = 0.0;
    return x_functor<D>(op, du, rh);
}

}  // namespace sfb
