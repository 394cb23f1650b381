/*
 * sf_oracle.c -- CPU oracle for the pair-histogram hot path. TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library, and
 * only as the checker / the timed CPU reference. The product path (libsfb200.so) never links it.
 *
 * It restates, in plain C with IEEE double arithmetic and no FMA contraction
 * (-ffp-contract=off), the Float64 SerialBackend arithmetic of jbphyswx/StructureFunctions.jl
 * v0.4.0. Inputs given as Float32 are widened exactly to double before any arithmetic (the
 * "FP64 oracle on widened inputs" semantics). Citations are path:line in that repository:
 *
 *   Euclidean 1D pair loop         src/Calculations/serial.jl:68-101   (_pf_simd_pairs!)
 *   Euclidean joint pair loop      src/Calculations/serial_2d.jl:49-85 (_pf_2d_simd_pairs!)
 *   non-Euclidean 1D pair loop     src/Calculations/serial.jl:228-267  (calculate_structure_function_i!)
 *   non-Euclidean joint pair loop  src/Calculations/serial_2d.jl:260-303
 *   threaded baseline              ext/StructureFunctionsOhMyThreadsExt.jl:171-193 (round-robin chunks,
 *                                  per-task histograms merged by +)
 *   squared-edge table             src/BinEdges.jl:440 (_sq_edges), 460-463, 517 (SquaredGeneralPlan)
 *   squared linear plan            src/BinEdges.jl:455-458, 506, 516 (key = sqrt(r2), FMA search)
 *   LinearBinEdges search          src/BinEdges.jl:114-131
 *   generic vector search          Base.searchsortedfirst (binary search with isless), via
 *                                  src/BinEdges.jl:56 and src/HelperFunctions.jl:77-84 (digitize)
 *   raw-geometry operator values   src/StructureFunctionTypes.jl:227-245 (_sf_raw)
 *   operator functors              src/StructureFunctionTypes.jl:58-151
 *   projections, n-hat             src/HelperFunctions.jl:450-468, 624-683
 *   spherical frame                src/HelperFunctions.jl:133-153, 186-200, 265-276, 324-348
 *   bin average                    src/Calculations/serial.jl:132-141
 *   six-invariant single pass      src/Calculations/serial_single_pass.jl:238-270 (Euclidean SIMD loop),
 *                                  321-350 (other metrics), 209-219 (derived rows T2, L1T2)
 *   two-dimensional single pass    src/Calculations/serial_single_pass.jl:876-909 (Euclidean SIMD loop:
 *                                  du_L and |du|^2 once per pair), _sp2d_scatter! :852-864 (one cell
 *                                  per row); a joint description of consecutive SFB200_OP_SP2D rows
 *
 * Third-party arithmetic that is not in the reference tree: StaticArrays `dot`/`cross` (compat 1.9,
 * plain left-to-right products and sums, restated literally), StaticArrays `normalize` (restated as
 * v / sqrt(sum of squares)), the @fastmath `norm2` (restated left to right, no FMA; Julia may
 * contract it, so S2/T2 sums are pinned to ~1 ulp, not bit-for-bit), Julia's libm `sincosd`, `sincos`
 * and `atan(y, x)` (replaced by the shared, mpmath-validated sfb200_sphmath.h, <= 1.5 ulp; the ulp of
 * a spherical separation is therefore unpinned against Julia itself, and deterministic against the
 * GPU library, which uses the same header).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/sfb200.h"
#include "../structurefunctions.jl_b200/csrc/sfb200_sphmath.h"

#define OR_EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------- digitize (src/BinEdges.jl) */

/* Julia's isless for floats: -0.0 < 0.0, NaN above everything. */
static int jl_isless(double a, double b)
{
    if (a != a) return 0;
    if (b != b) return 1;
    if (a < b) return 1;
    if (a == b && a == 0.0 && signbit(a) && !signbit(b)) return 1;
    return 0;
}

/* Base.searchsortedfirst(v, x) with Forward ordering: 1-based index of the first element not
 * isless than x, by the same binary search (lo = 0, hi = n + 1). */
OR_EXPORT int64_t oracle_searchsortedfirst_vec(const double* v, int64_t n, double x)
{
    int64_t lo = 0, hi = n + 1;
    while (lo < hi - 1) {
        const int64_t m = lo + ((hi - lo) >> 1);
        if (jl_isless(v[m - 1], x)) lo = m; else hi = m;
    }
    return hi;
}

/* searchsortedfirst(::LinearBinEdges, x), src/BinEdges.jl:114-131. NaN: the reference throws
 * (floor(Int, NaN)); the oracle reports n + 1 (out of range), as the library does. */
OR_EXPORT int64_t oracle_searchsortedfirst_linear(double f, double l, double inv_step, double step,
                                                  int64_t n, double x)
{
    if (x <= f) return 1;
    if (x > l) return n + 1;
    if (x != x) return n + 1;
    const double t = fma(x, inv_step, -f * inv_step);
    int64_t idx = (int64_t)floor(t) + 1;
    if (idx < 1) idx = 1;
    if (idx > n) idx = n;
    const double u = fma((double)(idx - 1), step, f);
    return u < x ? idx + 1 : idx;
}

/* digitize(x, BinEdges(edges)) = searchsortedfirst - 1 (src/HelperFunctions.jl:77-84). */
OR_EXPORT int64_t oracle_digitize(const sfb200_bins* b, double x)
{
    if (b->kind == SFB200_BINS_LINEAR)
        return oracle_searchsortedfirst_linear(b->first, b->last, b->inv_step, b->step, b->n_edges, x) - 1;
    return oracle_searchsortedfirst_vec(b->edges, b->n_edges, x) - 1;
}

/* Bin of a Euclidean pair from r^2 (src/BinEdges.jl:515-517, 549-550). `sq` is the squared-edge
 * table for TABLE / SQTABLE plans. */
static int64_t squared_bin(const sfb200_bins* b, const double* sq, double r2)
{
    if (b->kind == SFB200_BINS_LINEAR)
        return oracle_searchsortedfirst_linear(b->first, b->last, b->inv_step, b->step, b->n_edges,
                                               sqrt(r2)) - 1;
    return oracle_searchsortedfirst_vec(sq, b->n_edges, r2) - 1;
}

/* ---------------------------------------------------------------- operators */

static double dotn(const double* a, const double* b, int n)
{
    double s = a[0] * b[0];
    for (int k = 1; k < n; ++k) s = s + a[k] * b[k];
    return s;
}

/* norm2 (src/StructureFunctionTypes.jl:23-31): out = 0; out += x[i]^2 */
static double norm2(const double* x, int n)
{
    double out = 0.0;
    for (int k = 0; k < n; ++k) out = out + x[k] * x[k];
    return out;
}

/* x^p for an integer literal power (Base.literal_pow: p = 2 -> x*x, p = 3 -> x*x*x). */
static double lit_pow(double x, int p)
{
    if (p == 0) return 1.0;
    double r = x;
    for (int k = 1; k < p; ++k) r = r * x;
    return r;
}

/* n-hat(r_hat) (src/HelperFunctions.jl:450-468). */
static void nhat(const double* r, int D, double* n)
{
    if (D == 2) {
        n[0] = -r[1];
        n[1] = r[0];
        return;
    }
    /* normalize(cross(z-hat, r_hat)) with z-hat = (0, 0, 1), written out as StaticArrays does */
    const double v0 = 0.0 * r[2] - 1.0 * r[1];
    const double v1 = 1.0 * r[0] - 0.0 * r[2];
    const double v2 = 0.0 * r[1] - 0.0 * r[0];
    const double nr = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    n[0] = v0 / nr;
    n[1] = v1 / nr;
    n[2] = v2 / nr;
}

/* transverse_norm2 (src/HelperFunctions.jl:668-671): _sum_abs2(du) - du_l^2 */
static double transverse_norm2(const double* du, const double* r, int D)
{
    const double dl = dotn(du, r, D);
    double s = 0.0;
    for (int k = 0; k < D; ++k) s = s + du[k] * du[k];
    return s - dl * dl;
}

/* Row t of the two-dimensional single pass from du_L and |du|^2: (dn2, duL2, dn2 - duL2, duL dn2,
 * duL duL2, duL (dn2 - duL2)) (src/Calculations/serial_single_pass.jl:840-843, 901-905). */
static double sp2d_row(int t, double duL, double dn2)
{
    const double duL2 = duL * duL;
    switch (t) {
    case 0: return dn2;
    case 1: return duL2;
    case 2: return dn2 - duL2;
    case 3: return duL * dn2;
    case 4: return duL * duL2;
    case 5: return duL * (dn2 - duL2);
    }
    return NAN;
}

/* The operator functor sf(du, r_hat) (src/StructureFunctionTypes.jl:58-151). The single-pass rows
 * take du_L = du . r_hat and |du|^2 = du . du (src/Calculations/serial_single_pass.jl:839-841). */
static double sf_functor(const sfb200_operator* op, int D, const double* du, const double* r)
{
    switch (op->kind) {
    case SFB200_OP_SP2D:
        return sp2d_row(op->nl, dotn(du, r, D), dotn(du, du, D));
    case SFB200_OP_PROJECTED: {
        double ex = 1.0;
        if (op->nl != 0) ex = ex * lit_pow(dotn(du, r, D), op->nl);
        if (op->nt != 0) {
            if (op->nt == 2) {
                ex = ex * transverse_norm2(du, r, D);
            } else {
                double n[3];
                nhat(r, D, n);
                ex = ex * lit_pow(dotn(du, n, D), op->nt);
            }
        }
        return ex;
    }
    case SFB200_OP_S2:
        return norm2(du, D);
    case SFB200_OP_S3:
        return dotn(du, r, D) * norm2(du, D);
    case SFB200_OP_FULLVEC:
        if (op->nf == 2) return norm2(du, D);
        return lit_pow(sqrt(norm2(du, D)), op->nf);
    case SFB200_OP_T2C:
        return transverse_norm2(du, r, D) / (double)(D - 1);
    case SFB200_OP_L1T2C:
        return dotn(du, r, D) * (transverse_norm2(du, r, D) / (double)(D - 1));
    }
    return NAN;
}

/* _sf_raw(sf, du, dx, r2) (src/StructureFunctionTypes.jl:227-245). */
static double sf_raw(const sfb200_operator* op, int D, const double* du, const double* dx, double r2)
{
    if (op->kind == SFB200_OP_SP2D) { /* flat single pass (src/Calculations/serial_single_pass.jl:889-893) */
        const double inv_r = 1.0 / sqrt(r2);
        return sp2d_row(op->nl, dotn(du, dx, D) * inv_r, dotn(du, du, D));
    }
    if (op->kind == SFB200_OP_S2) return norm2(du, D);
    if (op->kind == SFB200_OP_PROJECTED && op->nl == 2 && op->nt == 0) {
        const double p = dotn(du, dx, D);
        return p * p / r2;
    }
    if (op->kind == SFB200_OP_PROJECTED && op->nl == 0 && op->nt == 2) {
        const double p = dotn(du, dx, D);
        return norm2(du, D) - p * p / r2;
    }
    if (op->kind == SFB200_OP_T2C) {
        const double p = dotn(du, dx, D);
        return (norm2(du, D) - p * p / r2) / (double)(D - 1);
    }
    const double s = sqrt(r2);
    double r[3];
    for (int k = 0; k < D; ++k) r[k] = dx[k] / s;
    return sf_functor(op, D, du, r);
}

/* ---------------------------------------------------------------- flat (Euclidean) path */

typedef struct {
    const sfb200_plan_desc* d;
    const double* sq;   /* squared distance edges (TABLE/SQTABLE) */
    int64_t nd, nv;     /* distance bins, value bins */
} plan_view;

static void plan_view_init(plan_view* pv, const sfb200_plan_desc* d, double* sqbuf)
{
    pv->d = d;
    pv->nd = d->distance.n_edges - 1;
    pv->nv = d->joint ? d->value.n_edges - 1 : 0;
    pv->sq = NULL;
    if (d->geometry == SFB200_GEOM_FLAT && d->distance.kind != SFB200_BINS_LINEAR) {
        if (d->distance.kind == SFB200_BINS_SQTABLE) {
            pv->sq = d->distance.edges;
        } else {
            for (int k = 0; k < d->distance.n_edges; ++k)
                sqbuf[k] = d->distance.edges[k] * d->distance.edges[k];
            pv->sq = sqbuf;
        }
    }
}

/* One outer index i of the Euclidean loop, pairs (i, j > i). x is (D, N), u is (D, N). */
static void flat_row(const plan_view* pv, const double* x, const double* u, int64_t N, int64_t i,
                     double* sums, uint64_t* counts, double* abss)
{
    const sfb200_plan_desc* d = pv->d;
    const int D = d->dim;
    const double* xi = x + (size_t)D * i;
    const double* ui = u + (size_t)D * i;
    for (int64_t j = i + 1; j < N; ++j) {
        const double* xj = x + (size_t)D * j;
        const double* uj = u + (size_t)D * j;
        double dx[3] = {0.0, 0.0, 0.0}, du[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < D; ++k) dx[k] = xj[k] - xi[k];
        const double r2 = dotn(dx, dx, D);
        const int64_t b = squared_bin(&d->distance, pv->sq, r2);
        if (!(b >= 1 && b <= pv->nd)) continue;
        for (int k = 0; k < D; ++k) du[k] = uj[k] - ui[k];
        if (!d->joint) {
            for (int o = 0; o < d->n_ops; ++o) {
                const double val = sf_raw(&d->ops[o], D, du, dx, r2);
                sums[(size_t)o * pv->nd + (b - 1)] += val;
                if (abss) abss[(size_t)o * pv->nd + (b - 1)] += fabs(val);
            }
            counts[b - 1] += 1;
        } else if (d->n_ops > 1) {
            /* consecutive rows of the two-dimensional single pass on one value axis: the pass's own
             * du_L = (du . dx) * inv(sqrt(r2)) and |du|^2 once, then each row's scatter; row o's cells
             * follow row o - 1's (the same arithmetic as sf_raw's SFB200_OP_SP2D case) */
            const double inv_r = 1.0 / sqrt(r2);
            const double duL = dotn(du, dx, D) * inv_r;
            const double dn2 = dotn(du, du, D);
            for (int o = 0; o < d->n_ops; ++o) {
                const double val = sp2d_row(d->ops[o].nl, duL, dn2);
                const int64_t vb = oracle_digitize(&d->value, val);
                if (vb >= 1 && vb <= pv->nv) {
                    const size_t cell = (size_t)o * (size_t)(pv->nd * pv->nv) + (size_t)(b - 1) +
                                        (size_t)pv->nd * (size_t)(vb - 1);
                    sums[cell] += val;
                    counts[cell] += 1;
                    if (abss) abss[cell] += fabs(val);
                }
            }
        } else {
            const double val = sf_raw(&d->ops[0], D, du, dx, r2);
            const int64_t vb = oracle_digitize(&d->value, val);
            if (vb >= 1 && vb <= pv->nv) {
                const size_t cell = (size_t)(b - 1) + (size_t)pv->nd * (size_t)(vb - 1);
                sums[cell] += val;
                counts[cell] += 1;
                if (abss) abss[cell] += fabs(val);
            }
        }
    }
}

/* ---------------------------------------------------------------- sphere path */

typedef struct {
    double p[3];  /* unit position */
    double E[3];  /* local east */
    double Nn[3]; /* local north */
} sph_point;

/* unit_position / local_east_north (src/HelperFunctions.jl:133-153, 404-409). */
static void sph_point_init(sph_point* P, double lon, double lat, int unit)
{
    double sl, cl, sp, cp;
    if (unit == SFB200_ANGLE_DEG) {
        sfb_sincosd(lon, &sl, &cl);
        sfb_sincosd(lat, &sp, &cp);
    } else {
        sfb_sincos(lon, &sl, &cl);
        sfb_sincos(lat, &sp, &cp);
    }
    P->p[0] = cp * cl; P->p[1] = cp * sl; P->p[2] = sp;
    P->E[0] = -sl; P->E[1] = cl; P->E[2] = 0.0;
    P->Nn[0] = -sp * cl; P->Nn[1] = -sp * sl; P->Nn[2] = cp;
}

static double dot3(const double* a, const double* b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* pair_frame(::SphericalGeometry) + geodesic_frame (src/HelperFunctions.jl:186-200, 265-276).
 * Returns ok; writes r, and the local longitudinal tangents tA, tB (2 components each). */
OR_EXPORT int oracle_sphere_frame(const double* A /*p,E,N*/, const double* B, double radius,
                                  double* r_out, double* tA, double* tB)
{
    const double* p = A;
    const double* EA = A + 3;
    const double* NA = A + 6;
    const double* q = B;
    const double* EB = B + 3;
    const double* NB = B + 6;
    double d[3], s[3], t_A[3], t_B[3], w[3];
    for (int k = 0; k < 3; ++k) d[k] = q[k] - p[k];
    for (int k = 0; k < 3; ++k) s[k] = p[k] + q[k];
    const double dp = dot3(d, p);
    for (int k = 0; k < 3; ++k) t_A[k] = d[k] - dp * p[k];
    for (int k = 0; k < 3; ++k) t_B[k] = dp * q[k] + d[k];
    w[0] = p[1] * d[2] - p[2] * d[1];
    w[1] = p[2] * d[0] - p[0] * d[2];
    w[2] = p[0] * d[1] - p[1] * d[0];
    const double s2 = dot3(w, w);
    const double sigma = 2.0 * sfb_atan2_pos(sqrt(dot3(d, d)), sqrt(dot3(s, s)));
    const int ok = s2 > 2.2250738585072014e-308; /* floatmin(Float64) */
    const double inv_s = ok ? 1.0 / sqrt(s2) : 0.0;
    double ta[3], tb[3];
    for (int k = 0; k < 3; ++k) { ta[k] = t_A[k] * inv_s; tb[k] = t_B[k] * inv_s; }
    tA[0] = dot3(ta, EA); tA[1] = dot3(ta, NA);
    tB[0] = dot3(tb, EB); tB[1] = dot3(tb, NB);
    *r_out = radius * sigma;
    return ok;
}

/* pair_delta(::SphericalGeometry{2|3}) (src/HelperFunctions.jl:324-348); du in the pair frame. */
static void sphere_delta(int D, const double* tA, const double* tB, const double* uA,
                         const double* uB, double* du)
{
    const double nA[2] = {-tA[1], tA[0]};
    const double nB[2] = {-tB[1], tB[0]};
    du[0] = (uB[0] * tB[0] + uB[1] * tB[1]) - (uA[0] * tA[0] + uA[1] * tA[1]);
    du[1] = (uB[0] * nB[0] + uB[1] * nB[1]) - (uA[0] * nA[0] + uA[1] * nA[1]);
    if (D == 3) du[2] = uB[2] - uA[2];
}

static void sphere_row(const plan_view* pv, const sph_point* P, const double* u, int64_t N,
                       int64_t i, double* sums, uint64_t* counts, double* abss)
{
    const sfb200_plan_desc* d = pv->d;
    const int D = d->dim;
    const double rh[3] = {1.0, 0.0, 0.0}; /* pair_direction(::SphericalGeometry) = e1 */
    const double* ui = u + (size_t)D * i;
    for (int64_t j = i + 1; j < N; ++j) {
        double r, tA[2], tB[2];
        const int ok = oracle_sphere_frame((const double*)&P[i], (const double*)&P[j], d->radius,
                                           &r, tA, tB);
        const int64_t b = oracle_digitize(&d->distance, r);
        if (!(ok && b >= 1 && b <= pv->nd)) continue;
        double du[3];
        sphere_delta(D, tA, tB, ui, u + (size_t)D * j, du);
        if (!d->joint) {
            for (int o = 0; o < d->n_ops; ++o) {
                const double val = sf_functor(&d->ops[o], D, du, rh);
                sums[(size_t)o * pv->nd + (b - 1)] += val;
                if (abss) abss[(size_t)o * pv->nd + (b - 1)] += fabs(val);
            }
            counts[b - 1] += 1;
        } else {
            const double val = sf_functor(&d->ops[0], D, du, rh);
            const int64_t vb = oracle_digitize(&d->value, val);
            if (vb >= 1 && vb <= pv->nv) {
                const size_t cell = (size_t)(b - 1) + (size_t)pv->nd * (size_t)(vb - 1);
                sums[cell] += val;
                counts[cell] += 1;
                if (abss) abss[cell] += fabs(val);
            }
        }
    }
}

/* ---------------------------------------------------------------- drivers */

/* a joint description of several operators: consecutive flat single-pass 2D rows (one matrix each) */
static int64_t out_len(const plan_view* pv)
{
    return pv->d->joint ? pv->nd * pv->nv * pv->d->n_ops : pv->nd * pv->d->n_ops;
}

static int64_t count_len(const plan_view* pv)
{
    return pv->d->joint ? pv->nd * pv->nv * pv->d->n_ops : pv->nd;
}

/* A joint description of several operators must be consecutive flat single-pass 2D rows. */
static int joint_ops_ok(const sfb200_plan_desc* d)
{
    if (!d->joint || d->n_ops == 1) return 1;
    if (d->geometry != SFB200_GEOM_FLAT || d->n_ops < 2 || d->n_ops > 6) return 0;
    for (int o = 0; o < d->n_ops; ++o)
        if (d->ops[o].kind != SFB200_OP_SP2D || d->ops[o].nl != d->ops[0].nl + o || d->ops[o].nl > 5) return 0;
    return 1;
}

/* Rows i = i0, i0 + istep, ... (the round-robin share of src/Calculations/serial.jl:372-377 and
 * ext/StructureFunctionsOhMyThreadsExt.jl:33-34), accumulated into sums / counts. */
static void run_rows(const plan_view* pv, const double* x, const double* u, const sph_point* P,
                     int64_t N, int64_t i0, int64_t istep, double* sums, uint64_t* counts, double* abss)
{
    for (int64_t i = i0; i < N - 1; i += istep) {
        if (pv->d->geometry == SFB200_GEOM_FLAT)
            flat_row(pv, x, u, N, i, sums, counts, abss);
        else
            sphere_row(pv, P, u, N, i, sums, counts, abss);
    }
}

static sph_point* sphere_points(const sfb200_plan_desc* d, const double* x, int64_t N)
{
    sph_point* P = (sph_point*)malloc(sizeof(sph_point) * (size_t)(N > 0 ? N : 1));
    if (!P) return NULL;
    for (int64_t i = 0; i < N; ++i) sph_point_init(&P[i], x[2 * i], x[2 * i + 1], d->angle_unit);
    return P;
}

/* Serial oracle: accumulates (adds) into sums / counts, which the caller zeroes. When `abss` is
 * not NULL it also accumulates the per-bin sum of |value| (the tolerance scale of the parity tests).
 * x: (W, N) doubles, u: (D, N) doubles. Returns 0, or -1 on allocation failure. */
OR_EXPORT int oracle_run(const sfb200_plan_desc* d, const double* x, const double* u, int64_t N,
                         int64_t i0, int64_t istep, double* sums, uint64_t* counts, double* abss)
{
    double sqbuf[4096];
    if (d->distance.n_edges > 4096 || !joint_ops_ok(d)) return -1;
    plan_view pv;
    plan_view_init(&pv, d, sqbuf);
    sph_point* P = NULL;
    if (d->geometry == SFB200_GEOM_SPHERE) {
        P = sphere_points(d, x, N);
        if (!P) return -1;
    }
    run_rows(&pv, x, u, P, N, i0, istep > 0 ? istep : 1, sums, counts, abss);
    free(P);
    return 0;
}

/* Threaded oracle (restates _threaded_pf_simd!, ext/StructureFunctionsOhMyThreadsExt.jl:171-193):
 * `nthreads` round-robin outer-index chunks, one private histogram per chunk, merged with +.
 * Used as the timed CPU baseline. */
OR_EXPORT int oracle_run_threaded(const sfb200_plan_desc* d, const double* x, const double* u,
                                  int64_t N, int nthreads, double* sums, uint64_t* counts)
{
    double sqbuf[4096];
    if (d->distance.n_edges > 4096 || !joint_ops_ok(d)) return -1;
    plan_view pv;
    plan_view_init(&pv, d, sqbuf);
    sph_point* P = NULL;
    if (d->geometry == SFB200_GEOM_SPHERE) {
        P = sphere_points(d, x, N);
        if (!P) return -1;
    }
    if (nthreads < 1) nthreads = 1;
    const int64_t ns = out_len(&pv), nc = count_len(&pv);
    double* ls = (double*)calloc((size_t)ns * nthreads, sizeof(double));
    uint64_t* lc = (uint64_t*)calloc((size_t)nc * nthreads, sizeof(uint64_t));
    if (!ls || !lc) { free(ls); free(lc); free(P); return -1; }
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
#endif
    for (int t = 0; t < nthreads; ++t)
        run_rows(&pv, x, u, P, N, t, nthreads, ls + (size_t)ns * t, lc + (size_t)nc * t, NULL);
    for (int t = 0; t < nthreads; ++t) {
        for (int64_t k = 0; k < ns; ++k) sums[k] += ls[(size_t)ns * t + k];
        for (int64_t k = 0; k < nc; ++k) counts[k] += lc[(size_t)nc * t + k];
    }
    free(ls); free(lc); free(P);
    return 0;
}

/* ---------------------------------------------------------------- six-invariant single pass */

/* Rows of the single-pass accumulator (src/Calculations/batch_api.jl:98, serial_single_pass.jl:593-600):
 * 0 S2 = |du|^2, 1 L2 = du_L^2, 2 T2 = S2 - L2 (derived), 3 S3 = du_L |du|^2, 4 L3 = du_L^3,
 * 5 L1T2 = S3 - L3 (derived). Sums and counts are (6, nb) column-major: element (t, b) at t + 6 b. */
#define SP_N 6

static void sp_add(double* sums, uint64_t* counts, double* abss, int64_t b, double duL, double dn2)
{
    const double duL2 = duL * duL;
    const double v[4] = {dn2, duL2, duL * dn2, duL * duL2};
    const int row[4] = {0, 1, 3, 4};
    for (int k = 0; k < 4; ++k) {
        sums[row[k] + SP_N * b] += v[k];
        if (abss) abss[row[k] + SP_N * b] += fabs(v[k]);
    }
    counts[SP_N * b] += 1;
}

/* _pf_sp_simd_pairs! (serial_single_pass.jl:238-270): du_L = dot(du, dx) * inv(sqrt(r2)),
 * dn2 = dot(du, du); the bin from r2 by the squared plan. Other metrics: _sp1d_pairs!
 * (serial_single_pass.jl:321-350), du_L = du . r_hat in the pair frame (r_hat = e1 on the sphere). */
static void sp_rows(const plan_view* pv, const double* x, const double* u, const sph_point* P, int64_t N,
                    int64_t i0, int64_t istep, double* sums, uint64_t* counts, double* abss)
{
    const sfb200_plan_desc* d = pv->d;
    const int D = d->dim;
    for (int64_t i = i0; i < N - 1; i += istep) {
        const double* ui = u + (size_t)D * i;
        for (int64_t j = i + 1; j < N; ++j) {
            const double* uj = u + (size_t)D * j;
            double du[3] = {0.0, 0.0, 0.0}, duL;
            int64_t b;
            if (d->geometry == SFB200_GEOM_FLAT) {
                const double* xi = x + (size_t)D * i;
                const double* xj = x + (size_t)D * j;
                double dx[3] = {0.0, 0.0, 0.0};
                for (int k = 0; k < D; ++k) dx[k] = xj[k] - xi[k];
                const double r2 = dotn(dx, dx, D);
                b = squared_bin(&d->distance, pv->sq, r2);
                if (!(b >= 1 && b <= pv->nd)) continue;
                for (int k = 0; k < D; ++k) du[k] = uj[k] - ui[k];
                const double inv_r = 1.0 / sqrt(r2);
                duL = dotn(du, dx, D) * inv_r;
            } else {
                double r, tA[2], tB[2];
                const int ok = oracle_sphere_frame((const double*)&P[i], (const double*)&P[j], d->radius, &r, tA, tB);
                b = oracle_digitize(&d->distance, r);
                if (!(ok && b >= 1 && b <= pv->nd)) continue;
                sphere_delta(D, tA, tB, ui, uj, du);
                duL = du[0];  /* dot(du, e1) */
            }
            sp_add(sums, counts, abss, b - 1, duL, dotn(du, du, D));
        }
    }
}

/* _sp1d_derive_rows! (serial_single_pass.jl:209-219): T2 = S2 - L2, L1T2 = S3 - L3, counts of row 0
 * copied to every row. Idempotent (assignments). */
OR_EXPORT void oracle_single_pass_derive(double* sums, uint64_t* counts, int64_t nb)
{
    for (int64_t b = 0; b < nb; ++b) {
        sums[2 + SP_N * b] = sums[0 + SP_N * b] - sums[1 + SP_N * b];
        sums[5 + SP_N * b] = sums[3 + SP_N * b] - sums[4 + SP_N * b];
        for (int t = 1; t < SP_N; ++t) counts[t + SP_N * b] = counts[SP_N * b];
    }
}

/* The six-invariant single pass over rows i0, i0 + istep, ... accumulated into (6, nb) sums/counts
 * (and, if abss is not NULL, the per-bin sums of |value| of the four accumulated rows). The derived
 * rows are NOT filled here: a caller that splits the rows over workers adds the partial results first
 * and then calls oracle_single_pass_derive once. `desc` supplies geometry, distance bins and
 * dimension; its operators are ignored. */
OR_EXPORT int oracle_run_single_pass(const sfb200_plan_desc* d, const double* x, const double* u, int64_t N,
                                     int64_t i0, int64_t istep, double* sums, uint64_t* counts, double* abss)
{
    double sqbuf[4096];
    if (d->distance.n_edges > 4096 || d->joint) return -1;
    plan_view pv;
    plan_view_init(&pv, d, sqbuf);
    sph_point* P = NULL;
    if (d->geometry == SFB200_GEOM_SPHERE) {
        P = sphere_points(d, x, N);
        if (!P) return -1;
    }
    sp_rows(&pv, x, u, P, N, i0, istep > 0 ? istep : 1, sums, counts, abss);
    free(P);
    return 0;
}

/* Single-pair evaluations for known-answer tests of the operator layer. */
OR_EXPORT double oracle_sf_functor(const sfb200_operator* op, int D, const double* du, const double* rhat)
{
    return sf_functor(op, D, du, rhat);
}

OR_EXPORT double oracle_sf_raw(const sfb200_operator* op, int D, const double* du, const double* dx, double r2)
{
    return sf_raw(op, D, du, dx, r2);
}

/* Per-point spherical basis (p, E, N as 9 doubles) for geometry tests. */
OR_EXPORT void oracle_sphere_point(double lon, double lat, int unit, double* out9)
{
    sph_point P;
    sph_point_init(&P, lon, lat, unit);
    memcpy(out9, &P, sizeof(P));
}

/* The shared transcendentals, exported so the tests can check them against mpmath. */
OR_EXPORT void oracle_sincosd(double x, double* s, double* c) { sfb_sincosd(x, s, c); }
OR_EXPORT void oracle_sincos(double x, double* s, double* c) { sfb_sincos(x, s, c); }
OR_EXPORT double oracle_atan2(double y, double x) { return sfb_atan2(y, x); }

OR_EXPORT int oracle_threads_available(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
