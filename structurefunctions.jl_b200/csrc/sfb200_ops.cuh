// sfb200_ops.cuh -- operator values from per-pair primitives.
//
// Every operator of src/StructureFunctionTypes.jl:43-151 is a polynomial in four per-pair
// primitives, all in the pair's own frame:
//   L  = du . r_hat                    (signed longitudinal increment, mdu_l)
//   T  = du . n_hat(r_hat)             (signed transverse increment, mdu_t; n_hat = z_hat x r_hat)
//   T2 = |du|^2 - L^2                  (transverse energy, transverse_norm2, src/HelperFunctions.jl:668-671)
//   Q  = |du|^2                        (norm2 / _sum_abs2)
// T2 is passed separately so that a kernel may form it without the cancellation of Q - L^2 (as
// |du x r_hat|^2); the FP64 kernels pass Q - L^2, the reference's own formula.
// Common operators get a compile-time code so a fused kernel evaluates exactly what it needs; any
// other ProjectedStructureFunctionType{NL,NT} / FullVector{NF} goes through the generic code.
#pragma once

#include "sfb200_common.cuh"

namespace sfb {

enum OpCode : int {
    OC_L1 = 0,    // {1,0}: du_L
    OC_L2 = 1,    // L2SF {2,0}
    OC_T2 = 2,    // T2SF {0,2}
    OC_S2 = 3,    // S2SF, FullVector{2}
    OC_L3 = 4,    // L3SF {3,0}
    OC_T3 = 5,    // T3SF {0,3}
    OC_S3 = 6,    // S3SF: du_L |du|^2
    OC_L1T2 = 7,  // L1T2SF {1,2}
    OC_L2T1 = 8,  // L2T1SF {2,1}
    OC_T2C = 9,   // T2ComponentSF
    OC_L1T2C = 10,// L1T2ComponentSF
    OC_GEN = 11   // anything else, from the runtime descriptor
};

template <int... K>
struct OpList {
    static constexpr int n = sizeof...(K);
};

template <int K>
constexpr bool op_needs_T() { return K == OC_T3 || K == OC_L2T1 || K == OC_GEN; }
template <int K>
constexpr bool op_needs_Q() {
    return K == OC_T2 || K == OC_S2 || K == OC_S3 || K == OC_L1T2 || K == OC_T2C || K == OC_L1T2C ||
           K == OC_GEN;
}
template <int K>
constexpr bool op_needs_L() { return K != OC_S2 && K != OC_T3; }

template <typename L> struct ListNeeds;
template <int... K>
struct ListNeeds<OpList<K...>> {
    static constexpr bool T = (op_needs_T<K>() || ...);
    static constexpr bool Q = (op_needs_Q<K>() || ...);
    static constexpr bool L = (op_needs_L<K>() || ...);
};

struct GenOps {
    sfb200_operator op[SFB200_MAX_OPS];
};

template <typename R>
__device__ __forceinline__ R ipow(R x, int p)
{
    R r = R(1);
    for (int k = 0; k < p; ++k) r = r * x;
    return r;
}

// Generic operator from its descriptor (runtime-uniform branches).
template <typename R>
__device__ __forceinline__ R gen_value(const sfb200_operator& o, R L, R T, R T2, R Q, int D)
{
    switch (o.kind) {
    case SFB200_OP_PROJECTED: {
        R ex = ipow(L, o.nl);
        if (o.nt == 2) ex = ex * T2;
        else if (o.nt != 0) ex = ex * ipow(T, o.nt);
        return ex;
    }
    case SFB200_OP_S2: return Q;
    case SFB200_OP_S3: return L * Q;
    case SFB200_OP_FULLVEC: return o.nf == 2 ? Q : ipow(sqrt(Q), o.nf);
    case SFB200_OP_T2C: return T2 / R(D - 1);
    case SFB200_OP_L1T2C: return L * (T2 / R(D - 1));
    case SFB200_OP_SP2D:  // rows S2, L2, T2, S3, L3, L1T2 of the two-dimensional single pass
        switch (o.nl) {
        case 0: return Q;
        case 1: return L * L;
        case 2: return T2;
        case 3: return L * Q;
        case 4: return L * L * L;
        case 5: return L * T2;
        }
    }
    return R(0) / R(0);
}

template <int K, typename R>
__device__ __forceinline__ R op_value(R L, R T, R T2, R Q, int D, const sfb200_operator& g)
{
    if constexpr (K == OC_L1) return L;
    else if constexpr (K == OC_L2) return L * L;
    else if constexpr (K == OC_T2) return T2;
    else if constexpr (K == OC_S2) return Q;
    else if constexpr (K == OC_L3) return L * L * L;
    else if constexpr (K == OC_T3) return T * T * T;
    else if constexpr (K == OC_S3) return L * Q;
    else if constexpr (K == OC_L1T2) return L * T2;
    else if constexpr (K == OC_L2T1) return L * L * T;
    else if constexpr (K == OC_T2C) return T2 / R(D - 1);
    else if constexpr (K == OC_L1T2C) return L * (T2 / R(D - 1));
    else return gen_value<R>(g, L, T, T2, Q, D);
}

template <typename R, int... K>
__device__ __forceinline__ void eval_ops(OpList<K...>, R L, R T, R T2, R Q, int D, const GenOps& g,
                                         R (&v)[sizeof...(K)])
{
    int k = 0;
    ((v[k] = op_value<K, R>(L, T, T2, Q, D, g.op[k]), ++k), ...);
}

// Which primitives an operator list needs, with T2 split out (the mixed kernels form T2 and Q
// from separate numerators).
template <int K>
constexpr bool op_needs_T2() { return K == OC_T2 || K == OC_L1T2 || K == OC_T2C || K == OC_L1T2C || K == OC_GEN; }
template <int K>
constexpr bool op_needs_Qonly() { return K == OC_S2 || K == OC_S3 || K == OC_GEN; }

template <typename L> struct ListNeeds2;
template <int... K>
struct ListNeeds2<OpList<K...>> {
    static constexpr bool T = (op_needs_T<K>() || ...);
    static constexpr bool T2 = (op_needs_T2<K>() || ...);
    static constexpr bool Q = (op_needs_Qonly<K>() || ...);
    static constexpr bool L = (op_needs_L<K>() || ...);
};

}  // namespace sfb
