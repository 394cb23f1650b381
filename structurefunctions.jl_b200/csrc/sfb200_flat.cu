// sfb200_flat.cu -- instantiations of the Euclidean 1D kernels.
#include "sfb200_internal.h"
#include "sfb200_kernels.cuh"

namespace sfb {

template <int D, int MODE, class OPS, int PRIV>  // MODE 0: FP64, 1: FP32-bulk on FP32 inputs, 2: FP32-bulk on FP64 inputs
static KernelChoice flat_kernel()
{
    if constexpr (MODE == 1) return {reinterpret_cast<const void*>(&k_flat1d_mixed<D, false, false, OPS, PRIV>), 256, PRIV};
    else if constexpr (MODE == 2) return {reinterpret_cast<const void*>(&k_flat1d_mixed<D, true, true, OPS, PRIV>), 256, PRIV};
    else return {reinterpret_cast<const void*>(&k_flat1d_fp64<D, OPS, PRIV>), 256, PRIV};
}

// Specialized operator lists get every privatization depth; generic lists warp-aggregated,
// run-length or per lane.
template <int D, int MODE, class OPS, bool ALL>
static KernelChoice flat_entry(int priv)
{
    switch (priv) {
    case 32: return flat_kernel<D, MODE, OPS, 32>();
    case 3: return flat_kernel<D, MODE, OPS, 3>();
    case 6: if constexpr (MODE == 0) return flat_kernel<D, MODE, OPS, 6>(); break;
    case 8: if constexpr (ALL) return flat_kernel<D, MODE, OPS, 8>(); break;
    case 4: if constexpr (ALL) return flat_kernel<D, MODE, OPS, 4>(); break;
    case 1: if constexpr (ALL) return flat_kernel<D, MODE, OPS, 1>(); break;
    case 2: if constexpr (ALL) return flat_kernel<D, MODE, OPS, 2>(); break;
    }
    return flat_kernel<D, MODE, OPS, 0>();
}

template <int D, int MODE>
static KernelChoice flat_by_list(int opl, int priv)
{
    switch (opl) {
    case OPL_L2: return flat_entry<D, MODE, OpList<OC_L2>, true>(priv);
    case OPL_L3: return flat_entry<D, MODE, OpList<OC_L3>, true>(priv);
    case OPL_L1: return flat_entry<D, MODE, OpList<OC_L1>, true>(priv);
    case OPL_QUAD: return flat_entry<D, MODE, OpList<OC_L2, OC_T2, OC_L3, OC_T3>, true>(priv);
    case OPL_SP: return flat_entry<D, MODE, OpList<OC_S2, OC_L2, OC_S3, OC_L3>, false>(priv);
    case OPL_GEN1: return flat_entry<D, MODE, OpList<OC_GEN>, false>(priv);
    case OPL_GEN2: return flat_entry<D, MODE, OpList<OC_GEN, OC_GEN>, false>(priv);
    case OPL_GEN4: return flat_entry<D, MODE, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv);
    case OPL_GEN8:
        return flat_entry<D, MODE, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv);
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_flat1d(int D, bool fp32, bool df, int opl, int priv)
{
    const int mode = fp32 ? (df ? 2 : 1) : 0;
    if (D == 2)
        return mode == 0 ? flat_by_list<2, 0>(opl, priv)
                         : (mode == 1 ? flat_by_list<2, 1>(opl, priv) : flat_by_list<2, 2>(opl, priv));
    if (D == 3)
        return mode == 0 ? flat_by_list<3, 0>(opl, priv)
                         : (mode == 1 ? flat_by_list<3, 1>(opl, priv) : flat_by_list<3, 2>(opl, priv));
    return {nullptr, 0, 0};
}

}  // namespace sfb
