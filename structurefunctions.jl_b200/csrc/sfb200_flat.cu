// sfb200_flat.cu -- instantiations of the Euclidean 1D kernels.
#include "sfb200_internal.h"
#include "sfb200_kernels.cuh"

namespace sfb {

template <int D, int MODE, class OPS>  // MODE 0: FP64, 1: mixed FP32 inputs, 2: mixed FP64 inputs
static KernelChoice flat_entry()
{
    if constexpr (MODE == 1) return {reinterpret_cast<const void*>(&k_flat1d_mixed<D, false, false, OPS>), 256};
    else if constexpr (MODE == 2) return {reinterpret_cast<const void*>(&k_flat1d_mixed<D, true, true, OPS>), 256};
    else return {reinterpret_cast<const void*>(&k_flat1d_fp64<D, OPS>), 256};
}

template <int D, int MODE>
static KernelChoice flat_by_list(int opl)
{
    switch (opl) {
    case OPL_L2: return flat_entry<D, MODE, OpList<OC_L2>>();
    case OPL_L3: return flat_entry<D, MODE, OpList<OC_L3>>();
    case OPL_L1: return flat_entry<D, MODE, OpList<OC_L1>>();
    case OPL_QUAD: return flat_entry<D, MODE, OpList<OC_L2, OC_T2, OC_L3, OC_T3>>();
    case OPL_GEN1: return flat_entry<D, MODE, OpList<OC_GEN>>();
    case OPL_GEN2: return flat_entry<D, MODE, OpList<OC_GEN, OC_GEN>>();
    case OPL_GEN4: return flat_entry<D, MODE, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>>();
    case OPL_GEN8:
        return flat_entry<D, MODE, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>>();
    }
    return {nullptr, 0};
}

KernelChoice pick_flat1d(int D, bool mixed, bool df, int opl)
{
    const int mode = mixed ? (df ? 2 : 1) : 0;
    if (D == 2) return mode == 0 ? flat_by_list<2, 0>(opl) : (mode == 1 ? flat_by_list<2, 1>(opl) : flat_by_list<2, 2>(opl));
    if (D == 3) return mode == 0 ? flat_by_list<3, 0>(opl) : (mode == 1 ? flat_by_list<3, 1>(opl) : flat_by_list<3, 2>(opl));
    return {nullptr, 0};
}

}  // namespace sfb
