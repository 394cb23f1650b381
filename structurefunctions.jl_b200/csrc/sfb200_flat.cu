// sfb200_flat.cu -- instantiations of the Euclidean 1D kernels.
#include "sfb200_internal.h"
#include "sfb200_kernels.cuh"

namespace sfb {

template <int D, bool MIXED, class OPS>
static KernelChoice flat_entry()
{
    if constexpr (MIXED) return {reinterpret_cast<const void*>(&k_flat1d_mixed<D, OPS>), 256};
    else return {reinterpret_cast<const void*>(&k_flat1d_fp64<D, OPS>), 256};
}

template <int D, bool MIXED>
static KernelChoice flat_by_list(int opl)
{
    switch (opl) {
    case OPL_L2: return flat_entry<D, MIXED, OpList<OC_L2>>();
    case OPL_L3: return flat_entry<D, MIXED, OpList<OC_L3>>();
    case OPL_L1: return flat_entry<D, MIXED, OpList<OC_L1>>();
    case OPL_QUAD: return flat_entry<D, MIXED, OpList<OC_L2, OC_T2, OC_L3, OC_T3>>();
    case OPL_GEN1: return flat_entry<D, MIXED, OpList<OC_GEN>>();
    case OPL_GEN2: return flat_entry<D, MIXED, OpList<OC_GEN, OC_GEN>>();
    case OPL_GEN4: return flat_entry<D, MIXED, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>>();
    case OPL_GEN8:
        return flat_entry<D, MIXED, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>>();
    }
    return {nullptr, 0};
}

KernelChoice pick_flat1d(int D, bool mixed, int opl)
{
    if (D == 2) return mixed ? flat_by_list<2, true>(opl) : flat_by_list<2, false>(opl);
    if (D == 3) return mixed ? flat_by_list<3, true>(opl) : flat_by_list<3, false>(opl);
    return {nullptr, 0};
}

}  // namespace sfb
