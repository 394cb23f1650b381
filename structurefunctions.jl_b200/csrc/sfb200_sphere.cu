// sfb200_sphere.cu -- instantiations of the spherical 1D kernels.
#include "sfb200_internal.h"
#include "sfb200_kernels.cuh"

namespace sfb {

template <int D, bool MIXED, class OPS>
static KernelChoice sphere_entry()
{
    if constexpr (MIXED) return {reinterpret_cast<const void*>(&k_sphere1d_mixed<D, OPS>), 256};
    else return {reinterpret_cast<const void*>(&k_sphere1d_fp64<D, OPS>), 256};
}

template <int D, bool MIXED>
static KernelChoice sphere_by_list(int opl)
{
    switch (opl) {
    case OPL_L2: return sphere_entry<D, MIXED, OpList<OC_L2>>();
    case OPL_L3: return sphere_entry<D, MIXED, OpList<OC_L3>>();
    case OPL_L1: return sphere_entry<D, MIXED, OpList<OC_L1>>();
    case OPL_QUAD: return sphere_entry<D, MIXED, OpList<OC_L2, OC_T2, OC_L3, OC_T3>>();
    case OPL_GEN1: return sphere_entry<D, MIXED, OpList<OC_GEN>>();
    case OPL_GEN2: return sphere_entry<D, MIXED, OpList<OC_GEN, OC_GEN>>();
    case OPL_GEN4: return sphere_entry<D, MIXED, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>>();
    case OPL_GEN8:
        return sphere_entry<D, MIXED, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>>();
    }
    return {nullptr, 0};
}

KernelChoice pick_sphere1d(int D, bool mixed, int opl)
{
    if (D == 2) return mixed ? sphere_by_list<2, true>(opl) : sphere_by_list<2, false>(opl);
    if (D == 3) return mixed ? sphere_by_list<3, true>(opl) : sphere_by_list<3, false>(opl);
    return {nullptr, 0};
}

}  // namespace sfb
