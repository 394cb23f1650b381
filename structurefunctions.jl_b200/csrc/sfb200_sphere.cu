// sfb200_sphere.cu -- instantiations of the spherical 1D kernels.
#include "sfb200_internal.h"
#include "sfb200_kernels.cuh"

namespace sfb {

template <int D, bool MIXED, class OPS, int PRIV>
static KernelChoice sphere_kernel()
{
    if constexpr (MIXED) return {reinterpret_cast<const void*>(&k_sphere1d_mixed<D, OPS, PRIV>), 256, PRIV};
    else return {reinterpret_cast<const void*>(&k_sphere1d_fp64<D, OPS, PRIV>), 256, PRIV};
}

template <int D, bool MIXED, class OPS, bool ALL>
static KernelChoice sphere_entry(int priv)
{
    switch (priv) {
    case 32: return sphere_kernel<D, MIXED, OPS, 32>();
    case 3: return sphere_kernel<D, MIXED, OPS, 3>();
    case 8: if constexpr (ALL) return sphere_kernel<D, MIXED, OPS, 8>(); break;
    case 4: if constexpr (ALL) return sphere_kernel<D, MIXED, OPS, 4>(); break;
    case 1: if constexpr (ALL) return sphere_kernel<D, MIXED, OPS, 1>(); break;
    case 2: if constexpr (ALL) return sphere_kernel<D, MIXED, OPS, 2>(); break;
    }
    return sphere_kernel<D, MIXED, OPS, 0>();
}

template <int D, bool MIXED>
static KernelChoice sphere_by_list(int opl, int priv)
{
    switch (opl) {
    case OPL_L2: return sphere_entry<D, MIXED, OpList<OC_L2>, true>(priv);
    case OPL_L3: return sphere_entry<D, MIXED, OpList<OC_L3>, true>(priv);
    case OPL_L1: return sphere_entry<D, MIXED, OpList<OC_L1>, true>(priv);
    case OPL_QUAD: return sphere_entry<D, MIXED, OpList<OC_L2, OC_T2, OC_L3, OC_T3>, true>(priv);
    case OPL_SP: return sphere_entry<D, MIXED, OpList<OC_S2, OC_L2, OC_S3, OC_L3>, false>(priv);
    case OPL_GEN1: return sphere_entry<D, MIXED, OpList<OC_GEN>, false>(priv);
    case OPL_GEN2: return sphere_entry<D, MIXED, OpList<OC_GEN, OC_GEN>, false>(priv);
    case OPL_GEN4: return sphere_entry<D, MIXED, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv);
    case OPL_GEN8:
        return sphere_entry<D, MIXED, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv);
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_sphere1d(int D, bool fp32, int opl, int priv)
{
    if (D == 2) return fp32 ? sphere_by_list<2, true>(opl, priv) : sphere_by_list<2, false>(opl, priv);
    if (D == 3) return fp32 ? sphere_by_list<3, true>(opl, priv) : sphere_by_list<3, false>(opl, priv);
    return {nullptr, 0, 0};
}

}  // namespace sfb
