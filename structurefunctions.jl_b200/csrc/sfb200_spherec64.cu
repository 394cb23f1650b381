// sfb200_spherec64.cu -- instantiations of the FP64 chord-formulation spherical 1D kernels (the plain
// FP64 form of the mixed sphere kernel; precision FP64, default formulation on the sphere).
#include "sfb200_internal.h"
#include "sfb200_mixed.cuh"

namespace sfb {

template <int D, class OPS, int PRIV>
static KernelChoice chord64_kernel()
{
    return {reinterpret_cast<const void*>(&k_sphere1d_chord64<D, OPS, PRIV>), 256, PRIV};
}

// run-length table (the default) or warp-aggregated histograms
template <int D, class OPS>
static KernelChoice chord64_entry(int priv)
{
    return priv == 0 ? chord64_kernel<D, OPS, 0>() : chord64_kernel<D, OPS, 3>();
}

template <int D>
static KernelChoice chord64_by_list(int opl, int priv)
{
    switch (opl) {
    case OPL_L2: return chord64_entry<D, OpList<OC_L2>>(priv);
    case OPL_L3: return chord64_entry<D, OpList<OC_L3>>(priv);
    case OPL_L1: return chord64_entry<D, OpList<OC_L1>>(priv);
    case OPL_QUAD: return chord64_entry<D, OpList<OC_L2, OC_T2, OC_L3, OC_T3>>(priv);
    case OPL_SP: return chord64_entry<D, OpList<OC_S2, OC_L2, OC_S3, OC_L3>>(priv);
    case OPL_GEN1: return chord64_entry<D, OpList<OC_GEN>>(priv);
    case OPL_GEN2: return chord64_entry<D, OpList<OC_GEN, OC_GEN>>(priv);
    case OPL_GEN4: return chord64_entry<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>>(priv);
    case OPL_GEN8:
        return chord64_entry<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>>(priv);
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_sphere1d_chord64(int D, int opl, int priv)
{
    if (D == 2) return chord64_by_list<2>(opl, priv);
    if (D == 3) return chord64_by_list<3>(opl, priv);
    return {nullptr, 0, 0};
}

}  // namespace sfb
