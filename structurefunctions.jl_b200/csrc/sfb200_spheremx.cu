// sfb200_spheremx.cu -- instantiations of the mixed-precision spherical 1D kernels.
#include "sfb200_internal.h"
#include "sfb200_mixed.cuh"

namespace sfb {

template <int D, class OPS, int PRIV>
static KernelChoice spheremx_kernel()
{
    return {reinterpret_cast<const void*>(&k_sphere1d_mx<D, OPS, PRIV>), 256, PRIV};
}

template <int D, class OPS, bool ALL>
static KernelChoice spheremx_entry(int priv)
{
    switch (priv) {
    case 3: return spheremx_kernel<D, OPS, 3>();
    case 32: return spheremx_kernel<D, OPS, 32>();
    case 2: if constexpr (ALL) return spheremx_kernel<D, OPS, 2>(); break;
    case 8: if constexpr (ALL) return spheremx_kernel<D, OPS, 8>(); break;
    case 4: if constexpr (ALL) return spheremx_kernel<D, OPS, 4>(); break;
    case 1: if constexpr (ALL) return spheremx_kernel<D, OPS, 1>(); break;
    }
    return spheremx_kernel<D, OPS, 0>();
}

template <int D>
static KernelChoice spheremx_by_list(int opl, int priv)
{
    switch (opl) {
    case OPL_L2: return spheremx_entry<D, OpList<OC_L2>, true>(priv);
    case OPL_L3: return spheremx_entry<D, OpList<OC_L3>, true>(priv);
    case OPL_L1: return spheremx_entry<D, OpList<OC_L1>, true>(priv);
    case OPL_QUAD: return spheremx_entry<D, OpList<OC_L2, OC_T2, OC_L3, OC_T3>, true>(priv);
    case OPL_SP: return spheremx_entry<D, OpList<OC_S2, OC_L2, OC_S3, OC_L3>, false>(priv);
    case OPL_GEN1: return spheremx_entry<D, OpList<OC_GEN>, false>(priv);
    case OPL_GEN2: return spheremx_entry<D, OpList<OC_GEN, OC_GEN>, false>(priv);
    case OPL_GEN4: return spheremx_entry<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv);
    case OPL_GEN8:
        return spheremx_entry<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv);
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_sphere1d_mx(int D, int opl, int priv)
{
    if (D == 2) return spheremx_by_list<2>(opl, priv);
    if (D == 3) return spheremx_by_list<3>(opl, priv);
    return {nullptr, 0, 0};
}

// Batched (serving) form: run-length histogram only.
template <int D>
static KernelChoice sphere1d_mx_batch_by_list(int opl)
{
    switch (opl) {
    case OPL_L2: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_L2>, 3>), 256, 3};
    case OPL_L3: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_L3>, 3>), 256, 3};
    case OPL_L1: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_L1>, 3>), 256, 3};
    case OPL_QUAD: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_L2, OC_T2, OC_L3, OC_T3>, 3>), 256, 3};
    case OPL_SP: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_S2, OC_L2, OC_S3, OC_L3>, 3>), 256, 3};
    case OPL_GEN1: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_GEN>, 3>), 256, 3};
    case OPL_GEN2: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_GEN, OC_GEN>, 3>), 256, 3};
    case OPL_GEN4: return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>, 3>), 256, 3};
    case OPL_GEN8:
        return {reinterpret_cast<const void*>(&k_sphere1d_mx_batch<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>, 3>), 256, 3};
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_sphere1d_mx_batch(int D, int opl)
{
    if (D == 2) return sphere1d_mx_batch_by_list<2>(opl);
    if (D == 3) return sphere1d_mx_batch_by_list<3>(opl);
    return {nullptr, 0, 0};
}

}  // namespace sfb
