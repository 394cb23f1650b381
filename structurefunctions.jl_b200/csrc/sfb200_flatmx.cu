// sfb200_flatmx.cu -- instantiations of the mixed-precision Euclidean 1D kernels.
#include "sfb200_internal.h"
#include "sfb200_mixed.cuh"

namespace sfb {

template <int D, class OPS, int PRIV, bool LIN = false>
static KernelChoice flatmx_kernel()
{
    return {reinterpret_cast<const void*>(&k_flat1d_mx<D, OPS, PRIV, LIN>), 256, PRIV};
}

// `lin`: a LinearBinEdges distance axis; the specialised lists (LINF) have a form compiled for it in the
// default histogram modes (3, 6)
template <int D, class OPS, bool ALL, bool LINF = ALL>
static KernelChoice flatmx_entry(int priv, bool lin)
{
    if constexpr (LINF) {
        if (lin && priv == 3) return flatmx_kernel<D, OPS, 3, true>();
        if (lin && priv == 6) return flatmx_kernel<D, OPS, 6, true>();
    }
    switch (priv) {
    case 3: return flatmx_kernel<D, OPS, 3>();
    case 6: return flatmx_kernel<D, OPS, 6>();
    case 32: return flatmx_kernel<D, OPS, 32>();
    case 2: if constexpr (ALL) return flatmx_kernel<D, OPS, 2>(); break;
    case 8: if constexpr (ALL) return flatmx_kernel<D, OPS, 8>(); break;
    case 4: if constexpr (ALL) return flatmx_kernel<D, OPS, 4>(); break;
    case 1: if constexpr (ALL) return flatmx_kernel<D, OPS, 1>(); break;
    }
    return flatmx_kernel<D, OPS, 0>();
}

template <int D>
static KernelChoice flatmx_by_list(int opl, int priv, bool lin)
{
    switch (opl) {
    case OPL_L2: return flatmx_entry<D, OpList<OC_L2>, true>(priv, lin);
    case OPL_L3: return flatmx_entry<D, OpList<OC_L3>, true>(priv, lin);
    case OPL_L1: return flatmx_entry<D, OpList<OC_L1>, true>(priv, lin);
    case OPL_QUAD: return flatmx_entry<D, OpList<OC_L2, OC_T2, OC_L3, OC_T3>, true>(priv, lin);
    case OPL_SP: return flatmx_entry<D, OpList<OC_S2, OC_L2, OC_S3, OC_L3>, false, true>(priv, lin);
    case OPL_GEN1: return flatmx_entry<D, OpList<OC_GEN>, false>(priv, lin);
    case OPL_GEN2: return flatmx_entry<D, OpList<OC_GEN, OC_GEN>, false>(priv, lin);
    case OPL_GEN4: return flatmx_entry<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv, lin);
    case OPL_GEN8:
        return flatmx_entry<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>, false>(priv, lin);
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_flat1d_mx(int D, int opl, int priv, bool lin)
{
    if (D == 2) return flatmx_by_list<2>(opl, priv, lin);
    if (D == 3) return flatmx_by_list<3>(opl, priv, lin);
    return {nullptr, 0, 0};
}

// Batched (serving) form: run-length histogram only.
template <int D>
static KernelChoice flat1d_mx_batch_by_list(int opl)
{
    switch (opl) {
    case OPL_L2: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_L2>, 3>), 256, 3};
    case OPL_L3: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_L3>, 3>), 256, 3};
    case OPL_L1: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_L1>, 3>), 256, 3};
    case OPL_QUAD: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_L2, OC_T2, OC_L3, OC_T3>, 3>), 256, 3};
    case OPL_SP: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_S2, OC_L2, OC_S3, OC_L3>, 3>), 256, 3};
    case OPL_GEN1: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_GEN>, 3>), 256, 3};
    case OPL_GEN2: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_GEN, OC_GEN>, 3>), 256, 3};
    case OPL_GEN4: return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN>, 3>), 256, 3};
    case OPL_GEN8:
        return {reinterpret_cast<const void*>(&k_flat1d_mx_batch<D, OpList<OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN, OC_GEN>, 3>), 256, 3};
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_flat1d_mx_batch(int D, int opl)
{
    if (D == 2) return flat1d_mx_batch_by_list<2>(opl);
    if (D == 3) return flat1d_mx_batch_by_list<3>(opl);
    return {nullptr, 0, 0};
}

}  // namespace sfb
