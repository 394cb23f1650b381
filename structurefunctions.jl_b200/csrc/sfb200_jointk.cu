// sfb200_jointk.cu -- instantiations of the joint (distance x value) kernels.
#include "sfb200_internal.h"
#include "sfb200_joint.cuh"

namespace sfb {

template <bool SPHERE, int D>
static KernelChoice joint_fp64(bool smem)
{
    if (smem) return {reinterpret_cast<const void*>(&k_joint_fp64<SPHERE, D, true>), 512, 0};
    return {reinterpret_cast<const void*>(&k_joint_fp64<SPHERE, D, false>), 512, 0};
}

template <bool SPHERE, int D, bool DF>
static KernelChoice joint_mixed(int opl)
{
    switch (opl) {
    case OPL_L1: return {reinterpret_cast<const void*>(&k_joint_mixed<SPHERE, D, DF, DF, OpList<OC_L1>>), 512, 0};
    case OPL_L2: return {reinterpret_cast<const void*>(&k_joint_mixed<SPHERE, D, DF, DF, OpList<OC_L2>>), 512, 0};
    case OPL_L3: return {reinterpret_cast<const void*>(&k_joint_mixed<SPHERE, D, DF, DF, OpList<OC_L3>>), 512, 0};
    case OPL_GEN1: return {reinterpret_cast<const void*>(&k_joint_mixed<SPHERE, D, DF, DF, OpList<OC_GEN>>), 512, 0};
    }
    return {nullptr, 0, 0};
}

KernelChoice pick_joint(bool sphere, int D, bool fp32, bool smem_hist, bool df, int opl)
{
    if (!fp32) {
        if (sphere) return D == 2 ? joint_fp64<true, 2>(smem_hist) : joint_fp64<true, 3>(smem_hist);
        return D == 2 ? joint_fp64<false, 2>(smem_hist) : joint_fp64<false, 3>(smem_hist);
    }
    if (sphere) return D == 2 ? joint_mixed<true, 2, true>(opl) : joint_mixed<true, 3, true>(opl);
    if (df) return D == 2 ? joint_mixed<false, 2, true>(opl) : joint_mixed<false, 3, true>(opl);
    return D == 2 ? joint_mixed<false, 2, false>(opl) : joint_mixed<false, 3, false>(opl);
}

// Consecutive rows of the flat two-dimensional single pass in one launch (FP64); `split` threads per
// point of the tile (1 or 2).
template <int D, bool SMEM>
static KernelChoice sp2d_kernel(int split)
{
    if (split == 2) return {reinterpret_cast<const void*>(&k_sp2d_fp64<D, SMEM, 2>), 1024, 0};
    return {reinterpret_cast<const void*>(&k_sp2d_fp64<D, SMEM, 1>), 512, 0};
}

KernelChoice pick_sp2d(int D, bool smem_hist, int split)
{
    if (D == 2) return smem_hist ? sp2d_kernel<2, true>(split) : sp2d_kernel<2, false>(split);
    if (D == 3) return smem_hist ? sp2d_kernel<3, true>(split) : sp2d_kernel<3, false>(split);
    return {nullptr, 0, 0};
}

}  // namespace sfb
