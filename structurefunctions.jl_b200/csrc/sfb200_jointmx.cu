// sfb200_jointmx.cu -- instantiations of the mixed-precision joint (distance x value) kernels.
#include "sfb200_internal.h"
#include "sfb200_mixed.cuh"

namespace sfb {

template <bool SPHERE, int D, int NT>
static KernelChoice jointmx_by_list(int opl)
{
    switch (opl) {
    case OPL_L1: return {reinterpret_cast<const void*>(&k_joint_mx<SPHERE, D, OpList<OC_L1>, NT>), NT, 0};
    case OPL_L2: return {reinterpret_cast<const void*>(&k_joint_mx<SPHERE, D, OpList<OC_L2>, NT>), NT, 0};
    case OPL_L3: return {reinterpret_cast<const void*>(&k_joint_mx<SPHERE, D, OpList<OC_L3>, NT>), NT, 0};
    case OPL_GEN1: return {reinterpret_cast<const void*>(&k_joint_mx<SPHERE, D, OpList<OC_GEN>, NT>), NT, 0};
    }
    return {nullptr, 0, 0};
}

template <int NT>
static KernelChoice jointmx_pick(bool sphere, int D, int opl)
{
    if (sphere) return D == 2 ? jointmx_by_list<true, 2, NT>(opl) : jointmx_by_list<true, 3, NT>(opl);
    return D == 2 ? jointmx_by_list<false, 2, NT>(opl) : jointmx_by_list<false, 3, NT>(opl);
}

// Tiles above 512 points take the kernel compiled for 768 threads per block.
KernelChoice pick_joint_mx(bool sphere, int D, int opl, int T)
{
    return T > 512 ? jointmx_pick<768>(sphere, D, opl) : jointmx_pick<512>(sphere, D, opl);
}

template <bool SPHERE, int D, int NT>
static KernelChoice jointmx_batch_by_list(int opl)
{
    switch (opl) {
    case OPL_L1: return {reinterpret_cast<const void*>(&k_joint_mx_batch<SPHERE, D, OpList<OC_L1>, NT>), NT, 0};
    case OPL_L2: return {reinterpret_cast<const void*>(&k_joint_mx_batch<SPHERE, D, OpList<OC_L2>, NT>), NT, 0};
    case OPL_L3: return {reinterpret_cast<const void*>(&k_joint_mx_batch<SPHERE, D, OpList<OC_L3>, NT>), NT, 0};
    case OPL_GEN1: return {reinterpret_cast<const void*>(&k_joint_mx_batch<SPHERE, D, OpList<OC_GEN>, NT>), NT, 0};
    }
    return {nullptr, 0, 0};
}

// Batched joint kernels: 768-thread blocks for the flat histogram, 512 on the sphere (whose 768-thread
// form spills registers).
KernelChoice pick_joint_mx_batch(bool sphere, int D, int opl)
{
    if (sphere) return D == 2 ? jointmx_batch_by_list<true, 2, 512>(opl) : jointmx_batch_by_list<true, 3, 512>(opl);
    return D == 2 ? jointmx_batch_by_list<false, 2, 768>(opl) : jointmx_batch_by_list<false, 3, 768>(opl);
}

}  // namespace sfb
