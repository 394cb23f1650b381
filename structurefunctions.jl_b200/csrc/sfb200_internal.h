// sfb200_internal.h -- declarations shared by the API translation unit and the kernel
// instantiation units.
#pragma once

#include <cuda_runtime.h>

#include "sfb200_common.cuh"

namespace sfb {

struct PairArgs;

// Operator lists with a dedicated (compile-time fused) kernel; anything else runs the generic
// kernel with the operator count padded to 1, 2, 4 or 8.
enum OpListId : int {
    OPL_L2 = 0,        // {L2SF}
    OPL_L3 = 1,        // {L3SF}
    OPL_L1 = 2,        // {ProjectedStructureFunctionType{1,0}} (du_L; joint value axis)
    OPL_QUAD = 3,      // {L2SF, T2SF, L3SF, T3SF}
    OPL_GEN1 = 4,
    OPL_GEN2 = 5,
    OPL_GEN4 = 6,
    OPL_GEN8 = 7,
    OPL_SP = 8         // {S2SF, L2SF, S3SF, L3SF}: the accumulated rows of the six-invariant single pass
};

struct KernelChoice {
    const void* fn;   // kernel entry
    int max_threads;  // launch bound
    int priv;         // histogram privatization depth the kernel was built with (1D kernels)
};

// Kernel lookup: returns nullptr fn for an unsupported combination. `fp32` selects the
// FP32-bulk kernels (precision SFB200_PREC_FP32); `df`: their FP32 records carry (hi, lo) pairs
// because an input is FP64.
KernelChoice pick_flat1d(int D, bool fp32, bool df, int opl, int priv);
KernelChoice pick_sphere1d(int D, bool fp32, int opl, int priv);
KernelChoice pick_joint(bool sphere, int D, bool fp32, bool smem_hist, bool df, int opl);
// flat single-pass 2D, rows r0 .. r0 + n_ops - 1 (FP64), `split` (1 or 2) threads per tile point
KernelChoice pick_sp2d(int D, bool smem_hist, int split);
// Mixed-precision kernels (FP64 differences and numerators, FP32 normalisation and accumulation).
KernelChoice pick_flat1d_mx(int D, int opl, int priv, bool lin = false);
KernelChoice pick_sphere1d_mx(int D, int opl, int priv);
KernelChoice pick_joint_mx(bool sphere, int D, int opl, int T = 512);
// FP64 chord-formulation sphere kernels (the mixed sphere kernel's algorithm in FP64).
KernelChoice pick_sphere1d_chord64(int D, int opl, int priv);
// Batched (serving) forms of the mixed kernels: BatchArgs parameter, run-length histogram.
KernelChoice pick_flat1d_mx_batch(int D, int opl);
KernelChoice pick_sphere1d_mx_batch(int D, int opl);
KernelChoice pick_joint_mx_batch(bool sphere, int D, int opl);

}  // namespace sfb
