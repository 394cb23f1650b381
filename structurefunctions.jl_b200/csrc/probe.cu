// probe.cu -- FP32 / FP64 FMA throughput probe (libsfb200_probe.so), used only to measure the
// roofline denominator of the pair kernels on the machine they run on. Not part of the C ABI of
// include/sfb200.h.
//
// Each thread runs 8 independent FMA chains for `iters` iterations; the grid is a multiple of the SM
// count. Reported rate: 2 * 8 * iters * threads flops / elapsed time (CUDA events).
#include <cuda_runtime.h>

template <typename T>
__global__ void k_fma(T* out, int iters, T a, T b)
{
    T r0 = (T)threadIdx.x, r1 = r0 + 1, r2 = r0 + 2, r3 = r0 + 3, r4 = r0 + 4, r5 = r0 + 5, r6 = r0 + 6, r7 = r0 + 7;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            r0 = r0 * a + b; r1 = r1 * a + b; r2 = r2 * a + b; r3 = r3 * a + b;
            r4 = r4 * a + b; r5 = r5 * a + b; r6 = r6 * a + b; r7 = r7 * a + b;
        }
    }
    const T s = r0 + r1 + r2 + r3 + r4 + r5 + r6 + r7;
    if (s == (T)-1.2345) out[blockIdx.x] = s;  // keeps the chains live; never true in practice
}

extern "C" __attribute__((visibility("default"))) int sfb200_probe_fma(int device, int fp64, double* tflops,
                                                                        double* ms_out)
{
    if (cudaSetDevice(device) != cudaSuccess) return -4;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    void* buf = nullptr;
    if (cudaMalloc(&buf, 1 << 20) != cudaSuccess) return -3;
    const int threads = 256, blocks = nsm * 8;
    const int iters = fp64 ? 512 : 2048;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (fp64) k_fma<double><<<blocks, threads>>>((double*)buf, iters, 0.999999, 1e-7);
        else k_fma<float><<<blocks, threads>>>((float*)buf, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    const double flops = 2.0 * 8.0 * 16.0 * (double)iters * (double)threads * (double)blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    if (ms_out) *ms_out = best;
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}
