// sfb200_acc.cuh -- per-block histogram accumulation for the 1D kernels, with a selectable
// privatization depth (the autotuner's histogram knob).
//
//   PRIV = 0  warp-private histogram, warp-aggregated: lanes holding the same bin are grouped with
//             __match_any_sync, their values reduced by a shuffle tree, and the group leader updates
//             the warp's row (no atomics: leaders of one step hold distinct bins). FP32 kernels keep
//             each cell as a two-sum (hi, lo) pair.
//   PRIV = C  C private copies per warp, lane l updating copy l % C. C = 32 gives every lane its own
//             column (plain read-modify-write, conflict-free: column = bank); 1 <= C < 32 uses
//             shared-memory atomics on the copy. Copies are folded every `flush_every` tile pairs
//             into a per-block FP64 histogram (and at the end), so an FP32 copy never carries more
//             than a few hundred terms before it is added in FP64.
//
// Rows 0 and nb+1 of every histogram collect out-of-range pairs and are dropped at the merge.
#pragma once

#include <type_traits>

#include "sfb200_common.cuh"

namespace sfb {

//   PRIV = 2  warp-aggregated as PRIV = 0, but the group leader adds into the warp's copy with a
//             shared-memory atomic (no read-modify-write chain on the leader; FP32 cells, folded into
//             the block FP64 histogram like the copies).
template <typename R, int NV, int PRIV>
struct BlockHist {
    static constexpr bool AGG = PRIV == 0;
    static constexpr bool AGG_RED = PRIV == 2;
    static constexpr int C = (PRIV == 0 || PRIV == 2) ? 1 : PRIV;
    using CountT = typename std::conditional<AGG && sizeof(R) == 8, unsigned long long, unsigned>::type;

    R* hv;          // values: AGG: [warp][o][bin] (+ lo plane for FP32); else [warp][o][bin][copy]
    R* hlo;         // AGG FP32 only
    CountT* hc;     // counts: AGG: [warp][bin]; else [warp][bin][copy]
    double* sblk;   // !AGG: block FP64 values [o][bin]
    unsigned long long* scnt;  // !AGG: block counts [bin]
    int NBP, NW;

    // Bytes of shared memory this accumulator needs (mirrored on the host by hist_bytes()).
    static __host__ __device__ size_t bytes(int NW_, int NBP_)
    {
        if (AGG) {
            size_t b = (size_t)NW_ * NV * NBP_ * sizeof(R) * (sizeof(R) == 4 ? 2 : 1);
            b += (size_t)NW_ * NBP_ * sizeof(CountT);
            return (b + 15) & ~(size_t)15;
        }
        size_t b = (size_t)NV * NBP_ * 8 + (size_t)NBP_ * 8;  // sblk, scnt (8-byte aligned first)
        b += (size_t)NW_ * NV * NBP_ * C * sizeof(R);
        b += (size_t)NW_ * NBP_ * C * sizeof(unsigned);
        return (b + 15) & ~(size_t)15;
    }

    __device__ void init(unsigned char* base, int NW_, int NBP_)
    {
        NW = NW_;
        NBP = NBP_;
        const int T = blockDim.x;
        if constexpr (AGG) {
            hv = reinterpret_cast<R*>(base);
            hlo = hv + (size_t)NW * NV * NBP;
            hc = reinterpret_cast<CountT*>(hv + (size_t)NW * NV * NBP * (sizeof(R) == 4 ? 2 : 1));
            for (int k = threadIdx.x; k < NW * NV * NBP * (sizeof(R) == 4 ? 2 : 1); k += T) hv[k] = R(0);
            for (int k = threadIdx.x; k < NW * NBP; k += T) hc[k] = 0;
        } else {
            sblk = reinterpret_cast<double*>(base);
            scnt = reinterpret_cast<unsigned long long*>(sblk + (size_t)NV * NBP);
            hv = reinterpret_cast<R*>(scnt + NBP);
            hc = reinterpret_cast<CountT*>(hv + (size_t)NW * NV * NBP * C);
            for (int k = threadIdx.x; k < NV * NBP; k += T) sblk[k] = 0.0;
            for (int k = threadIdx.x; k < NBP; k += T) scnt[k] = 0ull;
            for (int k = threadIdx.x; k < NW * NV * NBP * C; k += T) hv[k] = R(0);
            for (int k = threadIdx.x; k < NW * NBP * C; k += T) hc[k] = 0u;
        }
    }

    // One pair step of the warp: every lane adds its values v under bin `key` (all lanes call).
    __device__ __forceinline__ void add(int key, R (&v)[NV], int lane, int warp)
    {
        if constexpr (AGG) {
            const unsigned peers = __match_any_sync(FULL, key);
            reduce_peers<NV>(peers, lane, v);
            if (lane == __ffs(peers) - 1) {
                CountT* whc = hc + warp * NBP;
                whc[key] += (CountT)__popc(peers);
                R* wv = hv + (size_t)warp * NV * NBP;
                if constexpr (sizeof(R) == 4) {
                    R* wl = hlo + (size_t)warp * NV * NBP;
#pragma unroll
                    for (int o = 0; o < NV; ++o) two_sum_acc(wv[o * NBP + key], wl[o * NBP + key], v[o]);
                } else {
#pragma unroll
                    for (int o = 0; o < NV; ++o) wv[o * NBP + key] += v[o];
                }
            }
            __syncwarp();
        } else if constexpr (AGG_RED) {
            const unsigned peers = __match_any_sync(FULL, key);
            reduce_peers<NV>(peers, lane, v);
            if (lane == __ffs(peers) - 1) {
                R* wv = hv + (size_t)warp * NV * NBP;
#pragma unroll
                for (int o = 0; o < NV; ++o) atomicAdd(&wv[o * NBP + key], v[o]);
                atomicAdd(&hc[warp * NBP + key], (unsigned)__popc(peers));
            }
        } else {
            const int col = (C == 32) ? lane : (lane % C);
            R* wv = hv + (size_t)warp * NV * NBP * C;
            unsigned* wc = hc + (size_t)warp * NBP * C;
            if constexpr (C == 32) {
#pragma unroll
                for (int o = 0; o < NV; ++o) wv[((size_t)o * NBP + key) * C + col] += v[o];
                wc[key * C + col] += 1u;
            } else {
#pragma unroll
                for (int o = 0; o < NV; ++o) atomicAdd(&wv[((size_t)o * NBP + key) * C + col], v[o]);
                atomicAdd(&wc[key * C + col], 1u);
            }
        }
    }

    // Fold the copies into the block FP64 histogram (all threads of the block call; !AGG only).
    __device__ void fold()
    {
        if constexpr (!AGG) {
            const int T = blockDim.x;
            __syncthreads();
            for (int k = threadIdx.x; k < NV * NBP; k += T) {
                const int o = k / NBP, b = k - o * NBP;
                double s = 0.0;
                for (int w = 0; w < NW; ++w) {
                    R* row = hv + (((size_t)w * NV + o) * NBP + b) * C;
#pragma unroll 4
                    for (int c = 0; c < C; ++c) {
                        s += (double)row[c];
                        row[c] = R(0);
                    }
                }
                sblk[k] += s;
            }
            for (int b = threadIdx.x; b < NBP; b += T) {
                unsigned long long cnt = 0;
                for (int w = 0; w < NW; ++w) {
                    unsigned* row = hc + ((size_t)w * NBP + b) * C;
                    for (int c = 0; c < C; ++c) {
                        cnt += row[c];
                        row[c] = 0u;
                    }
                }
                scnt[b] += cnt;
            }
            __syncthreads();
        }
    }

    // Merge into the global FP64 sums / uint64 counts (all threads call, after the pair loop).
    __device__ void merge(double* g_sums, unsigned long long* g_counts, int nops, int nb)
    {
        const int T = blockDim.x;
        if constexpr (AGG) {
            __syncthreads();
            for (int k = threadIdx.x; k < min(NV, nops) * nb; k += T) {
                const int o = k / nb, b = k - o * nb + 1;
                double s = 0.0;
                for (int w = 0; w < NW; ++w) {
                    const size_t idx = ((size_t)w * NV + o) * NBP + b;
                    s += (double)hv[idx];
                    if constexpr (sizeof(R) == 4) s += (double)hlo[idx];
                }
                if (s != 0.0) atomicAdd(&g_sums[(size_t)o * nb + b - 1], s);
            }
            for (int b = threadIdx.x + 1; b <= nb; b += T) {
                unsigned long long c = 0;
                for (int w = 0; w < NW; ++w) c += hc[w * NBP + b];
                if (c) atomicAdd(&g_counts[b - 1], c);
            }
        } else {
            fold();
            for (int k = threadIdx.x; k < min(NV, nops) * nb; k += T) {
                const int o = k / nb, b = k - o * nb + 1;
                const double s = sblk[o * NBP + b];
                if (s != 0.0) atomicAdd(&g_sums[(size_t)o * nb + b - 1], s);
            }
            for (int b = threadIdx.x + 1; b <= nb; b += T) {
                const unsigned long long c = scnt[b];
                if (c) atomicAdd(&g_counts[b - 1], c);
            }
        }
    }
};

}  // namespace sfb
