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
//   PRIV = 3  run-length: every lane keeps its current bin, one running sum per operator and a count
//             in registers, and only when its bin changes adds the finished run into column
//             (lane % LC) of a block-wide [o][bin][column] table with shared-memory atomics (LC = 32:
//             the lanes of one warp hit 32 distinct banks; the atomics only order different warps).
//             Runs are closed at every tile-pair boundary (a run never holds more than one tile's
//             terms) and the table is folded into the block FP64 histogram every `flush_every` tile
//             pairs. With the points in space-filling-curve order, the j of consecutive steps are
//             neighbours, the pair distance changes little from step to step and most steps extend
//             the run: the per-pair cost is a compare and one add per operator. (The flat kernels also
//             stage each J tile sorted by distance from the I tile, so that a lane's bins rise almost
//             monotonically along its row and its runs last tens to hundreds of pairs.)
//   PRIV = 6  run-length with two open runs per lane (the same table as PRIV = 3): a lane keeps the
//             two bins it met most recently open at once, so that a row whose bin alternates between
//             two neighbours near a bin edge (the lanes of a warp differ in their i point, so the
//             distance order of a J tile is only approximately each lane's own) extends its runs
//             instead of ending one at every alternation; a third bin ends the least recently used.
template <typename R, int NV, int PRIV>
struct BlockHist {
    static constexpr bool AGG = PRIV == 0;
    static constexpr bool AGG_RED = PRIV == 2;
    static constexpr bool RUN2 = PRIV == 6;
    static constexpr bool RUN = PRIV == 3 || RUN2;
    static constexpr int C = (PRIV == 0 || PRIV == 2 || RUN) ? 1 : PRIV;
    using CountT = typename std::conditional<AGG && sizeof(R) == 8, unsigned long long, unsigned>::type;

    R* hv;          // values: AGG: [warp][o][bin] (+ lo plane for FP32); RUN: [o][bin][column];
                    // else [warp][o][bin][copy]
    R* hlo;         // AGG FP32 only
    CountT* hc;     // counts: AGG: [warp][bin]; RUN: [bin][column]; else [warp][bin][copy]
    double* sblk;   // !AGG: block FP64 values [o][bin]
    unsigned long long* scnt;  // !AGG: block counts [bin]
    int NBP, NW;
    int LC;         // RUN: table columns (power of two <= 32)
    // RUN: the lane's open run (RUN2: and its second open run, and which of the two was used last)
    int rkey;
    unsigned rc;
    R rs[NV];
    int rkey2;
    unsigned rc2;
    R rs2[NV];
    bool last2;

    // Bytes of shared memory this accumulator needs (mirrored on the host by hist_bytes()); `lc` is
    // the RUN table's column count.
    static __host__ __device__ size_t bytes(int NW_, int NBP_, int lc = 32)
    {
        if (AGG) {
            size_t b = (size_t)NW_ * NV * NBP_ * sizeof(R) * (sizeof(R) == 4 ? 2 : 1);
            b += (size_t)NW_ * NBP_ * sizeof(CountT);
            return (b + 15) & ~(size_t)15;
        }
        size_t b = (size_t)NV * NBP_ * 8 + (size_t)NBP_ * 8;  // sblk, scnt (8-byte aligned first)
        if (RUN) {
            b += (size_t)NV * NBP_ * lc * sizeof(R) + (size_t)NBP_ * lc * sizeof(unsigned);
            return (b + 15) & ~(size_t)15;
        }
        b += (size_t)NW_ * NV * NBP_ * C * sizeof(R);
        b += (size_t)NW_ * NBP_ * C * sizeof(unsigned);
        return (b + 15) & ~(size_t)15;
    }

    __device__ void init(unsigned char* base, int NW_, int NBP_, int lc = 32)
    {
        NW = NW_;
        NBP = NBP_;
        LC = lc;
        const int T = blockDim.x;
        if constexpr (RUN) {
            sblk = reinterpret_cast<double*>(base);
            scnt = reinterpret_cast<unsigned long long*>(sblk + (size_t)NV * NBP);
            hv = reinterpret_cast<R*>(scnt + NBP);
            hc = reinterpret_cast<CountT*>(hv + (size_t)NV * NBP * LC);
            for (int k = threadIdx.x; k < NV * NBP; k += T) sblk[k] = 0.0;
            for (int k = threadIdx.x; k < NBP; k += T) scnt[k] = 0ull;
            for (int k = threadIdx.x; k < NV * NBP * LC; k += T) hv[k] = R(0);
            for (int k = threadIdx.x; k < NBP * LC; k += T) hc[k] = 0u;
            open_empty();
        } else if constexpr (AGG) {
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

    // RUN: an empty run on the dropped overflow row, so that the first add may flush it unguarded.
    __device__ __forceinline__ void open_empty()
    {
        rkey = NBP - 1;
        rc = 0u;
#pragma unroll
        for (int o = 0; o < NV; ++o) rs[o] = R(0);
        if constexpr (RUN2) {
            rkey2 = NBP - 1;
            rc2 = 0u;
#pragma unroll
            for (int o = 0; o < NV; ++o) rs2[o] = R(0);
            last2 = false;
        }
    }

    // RUN: add a finished run (bin k, values s, count c) into the lane's table column.
    __device__ __forceinline__ void flush_one(int lane, int k, const R (&sv)[NV], unsigned c)
    {
        const int at = k * LC + (lane & (LC - 1));
        const int plane = NBP * LC;
#pragma unroll
        for (int o = 0; o < NV; ++o) atomicAdd(hv + (at + o * plane), sv[o]);
        atomicAdd(hc + at, c);
    }

    // RUN: add the lane's open run into its table column.
    __device__ __forceinline__ void flush_run(int lane)
    {
        const int at = rkey * LC + (lane & (LC - 1));
        const int plane = NBP * LC;
#pragma unroll
        for (int o = 0; o < NV; ++o) atomicAdd(hv + (at + o * plane), rs[o]);
        atomicAdd(hc + at, rc);
    }

    // RUN: close every lane's run (tile-pair boundary; before a fold or the merge).
    __device__ __forceinline__ void close_runs(int lane)
    {
        if constexpr (RUN) {
            if (rc) flush_run(lane);
            if constexpr (RUN2) {
                if (rc2) flush_one(lane, rkey2, rs2, rc2);
            }
            open_empty();
        }
    }

    // One pair step of the warp: every lane adds its values v under bin `key` (all lanes call).
    __device__ __forceinline__ void add(int key, R (&v)[NV], int lane, int warp)
    {
        if constexpr (RUN2) {
            bool in1 = key == rkey;
            if (!in1 && key != rkey2) {  // a third bin: end the least recently used run
                in1 = last2;
                R sv[NV];
#pragma unroll
                for (int o = 0; o < NV; ++o) sv[o] = in1 ? rs[o] : rs2[o];
                const unsigned c = in1 ? rc : rc2;
                if (c) flush_one(lane, in1 ? rkey : rkey2, sv, c);
                if (in1) {
                    rkey = key;
                    rc = 0u;
#pragma unroll
                    for (int o = 0; o < NV; ++o) rs[o] = R(0);
                } else {
                    rkey2 = key;
                    rc2 = 0u;
#pragma unroll
                    for (int o = 0; o < NV; ++o) rs2[o] = R(0);
                }
            }
            if (in1) {
#pragma unroll
                for (int o = 0; o < NV; ++o) rs[o] += v[o];
                ++rc;
            } else {
#pragma unroll
                for (int o = 0; o < NV; ++o) rs2[o] += v[o];
                ++rc2;
            }
            last2 = !in1;
        } else if constexpr (RUN) {
            if (key != rkey) {  // the run ends: add it to the table and open an empty one
                flush_run(lane);
#pragma unroll
                for (int o = 0; o < NV; ++o) rs[o] = R(0);
                rc = 0u;
                rkey = key;
            }
#pragma unroll
            for (int o = 0; o < NV; ++o) rs[o] += v[o];
            ++rc;
        } else if constexpr (AGG) {
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
        if constexpr (RUN) {
            // one warp per table row: lane c reads column c, a shuffle tree sums the row in FP64
            __syncthreads();
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            for (int r = warp; r < NV * NBP; r += NW) {
                double s = 0.0;
                if (lane < LC) {
                    s = (double)hv[(size_t)r * LC + lane];
                    hv[(size_t)r * LC + lane] = R(0);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
                if (lane == 0) sblk[r] += s;
            }
            for (int b = warp; b < NBP; b += NW) {
                unsigned c = 0u;
                if (lane < LC) {
                    c = hc[b * LC + lane];
                    hc[b * LC + lane] = 0u;
                }
                c = __reduce_add_sync(FULL, c);
                if (lane == 0) scnt[b] += c;
            }
            __syncthreads();
        } else if constexpr (!AGG) {
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
    // `oscale` (optional, NV entries): exact power-of-two factor applied to operator o's sums.
    __device__ void merge(double* g_sums, unsigned long long* g_counts, int nops, int nb,
                          const double* oscale = nullptr)
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
                if (oscale) s *= oscale[o];
                if (s != 0.0) atomicAdd(&g_sums[(size_t)o * nb + b - 1], s);
            }
            for (int b = threadIdx.x + 1; b <= nb; b += T) {
                unsigned long long c = 0;
                for (int w = 0; w < NW; ++w) c += hc[w * NBP + b];
                if (c) atomicAdd(&g_counts[b - 1], c);
            }
        } else {
            close_runs(threadIdx.x & 31);
            fold();
            for (int k = threadIdx.x; k < min(NV, nops) * nb; k += T) {
                const int o = k / nb, b = k - o * nb + 1;
                double s = sblk[o * NBP + b];
                if (oscale) s *= oscale[o];
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
