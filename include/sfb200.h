/*
 * sfb200.h -- C ABI of the B200 pair-histogram backend for structure functions.
 *
 * One library call replaces the O(N^2) pair loop that the reference runs behind
 * `calculate_structure_function` / `calculate_structure_function!`:
 *
 *   reference entry                         file:line (jbphyswx/StructureFunctions.jl)
 *   --------------------------------------  -------------------------------------------------------
 *   public 1D entry                         src/Calculations/dispatch.jl:64-91
 *   public joint (distance x value) entry   src/Calculations/dispatch.jl:108-136
 *   mutating entry (accumulate into)        src/Calculations/dispatch.jl:346-373
 *   backend routing (a B200Backend method)  src/Calculations/dispatch.jl:377-594
 *   Euclidean pair loop                     src/Calculations/serial.jl:68-101
 *   non-Euclidean (sphere) pair loop        src/Calculations/serial.jl:228-267
 *   joint pair loops                        src/Calculations/serial_2d.jl:49-85, 260-303
 *   squared-distance digitize plans         src/BinEdges.jl:410-558
 *   LinearBinEdges search                   src/BinEdges.jl:114-131
 *   result accumulators                     src/StructureFunctionObjects.jl:50-115
 *
 * Everything in this header is plain C: pointers, sizes, enums and POD structs. No CUDA or
 * torch type appears in a signature; CUDA streams travel as `void*`.
 *
 * Conventions
 *   - x is (W, N) column-major: x[k + W*i] is coordinate k of point i. W = D for flat geometry,
 *     W = 2 (lon, lat) for the sphere. u is (D, N) column-major, D in {2, 3}.
 *   - Bins are right-inclusive (a, b]; a pair lands in bin b (1-based in the reference) when
 *     edge[b-1] < key <= edge[b]. Out-of-range pairs are dropped, as in the reference.
 *   - Outputs: sums are double, counts are uint64. For a 1D plan with n_ops operators and nb
 *     distance bins, sums is (nb, n_ops) column-major (operator k at sums + k*nb) and counts
 *     has nb entries (shared by all operators: a pair is counted once per bin). For a joint plan
 *     (one operator), sums and counts are (n_dist, n_val) column-major, as the reference's
 *     StructureFunction2DSumsAndCounts matrices; a joint plan of r single-pass 2D rows holds r such
 *     matrices one after the other.
 *   - Every call returns 0 on success or a negative sfb200_status. Nothing aborts or traps.
 */
#ifndef SFB200_H
#define SFB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SFB200_ABI_VERSION 1
#define SFB200_MAX_OPS 8

#if defined(__GNUC__)
#define SFB200_API __attribute__((visibility("default")))
#else
#define SFB200_API
#endif

typedef enum {
    SFB200_OK = 0,
    SFB200_ERR_INVALID_ARG = -1,   /* maps to ArgumentError in the host glue */
    SFB200_ERR_UNSUPPORTED = -2,   /* maps to ArgumentError: shape/metric/operator not on this path */
    SFB200_ERR_OOM = -3,
    SFB200_ERR_CUDA = -4,
    SFB200_ERR_TIMEOUT = -5,
    SFB200_ERR_QUEUE_FULL = -6,
    SFB200_ERR_DIMENSION = -7      /* maps to DimensionMismatch */
} sfb200_status;

/* Pair geometry, chosen by the host from the distance metric (reference
 * src/HelperFunctions.jl:390-417 pair_geometry_for). */
typedef enum {
    SFB200_GEOM_FLAT = 0,    /* Distances.Euclidean -> FlatGeometry{D} */
    SFB200_GEOM_SPHERE = 1   /* Distances.Haversine(radius) / SphericalAngle -> SphericalGeometry{D} */
} sfb200_geometry;

/* Angle unit of sphere coordinates: Haversine takes degrees, SphericalAngle radians
 * (reference src/HelperFunctions.jl:404-409). */
typedef enum { SFB200_ANGLE_DEG = 0, SFB200_ANGLE_RAD = 1 } sfb200_angle_unit;

/* Operator kinds (reference src/StructureFunctionTypes.jl:43-151). */
typedef enum {
    SFB200_OP_PROJECTED = 0, /* ProjectedStructureFunctionType{NL,NT}: L2SF={2,0}, T2SF={0,2}, L3SF={3,0},
                                T3SF={0,3}, L2T1SF={2,1}, L1T2SF={1,2}, delta-u_L={1,0}, ... */
    SFB200_OP_S2 = 1,        /* SecondOrderStructureFunctionType: |du|^2 */
    SFB200_OP_S3 = 2,        /* ThirdOrderStructureFunctionType: du_L |du|^2 */
    SFB200_OP_FULLVEC = 3,   /* FullVectorStructureFunctionType{NF}: |du|^NF */
    SFB200_OP_T2C = 4,       /* TransverseComponentSecondOrderStructureFunctionType: |du_t|^2/(D-1) */
    SFB200_OP_L1T2C = 5,     /* LongitudinalTransverseComponentThirdOrderStructureFunctionType */
    SFB200_OP_SP2D = 6       /* one of the six invariants of the two-dimensional single pass, nl = its row
                                (0 S2, 1 L2, 2 T2, 3 S3, 4 L3, 5 L1T2), with that pass's own formulas: flat
                                du_L = (du . dx) * inv(sqrt(r2)), sphere du_L = du . r_hat, |du|^2 = du . du,
                                S2 = |du|^2, L2 = du_L^2, T2 = |du|^2 - L2, S3 = du_L |du|^2, L3 = du_L L2,
                                L1T2 = du_L T2 (src/Calculations/serial_single_pass.jl:886-905 flat,
                                :838-843 other metrics). A flat joint plan of this kind at precision
                                MIXED runs the FP64 joint kernel (faster for these rows, and within the
                                mixed tolerance); it cannot be a batched slice. A flat joint plan may
                                hold 2..6 consecutive rows (ops[k].nl = ops[0].nl + k, one value axis):
                                one FP64 launch forms each pair's arithmetic once for all of them, at
                                any precision, and its outputs are the rows' (n_dist, n_val) matrices
                                one after the other. */
} sfb200_op_kind;

typedef struct {
    int32_t kind; /* sfb200_op_kind */
    int32_t nl;   /* PROJECTED: longitudinal power NL >= 0 */
    int32_t nt;   /* PROJECTED: transverse power NT >= 0 */
    int32_t nf;   /* FULLVEC: power NF >= 0 */
} sfb200_operator;

/* Bin-edge descriptions (reference src/BinEdges.jl). */
typedef enum {
    SFB200_BINS_TABLE = 0,   /* sorted edge vector (BinEdges, binary search). For flat geometry the
                                library squares the edges in double (= _sq_edges(Float64, v),
                                src/BinEdges.jl:440). */
    SFB200_BINS_SQTABLE = 1, /* flat only: the caller passes the squared-edge table itself, as built by
                                squared_digitize_plan(...).sqedges (src/BinEdges.jl:447-463); this is
                                how Float32 edges and LogBinEdges keep the reference's exact table. */
    SFB200_BINS_LINEAR = 2   /* LinearBinEdges (an AbstractRange): FMA search of src/BinEdges.jl:114-131
                                with (first, last, inv_step, step, n_edges) as stored by the reference. */
} sfb200_bins_kind;

typedef struct {
    int32_t kind;        /* sfb200_bins_kind */
    int32_t n_edges;     /* number of edges (bins = n_edges - 1); >= 2 */
    const double* edges; /* TABLE / SQTABLE: n_edges values, copied at plan creation */
    double first, last, inv_step, step; /* LINEAR */
} sfb200_bins;

typedef enum {
    SFB200_PREC_FP64 = 0,  /* plain form: every pair in FP64 */
    SFB200_PREC_MIXED = 1, /* FP64 point differences, squared distance (exact bin) and projection
                              numerators; FP32 normalisation, operator powers and run accumulation;
                              FP64 merge. Sums within 1e-6 of the FP64 oracle per bin. */
    SFB200_PREC_FP32 = 2   /* FP32 bulk: FP32 differences ((hi, lo) records for FP64 inputs) and
                              binning with an FP64 recheck of near-edge / short / near-antipodal
                              pairs; counts exact, sums within FP32 accuracy of each pair (a pair
                              whose projection cancels carries ~1e-7 |du| absolute error) */
} sfb200_precision;

typedef enum { SFB200_F64 = 0, SFB200_F32 = 1 } sfb200_dtype;

typedef struct {
    int32_t geometry;    /* sfb200_geometry */
    int32_t dim;         /* velocity components D in {2, 3} */
    int32_t angle_unit;  /* sphere only */
    double radius;       /* sphere only: r = radius * central angle */
    int32_t n_ops;       /* 1..SFB200_MAX_OPS (joint plans: 1, or 2..6 consecutive flat SFB200_OP_SP2D rows) */
    sfb200_operator ops[SFB200_MAX_OPS];
    sfb200_bins distance;
    int32_t joint;       /* 0: 1D histogram; 1: joint (distance x value) histogram */
    sfb200_bins value;   /* joint only (TABLE or LINEAR) */
    int32_t precision;   /* sfb200_precision */
    int32_t x_dtype;     /* sfb200_dtype of x */
    int32_t u_dtype;     /* sfb200_dtype of u */
} sfb200_plan_desc;

/* sfb200_run flags */
#define SFB200_RUN_DEVICE_INPUT  0x1u /* x and u are device pointers (already in HBM) */
#define SFB200_RUN_DEVICE_OUTPUT 0x2u /* sums and counts are device pointers; the call is then
                                         asynchronous on the stream */
#define SFB200_RUN_ACCUMULATE    0x4u /* add into sums/counts (mutating API semantics) instead of
                                         overwriting them */

typedef struct {
    int64_t pairs;          /* N(N-1)/2 of the last run */
    int64_t rechecked;      /* pairs that took the FP64 recheck path (mixed precision) */
    double kernel_ms;       /* device time of the pair kernel(s), CUDA events */
    int32_t tile;           /* tile size the autotuner chose */
    int32_t blocks;         /* persistent blocks launched */
    int32_t threads;        /* threads per block */
    int32_t kernel_launches;/* kernels launched by the last run */
    int32_t privatization;  /* histogram privatization depth used (-1: joint kernel) */
} sfb200_stats;

typedef struct sfb200_ctx sfb200_ctx;
typedef struct sfb200_plan sfb200_plan;

/* Library ABI version (SFB200_ABI_VERSION). */
SFB200_API int sfb200_abi_version(void);

/* Context: one CUDA device, one stream, device workspace pool.
 * Replaces: the GPU workspace object of ext/gpu/workspace.jl:25-56. */
SFB200_API int sfb200_ctx_create(int device, sfb200_ctx** out);
SFB200_API int sfb200_ctx_destroy(sfb200_ctx* ctx);
/* Text of the calling thread's last failed call on this context (never NULL; empty if that thread's
 * last failure was on another context). Kept per thread, so threads sharing a context do not race. */
SFB200_API const char* sfb200_last_error(const sfb200_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work. */
SFB200_API void* sfb200_ctx_stream(sfb200_ctx* ctx);

/* Plan: validated operator set + bin tables + precision for one input layout.
 * Replaces: BinEdges / squared_digitize_plan construction (src/BinEdges.jl:362-469) and the
 * operator-to-kernel mapping of the GPU route (ext/StructureFunctionsKernelAbstractionsExt.jl:385-401). */
SFB200_API int sfb200_plan_create(sfb200_ctx* ctx, const sfb200_plan_desc* desc, sfb200_plan** out);
SFB200_API int sfb200_plan_destroy(sfb200_plan* plan);
/* Number of doubles in `sums` and of uint64 in `counts` that sfb200_run writes. */
SFB200_API int sfb200_plan_output_sizes(const sfb200_plan* plan, int64_t* n_sums, int64_t* n_counts);

/* Run the pair hot path over N points.
 * Replaces: _dispatch_execution_backend(::GPUBackend, ::PointField, ...) -> gpu_calculate_structure_function
 * (src/Calculations/dispatch.jl:537-544, ext/StructureFunctionsKernelAbstractionsExt.jl:385-401, 630-675)
 * and, with SFB200_RUN_ACCUMULATE, _dispatch_execution_backend! (dispatch.jl:399-404, accumulate-into
 * semantics of _accumulate_gpu_sf_host!, ext/StructureFunctionsKernelAbstractionsExt.jl:678-719).
 * `stream` may be NULL (context stream). With host outputs the call returns after the results are
 * copied back. */
SFB200_API int sfb200_run(sfb200_plan* plan, const void* x, const void* u, int64_t n, uint32_t flags,
               double* sums, uint64_t* counts, void* stream);

/* Smallest and largest pair distance over all pairs i < j of the N points, for automatic binning:
 * Euclidean sqrt(r^2) from the reference's squared distance; on the sphere the arc length R sigma
 * (SphericalAngle: sigma) from the pair frame's angle 2 atan(|q - p|, |q + p|). u is packed with x
 * (the plan's layout) but not used. flags may hold SFB200_RUN_DEVICE_INPUT. Synchronous.
 * Replaces: the min/max scan of the reference's auto-binning, _minmax_matrix_for_autobins / minmax_i
 * (src/Calculations/dispatch.jl:205-298). */
SFB200_API int sfb200_distance_range(sfb200_plan* plan, const void* x, const void* u, int64_t n, uint32_t flags,
                                     double* dmin, double* dmax, void* stream);

/* Statistics of the last sfb200_run on this plan. */
SFB200_API int sfb200_plan_last_stats(const sfb200_plan* plan, sfb200_stats* out);

/* Autotuner override of a plan's launch: tile size (points per tile = threads per block; 0 =
 * automatic; 32, 64, 128, 256, 512, and 768 for the mixed joint kernel), histogram privatization
 * depth of the 1D kernels (-1 = automatic; 0 = one warp-aggregated histogram per warp; 2 =
 * warp-aggregated with shared-memory atomics; 3 = per-lane runs added into a block table of lane
 * columns; 6 = the same with two open runs per lane (flat FP64 / MIXED kernels; the default for
 * 256-point tiles from 32768 points); 1, 4, 8 = copies per warp updated with shared-memory atomics;
 * 32 = one column per lane of every warp), and a cap on resident blocks per SM (0 = occupancy
 * limit). No counterpart in the reference (its GPU backend has no launch knobs). */
SFB200_API int sfb200_plan_set_launch(sfb200_plan* plan, int tile, int privatization, int blocks_per_sm);

/* Plan options for sfb200_plan_set_option. */
typedef enum {
    /* Point storage order on the device: -1 automatic (from 16384 points: Morton order for 1D
     * histograms, scattered for the flat joint histogram), 0 the caller's order, 1 Morton (Z-curve)
     * order, 2 scattered (slot i holds point (i m) mod N). Results are the same up to the rounding
     * of the sums (counts are identical); the joint sphere path always keeps the caller's order. */
    SFB200_OPT_POINT_ORDER = 1,
    /* Columns of the run-length histogram table (privatization 3): 0 automatic, else 1, 2, 4, 8,
     * 16 or 32. */
    SFB200_OPT_HIST_COLUMNS = 2,
    /* Multi-GPU sharding of sfb200_run: value = (count << 32) | index; the run then covers only
     * shard `index` of `count` contiguous ranges of the upper-triangle tile pairs holding equal numbers
     * of pairs (sfb200_shard_bounds; its outputs
     * hold that shard's partial histogram; the caller adds the shards, e.g. with one all-reduce).
     * Default 1 << 32 (one shard: everything). The partition of the pair set into tile pairs is
     * the reference's (i < j) pair set exactly, so the shard sums add up to the full histogram. */
    SFB200_OPT_SHARD = 3,
    /* J-tile order of the flat 1D kernels (precision FP64 and MIXED, 256-point tiles): -1 automatic
     * (sorted), 0 storage order, 1 each off-diagonal J tile staged in the order of its distance from
     * the I tile, so that each lane's run of equal bins is long. Counts are identical either way;
     * only the summation order of the sums changes. */
    SFB200_OPT_TILE_SORT = 4,
    /* Formulation of the FP64 spherical 1D kernel (other plans ignore it): -1 automatic (chord), 1 the
     * reference's own: the
     * pair frame (geodesic frame, parallel transport, atan2) for every pair
     * (src/HelperFunctions.jl:186-200, 265-276, 324-348), 2 the chord formulation of the mixed kernel
     * in FP64 (bin on the squared chord against the chord images of the edges, the reference frame only
     * for the pairs within 2^-40 of an edge image, coincident or antipodal; increments from the chord
     * and the tangent velocities). Counts are identical; sums agree to FP64 rounding. */
    SFB200_OPT_FORMULATION = 5
} sfb200_option;

/* Set a plan option (autotuning; no counterpart in the reference). */
SFB200_API int sfb200_plan_set_option(sfb200_plan* plan, int option, int64_t value);

/* Tile pairs [*tp_lo, *tp_hi) of shard `index` of `count` for n points in tiles of `tile` points (the
 * partition SFB200_OPT_SHARD uses; host arithmetic only, no device needed). Shard k begins at the
 * first tile pair before which k / count of the N(N-1)/2 pairs lie, so every shard is within one
 * tile pair of an equal share of the pairs. Replaces: the per-rank share of the outer index, _rank_share
 * (ext/StructureFunctionsMPIExt.jl:24-26), with tile pairs as the unit. */
SFB200_API int sfb200_shard_bounds(int64_t n, int32_t tile, int32_t index, int32_t count, int64_t* tp_lo,
                                   int64_t* tp_hi);

/* ------------------------------------------------------------------------------------ serving
 * Batched execution for many independent point sets (time slices, fields, requests) of uneven size.
 * No counterpart in the reference, which runs one call at a time; it serves the request loop of the
 * host glue (admission by free device memory, continuous batching).
 *
 * A slice is one point set made resident on the device with its own histogram: created from a plan
 * (precision SFB200_PREC_MIXED) and the inputs, it holds the packed points and a zeroed histogram.
 * Its work is `tile_pairs` independent units. sfb200_batch_run queues one round: for every listed
 * slice, the tile pairs [begin, end) are added into its histogram. Slices of different plans (2D/3D,
 * planar/spherical, 1D or joint) may share a round: the library groups them by kernel and runs each
 * group as one persistent launch whose blocks pull (slice, tile-pair range) items from a device
 * counter; the round is captured as a CUDA graph and replayed with updated parameters. Every tile
 * pair of a slice must be covered exactly once over the rounds; the result then equals sfb200_run's
 * (counts identical, sums up to summation order). Rounds are double-buffered: the next round may be
 * queued while one runs (the host prepares it meanwhile, and the device starts it as soon as the
 * running one ends); queuing a third waits for the first. Rounds queued on the same stream run one
 * after the other, so one slice may take part in consecutive rounds.
 *
 * Slice memory comes from a stream-ordered pool of the context: creating a slice allocates one block
 * in order on its preparation stream, destroying it frees the block in order after its preparation,
 * every round queued so far and its last read, without waiting on the host. Freed blocks stay in the
 * pool for later slices; sfb200_device_memory counts them as free. */
typedef struct sfb200_slice sfb200_slice;

typedef struct {
    int64_t n_points;
    int64_t pairs;          /* n (n - 1) / 2 */
    int64_t tile_pairs;     /* work units of the batched kernels */
    int64_t device_bytes;   /* device memory held by the slice */
} sfb200_slice_info;

/* Make one point set resident (copy if host input, order, pack, zero the histogram), queued on
 * `stream` (NULL: the context stream). The plan must outlive the slice. */
SFB200_API int sfb200_slice_create(sfb200_plan* plan, const void* x, const void* u, int64_t n, uint32_t flags,
                                   void* stream, sfb200_slice** out);
SFB200_API int sfb200_slice_get_info(const sfb200_slice* slice, sfb200_slice_info* out);
/* One round: tile pairs [tp_begin[k], tp_end[k]) of slices[k], k < n (each slice at most once). */
SFB200_API int sfb200_batch_run(sfb200_ctx* ctx, int32_t n, sfb200_slice* const* slices, const int64_t* tp_begin,
                                const int64_t* tp_end, void* stream);
/* Copy a slice's histogram out (host buffers: synchronous; SFB200_RUN_DEVICE_OUTPUT: queued on the
 * stream; SFB200_RUN_ACCUMULATE adds into the caller's buffers). The copy waits for the slice's
 * preparation and for the last round that listed it, not for rounds queued after that one; a NULL
 * stream means a side stream of the context that carries no rounds. Destroying a slice frees its
 * memory in the same order. */
SFB200_API int sfb200_slice_read(sfb200_slice* slice, double* sums, uint64_t* counts, uint32_t flags, void* stream);
SFB200_API int sfb200_slice_destroy(sfb200_slice* slice);
/* Wait for every queued round of the context (blocking) / ask whether all have finished (*done = 0
 * or 1). */
SFB200_API int sfb200_batch_wait(sfb200_ctx* ctx);
SFB200_API int sfb200_batch_query(sfb200_ctx* ctx, int32_t* done);
/* Wait for the oldest unfinished round only; *round (if not NULL) receives its number (rounds are
 * numbered 1, 2, ... in the order sfb200_batch_run queued them; 0 if none was unfinished). */
SFB200_API int sfb200_batch_wait_oldest(sfb200_ctx* ctx, int64_t* round);
/* Free and total device memory of the context's device (cudaMemGetInfo, plus blocks the context's
 * slice pool holds unused), for admission control. */
SFB200_API int sfb200_device_memory(sfb200_ctx* ctx, int64_t* free_bytes, int64_t* total_bytes);

/* ------------------------------------------------------------------------------ no allocation
 * sfb200_run over device inputs and device outputs that allocates no device memory: for callers that
 * must not allocate while they run -- a loop that reserved its whole device budget up front, or a
 * process sharing the device, where an allocation could fail under memory pressure or make the device
 * wait. No counterpart in the reference. Scratch is one fixed array per device inside the library
 * (3.4 MiB, held by every device that loads the library until the process exits): flat (Euclidean)
 * 1D plans of precision MIXED or FP64 only, at most 65536 points, at most 32768 sums (bins x
 * operators) and 4096 bins; larger calls return SFB200_ERR_UNSUPPORTED. Points are taken in the
 * caller's order. x, u, sums and counts are device pointers; flags may only hold
 * SFB200_RUN_ACCUMULATE. The first call on a context looks up the scratch array's device address
 * (and loads the kernels it uses), so make that first call before any stream capture; the context
 * keeps the address, and a device reset (cudaDeviceReset) invalidates it together with every other
 * context resource: destroy and re-create the context after one. All calls on one
 * device share the scratch: calls that overlap on the GPU (from several streams or threads) race on
 * it and must be serialised by the caller. */
SFB200_API int sfb200_run_noalloc(sfb200_plan* plan, const void* x, const void* u, int64_t n, uint32_t flags,
                                  double* sums, uint64_t* counts, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SFB200_H */
