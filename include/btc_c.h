/*
 * btc_c.h -- C ABI of the B200 (sm_100a) exact triangle-counting engine.
 *
 * The engine computes the masked product L (.) (L L^T) on Bit-BSR tiles, the path
 * of fanna1234/btc-tc-artifact's btc/btc.h (Bit-BSR build + hybrid count).  That
 * surface is a set of C++ templates; this header restates it as plain C: pointers,
 * sizes and status codes, no C++ or torch types.  Every entry point names the
 * reference interface it replaces (paths within fanna1234/btc-tc-artifact).
 *
 * Status codes: every int-returning call returns BTC_OK (0) or a negative BTC_E_*.
 * Streams: btc_stream_t is a cudaStream_t (NULL = legacy default stream).
 * Threading: calls on distinct handles are independent; calls that share a handle
 * must be ordered by the caller (one stream, or host synchronisation), because a
 * handle owns its build workspace and its count scratch.
 */
#ifndef BTC_C_H
#define BTC_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* btc_stream_t;

#if defined(__GNUC__)
#define BTC_API __attribute__((visibility("default")))
#else
#define BTC_API
#endif

#define BTC_OK 0
#define BTC_E_INVAL (-1)   /* bad argument: null pointer, tile width, size limit */
#define BTC_E_NOMEM (-2)   /* device or pinned-host allocation failed */
#define BTC_E_CUDA (-3)    /* CUDA runtime error (launch, copy, sync) */
#define BTC_E_TIMEOUT (-4) /* reserved: a bounded device wait gave up */
#define BTC_E_RANGE (-5)   /* an input vertex id lies outside [0, n) */
#define BTC_E_CAPACITY (-6) /* a rebuild enqueued with BTC_BUILD_ASYNC found more tiles
                               than the handle's arrays hold; nothing was built */

/* Build flags (btc_build_bitbsr, btc_rebuild_bitbsr, btc_convert_*). */
#define BTC_INPUT_ON_HOST 0x1u /* src/dst are host pointers (pinned or pageable) */
#define BTC_ORIENT_DEGREE 0x2u /* relabel vertices by descending degree (ties by id)
                                  before orienting each edge to (max, min) */
#define BTC_BUILD_RADIX 0x4u   /* number tiles with the radix-sort builder even when the
                                  (row block, column block) cell bitmap would fit */
#define BTC_BUILD_ASYNC 0x8u   /* rebuild without waiting (see btc_rebuild_bitbsr) */

/* Default dense/sparse switch: a tile takes the binary tensor-core path when its
 * popcount exceeds tau.  Pass BTC_TAU_DEFAULT to use the engine's value. */
#define BTC_TAU_DEFAULT (-1)
#define BTC_TAU_ALL_SPARSE 0x7fffffff

/* ======================================================================== */
/* Reference-shaped surface                                                  */
/* ======================================================================== */

/* Field order, types and bit layout of btc::BCSR_16x128_Device
 * (btc/operations/bcsr_16x128.h:24-32) and btc::BCSR_16x32_Device
 * (btc/operations/bcsr_16x32.h:109-117):
 *   indptr[n_row_blocks+1]  tile offsets per 16-row block
 *   indices[num_blocks]     column-block id of each tile, ascending within a row block
 *   row_indices[num_blocks] row-block id of each tile
 *   blocks[num_blocks*W]    tile bits, row-major, W = 64 (16x128) or 16 (16x32) words;
 *                           bit b of word (r*W/16 + w) is column 32w+b of tile row r
 *   result                  device uint64 that receives the count
 * All arrays are device memory owned by the engine (free with btc_bcsr_free). */
typedef struct btc_bcsr_device {
    uint32_t* indptr;
    uint32_t* indices;
    uint32_t* blocks;
    uint32_t* row_indices;
    unsigned long long* result;
    int n;
    int n_row_blocks;
    uint32_t num_blocks;
} btc_bcsr_device;

/* Replaces btc::convert_coo_to_bcsr_16x128_gpu (btc/operations/bcsr_16x128.h:136-241).
 * d_rows/d_cols: device COO of nnz entries on num_rows vertices.  The reference
 * expects the preprocessed lower triangle; this call orients, drops self-loops and
 * deduplicates itself, so any symmetric or one-sided edge list gives the same tiles.
 * Blocking (legacy default stream).  Returns BTC_OK or BTC_E_*. */
BTC_API int btc_convert_coo_to_bcsr_16x128_gpu(btc_bcsr_device* bcsr, const int32_t* d_rows,
                                       const int32_t* d_cols, int64_t nnz, int32_t num_rows);

/* Replaces btc::convert_coo_to_bcsr_16x32_gpu (btc/operations/bcsr_16x32.h:144-249). */
BTC_API int btc_convert_coo_to_bcsr_16x32_gpu(btc_bcsr_device* bcsr, const int32_t* d_rows,
                                      const int32_t* d_cols, int64_t nnz, int32_t num_rows);

/* Replaces btc::count_triangles_16x128_adaptive (btc/operations/tc_16x128_adaptive.h:12-29)
 * and count_triangles_16x128_v5/_v4.  threshold_blocks selected the reference's v4/v5
 * variant; the engine has one kernel and accepts the argument for signature parity.
 * kernel_ms (nullable) receives the kernel-only event time.  The count is written to
 * *out_count and to bcsr->result.  Blocking. */
BTC_API int btc_count_triangles_16x128_adaptive(btc_bcsr_device* bcsr, int threshold_blocks,
                                        float* kernel_ms, unsigned long long* out_count);

/* Replaces btc::count_triangles_16x32_adaptive (btc/operations/tc_16x32_adaptive.h:14-31). */
BTC_API int btc_count_triangles_16x32_adaptive(btc_bcsr_device* bcsr, int threshold_blocks,
                                       float* kernel_ms, unsigned long long* out_count);

/* Replaces BCSR_*_Device::free() (bcsr_16x128.h:34-42): releases every array and
 * nulls the pointers.  Safe on a zeroed or already freed struct. */
BTC_API void btc_bcsr_free(btc_bcsr_device* bcsr);

/* Replaces BCSR_*_Device::reset_result() / get_result() (bcsr_16x128.h:44-50). */
BTC_API int btc_bcsr_reset_result(btc_bcsr_device* bcsr);
BTC_API int btc_bcsr_get_result(const btc_bcsr_device* bcsr, unsigned long long* out);

/* Replaces btc::preprocess_for_triangle_counting (btc/operations/convert.h:600-612 with
 * BTC_REORDER=0): in place on device COO arrays, orient every entry to (max, min),
 * drop self-loops, sort lexicographically and drop duplicates; with remap != 0 also
 * compact vertex ids to [0, n_used) in ascending order (convert.h:386-425).  *nnz and
 * *num_rows are updated.  Blocking. */
BTC_API int btc_preprocess_for_triangle_counting(int32_t* d_rows, int32_t* d_cols, int64_t* nnz,
                                         int32_t* num_rows, int remap);

/* Replaces btc::reorder_hashorder_gpu (btc/operations/reorder.h:443-587; BTC_REORDER=8, and
 * what the default BTC_REORDER=9 runs when the automatic rule says so): relabels the
 * vertices of a device COO in place so that vertices with similar neighbourhoods get
 * nearby ids, then orients every entry to (max, min).  Signature of vertex v: num_hashes
 * MinHash values over its num_hops-hop closed neighbourhood, h_j(v) = (a_j v + b_j) mod
 * (2^32 - 5) with the reference's parameters (btc_hashorder_params); order: lexicographic
 * by signature, ties by id.  The reference's defaults are num_hashes 16, num_hops 1.
 * d_perm (nullable, num_rows int32) receives new id = d_perm[old id].  Ids outside
 * [0, num_rows) give BTC_E_RANGE and leave both the COO and d_perm unwritten.  Allocates
 * its workspace; blocking. */
BTC_API int btc_reorder_hashorder(int32_t* d_rows, int32_t* d_cols, int64_t nnz, int32_t num_rows,
                                  int num_hashes, int num_hops, int32_t* d_perm,
                                  btc_stream_t stream);

/* The hash parameters btc_reorder_hashorder uses (host only): a[j], b[j] for j <
 * num_hashes (at most 64), drawn as reorder.h:495-506 draws them. */
BTC_API int btc_hashorder_params(int num_hashes, uint32_t* a, uint32_t* b);

/* Replaces btc::should_reorder_gpu (btc/operations/convert.h:579-596, with
 * should_reorder_hopper_ampere 510-575 below sm_120 -- B200 is sm_100 -- and
 * should_reorder_blackwell 443-505 from sm_120): whether the default preprocess reorders
 * a graph of num_rows vertices and nnz COO entries.  dataset_hint (nullable) is the input
 * file's base name.  Returns 1 or 0. */
BTC_API int btc_should_reorder(int32_t num_rows, int64_t nnz, int sm_version,
                               const char* dataset_hint);

/* The BTC-Lite O(1) tile policy (apps/btc_tc_lite.cu:45-65): returns 32 or 128.
 * mode 1 forces 32, mode 2 forces 128 (the reference's BTC_MODE), 0 applies
 * "avg degree nnz/rows < 15 or rows < 50000 -> 32, else 128". */
BTC_API int btc_lite_select_tile_cols(int64_t nnz, int32_t num_rows, int mode);

/* The engine's tile policy: tile width and tau per graph class, chosen from cheap
 * features, in order -- the average degree 2m/n (>= 512: 16x32), BTC_ORIENT_DEGREE in
 * flags (power-law input ordered by degree: 16x128) and the id locality `locality` (the
 * share of edges with |u - v| < 128 over the share uniform ids would give; >= 16: 16x128,
 * else 16x32) -- set from a measured sweep of both widths over five graph families on a
 * B200.
 * No counterpart in the reference, whose policy is the fixed BTC-Lite rule above (kept
 * as the baseline this policy beats).  Host only; *tau (nullable) receives the measured
 * default tau of the chosen width. */
BTC_API int btc_tile_policy_from_features(int64_t m, int32_t n, uint32_t flags, double locality,
                                          int* tile_cols, int* tau);

/* The same policy with the locality sampled from the edge list itself (65,536 evenly
 * spaced edges): on the host for BTC_INPUT_ON_HOST arrays, else by one small kernel on
 * `stream` followed by one wait (16 bytes of device scratch, allocated and freed here).
 * btc_build_bitbsr and btc_batch_build apply it when tile_cols is 0.  No counterpart in
 * the reference. */
BTC_API int btc_select_tile_policy(const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                                   uint32_t flags, btc_stream_t stream, int* tile_cols, int* tau);

/* ======================================================================== */
/* Stream-ordered engine surface                                             */
/* ======================================================================== */

typedef struct btc_bitbsr btc_bitbsr; /* opaque, device-resident, owns its buffers */

typedef struct btc_bitbsr_view {
    btc_bcsr_device bcsr; /* the arrays, in the reference layout */
    int tile_cols;        /* 32 or 128 */
    int device;           /* CUDA ordinal the handle lives on */
    int64_t num_edges;    /* unique lower edges (r > c) after dedup */
    int64_t input_edges;  /* edges handed to the build, self-loops included */
    size_t device_bytes;  /* device memory held by the handle */
} btc_bitbsr_view;

/* Builds the Bit-BSR of an edge list (src[i], dst[i]), i < m, on n vertices with
 * 16 x tile_cols tiles (tile_cols 32 or 128; 0 applies btc_select_tile_policy -- an
 * asynchronous rebuild of an edge list not ordered by degree keeps the handle's current
 * width instead, since the policy's edge sample would wait).
 * Orientation to (max, min), self-loop removal and deduplication happen on the GPU.
 * With BTC_INPUT_ON_HOST the arrays are host memory and are copied on `stream`.
 * Synchronises `stream` once (to size the tile arrays, or at the end of a rebuild that
 * fits the handle's arrays).  *out receives a new handle.
 * Limits: n < 2^31, m <= 2^32 - 4096, tiles < 2^32.  Replaces the preprocess + convert pair
 * (convert.h:600, bcsr_16x128.h:136 / bcsr_16x32.h:144). */
BTC_API int btc_build_bitbsr(const int32_t* src, const int32_t* dst, int64_t m, int32_t n, int tile_cols,
                     uint32_t flags, btc_stream_t stream, btc_bitbsr** out);

/* Same as btc_build_bitbsr into an existing handle, reusing its device buffers
 * when they are large enough (no allocation in steady state).
 *
 * BTC_BUILD_ASYNC (no counterpart in the reference): when the handle already holds tile
 * arrays from an earlier build and the cell-bitmap builder applies, the whole build is
 * enqueued on `stream` against the arrays' capacity and the call returns without
 * waiting (otherwise the flag is ignored and the call waits as usual).  The inputs must
 * stay valid until `stream` has run the build.  A count enqueued after it reads the
 * tile count on the device.  The build's status arrives with the next call that waits
 * on the handle (btc_count, btc_bitbsr_info, btc_density_hist, btc_partition_tiles,
 * btc_count_tiles_async, a rebuild): BTC_E_RANGE for an out-of-range id, BTC_E_CAPACITY
 * for more tiles than the arrays hold (nothing built; rebuild without the flag).  Until
 * then a failed build makes btc_count_async write 0xFFFFFFFFFFFFFFFF. */
BTC_API int btc_rebuild_bitbsr(btc_bitbsr* g, const int32_t* src, const int32_t* dst, int64_t m,
                       int32_t n, int tile_cols, uint32_t flags, btc_stream_t stream);

/* Counts the triangles of a handle: enqueues the count on `stream`, waits, and
 * writes *out_count.  tau: dense/sparse switch (BTC_TAU_DEFAULT for the engine's).
 * kernel_ms (nullable): event time of the count kernel alone.  Replaces
 * count_triangles_16x{128,32}_adaptive (tc_16x128_adaptive.h:12, tc_16x32_adaptive.h:14). */
BTC_API int btc_count(btc_bitbsr* g, int tau, btc_stream_t stream, unsigned long long* out_count,
              float* kernel_ms);

/* Counts the triangles of a Bit-BSR without allocating any memory.  No counterpart in
 * the reference: it exists for callers that cannot let a library call cudaMalloc, such
 * as a serving process whose memory pool already holds the device's free memory, or a
 * latency-bound loop that must not call cudaMalloc/cudaFree because they can synchronise
 * the device.  The caller passes the Bit-BSR (reference layout, e.g. from
 * btc_bitbsr_info or btc_convert_*) and a device word d_out for the count (NULL: use
 * bcsr->result).  The count kernel's scratch (one partial sum per CTA plus a completion
 * counter) is a fixed array inside the library's device image: 2048 partial-sum slots
 * and two control words, 16,400 bytes, held by every GPU that loads the library until the process exits.  A GPU
 * whose count grid needs more than 2048 CTAs is rejected with BTC_E_INVAL and a message
 * on stderr (a B200 needs 592).  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  A device reset (cudaDeviceReset) gives the device a new
 * context, and the next call repeats that lookup, so it too should come before any
 * capture.  All calls share the one array: calls whose kernels overlap on the GPU
 * (different streams, or several host threads) race and give wrong counts, so order
 * them.  It always runs the count's light variant (it has no per-tile row masks), so on
 * power-law graphs, where btc_count picks the heavy variant, it is exact but slower.
 * Stream-ordered; does not wait for the result.  tau as in btc_count. */
BTC_API int btc_count_bcsr_noalloc(const btc_bcsr_device* bcsr, int tile_cols, int tau,
                                   btc_stream_t stream, unsigned long long* d_out);

/* Enqueues the count on `stream` without waiting; the uint64 count lands in device
 * memory at d_out (nullable: then only in the handle's result slot) when the
 * stream reaches it. */
BTC_API int btc_count_async(btc_bitbsr* g, int tau, btc_stream_t stream, unsigned long long* d_out);

/* ---- one graph on several GPUs ------------------------------------------------
 * No counterpart in the reference, which counts on one GPU.  Every rank builds the
 * same Bit-BSR (same input and flags, hence the same tiles in the same order), takes
 * its tile range from btc_partition_tiles, counts it with btc_count_tiles_async, and
 * the ranks add their counts (one int64 all-reduce).  The counts of any partition of
 * [0, num_tiles) add up to btc_count's result. */

/* bounds[0..parts]: tile ranges [bounds[r], bounds[r+1]) of about equal estimated count
 * cost, cut at multiples of 256 tiles.  One device pass over the tiles and one wait on
 * `stream`; allocates (and frees) 8 bytes per 256 tiles. */
BTC_API int btc_partition_tiles(const btc_bitbsr* g, int parts, btc_stream_t stream,
                                uint32_t* bounds);

/* The host half of btc_partition_tiles: bounds from per-bucket costs (bucket b holds
 * tiles [b*bucket_tiles, (b+1)*bucket_tiles)).  Needs no GPU. */
BTC_API int btc_partition_from_costs(const unsigned long long* bucket_cost, uint64_t n_buckets,
                                     uint32_t bucket_tiles, uint32_t num_tiles, int parts,
                                     uint32_t* bounds);

/* Counts the sample tiles [tile_begin, tile_end) into device memory at d_out, enqueued
 * on `stream` without waiting.  Uses the handle's count scratch: one count at a time
 * per handle. */
BTC_API int btc_count_tiles_async(btc_bitbsr* g, uint32_t tile_begin, uint32_t tile_end, int tau,
                                  btc_stream_t stream, unsigned long long* d_out);

/* Diagnostic (no counterpart in the reference): binary AND-popcount-accumulates per
 * second of mma.sync.m16n8k128...b1.and.popc on this GPU (the dense path's instruction),
 * measured with `iters` rounds of independent MMAs per warp on a persistent grid; the
 * denominator of the dense class's tensor-core utilisation. */
BTC_API int btc_b1_mma_peak(btc_stream_t stream, int iters, double* ops_per_s);

/* Fills *v with the handle's arrays and sizes. */
BTC_API int btc_bitbsr_info(const btc_bitbsr* g, btc_bitbsr_view* v);

/* Tile popcount histogram: hist[p] = number of tiles with exactly p bits set,
 * p in [0, 16*tile_cols] (hist holds 16*tile_cols+1 host uint64).  Blocking. */
BTC_API int btc_density_hist(btc_bitbsr* g, btc_stream_t stream, uint64_t* hist);

/* Releases the handle and every buffer it owns.  NULL is a no-op. */
BTC_API void btc_free(btc_bitbsr* g);

/* ======================================================================== */
/* Batches: many graphs, one build, one persistent count launch               */
/* (no counterpart in the reference, which counts one graph per process)      */
/* ======================================================================== */

typedef struct btc_batch btc_batch; /* opaque, device-resident */

/* Builds the Bit-BSR of num_graphs graphs at once.  Graph g's edges are
 * (src[i], dst[i]) for i in [edge_offsets[g], edge_offsets[g+1]) with local vertex ids in
 * [0, num_vertices[g]); edge_offsets (num_graphs+1 entries, edge_offsets[0] = 0) and
 * num_vertices are host arrays.  src/dst are device arrays, or host arrays with
 * BTC_INPUT_ON_HOST.  The batch is the block-diagonal union of the graphs (graph g's
 * vertex v is union vertex 16*R_<g + v, R_<g = row blocks of graphs 0..g-1), with one
 * tile width for all (32, 128, or 0 for btc_select_tile_policy over the whole batch, each
 * sampled edge's locality measured against its own graph's size).  Each graph has its own
 * cell bitmap of ceil(n/16) x ceil(ceil(n/tile_cols)/32) words; a batch whose graphs need
 * more than 2^29 words together returns BTC_E_INVAL (count such graphs one at a time).
 * Synchronises `stream` once. */
BTC_API int btc_batch_build(const int32_t* src, const int32_t* dst, const int64_t* edge_offsets,
                            const int32_t* num_vertices, int32_t num_graphs, int tile_cols,
                            uint32_t flags, btc_stream_t stream, btc_batch** out);

/* Rebuilds into an existing batch, reusing its device buffers when large enough.
 * With BTC_BUILD_ASYNC in flags, device input and the same graphs' sizes as the batch's
 * last successful build (num_graphs, edge_offsets, num_vertices, tile width; the edges may
 * differ), the rebuild is enqueued against the arrays the batch holds without host work,
 * allocation or a wait, so it can be captured in a CUDA graph together with
 * btc_batch_count(..., h_counts = NULL); its status comes with the next call that waits
 * (btc_batch_count with h_counts, btc_batch_info, a waiting rebuild): BTC_E_RANGE for an
 * out-of-range id, BTC_E_CAPACITY for more tiles than the arrays held (nothing built, the
 * counts are 0; rebuild without the flag).  Another enqueued rebuild before that call
 * replaces it (its status is not kept).  Otherwise the flag is ignored and the rebuild
 * waits once, as btc_batch_build does. */
BTC_API int btc_batch_rebuild(btc_batch* b, const int32_t* src, const int32_t* dst,
                              const int64_t* edge_offsets, const int32_t* num_vertices,
                              int32_t num_graphs, int tile_cols, uint32_t flags,
                              btc_stream_t stream);

/* Counts every graph of the batch in one launch.  d_counts (device, num_graphs uint64,
 * nullable: the batch's own buffer) receives graph g's count at index g; with h_counts
 * (host, nullable) the counts are also copied out and the call waits for them. */
BTC_API int btc_batch_count(btc_batch* b, int tau, btc_stream_t stream,
                            unsigned long long* d_counts, unsigned long long* h_counts);

/* The union graph's Bit-BSR (reference layout) and sizes. */
BTC_API int btc_batch_info(btc_batch* b, btc_bitbsr_view* v);

/* First row block of each graph in the union (num_graphs+1 host entries). */
BTC_API int btc_batch_row_offsets(const btc_batch* b, uint32_t* row_offsets);

/* Releases the batch.  NULL is a no-op. */
BTC_API void btc_batch_free(btc_batch* b);

/* ======================================================================== */
/* Serving: continuous batching over the batched path                        */
/* (no counterpart in the reference)                                          */
/* ======================================================================== */

typedef struct btc_server btc_server; /* opaque; owns one engine thread */

typedef struct btc_server_config {
    uint64_t hbm_budget_bytes; /* device memory all batch slots together may hold */
    int32_t max_batch_graphs;  /* requests per batch (1: no batching) */
    int32_t slots;             /* batches in flight at once (1..8; 2 overlaps them) */
    int64_t max_batch_edges;   /* input edges per batch */
    int tile_cols;             /* 32, 128, or 0 for the engine's tile policy per batch */
    int tau;                   /* dense/sparse switch, BTC_TAU_DEFAULT */
    int64_t solo_edges;        /* requests with at least this many edges (or a vertex
                                  range needing more than 2^26 cell-bitmap words) run
                                  alone, degree-ordered, with the engine's tile policy */
} btc_server_config;

typedef struct btc_server_result {
    uint64_t id;              /* from btc_server_submit */
    unsigned long long count; /* triangles (0 unless status == BTC_OK) */
    int32_t status;           /* BTC_OK, or BTC_E_NOMEM if the request alone exceeds
                                 the budget, or the failing call's status */
    int32_t n;                /* the request's vertex count */
    int64_t m;                /* the request's edge count */
    double submit_s;          /* server steady clock, seconds */
    double done_s;            /* when the result was published */
} btc_server_result;

typedef struct btc_server_stats {
    uint64_t batches, graphs, edges, rejected, queued, peak_device_bytes;
    double now_s;
    /* launches that ran one large request alone (the single-graph path), and the
     * stream time (first copy to the result's copy back, CUDA events) spent in those
     * and in batches; slots overlap, so the two may add up to more than wall time */
    uint64_t solo_launches;
    double solo_stream_ms, batch_stream_ms;
} btc_server_stats;

/* Fills the defaults: 150 GB budget, 4096 graphs and 256M edges per batch, 2 slots,
 * 16x32 tiles, default tau, requests of 2^20 edges or more run alone. */
BTC_API void btc_server_default_config(btc_server_config* cfg);

/* Starts a server on the current device.  A batch slot admits queued requests in
 * arrival order while the batch stays within the caps and all slots stay within the
 * budget; requests that arrive while batches are on the GPU join the next batch.  The
 * slots' device memory comes from a stream-ordered pool the server owns (freed memory
 * stays in the pool for later requests until btc_server_destroy). */
BTC_API int btc_server_create(const btc_server_config* cfg, btc_server** out);

/* Host-side allocation-failure injection, for tests of the server's recovery: when the
 * environment variable BTC_SERVER_FAIL_RESERVE holds comma-separated positive integers
 * at btc_server_create, the server's buffer reservations (six per launched batch,
 * numbered from 1 in the order the engine makes them) with those numbers report
 * BTC_E_NOMEM without allocating.  The requests of that batch complete with status
 * BTC_E_NOMEM; the server goes on with the next ones.  No GPU fault is involved. */

/* Queues a request (host edge arrays; local ids in [0, n)).  Returns at once;
 * *id_out identifies the result.  The edges are copied on submit, or, with
 * BTC_SUBMIT_BORROW, read in place when the request's batch is staged: the caller then
 * keeps src/dst unchanged until the request's result has been polled. */
#define BTC_SUBMIT_BORROW 0x1u
BTC_API int btc_server_submit(btc_server* s, const int32_t* src, const int32_t* dst, int64_t m,
                              int32_t n, uint32_t flags, uint64_t* id_out);

/* Moves up to max_results finished results to out (*n_out of them), waiting up to
 * wait_ms for the first one. */
BTC_API int btc_server_poll(btc_server* s, btc_server_result* out, int max_results, int* n_out,
                            int wait_ms);

BTC_API int btc_server_stats_get(btc_server* s, btc_server_stats* st);

/* Finishes every queued request, then stops the engine and frees the server. */
BTC_API void btc_server_destroy(btc_server* s);

/* Default tau for a tile width (the value BTC_TAU_DEFAULT resolves to). */
BTC_API int btc_default_tau(int tile_cols);

/* Static text for a status code. */
BTC_API const char* btc_strerror(int status);

/* ABI version: (major << 16) | minor. */
BTC_API int btc_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BTC_C_H */
