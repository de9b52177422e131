// capi.cu -- the C ABI (include/btc_c.h): handles, build pipeline, count calls and
// the reference-shaped struct surface.  Host code only; kernels live in radix.cu,
// build.cu and count.cu.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "common.cuh"
#include "handle.cuh"

#include <algorithm>

namespace btc200 {

int launch_degree(const int32_t*, const int32_t*, int64_t, int32_t, uint32_t*, cudaStream_t);
int launch_rank_keys(const uint32_t*, int32_t, uint32_t, uint64_t*, cudaStream_t);
int launch_rank_scatter(const uint64_t*, int32_t, int32_t*, cudaStream_t);
int launch_make_keys(const BuildGeom&, const int32_t*, const int32_t*, int64_t, const int32_t*,
                     uint64_t*, unsigned long long*, cudaStream_t);
int launch_segment(const BuildGeom&, const uint64_t*, size_t, const unsigned long long*, uint32_t*,
                   unsigned long long*, cudaStream_t);
int launch_fill(const BuildGeom&, const uint64_t*, size_t, const unsigned long long*,
                const uint32_t*, uint32_t*, uint32_t*, uint32_t*, cudaStream_t);
uint64_t bitmap_words_per_row(const BuildGeom&);
size_t bitmap_chunks(uint64_t W);
int bitmap_mark_and_count(const BuildGeom&, const int32_t*, const int32_t*, int64_t, const int32_t*,
                          uint32_t*, uint32_t*, unsigned long long*, unsigned long long*, cudaStream_t);
int bitmap_emit_and_fill(const BuildGeom&, const int32_t*, const int32_t*, int64_t, const int32_t*,
                         const uint32_t*, const uint32_t*, uint2*, uint32_t*, uint32_t*, uint32_t*,
                         uint32_t*, unsigned long long*, uint32_t, unsigned long long*,
                         cudaStream_t, uint32_t*);
int launch_popcount_sum(int, const uint32_t*, uint64_t, unsigned long long*, cudaStream_t);
int launch_indptr(const uint32_t*, uint32_t, int32_t, uint32_t*, cudaStream_t);
int launch_density(int, const uint32_t*, uint32_t, unsigned long long*, cudaStream_t);
int launch_set_u64(unsigned long long* p, unsigned long long v, cudaStream_t s);

void note_cuda_error(cudaError_t e, const char* what, const char* file, int line)
{
    static const bool verbose = std::getenv("BTC_DEBUG") != nullptr;
    if (verbose)
        std::fprintf(stderr, "[btc] CUDA error %s (%s) at %s:%d: %s\n", cudaGetErrorName(e),
                     cudaGetErrorString(e), file, line, what);
}

int device_sm_count()
{
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}

}  // namespace btc200

using namespace btc200;

// Engine's default dense/sparse switch.  A tile takes the binary tensor-core path
// when its popcount exceeds tau.
// Measured on sm_100a (policy.cu, the tau sweep): 16x128 tiles switch to the binary
// tensor core above 1024 bits (half full), 16x32 tiles above 64 (the reference's value).
int default_tau(int tile_cols) { return tile_cols == 128 ? 1024 : 64; }

static constexpr uint64_t kMaxEdges = (1ull << 32) - (uint64_t)kSortTile;

int ensure_count_scratch(btc_bitbsr* g)
{
    const int grid = count_grid_size(128) > count_grid_size(32) ? count_grid_size(128)
                                                                 : count_grid_size(32);
    const size_t need = sizeof(unsigned long long) * (size_t)grid;
    if (g->partials.bytes < need) BTC_TRY(g->partials.reserve(need));
    if (!g->done.ptr) {
        BTC_TRY(g->done.reserve(kCountCtlBytes));
        BTC_CUDA_TRY(g->done.zero(kCountCtlBytes));
    }
    if (!g->result.ptr) {
        BTC_TRY(g->result.reserve(sizeof(unsigned long long)));
        BTC_CUDA_TRY(g->result.zero(sizeof(unsigned long long)));
    }
    return BTC_OK;
}

// Pinned host slots the device writes directly (mapped): build status, tile count and
// the count result reach the host without a copy-engine hop.
int ensure_host_meta(btc_bitbsr* g)
{
    if (g->h_meta) return BTC_OK;
    void* p = nullptr;
    if (cudaHostAlloc(&p, sizeof(unsigned long long) * kMetaSlots,
                      cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return BTC_E_NOMEM;
    }
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeHost(p);
        return BTC_E_CUDA;
    }
    std::memset(p, 0, sizeof(unsigned long long) * kMetaSlots);
    g->h_meta = static_cast<unsigned long long*>(p);
    g->d_hmeta = static_cast<unsigned long long*>(d);
    return BTC_OK;
}

// What one build enqueues, fixed before anything is enqueued (every buffer reserved).
struct BuildPlan {
    BuildGeom geom;
    const int32_t* src;  // caller's arrays (host with BTC_INPUT_ON_HOST)
    const int32_t* dst;
    const int32_t* d_src;  // device arrays the kernels read
    const int32_t* d_dst;
    int64_t m;
    int32_t n;
    uint32_t flags;
    bool use_bitmap;
    bool degree;
    uint64_t bm_words;
    uint32_t cap;  // > 0: the post-count steps run against this tile capacity
    bool row_index = false;  // build the row-wise count's row index (rowindex.cu)
};

static bool row_index_possible(int64_t m, int32_t n_row_blocks)
{
    return n_row_blocks > 0 && m >= 8 * (int64_t)n_row_blocks && m < (int64_t)0xffffffffll;
}

static int reserve_row_index(btc_bitbsr* g, int64_t m, uint64_t R)
{
    BTC_TRY(g->row_off.reserve(sizeof(uint32_t) * (16 * R + 1)));
    BTC_TRY(g->row_ent.reserve(sizeof(uint2) * (size_t)m));
    BTC_TRY(g->row_tot.reserve(sizeof(uint32_t) * R));
    return g->row_bsum.reserve(sizeof(unsigned long long) +
                               sizeof(uint32_t) * ((size_t)ri_scan_blocks((uint32_t)R) + 1));
}

// The row index after the row masks (T = *d_tiles bounded by cap, or cap itself).
static int enqueue_row_index(btc_bitbsr* g, const unsigned long long* d_tiles, uint32_t cap,
                             cudaStream_t s)
{
    unsigned long long* total = g->row_bsum.as<unsigned long long>();
    return launch_rowindex(g->indptr.as<uint32_t>(), g->indices.as<uint32_t>(), g->n_row_blocks,
                           g->rowmask.as<uint32_t>(), d_tiles, cap, g->row_tot.as<uint32_t>(),
                           reinterpret_cast<uint32_t*>(total + 1), total, g->row_off.as<uint32_t>(),
                           g->row_ent.as<uint2>(), g->row_ent.bytes / sizeof(uint2), s);
}

// Enqueues the build up to the tile count (bitmap path) or up to the tile segmentation
// (radix path), and with plan.cap > 0 the whole bitmap build.  No waits, no allocation:
// this sequence is what a cached CUDA graph replays.
static int enqueue_build(btc_bitbsr* g, const BuildPlan& P, uint64_t** sorted_out, cudaStream_t s)
{
    const BuildGeom& geom = P.geom;
    unsigned long long* meta = g->meta.as<unsigned long long>();
    BTC_CUDA_TRY(cudaMemsetAsync(meta, 0, sizeof(unsigned long long) * kMetaSlots, s));
    if ((P.flags & BTC_INPUT_ON_HOST) && P.m > 0) {
        BTC_CUDA_TRY(cudaMemcpyAsync(g->in_src.ptr, P.src, sizeof(int32_t) * (size_t)P.m,
                                     cudaMemcpyHostToDevice, s));
        BTC_CUDA_TRY(cudaMemcpyAsync(g->in_dst.ptr, P.dst, sizeof(int32_t) * (size_t)P.m,
                                     cudaMemcpyHostToDevice, s));
    }
    uint64_t* k0 = g->keys0.as<uint64_t>();
    uint64_t* k1 = g->keys1.as<uint64_t>();
    int st = BTC_OK;

    // ---- optional descending-degree relabel ---------------------------------
    const int32_t* rank = nullptr;
    if (P.degree) {
        const int32_t n = P.n;
        BTC_CUDA_TRY(cudaMemsetAsync(g->deg.ptr, 0, sizeof(uint32_t) * (size_t)n, s));
        BTC_TRY(launch_degree(P.d_src, P.d_dst, P.m, n, g->deg.as<uint32_t>(), s));
        int db = bit_length_u64(2ull * (uint64_t)P.m);  // degrees fit in db bits
        if (db > 32) db = 32;
        const uint32_t dmax = db >= 32 ? 0xffffffffu : ((1u << db) - 1u);
        BTC_TRY(launch_rank_keys(g->deg.as<uint32_t>(), n, dmax, k0, s));
        BTC_TRY(launch_set_u64(meta + kMetaN, (unsigned long long)n, s));
        uint64_t* sorted = radix_sort_u64(k0, k1, (size_t)n, meta + kMetaN, 32, 32 + (db ? db : 1),
                                          g->sort_scratch.as<uint32_t>(), s, &st);
        BTC_TRY(st);
        BTC_TRY(launch_rank_scatter(sorted, n, g->rank.as<int32_t>(), s));
        rank = g->rank.as<int32_t>();
    }

    if (P.use_bitmap) {
        BTC_TRY(bitmap_mark_and_count(geom, P.d_src, P.d_dst, P.m, rank, g->bitmap.as<uint32_t>(),
                                      g->tile_base.as<uint32_t>(), meta + kMetaBad,
                                      meta + kMetaTiles, s));
        if (P.cap) {
            BTC_TRY(bitmap_emit_and_fill(geom, P.d_src, P.d_dst, P.m, rank,
                                         g->bitmap.as<uint32_t>(), g->tile_base.as<uint32_t>(),
                                         g->prefix.as<uint2>(), g->indices.as<uint32_t>(),
                                         g->row_indices.as<uint32_t>(), g->indptr.as<uint32_t>(),
                                         g->blocks.as<uint32_t>(), meta, P.cap, g->d_hmeta, s,
                                         g->rowmask.as<uint32_t>()));
            // the fill pass set the row masks; this pass finds the longest row-block list
            BTC_TRY(launch_rowmask(geom.tile_cols, g->blocks.as<uint32_t>(), P.cap,
                                   meta + kMetaTiles, g->indptr.as<uint32_t>(), geom.n_row_blocks,
                                   g->rowmask.as<uint32_t>(), meta + kMetaRowMax, s, false));
            if (P.row_index) BTC_TRY(enqueue_row_index(g, meta + kMetaTiles, P.cap, s));
        }
    } else {
        // ---- keys, sort, segmentation ---------------------------------------
        BTC_TRY(launch_make_keys(geom, P.d_src, P.d_dst, P.m, rank, k0, meta, s));
        uint64_t* sorted = radix_sort_u64(k0, k1, (size_t)P.m, meta + kMetaValid,
                                          geom.payload_bits, geom.payload_bits + geom.t_bits,
                                          g->sort_scratch.as<uint32_t>(), s, &st);
        BTC_TRY(st);
        BTC_TRY(launch_segment(geom, sorted, (size_t)P.m, meta + kMetaValid,
                               g->tile_base.as<uint32_t>(), meta + kMetaTiles, s));
        *sorted_out = sorted;
    }
    return BTC_OK;
}

// Everything an enqueued build reads or writes, plus its arguments: a graph captured
// from enqueue_build replays only under the same key.
static void build_key(const btc_bitbsr* g, const BuildPlan& P, BuildGraphKey* k)
{
    std::memset(k, 0, sizeof(*k));
    const void* w[] = {P.src, P.dst, g->meta.ptr, g->in_src.ptr, g->in_dst.ptr, g->keys0.ptr,
                       g->keys1.ptr, g->sort_scratch.ptr, g->deg.ptr, g->rank.ptr, g->bitmap.ptr,
                       g->prefix.ptr, g->tile_base.ptr, g->indices.ptr, g->row_indices.ptr,
                       g->indptr.ptr, g->blocks.ptr, g->rowmask.ptr, g->d_hmeta, g->row_off.ptr,
                       g->row_ent.ptr, g->row_tot.ptr, g->row_bsum.ptr};
    static_assert(sizeof(w) / sizeof(w[0]) == kBuildKeyPtrs, "key layout");
    for (int i = 0; i < kBuildKeyPtrs; ++i) k->ptr[i] = w[i];
    k->m = P.m;
    k->n = P.n;
    k->tile_cols = P.geom.tile_cols;
    k->flags = P.flags;
    k->cap = P.cap;
}

// Replays (or, on the second identical call, captures) the enqueued build as a CUDA
// graph: one launch instead of about a dozen.  Returns false when it did not enqueue.
static bool launch_build_graph(btc_bitbsr* g, const BuildPlan& P, cudaStream_t s)
{
    BuildGraphKey key;
    build_key(g, P, &key);
    if (g->graph_exec && std::memcmp(&key, &g->graph_key, sizeof(key)) == 0)
        return cudaGraphLaunch(g->graph_exec, s) == cudaSuccess;
    const bool repeat = std::memcmp(&key, &g->last_key, sizeof(key)) == 0;
    g->last_key = key;
    if (!repeat) return false;
    if (!g->capture_stream &&
        cudaStreamCreateWithFlags(&g->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(g->capture_stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    uint64_t* unused = nullptr;
    const int st = enqueue_build(g, P, &unused, g->capture_stream);
    const cudaError_t e = cudaStreamEndCapture(g->capture_stream, &graph);
    cudaGraphExec_t exec = nullptr;
    const bool ok = st == BTC_OK && e == cudaSuccess && graph &&
                    cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return false;
    }
    if (g->graph_exec) cudaGraphExecDestroy(g->graph_exec);
    g->graph_exec = exec;
    g->graph_key = key;
    return cudaGraphLaunch(g->graph_exec, s) == cudaSuccess;
}

static int build_into(btc_bitbsr* g, const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                      int tile_cols, uint32_t flags, cudaStream_t s)
{
    if (n < 0 || m < 0 || (uint64_t)m > kMaxEdges) return BTC_E_INVAL;
    if (m > 0 && (!src || !dst)) return BTC_E_INVAL;
    if (flags & ~(BTC_INPUT_ON_HOST | BTC_ORIENT_DEGREE | BTC_BUILD_RADIX | BTC_BUILD_ASYNC))
        return BTC_E_INVAL;
    if (g->pending) resolve_build(g);  // an enqueued build still owns the buffers
    if (tile_cols == 0) {
        // the engine's tile policy (policy.cu).  With degree ordering it needs only m and
        // n; otherwise it samples the edges (a wait), which an enqueued rebuild skips by
        // keeping the handle's width.
        if (flags & BTC_ORIENT_DEGREE)
            BTC_TRY(btc_tile_policy_from_features(m, n, BTC_ORIENT_DEGREE, 0.0, &tile_cols, nullptr));
        else if ((flags & BTC_BUILD_ASYNC) && (g->tile_cols == 32 || g->tile_cols == 128))
            tile_cols = g->tile_cols;
        else
            BTC_TRY(btc_select_tile_policy(src, dst, m, n, flags & BTC_INPUT_ON_HOST, s, &tile_cols,
                                           nullptr));
    }
    if (tile_cols != 32 && tile_cols != 128) return BTC_E_INVAL;
    BTC_CUDA_TRY(cudaGetDevice(&g->device));

    BuildPlan P{};
    P.geom = make_geom(n, tile_cols);
    const BuildGeom& geom = P.geom;
    // the previous build of this handle, when it had the same geometry, predicts whether
    // the graph averages 8 or more tiles per row block (the row index's condition)
    const bool prev_light = g->tile_cols == tile_cols && g->n_row_blocks == geom.n_row_blocks &&
                            g->num_tiles > 0 &&
                            (uint64_t)g->num_tiles < 8ull * (uint64_t)geom.n_row_blocks;
    g->tile_cols = tile_cols;
    g->n = n;
    g->n_row_blocks = geom.n_row_blocks;
    g->input_edges = m;
    g->edges_known = false;
    g->num_edges = 0;

    // ---- reserve every buffer the enqueued steps use ---------------------------
    BTC_TRY(ensure_host_meta(g));
    BTC_TRY(g->meta.reserve(sizeof(unsigned long long) * kMetaSlots));
    unsigned long long* meta = g->meta.as<unsigned long long>();
    P.src = src;
    P.dst = dst;
    P.d_src = src;
    P.d_dst = dst;
    P.m = m;
    P.n = n;
    P.flags = flags;
    if ((flags & BTC_INPUT_ON_HOST) && m > 0) {
        BTC_TRY(g->in_src.reserve(sizeof(int32_t) * (size_t)m));
        BTC_TRY(g->in_dst.reserve(sizeof(int32_t) * (size_t)m));
        P.d_src = g->in_src.as<int32_t>();
        P.d_dst = g->in_dst.as<int32_t>();
    }
    // The cell bitmap (one bit per (row block, column block)) replaces the sort when it
    // is small next to the edge list; otherwise the radix path sorts tile keys.
    const uint64_t wpr = bitmap_words_per_row(geom);
    P.bm_words = wpr * (uint64_t)geom.n_row_blocks;
    const uint64_t bm_bytes = 4 * P.bm_words;
    P.use_bitmap = !(flags & BTC_BUILD_RADIX) && bm_bytes <= (4ull << 30) &&
                   bm_bytes <= 32ull * (uint64_t)m + (64ull << 20);
    g->used_bitmap = P.use_bitmap;
    g->row_index = false;
    P.degree = (flags & BTC_ORIENT_DEGREE) && n > 0;
    size_t key_cap = P.use_bitmap ? 0 : (size_t)m;
    if (P.degree && (size_t)n > key_cap) key_cap = (size_t)n;
    if (key_cap) {
        BTC_TRY(g->keys0.reserve(sizeof(uint64_t) * key_cap));
        BTC_TRY(g->keys1.reserve(sizeof(uint64_t) * key_cap));
        BTC_TRY(g->sort_scratch.reserve(sizeof(uint32_t) * radix_scratch_words(key_cap)));
    }
    const size_t chunk_slots = P.use_bitmap ? bitmap_chunks(P.bm_words) : sort_tiles((size_t)m);
    BTC_TRY(g->tile_base.reserve(sizeof(uint32_t) * (chunk_slots + 1)));
    if (P.degree) {
        BTC_TRY(g->deg.reserve(sizeof(uint32_t) * (size_t)n));
        BTC_TRY(g->rank.reserve(sizeof(int32_t) * (size_t)n));
    }
    if (P.use_bitmap) {
        BTC_TRY(g->bitmap.reserve(sizeof(uint32_t) * (P.bm_words ? P.bm_words : 1)));
        BTC_TRY(g->prefix.reserve(sizeof(uint2) * (P.bm_words ? P.bm_words : 1)));
        // the row-wise count's row index: only a graph with at least 8 edges per row block
        // can average 8 tiles per row block (every tile holds an edge).  A rebuild whose
        // previous graph of the same geometry averaged fewer skips it (a mesh would pay
        // five launches that find nothing to do); should this graph average more after
        // all, the count takes the tile-wise kernel, which needs no index.
        P.row_index = row_index_possible(m, geom.n_row_blocks) && !prev_light;
        if (P.row_index) BTC_TRY(reserve_row_index(g, m, (uint64_t)geom.n_row_blocks));
        g->row_index = P.row_index;
    }
    BTC_TRY(g->indptr.reserve(sizeof(uint32_t) * ((size_t)geom.n_row_blocks + 1)));
    BTC_TRY(ensure_count_scratch(g));

    const size_t TW = (size_t)16 * (tile_cols / 32);
    // Tiles the arrays already hold room for (a rebuild): the bitmap path then enqueues
    // the whole build against that capacity, with every post-count kernel checking the
    // device tile count, and waits once at the end (or not at all with BTC_BUILD_ASYNC);
    // a count above the capacity is redone below at the right size.  A first build
    // waits for the count in between.
    if (P.use_bitmap && g->indices.ptr && g->row_indices.ptr && g->blocks.ptr && g->rowmask.ptr) {
        uint64_t c = g->indices.bytes / 4;
        c = std::min<uint64_t>(c, g->row_indices.bytes / 4);
        c = std::min<uint64_t>(c, g->blocks.bytes / (4 * TW));
        c = std::min<uint64_t>(c, g->rowmask.bytes / 4);
        P.cap = (uint32_t)std::min<uint64_t>(c, 0xffffffffull);
    }

    uint64_t* sorted = nullptr;
    if (P.cap) {
        // repeated identical asynchronous rebuilds of device input replay a CUDA graph
        const bool graphed = (flags & BTC_BUILD_ASYNC) && !(flags & BTC_INPUT_ON_HOST) &&
                             launch_build_graph(g, P, s);
        if (!graphed) BTC_TRY(enqueue_build(g, P, &sorted, s));
        // the build's status and tile count are in h_meta once the stream has run it
        // (k_set_last writes them through the mapping)
        if (!g->meta_event)
            BTC_CUDA_TRY(cudaEventCreateWithFlags(&g->meta_event, cudaEventDisableTiming));
        BTC_CUDA_TRY(cudaEventRecord(g->meta_event, s));
        g->pending = true;
        g->pending_cap = P.cap;
        if (flags & BTC_BUILD_ASYNC) return BTC_OK;  // resolved by the next wait
        const int st2 = resolve_build(g);
        if (st2 != BTC_E_CAPACITY) return st2;
        // more tiles than the arrays hold: redo the post-count steps at the right size
        BTC_CUDA_TRY(cudaMemsetAsync(meta + kMetaOverflow, 0, sizeof(unsigned long long), s));
    } else {
        BTC_TRY(enqueue_build(g, P, &sorted, s));
    }
    BTC_CUDA_TRY(cudaMemcpyAsync(g->h_meta, meta, sizeof(unsigned long long) * 3,
                                 cudaMemcpyDeviceToHost, s));
    BTC_CUDA_TRY(cudaStreamSynchronize(s));
    if (g->h_meta[kMetaBad] != 0) return BTC_E_RANGE;
    const unsigned long long tiles = g->h_meta[kMetaTiles];
    if (tiles > 0xffffffffull) return BTC_E_INVAL;
    g->num_tiles = (uint32_t)tiles;

    // ---- tile arrays ----------------------------------------------------------
    BTC_TRY(g->indices.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    BTC_TRY(g->row_indices.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    BTC_TRY(g->blocks.reserve(sizeof(uint32_t) * TW * (tiles ? tiles : 1)));
    BTC_TRY(g->rowmask.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    if (P.use_bitmap) {
        BTC_TRY(bitmap_emit_and_fill(geom, P.d_src, P.d_dst, m, P.degree ? g->rank.as<int32_t>() : nullptr,
                                     g->bitmap.as<uint32_t>(), g->tile_base.as<uint32_t>(),
                                     g->prefix.as<uint2>(), g->indices.as<uint32_t>(),
                                     g->row_indices.as<uint32_t>(), g->indptr.as<uint32_t>(),
                                     g->blocks.as<uint32_t>(), meta, (uint32_t)tiles, nullptr, s,
                                     g->rowmask.as<uint32_t>()));
    } else {
        if (tiles)
            BTC_CUDA_TRY(cudaMemsetAsync(g->blocks.ptr, 0, sizeof(uint32_t) * TW * tiles, s));
        BTC_TRY(launch_fill(geom, sorted, (size_t)m, meta + kMetaValid, g->tile_base.as<uint32_t>(),
                            g->indices.as<uint32_t>(), g->row_indices.as<uint32_t>(),
                            g->blocks.as<uint32_t>(), s));
        BTC_TRY(launch_indptr(g->row_indices.as<uint32_t>(), g->num_tiles, geom.n_row_blocks,
                              g->indptr.as<uint32_t>(), s));
    }
    // the bitmap path's fill pass set the row masks; the radix path's are computed here
    BTC_TRY(launch_rowmask(tile_cols, g->blocks.as<uint32_t>(), g->num_tiles, nullptr,
                           g->indptr.as<uint32_t>(), g->n_row_blocks, g->rowmask.as<uint32_t>(),
                           meta + kMetaRowMax, s, !P.use_bitmap));
    // the tile count is known here: the index exactly when the graph averages 8 or more
    // tiles per row block
    P.row_index = P.use_bitmap && row_index_possible(m, geom.n_row_blocks) &&
                  (uint64_t)g->num_tiles >= 8ull * (uint64_t)geom.n_row_blocks;
    if (P.row_index) {
        BTC_TRY(reserve_row_index(g, m, (uint64_t)geom.n_row_blocks));
        BTC_TRY(enqueue_row_index(g, nullptr, g->num_tiles, s));
    }
    g->row_index = P.row_index;
    return BTC_OK;
}

int count_handle(btc_bitbsr* g, int tau, cudaStream_t s, unsigned long long* d_out2,
                 uint32_t tile_begin, uint32_t tile_end, bool to_host)
{
    if (!g) return BTC_E_INVAL;
    if (tau == BTC_TAU_DEFAULT) tau = default_tau(g->tile_cols);
    if (tau < 0) return BTC_E_INVAL;
    if (!g->pending && g->failed != BTC_OK) return g->failed;
    BTC_TRY(ensure_count_scratch(g));
    CountScratch scr{g->partials.as<unsigned long long>(), g->done.as<unsigned int>(),
                     reinterpret_cast<unsigned long long*>(g->done.as<char>() + 8),
                     g->result.as<unsigned long long>(), d_out2};
    if (to_host) {
        BTC_TRY(ensure_host_meta(g));
        scr.result_host = g->d_hmeta + 7;
    }
    // after an enqueued build the kernel reads the tile count (and the build's status)
    // from the device; the capacity bounds it
    const unsigned long long* build_meta = g->pending ? g->meta.as<unsigned long long>() : nullptr;
    return launch_count(g->tile_cols, g->indptr.as<uint32_t>(), g->indices.as<uint32_t>(),
                        g->row_indices.as<uint32_t>(), g->blocks.as<uint32_t>(),
                        g->pending ? g->pending_cap : g->num_tiles, g->n_row_blocks, tau, scr, s,
                        nullptr, 0, nullptr, g->rowmask.as<uint32_t>(),
                        g->used_bitmap ? g->prefix.as<uint2>() : nullptr,
                        bitmap_words_per_row(make_geom(g->n, g->tile_cols)),
                        g->meta.as<unsigned long long>() + kMetaRowMax, tile_begin, tile_end,
                        build_meta, g->num_tiles,
                        g->used_bitmap && g->row_index ? g->row_off.as<uint32_t>() : nullptr,
                        g->used_bitmap && g->row_index ? g->row_ent.as<uint2>() : nullptr,
                        // tiles averaging more than half of tau's bits: the kernel variant
                        // that keeps the tensor-core path's registers
                        (uint64_t)g->input_edges * 2 > (uint64_t)tau * (uint64_t)g->num_tiles);
}

int resolve_build(btc_bitbsr* g)
{
    if (!g->pending) return g->failed;
    g->pending = false;
    if (cudaEventSynchronize(g->meta_event) != cudaSuccess) {
        cudaGetLastError();
        return g->failed = BTC_E_CUDA;
    }
    const unsigned long long* h = g->h_meta;
    if (h[kMetaBad] != 0) {
        g->failed = BTC_E_RANGE;
    } else if (h[kMetaOverflow] != 0 || h[kMetaTiles] > g->pending_cap) {
        g->failed = BTC_E_CAPACITY;
    } else {
        g->num_tiles = (uint32_t)h[kMetaTiles];
        g->failed = BTC_OK;
    }
    return g->failed;
}

// ===========================================================================
// C ABI
// ===========================================================================
namespace btc200 {
// An empty handle whose allocations are all stream-ordered on `s` from `pool`, for an
// owner that uses it on `s` only (a server slot); its first (re)build sizes it.
btc_bitbsr* bitbsr_new_pooled(cudaMemPool_t pool, cudaStream_t s)
{
    btc_bitbsr* g = new (std::nothrow) btc_bitbsr();
    if (g) g->set_pool(pool, s);
    return g;
}
}  // namespace btc200

extern "C" {

int btc_abi_version(void) { return (1 << 16) | 0; }

int btc_default_tau(int tile_cols) { return default_tau(tile_cols); }

const char* btc_strerror(int status)
{
    switch (status) {
    case BTC_OK: return "ok";
    case BTC_E_INVAL: return "invalid argument";
    case BTC_E_NOMEM: return "out of memory";
    case BTC_E_CUDA: return "CUDA error";
    case BTC_E_TIMEOUT: return "device wait timed out";
    case BTC_E_RANGE: return "vertex id out of range";
    case BTC_E_CAPACITY: return "an enqueued rebuild needed more tiles than the handle held";
    default: return "unknown status";
    }
}

int btc_lite_select_tile_cols(int64_t nnz, int32_t num_rows, int mode)
{
    if (mode == 1) return 32;
    if (mode == 2) return 128;
    const float avg = num_rows > 0 ? (float)nnz / (float)num_rows : 0.0f;
    return (avg < 15.0f || num_rows < 50000) ? 32 : 128;
}

int btc_build_bitbsr(const int32_t* src, const int32_t* dst, int64_t m, int32_t n, int tile_cols,
                     uint32_t flags, btc_stream_t stream, btc_bitbsr** out)
{
    if (!out) return BTC_E_INVAL;
    *out = nullptr;
    btc_bitbsr* g = new (std::nothrow) btc_bitbsr();
    if (!g) return BTC_E_NOMEM;
    const int st = build_into(g, src, dst, m, n, tile_cols, flags, stream);
    if (st != BTC_OK) {
        g->release_all();
        delete g;
        return st;
    }
    *out = g;
    return BTC_OK;
}

int btc_rebuild_bitbsr(btc_bitbsr* g, const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                       int tile_cols, uint32_t flags, btc_stream_t stream)
{
    if (!g) return BTC_E_INVAL;
    const int st = build_into(g, src, dst, m, n, tile_cols, flags, stream);
    if (!g->pending) g->failed = st;  // an enqueued build's status comes with resolve_build
    return st;
}

int btc_count_async(btc_bitbsr* g, int tau, btc_stream_t stream, unsigned long long* d_out)
{
    return count_handle(g, tau, stream, d_out);
}

int btc_count(btc_bitbsr* g, int tau, btc_stream_t stream, unsigned long long* out_count,
              float* kernel_ms)
{
    if (!g || !out_count) return BTC_E_INVAL;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernel_ms) {
        BTC_CUDA_TRY(cudaEventCreate(&e0));
        BTC_CUDA_TRY(cudaEventCreate(&e1));
        BTC_CUDA_TRY(cudaEventRecord(e0, stream));
    }
    // the count kernel's last CTA writes the result into h_meta[7] through the mapping
    int st = count_handle(g, tau, stream, nullptr, 0, 0xffffffffu, true);
    if (st == BTC_OK && kernel_ms && cudaEventRecord(e1, stream) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK) st = resolve_build(g);
    if (st == BTC_OK) {
        *out_count = g->h_meta[7];
        if (kernel_ms) cudaEventElapsedTime(kernel_ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return st;
}

int btc_bitbsr_info(const btc_bitbsr* gc, btc_bitbsr_view* v)
{
    if (!gc || !v) return BTC_E_INVAL;
    btc_bitbsr* g = const_cast<btc_bitbsr*>(gc);
    BTC_TRY(resolve_build(g));
    if (!g->edges_known) {
        // unique lower edges = bits set in the tiles (duplicates OR the same bit); the
        // build may have run on any stream, so wait for the device first
        BTC_CUDA_TRY(cudaDeviceSynchronize());
        unsigned long long u = 0;
        unsigned long long* d = g->meta.as<unsigned long long>() + kMetaUniq;
        BTC_TRY(launch_popcount_sum(g->tile_cols, g->blocks.as<uint32_t>(), g->num_tiles, d, nullptr));
        BTC_CUDA_TRY(cudaMemcpy(&u, d, sizeof(u), cudaMemcpyDeviceToHost));
        g->num_edges = (int64_t)u;
        g->edges_known = true;
    }
    std::memset(v, 0, sizeof(*v));
    v->bcsr.indptr = g->indptr.as<uint32_t>();
    v->bcsr.indices = g->indices.as<uint32_t>();
    v->bcsr.blocks = g->blocks.as<uint32_t>();
    v->bcsr.row_indices = g->row_indices.as<uint32_t>();
    v->bcsr.result = g->result.as<unsigned long long>();
    v->bcsr.n = g->n;
    v->bcsr.n_row_blocks = g->n_row_blocks;
    v->bcsr.num_blocks = g->num_tiles;
    v->tile_cols = g->tile_cols;
    v->device = g->device;
    v->num_edges = g->num_edges;
    v->input_edges = g->input_edges;
    v->device_bytes = g->device_bytes();
    return BTC_OK;
}

int btc_density_hist(btc_bitbsr* g, btc_stream_t stream, uint64_t* hist)
{
    if (!g || !hist) return BTC_E_INVAL;
    BTC_TRY(resolve_build(g));
    const size_t nb = (size_t)16 * g->tile_cols + 1;
    DevBuf d;
    BTC_TRY(d.reserve(sizeof(unsigned long long) * nb));
    int st = BTC_OK;
    if (cudaMemsetAsync(d.ptr, 0, sizeof(unsigned long long) * nb, stream) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK)
        st = launch_density(g->tile_cols, g->blocks.as<uint32_t>(), g->num_tiles,
                            d.as<unsigned long long>(), stream);
    if (st == BTC_OK && cudaMemcpyAsync(hist, d.ptr, sizeof(unsigned long long) * nb,
                                        cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        st = BTC_E_CUDA;
    if (st == BTC_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = BTC_E_CUDA;
    d.release();
    return st;
}

void btc_free(btc_bitbsr* g)
{
    if (!g) return;
    g->release_all();
    delete g;
}

// ---------------------------------------------------------------------------
// reference-shaped struct surface
// ---------------------------------------------------------------------------
static int convert_struct(btc_bcsr_device* b, const int32_t* d_rows, const int32_t* d_cols,
                          int64_t nnz, int32_t num_rows, int tile_cols)
{
    if (!b) return BTC_E_INVAL;
    std::memset(b, 0, sizeof(*b));
    btc_bitbsr* g = nullptr;
    const int st = btc_build_bitbsr(d_rows, d_cols, nnz, num_rows, tile_cols, 0, nullptr, &g);
    if (st != BTC_OK) return st;
    // hand the arrays to the struct; it frees them one by one (btc_bcsr_free)
    b->indptr = g->indptr.as<uint32_t>();
    b->indices = g->indices.as<uint32_t>();
    b->blocks = g->blocks.as<uint32_t>();
    b->row_indices = g->row_indices.as<uint32_t>();
    b->result = g->result.as<unsigned long long>();
    b->n = g->n;
    b->n_row_blocks = g->n_row_blocks;
    b->num_blocks = g->num_tiles;
    g->indptr.ptr = g->indices.ptr = g->blocks.ptr = g->row_indices.ptr = g->result.ptr = nullptr;
    g->indptr.bytes = g->indices.bytes = g->blocks.bytes = g->row_indices.bytes = g->result.bytes = 0;
    btc_free(g);
    return BTC_OK;
}

int btc_convert_coo_to_bcsr_16x128_gpu(btc_bcsr_device* b, const int32_t* d_rows,
                                       const int32_t* d_cols, int64_t nnz, int32_t num_rows)
{
    return convert_struct(b, d_rows, d_cols, nnz, num_rows, 128);
}

int btc_convert_coo_to_bcsr_16x32_gpu(btc_bcsr_device* b, const int32_t* d_rows,
                                      const int32_t* d_cols, int64_t nnz, int32_t num_rows)
{
    return convert_struct(b, d_rows, d_cols, nnz, num_rows, 32);
}

void btc_bcsr_free(btc_bcsr_device* b)
{
    if (!b) return;
    if (b->indptr) cudaFree(b->indptr);
    if (b->indices) cudaFree(b->indices);
    if (b->blocks) cudaFree(b->blocks);
    if (b->row_indices) cudaFree(b->row_indices);
    if (b->result) cudaFree(b->result);
    b->indptr = b->indices = b->blocks = b->row_indices = nullptr;
    b->result = nullptr;
}

int btc_bcsr_reset_result(btc_bcsr_device* b)
{
    if (!b || !b->result) return BTC_E_INVAL;
    BTC_CUDA_TRY(cudaMemset(b->result, 0, sizeof(unsigned long long)));
    return BTC_OK;
}

int btc_bcsr_get_result(const btc_bcsr_device* b, unsigned long long* out)
{
    if (!b || !b->result || !out) return BTC_E_INVAL;
    BTC_CUDA_TRY(cudaMemcpy(out, b->result, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return BTC_OK;
}

}  // extern "C"

// Per-device count scratch for the struct surface, whose calls are blocking; a mutex
// serialises them.
namespace {
struct StructScratch {
    std::mutex mu;
    DevBuf partials[64];
    DevBuf done[64];
};
StructScratch& struct_scratch()
{
    static StructScratch s;
    return s;
}
}  // namespace

static int count_struct(btc_bcsr_device* b, int tile_cols, float* kernel_ms,
                        unsigned long long* out)
{
    if (!b || !b->result || !out) return BTC_E_INVAL;
    if (b->num_blocks && (!b->indptr || !b->indices || !b->blocks || !b->row_indices))
        return BTC_E_INVAL;
    int dev = 0;
    BTC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return BTC_E_INVAL;
    StructScratch& ss = struct_scratch();
    std::lock_guard<std::mutex> lock(ss.mu);
    const size_t need = sizeof(unsigned long long) * (size_t)count_grid_size(tile_cols);
    if (ss.partials[dev].bytes < need) BTC_TRY(ss.partials[dev].reserve(need));
    if (!ss.done[dev].ptr) {
        BTC_TRY(ss.done[dev].reserve(kCountCtlBytes));
        BTC_CUDA_TRY(cudaMemset(ss.done[dev].ptr, 0, kCountCtlBytes));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernel_ms) {
        BTC_CUDA_TRY(cudaEventCreate(&e0));
        BTC_CUDA_TRY(cudaEventCreate(&e1));
        BTC_CUDA_TRY(cudaEventRecord(e0, nullptr));
    }
    CountScratch scr{ss.partials[dev].as<unsigned long long>(), ss.done[dev].as<unsigned int>(),
                     reinterpret_cast<unsigned long long*>(ss.done[dev].as<char>() + 8), b->result,
                     nullptr};
    int st = launch_count(tile_cols, b->indptr, b->indices, b->row_indices, b->blocks, b->num_blocks,
                          b->n_row_blocks, default_tau(tile_cols), scr, nullptr);
    if (st == BTC_OK && kernel_ms && cudaEventRecord(e1, nullptr) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK && cudaMemcpy(out, b->result, sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost) != cudaSuccess)
        st = BTC_E_CUDA;
    if (st == BTC_OK && kernel_ms) cudaEventElapsedTime(kernel_ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return st;
}

extern "C" int btc_count_triangles_16x128_adaptive(btc_bcsr_device* b, int threshold_blocks,
                                                   float* kernel_ms, unsigned long long* out)
{
    (void)threshold_blocks;
    return count_struct(b, 128, kernel_ms, out);
}

extern "C" int btc_count_triangles_16x32_adaptive(btc_bcsr_device* b, int threshold_blocks,
                                                  float* kernel_ms, unsigned long long* out)
{
    (void)threshold_blocks;
    return count_struct(b, 32, kernel_ms, out);
}
