// batch.cu -- many graphs in one build and one persistent count launch.
//
// A batch is the block-diagonal union of its graphs: graph g's local vertex v becomes
// global vertex V_g + v with V_g = 16 * (row blocks of graphs 0..g-1), so every row block
// belongs to exactly one graph and no tile holds edges of two graphs.  The union's
// Bit-BSR is the reference layout and the count kernel runs on it unchanged; it adds each
// tile's sum to the graph owning the tile's row block (k_count's graph attribution).
//
// The cell bitmap is segmented: graph g has its own R_g x ceil(ncb_g/32)-word grid over
// the column blocks its vertices touch, so the bitmap grows with the sum of the graphs'
// squared sizes, not with the square of the batch's total vertex count.  Build passes are
// those of bitmap.cu (mark, count, scan, emit, fill), with the graph of an edge found by
// a binary search over the edge offsets and the graph of a bitmap word by a search over
// the segment offsets.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "handle.cuh"

namespace btc200 {

namespace bt {

constexpr int kThreads = 256;
constexpr int kWordsPerThread = 16;
constexpr int kChunk = kThreads * kWordsPerThread;

// last g in [0, G) with off[g] <= x (off[0] == 0; equal offsets are empty graphs)
template <class T>
__device__ __forceinline__ uint32_t last_le(const T* __restrict__ off, uint32_t G, T x)
{
    uint32_t lo = 0, hi = G;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Orients edge i of its graph to local (r, c), r > c.  false: self-loop or bad id.
__device__ __forceinline__ bool local_edge(const int32_t* __restrict__ src,
                                           const int32_t* __restrict__ dst, int64_t i,
                                           const GraphSeg& s, uint32_t& r, uint32_t& c, bool& bad)
{
    const int32_t u = src[i], v = dst[i];
    bad = (u < 0) | (v < 0) | (u >= s.n) | (v >= s.n);
    if (bad || u == v) return false;
    r = (uint32_t)max(u, v);
    c = (uint32_t)min(u, v);
    return true;
}

template <int LOG2C>
__device__ __forceinline__ uint64_t cell_word(const GraphSeg& s, uint32_t r, uint32_t c,
                                              uint32_t& bit)
{
    const uint32_t cb = ((s.vbase + c) >> LOG2C) - s.cb_lo;
    bit = 1u << (cb & 31u);
    return s.bm_off + (uint64_t)(r >> 4) * s.wpr + (cb >> 5);
}

template <int LOG2C>
__global__ void __launch_bounds__(kThreads)
k_mark_b(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t m,
         const GraphSeg* __restrict__ segs, const int64_t* __restrict__ e_off, uint32_t G,
         uint32_t* bitmap, unsigned long long* __restrict__ bad_count)
{
    uint32_t nbad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const GraphSeg s = segs[last_le<int64_t>(e_off, G, i)];
        uint32_t r, c, bit;
        bool bad;
        if (local_edge(src, dst, i, s, r, c, bad)) {
            const uint64_t w = cell_word<LOG2C>(s, r, c, bit);
            if (!(bitmap[w] & bit)) atomicOr(&bitmap[w], bit);
        }
        nbad += bad;
    }
    nbad = __reduce_add_sync(kFull, nbad);
    if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(bad_count, (unsigned long long)nbad);
}

__global__ void __launch_bounds__(kThreads)
k_emit_b(const uint32_t* __restrict__ bitmap, uint64_t W, const GraphSeg* __restrict__ segs,
         const uint64_t* __restrict__ bm_off, uint32_t G, const uint32_t* __restrict__ chunk_base,
         uint2* __restrict__ cellpp, uint32_t* __restrict__ indices,
         uint32_t* __restrict__ row_indices, uint32_t* __restrict__ indptr,
         const unsigned long long* __restrict__ tiles, uint32_t cap, uint4* __restrict__ blocks,
         uint32_t tile_vec4)
{
    __shared__ uint32_t s_warp[kThreads / kWarp];
    const unsigned long long T = *tiles;
    if (T > cap) return;  // more tiles than the arrays hold: nothing is built
    {
        // zero this chunk's tiles before k_fill_b ORs bits into them
        const uint64_t tb = chunk_base[blockIdx.x];
        const uint64_t te = blockIdx.x + 1 < gridDim.x ? chunk_base[blockIdx.x + 1] : T;
        for (uint64_t i = tb * tile_vec4 + threadIdx.x; i < te * tile_vec4; i += kThreads)
            blocks[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t w0 = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kWordsPerThread;
    uint32_t x[kWordsPerThread];
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) x[k] = (w0 + k < W) ? bitmap[w0 + k] : 0u;
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) mine += __popc(x[k]);
    uint32_t incl = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, d);
        if (lane >= d) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t base = chunk_base[blockIdx.x] + incl - mine;
#pragma unroll
    for (int w = 0; w < kThreads / kWarp; ++w) base += (w < warp) ? s_warp[w] : 0u;
    if (w0 >= W) return;

    uint32_t g = last_le<uint64_t>(bm_off, G, w0);
    GraphSeg s = segs[g];
    uint64_t lw = w0 - s.bm_off;
    uint32_t rb = (uint32_t)(lw / s.wpr);
    uint32_t cw = (uint32_t)(lw - (uint64_t)rb * s.wpr);
    for (int k = 0; k < kWordsPerThread; ++k) {
        const uint64_t w = w0 + k;
        if (w >= W) break;
        while (w >= bm_off[g + 1]) {  // next non-empty graph
            ++g;
            s = segs[g];
            rb = 0;
            cw = 0;
        }
        cellpp[w] = make_uint2(x[k], base);
        if (cw == 0) indptr[s.row_off + rb] = base;
        uint32_t bits = x[k];
        while (bits) {
            const uint32_t b = __ffs(bits) - 1;
            bits &= bits - 1;
            indices[base] = s.cb_lo + cw * 32 + b;
            row_indices[base] = s.row_off + rb;
            ++base;
        }
        if (++cw == s.wpr) {
            cw = 0;
            ++rb;
        }
    }
}

template <int LOG2C>
__global__ void __launch_bounds__(kThreads)
k_fill_b(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t m,
         const GraphSeg* __restrict__ segs, const int64_t* __restrict__ e_off, uint32_t G,
         const uint2* __restrict__ cellpp, uint32_t* __restrict__ blocks,
         const unsigned long long* __restrict__ tiles, uint32_t cap)
{
    if (*tiles > cap) return;  // nothing was emitted
    constexpr int C = 1 << LOG2C;
    constexpr int WPR = C / 32;
    constexpr int TW = 16 * WPR;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const GraphSeg s = segs[last_le<int64_t>(e_off, G, i)];
        uint32_t r, c, bit;
        bool bad;
        if (!local_edge(src, dst, i, s, r, c, bad)) continue;
        const uint64_t w = cell_word<LOG2C>(s, r, c, bit);
        const uint2 cp = cellpp[w];
        const uint32_t t = cp.y + __popc(cp.x & (bit - 1u));
        const uint32_t cl = (s.vbase + c) & (C - 1);
        atomicOr(&blocks[(size_t)t * TW + (r & 15u) * WPR + (cl >> 5)], 1u << (cl & 31u));
    }
}

__global__ void k_set_last_b(uint32_t* __restrict__ indptr, uint32_t R,
                             unsigned long long* __restrict__ meta, uint32_t cap)
{
    const unsigned long long T = meta[kMetaTiles];
    indptr[R] = (uint32_t)T;
    meta[kMetaOverflow] = T > cap ? 1ull : 0ull;
}

}  // namespace bt

int grid_for(int64_t work, int threads);
int launch_tile_scan(uint32_t* per_tile, uint32_t ntiles, unsigned long long* total, cudaStream_t s);
int launch_bitmap_count(const uint32_t* bitmap, uint64_t W, uint32_t* chunk_count, cudaStream_t s);

}  // namespace btc200

using namespace btc200;

struct btc_batch {
    btc_bitbsr g;  // the union graph's Bit-BSR, workspace and count scratch
    int32_t num_graphs = 0;
    DevBuf segs, e_off, bm_off, row_off, counts;
    std::vector<GraphSeg> h_segs;
    std::vector<int64_t> h_eoff;
    std::vector<uint64_t> h_bmoff;
    std::vector<uint32_t> h_rowoff;
    std::vector<int32_t> h_nv;
    bool built = false;        // the geometry above belongs to a build that succeeded
    bool row_index = false;    // the builds enqueue the row index (row-wise count)
    bool pending = false;      // an enqueued rebuild's status is not known yet
    uint32_t pending_cap = 0;  // the tile capacity that rebuild ran against
    cudaStream_t pending_stream = nullptr;
    void release()
    {
        g.release_all();
        segs.release();
        e_off.release();
        bm_off.release();
        row_off.release();
        counts.release();
        built = pending = false;
    }
};

// Waits for an enqueued rebuild's metadata and returns its status: BTC_E_RANGE for an
// out-of-range id, BTC_E_CAPACITY for more tiles than the arrays held (nothing built),
// BTC_OK (the tile count is then known).
static int batch_resolve(btc_batch* b)
{
    if (!b->pending) return BTC_OK;
    b->pending = false;
    btc_bitbsr* g = &b->g;
    unsigned long long* meta = g->meta.as<unsigned long long>();
    BTC_CUDA_TRY(cudaMemcpyAsync(g->h_meta, meta, sizeof(unsigned long long) * kMetaSlots,
                                 cudaMemcpyDeviceToHost, b->pending_stream));
    BTC_CUDA_TRY(cudaStreamSynchronize(b->pending_stream));
    if (g->h_meta[kMetaBad] != 0) {
        b->built = false;
        return BTC_E_RANGE;
    }
    if (g->h_meta[kMetaOverflow] != 0) {
        b->built = false;
        return BTC_E_CAPACITY;
    }
    g->num_tiles = (uint32_t)g->h_meta[kMetaTiles];
    return BTC_OK;
}

// Tiles the batch's arrays hold room for.
static uint32_t batch_capacity(const btc_batch* b)
{
    const btc_bitbsr* g = &b->g;
    const size_t TW = (size_t)16 * (g->tile_cols / 32);
    uint64_t c = g->indices.bytes / 4;
    c = std::min<uint64_t>(c, g->row_indices.bytes / 4);
    c = std::min<uint64_t>(c, g->blocks.bytes / (4 * TW));
    c = std::min<uint64_t>(c, g->rowmask.bytes / 4);
    return (uint32_t)std::min<uint64_t>(c, 0xffffffffull);
}

// The build after the tile count: emit (indices, row_indices, indptr, the (cell word, tile
// prefix) pairs, the tiles zeroed), fill, row masks and, when reserved, the row index of
// the row-wise count (built on the device when the union averages 8 or more tiles per row
// block) -- all against `cap` tiles, the device tile count deciding (more than cap:
// nothing is built and the overflow flag is set).
static int batch_enqueue_tiles(btc_batch* b, const int32_t* d_src, const int32_t* d_dst, int64_t m,
                               uint32_t cap, cudaStream_t s)
{
    btc_bitbsr* g = &b->g;
    unsigned long long* meta = g->meta.as<unsigned long long>();
    const uint64_t words = b->h_bmoff[(size_t)b->num_graphs];
    const size_t chunks = (size_t)((words + bt::kChunk - 1) / bt::kChunk);
    const GraphSeg* dsegs = b->segs.as<GraphSeg>();
    const int64_t* deoff = b->e_off.as<int64_t>();
    const uint32_t G = (uint32_t)b->num_graphs;
    const uint32_t rows = (uint32_t)g->n_row_blocks;
    const uint32_t vec4 = 4u * (uint32_t)(g->tile_cols / 32);
    if (words)
        bt::k_emit_b<<<(unsigned)chunks, bt::kThreads, 0, s>>>(
            g->bitmap.as<uint32_t>(), words, dsegs, b->bm_off.as<uint64_t>(), G,
            g->tile_base.as<uint32_t>(), g->prefix.as<uint2>(), g->indices.as<uint32_t>(),
            g->row_indices.as<uint32_t>(), g->indptr.as<uint32_t>(), meta + kMetaTiles, cap,
            g->blocks.as<uint4>(), vec4);
    bt::k_set_last_b<<<1, 1, 0, s>>>(g->indptr.as<uint32_t>(), rows, meta, cap);
    if (m > 0 && words) {
        const int egrid = grid_for((m + 3) / 4, bt::kThreads);
        if (g->tile_cols == 128)
            bt::k_fill_b<7><<<egrid, bt::kThreads, 0, s>>>(d_src, d_dst, m, dsegs, deoff, G,
                                                           g->prefix.as<uint2>(), g->blocks.as<uint32_t>(),
                                                           meta + kMetaTiles, cap);
        else
            bt::k_fill_b<5><<<egrid, bt::kThreads, 0, s>>>(d_src, d_dst, m, dsegs, deoff, G,
                                                           g->prefix.as<uint2>(), g->blocks.as<uint32_t>(),
                                                           meta + kMetaTiles, cap);
    }
    BTC_TRY(launch_rowmask(g->tile_cols, g->blocks.as<uint32_t>(), cap, meta + kMetaTiles,
                           g->indptr.as<uint32_t>(), g->n_row_blocks, g->rowmask.as<uint32_t>(),
                           meta + kMetaRowMax, s));
    if (b->row_index) {
        unsigned long long* total = g->row_bsum.as<unsigned long long>();
        BTC_TRY(launch_rowindex(g->indptr.as<uint32_t>(), g->indices.as<uint32_t>(), g->n_row_blocks,
                                g->rowmask.as<uint32_t>(), meta + kMetaTiles, cap,
                                g->row_tot.as<uint32_t>(), reinterpret_cast<uint32_t*>(total + 1), total,
                                g->row_off.as<uint32_t>(), g->row_ent.as<uint2>(),
                                g->row_ent.bytes / sizeof(uint2), s));
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

// Mark and count: the cell bitmap of every graph and the tile count (meta[kMetaTiles]).
static int batch_enqueue_mark(btc_batch* b, const int32_t* d_src, const int32_t* d_dst, int64_t m,
                              cudaStream_t s)
{
    btc_bitbsr* g = &b->g;
    unsigned long long* meta = g->meta.as<unsigned long long>();
    const uint64_t words = b->h_bmoff[(size_t)b->num_graphs];
    const size_t chunks = (size_t)((words + bt::kChunk - 1) / bt::kChunk);
    BTC_CUDA_TRY(cudaMemsetAsync(meta, 0, sizeof(unsigned long long) * kMetaSlots, s));
    if (!words) return BTC_OK;
    BTC_CUDA_TRY(cudaMemsetAsync(g->bitmap.ptr, 0, sizeof(uint32_t) * words, s));
    if (m > 0) {
        const int egrid = grid_for((m + 3) / 4, bt::kThreads);
        if (g->tile_cols == 128)
            bt::k_mark_b<7><<<egrid, bt::kThreads, 0, s>>>(d_src, d_dst, m, b->segs.as<GraphSeg>(),
                                                           b->e_off.as<int64_t>(), (uint32_t)b->num_graphs,
                                                           g->bitmap.as<uint32_t>(), meta + kMetaBad);
        else
            bt::k_mark_b<5><<<egrid, bt::kThreads, 0, s>>>(d_src, d_dst, m, b->segs.as<GraphSeg>(),
                                                           b->e_off.as<int64_t>(), (uint32_t)b->num_graphs,
                                                           g->bitmap.as<uint32_t>(), meta + kMetaBad);
    }
    BTC_TRY(launch_bitmap_count(g->bitmap.as<uint32_t>(), words, g->tile_base.as<uint32_t>(), s));
    BTC_TRY(launch_tile_scan(g->tile_base.as<uint32_t>(), (uint32_t)chunks, meta + kMetaTiles, s));
    return BTC_OK;
}

static int batch_build_into(btc_batch* b, const int32_t* src, const int32_t* dst,
                            const int64_t* edge_offsets, const int32_t* num_vertices, int32_t G,
                            int tile_cols, uint32_t flags, cudaStream_t s)
{
    if (G < 1 || !edge_offsets || !num_vertices) return BTC_E_INVAL;
    if (flags & ~(BTC_INPUT_ON_HOST | BTC_BUILD_ASYNC)) return BTC_E_INVAL;
    const int64_t m = edge_offsets[G];
    if (edge_offsets[0] != 0 || m < 0 || (uint64_t)m > (1ull << 32) - (uint64_t)kSortTile)
        return BTC_E_INVAL;
    if (m > 0 && (!src || !dst)) return BTC_E_INVAL;
    int64_t n_sum = 0;
    for (int32_t i = 0; i < G; ++i) {
        if (num_vertices[i] < 0 || edge_offsets[i + 1] < edge_offsets[i]) return BTC_E_INVAL;
        n_sum += num_vertices[i];
    }
    btc_bitbsr* g = &b->g;

    // ---- an enqueued rebuild: same graphs' sizes, device input, room for the tiles ------
    // (no host work, no allocation, no wait: the tile count stays on the device)
    // (a previous enqueued rebuild still pending is superseded: its status is not kept)
    const bool same_geometry =
        b->built && G == b->num_graphs &&
        (tile_cols == 0 || tile_cols == g->tile_cols) &&
        std::equal(edge_offsets, edge_offsets + G + 1, b->h_eoff.begin()) &&
        std::equal(num_vertices, num_vertices + G, b->h_nv.begin());
    if ((flags & BTC_BUILD_ASYNC) && !(flags & BTC_INPUT_ON_HOST) && same_geometry) {
        const uint32_t cap = batch_capacity(b);
        BTC_TRY(batch_enqueue_mark(b, src, dst, m, s));
        BTC_TRY(batch_enqueue_tiles(b, src, dst, m, cap, s));
        b->pending = true;
        b->pending_cap = cap;
        b->pending_stream = s;
        return BTC_OK;
    }
    if (b->pending) batch_resolve(b);  // an enqueued build still owns the buffers
    b->built = false;

    if (tile_cols == 0) {
        // the engine's tile policy over the whole batch (policy.cu), each sampled edge's
        // locality measured against its own graph's size
        double L = 0.0;
        if (flags & BTC_INPUT_ON_HOST) {
            BTC_TRY(policy_locality(src, dst, m, 0, true, edge_offsets, num_vertices, (uint32_t)G, s, &L));
        } else if (m > 0) {
            DevBuf tmp;
            const size_t eb = sizeof(int64_t) * ((size_t)G + 1), nb = sizeof(int32_t) * (size_t)G;
            int st = tmp.reserve(eb + nb);
            if (st == BTC_OK && (cudaMemcpyAsync(tmp.ptr, edge_offsets, eb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                                 cudaMemcpyAsync(tmp.as<char>() + eb, num_vertices, nb, cudaMemcpyHostToDevice, s) != cudaSuccess))
                st = BTC_E_CUDA;
            if (st == BTC_OK)
                st = policy_locality(src, dst, m, 0, false, tmp.as<int64_t>(),
                                     reinterpret_cast<const int32_t*>(tmp.as<char>() + eb), (uint32_t)G, s, &L);
            tmp.release();
            BTC_TRY(st);
        }
        BTC_TRY(btc_tile_policy_from_features(m, (int32_t)(n_sum > 0x7fffffff ? 0x7fffffff : n_sum), 0, L,
                                              &tile_cols, nullptr));
    }
    if (tile_cols != 32 && tile_cols != 128) return BTC_E_INVAL;
    const int log2c = tile_cols == 128 ? 7 : 5;

    // ---- host geometry ----------------------------------------------------------
    b->num_graphs = G;
    b->h_segs.resize((size_t)G);
    b->h_eoff.assign(edge_offsets, edge_offsets + G + 1);
    b->h_nv.assign(num_vertices, num_vertices + G);
    b->h_bmoff.resize((size_t)G + 1);
    b->h_rowoff.resize((size_t)G + 1);
    uint64_t rows = 0, words = 0;
    for (int32_t i = 0; i < G; ++i) {
        GraphSeg& sg = b->h_segs[(size_t)i];
        const uint64_t Ri = ((uint64_t)num_vertices[i] + 15) / 16;
        sg.row_off = (uint32_t)rows;
        sg.n = num_vertices[i];
        sg.vbase = (uint32_t)(rows * 16);
        sg.cb_lo = (uint32_t)((rows * 16) >> log2c);
        const uint64_t hi = num_vertices[i] > 0 ? ((rows * 16 + num_vertices[i] - 1) >> log2c) : sg.cb_lo;
        const uint64_t ncb = hi - sg.cb_lo + 1;
        sg.wpr = (uint32_t)((ncb + 31) / 32);
        sg.pad = 0;
        sg.bm_off = words;
        b->h_rowoff[(size_t)i] = (uint32_t)rows;
        b->h_bmoff[(size_t)i] = words;
        rows += Ri;
        words += Ri * sg.wpr;
        if (rows * 16 > 0x7fffffffull) return BTC_E_INVAL;
    }
    b->h_rowoff[(size_t)G] = (uint32_t)rows;
    b->h_bmoff[(size_t)G] = words;
    if (words * 8 > (4ull << 30)) return BTC_E_INVAL;  // cell words: at most 512M (bitmap + pairs 6 GB)

    BTC_CUDA_TRY(cudaGetDevice(&g->device));
    g->tile_cols = tile_cols;
    g->n = (int32_t)(rows * 16);
    g->n_row_blocks = (int32_t)rows;
    g->input_edges = m;
    g->edges_known = false;
    if (!g->h_meta) {
        void* p = nullptr;
        if (cudaMallocHost(&p, sizeof(unsigned long long) * kMetaSlots) != cudaSuccess) {
            cudaGetLastError();
            return BTC_E_NOMEM;
        }
        g->h_meta = static_cast<unsigned long long*>(p);
    }
    BTC_TRY(g->meta.reserve(sizeof(unsigned long long) * kMetaSlots));
    unsigned long long* meta = g->meta.as<unsigned long long>();

    BTC_TRY(b->segs.reserve(sizeof(GraphSeg) * (size_t)G));
    BTC_TRY(b->e_off.reserve(sizeof(int64_t) * ((size_t)G + 1)));
    BTC_TRY(b->bm_off.reserve(sizeof(uint64_t) * ((size_t)G + 1)));
    BTC_TRY(b->row_off.reserve(sizeof(uint32_t) * ((size_t)G + 1)));
    // pageable sources: the copies are staged before cudaMemcpyAsync returns
    BTC_CUDA_TRY(cudaMemcpyAsync(b->segs.ptr, b->h_segs.data(), sizeof(GraphSeg) * (size_t)G,
                                 cudaMemcpyHostToDevice, s));
    BTC_CUDA_TRY(cudaMemcpyAsync(b->e_off.ptr, b->h_eoff.data(), sizeof(int64_t) * ((size_t)G + 1),
                                 cudaMemcpyHostToDevice, s));
    BTC_CUDA_TRY(cudaMemcpyAsync(b->bm_off.ptr, b->h_bmoff.data(),
                                 sizeof(uint64_t) * ((size_t)G + 1), cudaMemcpyHostToDevice, s));
    BTC_CUDA_TRY(cudaMemcpyAsync(b->row_off.ptr, b->h_rowoff.data(),
                                 sizeof(uint32_t) * ((size_t)G + 1), cudaMemcpyHostToDevice, s));

    const int32_t* d_src = src;
    const int32_t* d_dst = dst;
    if ((flags & BTC_INPUT_ON_HOST) && m > 0) {
        BTC_TRY(g->in_src.reserve(sizeof(int32_t) * (size_t)m));
        BTC_TRY(g->in_dst.reserve(sizeof(int32_t) * (size_t)m));
        BTC_CUDA_TRY(cudaMemcpyAsync(g->in_src.ptr, src, sizeof(int32_t) * (size_t)m,
                                     cudaMemcpyHostToDevice, s));
        BTC_CUDA_TRY(cudaMemcpyAsync(g->in_dst.ptr, dst, sizeof(int32_t) * (size_t)m,
                                     cudaMemcpyHostToDevice, s));
        d_src = g->in_src.as<int32_t>();
        d_dst = g->in_dst.as<int32_t>();
    }

    // ---- mark, count, scan; the tile count to size the arrays ----------------------
    const size_t chunks = (size_t)((words + bt::kChunk - 1) / bt::kChunk);
    BTC_TRY(g->bitmap.reserve(sizeof(uint32_t) * (words ? words : 1)));
    BTC_TRY(g->prefix.reserve(sizeof(uint2) * (words ? words : 1)));
    BTC_TRY(g->tile_base.reserve(sizeof(uint32_t) * (chunks + 1)));
    BTC_TRY(batch_enqueue_mark(b, d_src, d_dst, m, s));
    if (!words && m > 0) return BTC_E_RANGE;  // only empty graphs: every edge is out of range
    BTC_CUDA_TRY(cudaMemcpyAsync(g->h_meta, meta, sizeof(unsigned long long) * 3,
                                 cudaMemcpyDeviceToHost, s));
    BTC_CUDA_TRY(cudaStreamSynchronize(s));
    if (g->h_meta[kMetaBad] != 0) return BTC_E_RANGE;
    const unsigned long long tiles = g->h_meta[kMetaTiles];
    if (tiles > 0xffffffffull) return BTC_E_INVAL;
    g->num_tiles = (uint32_t)tiles;

    // ---- tiles ------------------------------------------------------------------
    const size_t TW = (size_t)16 * (tile_cols / 32);
    BTC_TRY(g->indptr.reserve(sizeof(uint32_t) * ((size_t)rows + 1)));
    BTC_TRY(g->indices.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    BTC_TRY(g->row_indices.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    BTC_TRY(g->blocks.reserve(sizeof(uint32_t) * TW * (tiles ? tiles : 1)));
    BTC_TRY(g->rowmask.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    // the row-wise count's row index, when the union averages 8 or more tiles per row
    // block (then it has at least 8 edges per row block)
    b->row_index = rows > 0 && (uint64_t)tiles >= 8ull * rows && m < (int64_t)0xffffffffll;
    if (b->row_index) {
        BTC_TRY(g->row_off.reserve(sizeof(uint32_t) * (16 * (size_t)rows + 1)));
        BTC_TRY(g->row_ent.reserve(sizeof(uint2) * (size_t)m));
        BTC_TRY(g->row_tot.reserve(sizeof(uint32_t) * (size_t)rows));
        BTC_TRY(g->row_bsum.reserve(sizeof(unsigned long long) +
                                    sizeof(uint32_t) * ((size_t)ri_scan_blocks((uint32_t)rows) + 1)));
    }
    BTC_TRY(ensure_count_scratch(g));
    BTC_TRY(b->counts.reserve(sizeof(unsigned long long) * (size_t)G));
    BTC_TRY(batch_enqueue_tiles(b, d_src, d_dst, m, (uint32_t)tiles, s));
    b->built = true;
    return BTC_OK;
}

namespace btc200 {
size_t batch_device_bytes(const btc_batch* b)
{
    return b->g.device_bytes() + b->segs.bytes + b->e_off.bytes + b->bm_off.bytes +
           b->row_off.bytes + b->counts.bytes;
}
}  // namespace btc200

namespace btc200 {
// An empty batch whose allocations are all stream-ordered on `s` from `pool` (see
// bitbsr_new_pooled); its first (re)build sizes it.
btc_batch* batch_new_pooled(cudaMemPool_t pool, cudaStream_t s)
{
    btc_batch* b = new (std::nothrow) btc_batch();
    if (!b) return nullptr;
    b->g.set_pool(pool, s);
    for (DevBuf* d : {&b->segs, &b->e_off, &b->bm_off, &b->row_off, &b->counts}) {
        d->pool = pool;
        d->stream = s;
    }
    return b;
}
}  // namespace btc200

extern "C" {

int btc_batch_build(const int32_t* src, const int32_t* dst, const int64_t* edge_offsets,
                    const int32_t* num_vertices, int32_t num_graphs, int tile_cols, uint32_t flags,
                    btc_stream_t stream, btc_batch** out)
{
    if (!out) return BTC_E_INVAL;
    *out = nullptr;
    btc_batch* b = new (std::nothrow) btc_batch();
    if (!b) return BTC_E_NOMEM;
    const int st = batch_build_into(b, src, dst, edge_offsets, num_vertices, num_graphs, tile_cols,
                                    flags, stream);
    if (st != BTC_OK) {
        b->release();
        delete b;
        return st;
    }
    *out = b;
    return BTC_OK;
}

int btc_batch_rebuild(btc_batch* b, const int32_t* src, const int32_t* dst,
                      const int64_t* edge_offsets, const int32_t* num_vertices, int32_t num_graphs,
                      int tile_cols, uint32_t flags, btc_stream_t stream)
{
    if (!b) return BTC_E_INVAL;
    return batch_build_into(b, src, dst, edge_offsets, num_vertices, num_graphs, tile_cols, flags,
                            stream);
}

int btc_batch_count(btc_batch* b, int tau, btc_stream_t stream, unsigned long long* d_counts,
                    unsigned long long* h_counts)
{
    if (!b) return BTC_E_INVAL;
    btc_bitbsr* g = &b->g;
    if (tau == BTC_TAU_DEFAULT) tau = default_tau(g->tile_cols);
    if (tau < 0) return BTC_E_INVAL;
    BTC_TRY(ensure_count_scratch(g));
    if (!b->built && !b->pending) return BTC_E_INVAL;  // the last build failed
    unsigned long long* counts = d_counts ? d_counts : b->counts.as<unsigned long long>();
    const size_t bytes = sizeof(unsigned long long) * (size_t)b->num_graphs;
    BTC_CUDA_TRY(cudaMemsetAsync(counts, 0, bytes, stream));
    CountScratch scr{g->partials.as<unsigned long long>(), g->done.as<unsigned int>(),
                     reinterpret_cast<unsigned long long*>(g->done.as<char>() + 8),
                     g->result.as<unsigned long long>(), nullptr};
    // after an enqueued rebuild the kernel reads the tile count (and the build's status)
    // from the device, within the capacity; the schedule follows the previous count
    const unsigned long long* build_meta = b->pending ? g->meta.as<unsigned long long>() : nullptr;
    BTC_TRY(launch_count(g->tile_cols, g->indptr.as<uint32_t>(), g->indices.as<uint32_t>(),
                         g->row_indices.as<uint32_t>(), g->blocks.as<uint32_t>(),
                         b->pending ? b->pending_cap : g->num_tiles, g->n_row_blocks, tau, scr,
                         stream, b->row_off.as<uint32_t>(), (uint32_t)b->num_graphs, counts,
                         g->rowmask.as<uint32_t>(), g->prefix.as<uint2>(), 0,
                         g->meta.as<unsigned long long>() + kMetaRowMax, 0, 0xffffffffu, build_meta,
                         g->num_tiles,
                         b->row_index ? g->row_off.as<uint32_t>() : nullptr,
                         b->row_index ? g->row_ent.as<uint2>() : nullptr, false,
                         b->segs.as<GraphSeg>()));
    if (h_counts) {
        BTC_CUDA_TRY(cudaMemcpyAsync(h_counts, counts, bytes, cudaMemcpyDeviceToHost, stream));
        BTC_CUDA_TRY(cudaStreamSynchronize(stream));
        return batch_resolve(b);  // an enqueued rebuild's failure shows here
    }
    return BTC_OK;
}

int btc_batch_info(btc_batch* b, btc_bitbsr_view* v)
{
    if (!b) return BTC_E_INVAL;
    BTC_TRY(batch_resolve(b));
    return btc_bitbsr_info(&b->g, v);
}

int btc_batch_row_offsets(const btc_batch* b, uint32_t* row_offsets)
{
    if (!b || !row_offsets) return BTC_E_INVAL;
    std::memcpy(row_offsets, b->h_rowoff.data(), sizeof(uint32_t) * ((size_t)b->num_graphs + 1));
    return BTC_OK;
}

void btc_batch_free(btc_batch* b)
{
    if (!b) return;
    b->release();
    delete b;
}

}  // extern "C"
