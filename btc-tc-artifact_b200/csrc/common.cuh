// common.cuh -- shared definitions for the engine's CUDA sources (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "btc_c.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "this engine is written for sm_100a (B200) only"
#endif

namespace btc200 {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Status propagation for host code: evaluate a CUDA call, map failure to BTC_E_CUDA
// (or BTC_E_NOMEM for allocation failures) and return from the enclosing function.
#define BTC_CUDA_TRY(expr)                                                      \
    do {                                                                        \
        cudaError_t _e = (expr);                                                \
        if (_e != cudaSuccess) {                                                \
            ::btc200::note_cuda_error(_e, #expr, __FILE__, __LINE__);           \
            return _e == cudaErrorMemoryAllocation ? BTC_E_NOMEM : BTC_E_CUDA;  \
        }                                                                       \
    } while (0)

#define BTC_TRY(expr)                 \
    do {                              \
        int _s = (expr);              \
        if (_s != BTC_OK) return _s;  \
    } while (0)

void note_cuda_error(cudaError_t e, const char* what, const char* file, int line);

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__host__ __device__ __forceinline__ int bit_length_u64(uint64_t x)
{
#ifdef __CUDA_ARCH__
    return x ? 64 - __clzll((long long)x) : 0;
#else
    return x ? 64 - __builtin_clzll(x) : 0;
#endif
}

__host__ __device__ __forceinline__ int log2_exact(int x)
{
    int k = 0;
    while ((1 << k) < x) ++k;
    return k;
}

// A grow-only device buffer.  reserve() keeps contents only when no reallocation
// happens; callers treat it as scratch.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    // Stream-ordered allocation, for an owner that uses the buffer on one stream only:
    // with `pool` and `stream` set, a growth frees and allocates in that stream's order
    // (cudaFreeAsync / cudaMallocFromPoolAsync) instead of cudaFree's wait for the whole
    // device.  `pooled` records how the current allocation was made.
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    bool pooled = false;
    int reserve(size_t need)
    {
        if (need <= bytes && ptr) return BTC_OK;
        release();
        if (need == 0) return BTC_OK;
        size_t want = need + need / 8;  // headroom for slowly growing rebuilds
        if (allocate(want) != cudaSuccess) {
            cudaGetLastError();
            if (allocate(need) != cudaSuccess) {
                cudaGetLastError();
                ptr = nullptr;
                return BTC_E_NOMEM;
            }
            want = need;
        }
        bytes = want;
        return BTC_OK;
    }
    cudaError_t allocate(size_t b)
    {
        pooled = pool != nullptr && stream != nullptr;
        return pooled ? cudaMallocFromPoolAsync(&ptr, b, pool, stream) : cudaMalloc(&ptr, b);
    }
    void release()
    {
        if (ptr) {
            if (pooled) cudaFreeAsync(ptr, stream);
            else cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
    // zeroes the first n bytes, ordered with the buffer's stream when it has one
    cudaError_t zero(size_t n) const
    {
        return pooled ? cudaMemsetAsync(ptr, 0, n, stream) : cudaMemset(ptr, 0, n);
    }
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

// ---------------------------------------------------------------------------
// Sort (radix.cu)
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per CTA tile
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

inline size_t sort_tiles(size_t n) { return (n + kSortTile - 1) / kSortTile; }

// Scratch words needed by radix_sort_u64 for up to n keys.
size_t radix_scratch_words(size_t n);

// Stable LSD sort of keys[0, *d_count) by bits [lo_bit, hi_bit).  d_count lives in
// device memory (at most max_n); alt is a second buffer of max_n keys.  Returns the
// buffer holding the sorted keys (keys or alt).
uint64_t* radix_sort_u64(uint64_t* keys, uint64_t* alt, size_t max_n,
                         const unsigned long long* d_count, int lo_bit, int hi_bit,
                         uint32_t* scratch, cudaStream_t s, int* status);

// ---------------------------------------------------------------------------
// Build (build.cu)
// ---------------------------------------------------------------------------
struct BuildGeom {
    int32_t n;
    int tile_cols;      // C
    int log2c;          // log2(C)
    int payload_bits;   // 4 + log2(C): (row in tile, column in tile)
    int cb_bits;        // bits of the column-block id
    int t_bits;         // bits of the tile key (row block, column block)
    int32_t n_row_blocks;
    int64_t n_col_blocks;
};
BuildGeom make_geom(int32_t n, int tile_cols);

// ---------------------------------------------------------------------------
// Count (count.cu)
// ---------------------------------------------------------------------------
// One graph of a batch union: its rows, vertex ids and the part of the cell bitmap (and
// of the (cell word, tile prefix) pairs) that covers it.  The cell of union row block J and
// union column block K is word bm_off + (J - row_off) * wpr + ((K - cb_lo) >> 5), bit
// (K - cb_lo) & 31; a single graph is the one segment {0, n, 0, 0, words per row, 0, 0}.
struct GraphSeg {
    uint32_t row_off;  // first global row block
    int32_t n;         // vertices (local ids are in [0, n))
    uint32_t vbase;    // first global vertex id (16 * row_off)
    uint32_t cb_lo;    // first global column block of the graph's vertex range
    uint32_t wpr;      // bitmap words per row block
    uint32_t pad;
    uint64_t bm_off;   // first bitmap word of the graph
};

struct CountScratch {
    unsigned long long* partials;  // one per CTA of the persistent grid
    unsigned int* done;            // CTAs finished (reset to 0 by the last one)
    unsigned long long* work;      // tile queue head (reset to 0 by the last CTA)
    unsigned long long* result;    // where the final count lands
    unsigned long long* result2;   // optional second destination (nullable)
    // optional device alias of mapped pinned host memory that also receives the count
    // (written by the last CTA, no copy-engine hop)
    unsigned long long* result_host = nullptr;
};

int count_grid_size(int tile_cols);
// graph_rows / graph_counts (nullable): per-graph attribution for batches; graph g
// owns row blocks [graph_rows[g], graph_rows[g+1]) and its count is added to
// graph_counts[g] (which the caller zeroes).
int launch_count(int tile_cols, const uint32_t* indptr, const uint32_t* indices,
                 const uint32_t* row_indices, const uint32_t* blocks, uint32_t num_tiles,
                 int32_t n_row_blocks, int tau, CountScratch scr, cudaStream_t s,
                 const uint32_t* graph_rows = nullptr, uint32_t num_graphs = 0,
                 unsigned long long* graph_counts = nullptr, const uint32_t* rowmask = nullptr,
                 const uint2* cellpp = nullptr,
                 uint64_t cell_wpr = 0, const unsigned long long* row_max = nullptr,
                 uint32_t tile_begin = 0, uint32_t tile_end = 0xffffffffu,
                 const unsigned long long* build_meta = nullptr, uint32_t tiles_hint = 0,
                 const uint32_t* row_off = nullptr, const uint2* row_ent = nullptr,
                 bool dense_tiles = false, const GraphSeg* segs = nullptr);

// rowmask[t] bit r = tile t's row r has a bit, for t < T = *d_tiles (T = cap when d_tiles
// is null) when T >= 8 * n_row_blocks (the heavy count variant's condition), and
// *row_max = max(*row_max, the most tiles in one row block), which picks the count
// kernel's schedule (the caller zeroes it).  Runs after the tiles are filled.  Writes
// nothing when T > cap (the tile arrays overflowed).
// masks = false: only *row_max (the bitmap builder's fill pass sets the masks itself).
int launch_rowmask(int tile_cols, const uint32_t* blocks, uint32_t cap,
                   const unsigned long long* d_tiles, const uint32_t* indptr, int32_t n_row_blocks,
                   uint32_t* rowmask, unsigned long long* row_max, cudaStream_t s, bool masks = true);

// Row index of the row-wise count kernel (rowindex.cu): for vertex u, ent[off[u],
// off[u+1]) lists (column block, tile) of the tiles whose row u % 16 holds a bit, in tile
// order.  Built when the row masks are (T >= 8 * n_row_blocks, T = *d_tiles or cap);
// tot: n_row_blocks words, bsum: ri_scan_blocks(n_row_blocks) words, total: one uint64 of
// scratch; off: 16 * n_row_blocks + 1 words; ent: ent_cap entries (>= the unique edges).
uint32_t ri_scan_blocks(uint32_t n_row_blocks);
int launch_rowindex(const uint32_t* indptr, const uint32_t* indices, int32_t n_row_blocks,
                    const uint32_t* rowmask, const unsigned long long* d_tiles, uint32_t cap,
                    uint32_t* tot, uint32_t* bsum, unsigned long long* total, uint32_t* off,
                    uint2* ent, uint64_t ent_cap, cudaStream_t s);

// Id locality of an edge list for the tile policy (policy.cu): sampled share of edges
// with |u - v| < 128 over the share uniform ids would give.  e_off / nv (nullable): the
// batch layout, each edge measured against its own graph's vertex count.
int policy_locality(const int32_t* src, const int32_t* dst, int64_t m, int32_t n, bool on_host,
                    const int64_t* e_off, const int32_t* nv, uint32_t G, cudaStream_t s, double* L);

// Device metadata slots of a build (uint64 each): valid keys, out-of-range flag, tile
// count, unique edges, sort length, longest row-block list, tile-capacity overflow flag,
// and the chunk-scan ticket (CTAs of the chunk popcount that have finished).
enum {
    kMetaValid = 0,
    kMetaBad = 1,
    kMetaTiles = 2,
    kMetaUniq = 3,
    kMetaN = 4,
    kMetaRowMax = 5,
    kMetaOverflow = 6,
    kMetaTicket = 7,
    kMetaSlots = 8
};

// Queue/completion words of the count kernel: done (u32) at byte 0, work (u64) at 8.
constexpr size_t kCountCtlBytes = 16;

int device_sm_count();

}  // namespace btc200
