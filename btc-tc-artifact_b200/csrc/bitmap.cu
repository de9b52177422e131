// bitmap.cu -- sort-free Bit-BSR builder.
//
// The tiles of L are the cells (row block rb, column block cb) that hold at least
// one edge.  When the R x ceil(ncb/32) word grid of those cells is small enough, the
// builder marks every edge's cell in a presence bitmap and numbers the tiles by a
// popcount prefix over it; row-major cell order is exactly the reference's tile order
// (indices ascending within a row block, row blocks ascending).  Then:
//
//   k_mark       one pass over the edges: orient (max,min), range-check, drop
//                self-loops, set the cell bit (fire-and-forget atomicOr)
//   k_bm_count_scan  popcount per 4096-word chunk; the last CTA to finish scans the
//                chunk counts into chunk bases and the tile total
//   k_bm_emit    per word: exclusive tile prefix (kept for k_fill_bm), indices /
//                row_indices of each set cell, indptr at row-block starts; each CTA
//                zeroes its chunk's tiles, the last one writes indptr[R]
//   k_fill_bm    second pass over the edges: tile = prefix[word] + popc(lower bits of
//                the word); OR the edge's bit into the tile; where the count wants row
//                masks (8 or more tiles per row block), the edge whose OR finds its tile
//                word empty also sets its row's bit in the tile's row mask
//
// Two reads of the edge list, one read and one write of the bitmap and its prefix
// array (their lower-triangle words only: the rest can hold no cell and is never looked
// up), one write of the tiles: no sort.  Duplicate edges OR the same bit.
#include "common.cuh"

namespace btc200 {
namespace bm {

constexpr int kThreads = 256;
constexpr int kWordsPerThread = 16;
constexpr int kChunk = kThreads * kWordsPerThread;  // 4096 words per CTA

__device__ __forceinline__ bool orient(int32_t u, int32_t v, int32_t n, const int32_t* rank,
                                       uint32_t& r, uint32_t& c, bool& bad)
{
    bad = (u < 0) | (v < 0) | (u >= n) | (v >= n);
    if (bad) return false;
    if (rank) {
        u = rank[u];
        v = rank[v];
    }
    if (u == v) return false;
    r = (uint32_t)max(u, v);
    c = (uint32_t)min(u, v);
    return true;
}

// Every cell bit is hit by all edges of its tile, so the word is read first and the
// atomic is skipped when the bit is already set.  Bits only go from 0 to 1, so a
// stale read can only cost a redundant atomic, never a missing one.
template <int LOG2C>
__global__ void __launch_bounds__(kThreads)
k_mark(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t m, int32_t n,
       const int32_t* __restrict__ rank, uint64_t wpr, uint32_t* bitmap,
       unsigned long long* __restrict__ bad_count)
{
    constexpr int U = 8;  // edges in flight per thread
    uint32_t nbad = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < m; i0 += U * stride) {
        int32_t u[U], v[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const int64_t i = i0 + k * stride;
            u[k] = i < m ? src[i] : 0;
            v[k] = i < m ? dst[i] : 0;
        }
        uint64_t w[U];
        uint32_t bit[U];
        bool ok[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            uint32_t r = 0, c = 0;
            bool bad = false;
            ok[k] = (i0 + k * stride < m) && orient(u[k], v[k], n, rank, r, c, bad);
            nbad += bad && (i0 + k * stride < m);
            const uint32_t cb = c >> LOG2C;
            w[k] = (uint64_t)(r >> 4) * wpr + (cb >> 5);
            bit[k] = 1u << (cb & 31u);
        }
        uint32_t cur[U];
#pragma unroll
        for (int k = 0; k < U; ++k) cur[k] = ok[k] ? bitmap[w[k]] : 0xffffffffu;
#pragma unroll
        for (int k = 0; k < U; ++k)
            if (!(cur[k] & bit[k])) atomicOr(&bitmap[w[k]], bit[k]);
    }
    nbad = __reduce_add_sync(kFull, nbad);
    if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(bad_count, (unsigned long long)nbad);
}

// Per-thread view of 16 consecutive bitmap words.
template <int WPT>
__device__ __forceinline__ void load_words(const uint32_t* __restrict__ bitmap, uint64_t w0,
                                           uint64_t W, uint32_t (&x)[WPT])
{
    if constexpr (WPT % 4 == 0) {
        if (w0 + WPT <= W) {
            const uint4* p = reinterpret_cast<const uint4*>(bitmap + w0);
#pragma unroll
            for (int q = 0; q < WPT / 4; ++q) {
                const uint4 v = p[q];
                x[4 * q] = v.x;
                x[4 * q + 1] = v.y;
                x[4 * q + 2] = v.z;
                x[4 * q + 3] = v.w;
            }
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < WPT; ++k) x[k] = (w0 + k < W) ? bitmap[w0 + k] : 0u;
}

// Division of word indices by the words per row without a divide instruction: for
// n < 2^31 and d > 1, n / d = umulhi(n, m) >> s with l = ceil(log2 d), m = ceil(2^(31+l) / d)
// (< 2^32) and s = l - 1 (Granlund and Montgomery, "Division by invariant integers using
// multiplication", 1994, theorem 4.2 with N = 31); d = 1 is passed through.
struct RowDiv {
    uint32_t d, m, s;
};

inline RowDiv make_row_div(uint64_t d)
{
    RowDiv v{(uint32_t)d, 0u, 0u};
    if (d > 1) {
        uint32_t l = 0;
        while ((1ull << l) < d) ++l;
        v.m = (uint32_t)(((1ull << (31 + l)) + d - 1) / d);
        v.s = l - 1;
    }
    return v;
}

__device__ __forceinline__ uint32_t row_of(uint32_t n, RowDiv v)
{
    return v.d == 1 ? n : (__umulhi(n, v.m) >> v.s);
}

// Reading only the words that can hold a cell.  Edges are oriented (max, min), so row
// block rb's cells lie in column blocks <= (16 rb + 15) >> LOG2C and its words past
// (16 rb + 15) >> (LOG2C + 5) (lshift = LOG2C + 5) stay zero: about half of the bitmap,
// which the chunk popcount need not read and k_bm_emit need not give pairs, since no
// lookup lands there (a lookup of row block J, column block K always has K within J's
// lower triangle).  Bit k of the result: word w0 + k can hold a cell.  The builder takes
// this path only for bitmaps of at most 2^30 words (4 GiB), so word and row indices fit
// 31 bits.  The usual thread's WPT words lie in one row and take the short path; per-word
// arithmetic with a divide instruction made the chunk popcount slower than reading
// everything (341 against 292 us at R-MAT s22).
template <int WPT>
__device__ __forceinline__ uint32_t load_lower_words(const uint32_t* __restrict__ bitmap, uint64_t w0,
                                                     uint64_t W, RowDiv wpr, uint32_t lshift,
                                                     uint32_t (&x)[WPT])
{
    constexpr uint32_t kAll = WPT == 32 ? 0xFFFFFFFFu : (1u << WPT) - 1u;
    uint32_t rb = row_of((uint32_t)w0, wpr);
    uint32_t cw = (uint32_t)w0 - rb * wpr.d;
    uint32_t lim = (16u * rb + 15u) >> lshift;
    uint32_t need = 0;
    if (w0 + WPT <= W && cw + WPT <= wpr.d) {
        // one row: the words up to lim
        if (cw <= lim) need = lim - cw + 1u >= (uint32_t)WPT ? kAll : (1u << (lim - cw + 1u)) - 1u;
    } else {
#pragma unroll
        for (int k = 0; k < WPT; ++k) {
            if (w0 + k < W && cw <= lim) need |= 1u << k;
            if (++cw == wpr.d) {
                cw = 0;
                ++rb;
                lim = (16u * rb + 15u) >> lshift;
            }
        }
    }
    if constexpr (WPT % 4 == 0) {
        if (w0 + WPT <= W) {
            const uint4* p = reinterpret_cast<const uint4*>(bitmap + w0);
#pragma unroll
            for (int q = 0; q < WPT / 4; ++q) {
                const uint4 v = ((need >> (4 * q)) & 0xFu) ? p[q] : make_uint4(0u, 0u, 0u, 0u);
                x[4 * q] = v.x;
                x[4 * q + 1] = v.y;
                x[4 * q + 2] = v.z;
                x[4 * q + 3] = v.w;
            }
            return need;
        }
    }
#pragma unroll
    for (int k = 0; k < WPT; ++k) x[k] = ((need >> k) & 1u) ? bitmap[w0 + k] : 0u;
    return need;
}

__global__ void __launch_bounds__(kThreads)
k_bm_count(const uint32_t* __restrict__ bitmap, uint64_t W, uint32_t* __restrict__ chunk_count)
{
    __shared__ uint32_t s_warp[kThreads / kWarp];
    const uint64_t w0 = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kWordsPerThread;
    uint32_t x[kWordsPerThread];
    load_words<kWordsPerThread>(bitmap, w0, W, x);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) s += __popc(x[k]);
    s = __reduce_add_sync(kFull, s);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kThreads / kWarp; ++w) t += s_warp[w];
        chunk_count[blockIdx.x] = t;
    }
}

// Chunk popcounts into chunk_base[b]; the last CTA to finish (a ticket in
// meta[kMetaTicket], zeroed with the metadata) scans them in place into exclusive chunk
// bases and writes the tile total to meta[kMetaTiles].  No CTA waits for another.
template <int WPT>
__global__ void __launch_bounds__(kThreads)
k_bm_count_scan(const uint32_t* __restrict__ bitmap, uint64_t W, RowDiv wpr, uint32_t lshift,
                uint32_t* chunk_base, unsigned long long* meta)
{
    __shared__ uint32_t s_warp[kThreads / kWarp];
    __shared__ unsigned long long s_tot[kThreads / kWarp];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t w0 = (uint64_t)blockIdx.x * (kThreads * WPT) + (uint64_t)threadIdx.x * WPT;
    uint32_t x[WPT];
    load_lower_words<WPT>(bitmap, w0, W, wpr, lshift, x);
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < WPT; ++k) sum += __popc(x[k]);
    sum = __reduce_add_sync(kFull, sum);
    if (lane == 0) s_warp[warp] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kThreads / kWarp; ++w) t += s_warp[w];
        chunk_base[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(&meta[kMetaTicket], 1ull) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // exclusive scan of the gridDim.x counts; thread t owns a contiguous run of them
    const uint32_t nch = gridDim.x;
    const uint32_t per = (nch + kThreads - 1) / kThreads;
    const uint32_t b0 = min((uint32_t)threadIdx.x * per, nch), b1 = min(b0 + per, nch);
    unsigned long long own = 0;
    for (uint32_t b = b0; b < b1; ++b) own += __ldcg(&chunk_base[b]);
    unsigned long long incl = own;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long t = __shfl_up_sync(kFull, incl, d);
        if (lane >= d) incl += t;
    }
    if (lane == 31) s_tot[warp] = incl;
    __syncthreads();
    unsigned long long run = incl - own;
    for (int w = 0; w < warp; ++w) run += s_tot[w];
    for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t c = __ldcg(&chunk_base[b]);
        chunk_base[b] = (uint32_t)run;
        run += c;
    }
    if (threadIdx.x == kThreads - 1) meta[kMetaTiles] = run;  // the total
}

// indptr[R] = tile count; the overflow flag; and, when host_meta (a device alias of
// mapped pinned memory) is given, the build's status slots copied to the host.
__device__ __forceinline__ void finish_tiles(uint32_t* indptr, int32_t R, unsigned long long* meta,
                                             uint32_t cap, unsigned long long* host_meta)
{
    const unsigned long long T = meta[kMetaTiles];
    indptr[R] = (uint32_t)T;
    if (T > cap) meta[kMetaOverflow] = 1ull;
    if (host_meta) {
        volatile unsigned long long* h = host_meta;
        h[kMetaBad] = meta[kMetaBad];
        h[kMetaTiles] = T;
        h[kMetaOverflow] = T > cap ? 1ull : 0ull;
        __threadfence_system();
    }
}

template <int WPT>
__global__ void __launch_bounds__(kThreads)
k_bm_emit(const uint32_t* __restrict__ bitmap, uint64_t W, RowDiv wpr, uint32_t lshift,
          const uint32_t* __restrict__ chunk_base, uint2* __restrict__ cellpp,
          uint32_t* __restrict__ indices, uint32_t* __restrict__ row_indices,
          uint32_t* __restrict__ indptr, unsigned long long* meta, uint32_t cap,
          unsigned long long* host_meta, int32_t R, uint4* __restrict__ blocks, uint32_t tile_vec4,
          uint32_t* __restrict__ rowmask)
{
    __shared__ uint32_t s_warp[kThreads / kWarp];
    const unsigned long long T = meta[kMetaTiles];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) finish_tiles(indptr, R, meta, cap, host_meta);
    if (T > cap) return;  // overflowed tile arrays: the builder redoes this step
    {
        // zero this chunk's tiles before k_fill_bm ORs bits into them
        const uint64_t tb = chunk_base[blockIdx.x];
        const uint64_t te = blockIdx.x + 1 < gridDim.x ? chunk_base[blockIdx.x + 1] : T;
        for (uint64_t i = tb * tile_vec4 + threadIdx.x; i < te * tile_vec4; i += kThreads)
            blocks[i] = make_uint4(0u, 0u, 0u, 0u);
        // and their row-occupancy masks, which k_fill_bm sets
        if (rowmask)
            for (uint64_t i = tb + threadIdx.x; i < te; i += kThreads) rowmask[i] = 0u;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t w0 = (uint64_t)blockIdx.x * (kThreads * WPT) + (uint64_t)threadIdx.x * WPT;
    uint32_t x[WPT];
    const uint32_t need = load_lower_words<WPT>(bitmap, w0, W, wpr, lshift, x);
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < WPT; ++k) mine += __popc(x[k]);
    // exclusive prefix of `mine` over the CTA (thread order = word order)
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

    uint32_t rb = row_of((uint32_t)w0, wpr);  // at most 2^30 words (load_lower_words)
    uint32_t col_word = (uint32_t)w0 - rb * wpr.d;
    uint32_t pre[WPT];
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
        pre[k] = base;
        if (w0 + k < W) {
            if (col_word == 0) indptr[rb] = base;
            uint32_t bits = x[k];
            uint32_t t = base;
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                indices[t] = (uint32_t)(col_word * 32 + b);
                row_indices[t] = (uint32_t)rb;
                ++t;
            }
            base = t;
        }
        if (++col_word == wpr.d) {
            col_word = 0;
            ++rb;
        }
    }
    // (word, prefix) pairs only where a lookup can land (the words load_lower_words read)
    if (WPT % 2 == 0 && w0 + WPT <= W) {
        uint4* p = reinterpret_cast<uint4*>(cellpp + w0);
#pragma unroll
        for (int q = 0; q < WPT / 2; ++q)
            if ((need >> (2 * q)) & 3u) p[q] = make_uint4(x[2 * q], pre[2 * q], x[2 * q + 1], pre[2 * q + 1]);
    } else {
#pragma unroll
        for (int k = 0; k < WPT; ++k)
            if ((need >> k) & 1u) cellpp[w0 + k] = make_uint2(x[k], pre[k]);
    }
}

// six CTAs per SM (40 registers): R-MAT s22 build 9.38 ms against 9.51 at the default five
template <int LOG2C>
__global__ void __launch_bounds__(kThreads, 6)
k_fill_bm(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t m, int32_t n,
          const int32_t* __restrict__ rank, uint64_t wpr, const uint32_t* __restrict__ bitmap,
          const uint2* __restrict__ cellpp, uint32_t* __restrict__ blocks,
          const unsigned long long* __restrict__ d_tiles, uint32_t cap, uint32_t* __restrict__ rowmask,
          int32_t R)
{
    const unsigned long long T = *d_tiles;
    if (T > cap) return;  // overflowed tile arrays: the builder redoes this step
    // row-occupancy masks: wanted when row blocks average 8 or more tiles (the row-wise
    // count's condition, on the device tile count)
    if (T < 8ull * (unsigned long long)(R > 0 ? R : 0)) rowmask = nullptr;
    constexpr int C = 1 << LOG2C;
    constexpr int WPR = C / 32;
    constexpr int TW = 16 * WPR;
    constexpr int U = 8;  // edges in flight per thread
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < m; i0 += U * stride) {
        int32_t u[U], v[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const int64_t i = i0 + k * stride;
            u[k] = i < m ? src[i] : 0;
            v[k] = i < m ? dst[i] : 0;
        }
        uint32_t r[U], c[U];
        bool ok[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            bool bad;
            r[k] = c[k] = 0;
            ok[k] = (i0 + k * stride < m) && orient(u[k], v[k], n, rank, r[k], c[k], bad);
        }
        uint32_t pre[U], word[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const uint64_t w = (uint64_t)(r[k] >> 4) * wpr + ((c[k] >> LOG2C) >> 5);
            const uint2 cp = ok[k] ? cellpp[w] : make_uint2(0u, 0u);
            word[k] = cp.x;
            pre[k] = cp.y;
        }
        uint32_t tile[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const uint32_t below = (1u << ((c[k] >> LOG2C) & 31u)) - 1u;
            tile[k] = pre[k] + __popc(word[k] & below);
        }
        if (rowmask) {
            // the edge that finds its tile word empty marks the row: one mask atomic per
            // non-empty word, none per edge of a busy row.  All U atomics are issued
            // before the first old value is looked at.
            uint32_t old[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const uint32_t cl = c[k] & (C - 1);
                old[k] = ok[k] ? atomicOr(&blocks[(size_t)tile[k] * TW + (r[k] & 15u) * WPR + (cl >> 5)],
                                          1u << (cl & 31u))
                               : 1u;
            }
#pragma unroll
            for (int k = 0; k < U; ++k)
                if (old[k] == 0u) atomicOr(&rowmask[tile[k]], 1u << (r[k] & 15u));
        } else {
#pragma unroll
            for (int k = 0; k < U; ++k) {
                if (!ok[k]) continue;
                const uint32_t cl = c[k] & (C - 1);
                atomicOr(&blocks[(size_t)tile[k] * TW + (r[k] & 15u) * WPR + (cl >> 5)], 1u << (cl & 31u));
            }
        }
    }
}

// indptr[R] = tile count; the overflow flag; and, when host_meta (a device alias of
// mapped pinned memory) is given, the build's status slots copied to the host.
// The same for a graph without cells (n = 0), where no k_bm_emit runs.
__global__ void k_set_last(uint32_t* __restrict__ indptr, int32_t R,
                           unsigned long long* __restrict__ meta, uint32_t cap,
                           unsigned long long* __restrict__ host_meta)
{
    finish_tiles(indptr, R, meta, cap, host_meta);
}

template <int TW>
__global__ void k_popcount_sum(const uint32_t* __restrict__ blocks, uint64_t words,
                               unsigned long long* __restrict__ out)
{
    unsigned long long s = 0;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4; i < words;
         i += (uint64_t)gridDim.x * blockDim.x * 4) {
        const uint4 v = *reinterpret_cast<const uint4*>(blocks + i);
        s += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(kFull, s, d);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

}  // namespace bm

int grid_for(int64_t work, int threads);
int launch_tile_scan(uint32_t* per_tile, uint32_t ntiles, unsigned long long* total, cudaStream_t s);

// one round of U = 8 edges per thread (the grid is capped at 16 CTAs per SM)
static int edge_grid(int64_t m) { return grid_for((m + 7) / 8, bm::kThreads); }

uint64_t bitmap_words_per_row(const BuildGeom& g)
{
    return (uint64_t)((g.n_col_blocks + 31) / 32);
}

// Words per thread of the chunk popcount/scan and emit: 16 when that still gives two CTAs
// per SM, else 4, else 1 (small bitmaps with many tiles per word: the per-CTA share of
// emitted and zeroed tiles stays small).
static int bitmap_wpt(uint64_t W)
{
    const uint64_t ctas = 2ull * (uint64_t)device_sm_count();
    if (W / (bm::kThreads * 16ull) >= ctas) return 16;
    if (W / (bm::kThreads * 4ull) >= ctas) return 4;
    return 1;
}

size_t bitmap_chunks(uint64_t W)
{
    const uint64_t chunk = (uint64_t)bm::kThreads * bitmap_wpt(W);
    return (size_t)((W + chunk - 1) / chunk);
}

int bitmap_mark_and_count(const BuildGeom& g, const int32_t* src, const int32_t* dst, int64_t m,
                          const int32_t* rank, uint32_t* bitmap, uint32_t* chunk_count,
                          unsigned long long* meta_bad, unsigned long long* meta_tiles,
                          cudaStream_t s)
{
    const uint64_t wpr = bitmap_words_per_row(g);
    const uint64_t W = wpr * (uint64_t)g.n_row_blocks;
    if (W == 0) {
        return cudaMemsetAsync(meta_tiles, 0, sizeof(unsigned long long), s) == cudaSuccess
                   ? BTC_OK
                   : BTC_E_CUDA;
    }
    if (cudaMemsetAsync(bitmap, 0, sizeof(uint32_t) * W, s) != cudaSuccess) return BTC_E_CUDA;
    if (m > 0) {
        if (g.tile_cols == 128)
            bm::k_mark<7><<<edge_grid(m), bm::kThreads, 0, s>>>(src, dst, m, g.n, rank, wpr, bitmap,
                                                                 meta_bad);
        else
            bm::k_mark<5><<<edge_grid(m), bm::kThreads, 0, s>>>(src, dst, m, g.n, rank, wpr, bitmap,
                                                                 meta_bad);
    }
    const size_t chunks = bitmap_chunks(W);
    // meta_tiles - kMetaTiles is the metadata base (its ticket slot is zero)
    unsigned long long* meta = meta_tiles - kMetaTiles;
    const bm::RowDiv rdiv = bm::make_row_div(wpr);
    const uint32_t lshift = (g.tile_cols == 128 ? 7u : 5u) + 5u;
    switch (bitmap_wpt(W)) {
    case 16:
        bm::k_bm_count_scan<16><<<(unsigned)chunks, bm::kThreads, 0, s>>>(bitmap, W, rdiv, lshift,
                                                                          chunk_count, meta);
        break;
    case 4:
        bm::k_bm_count_scan<4><<<(unsigned)chunks, bm::kThreads, 0, s>>>(bitmap, W, rdiv, lshift,
                                                                         chunk_count, meta);
        break;
    default:
        bm::k_bm_count_scan<1><<<(unsigned)chunks, bm::kThreads, 0, s>>>(bitmap, W, rdiv, lshift,
                                                                         chunk_count, meta);
        break;
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int bitmap_emit_and_fill(const BuildGeom& g, const int32_t* src, const int32_t* dst, int64_t m,
                         const int32_t* rank, const uint32_t* bitmap, const uint32_t* chunk_base,
                         uint2* cellpp, uint32_t* indices, uint32_t* row_indices,
                         uint32_t* indptr, uint32_t* blocks, unsigned long long* meta,
                         uint32_t cap, unsigned long long* host_meta, cudaStream_t s,
                         uint32_t* rowmask)
{
    const unsigned long long* meta_tiles = meta + kMetaTiles;
    const uint64_t wpr = bitmap_words_per_row(g);
    const uint64_t W = wpr * (uint64_t)g.n_row_blocks;
    const uint32_t vec4 = 4u * (uint32_t)(g.tile_cols / 32);  // 16-byte words per tile
    if (W > 0) {
        const unsigned grid = (unsigned)bitmap_chunks(W);
        uint4* b4 = reinterpret_cast<uint4*>(blocks);
        const int R = g.n_row_blocks;
        const uint32_t lshift = (g.tile_cols == 128 ? 7u : 5u) + 5u;
#define BTC_EMIT(WPT)                                                                         \
    bm::k_bm_emit<WPT><<<grid, bm::kThreads, 0, s>>>(bitmap, W, bm::make_row_div(wpr), lshift, chunk_base, \
                                                    cellpp, indices, \
                                                    row_indices, indptr, meta, cap, host_meta, R, \
                                                    b4, vec4, rowmask)
        switch (bitmap_wpt(W)) {
        case 16: BTC_EMIT(16); break;
        case 4: BTC_EMIT(4); break;
        default: BTC_EMIT(1); break;
        }
#undef BTC_EMIT
    }
    else
        bm::k_set_last<<<1, 1, 0, s>>>(indptr, g.n_row_blocks, meta, cap, host_meta);
    if (m > 0 && W > 0) {
        if (g.tile_cols == 128)
            bm::k_fill_bm<7><<<edge_grid(m), bm::kThreads, 0, s>>>(
                src, dst, m, g.n, rank, wpr, bitmap, cellpp, blocks, meta_tiles, cap, rowmask,
                g.n_row_blocks);
        else
            bm::k_fill_bm<5><<<edge_grid(m), bm::kThreads, 0, s>>>(
                src, dst, m, g.n, rank, wpr, bitmap, cellpp, blocks, meta_tiles, cap, rowmask,
                g.n_row_blocks);
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_popcount_sum(int tile_cols, const uint32_t* blocks, uint64_t num_tiles,
                        unsigned long long* out, cudaStream_t s)
{
    const uint64_t words = num_tiles * (uint64_t)(16 * (tile_cols / 32));
    if (cudaMemsetAsync(out, 0, sizeof(unsigned long long), s) != cudaSuccess) return BTC_E_CUDA;
    if (words) {
        const int grid = grid_for((int64_t)((words + 3) / 4), 256);
        if (tile_cols == 128)
            bm::k_popcount_sum<64><<<grid, 256, 0, s>>>(blocks, words, out);
        else
            bm::k_popcount_sum<16><<<grid, 256, 0, s>>>(blocks, words, out);
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

}  // namespace btc200

namespace btc200 {
// Popcount per fixed 4096-word chunk (bm::kChunk; the batch builder's chunking, which
// does not follow bitmap_chunks).
int launch_bitmap_count(const uint32_t* bitmap, uint64_t W, uint32_t* chunk_count, cudaStream_t s)
{
    const uint64_t chunks = (W + bm::kChunk - 1) / bm::kChunk;
    if (W) bm::k_bm_count<<<(unsigned)chunks, bm::kThreads, 0, s>>>(bitmap, W, chunk_count);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}
}  // namespace btc200

namespace btc200 {
namespace bm {
template <int WPR>
__global__ void k_rowmask(const uint32_t* __restrict__ blocks, uint32_t cap,
                          const unsigned long long* __restrict__ d_tiles,
                          const uint32_t* __restrict__ indptr, uint32_t R,
                          uint32_t* __restrict__ rowmask, unsigned long long* __restrict__ row_max,
                          bool masks)
{
    const unsigned long long T = d_tiles ? *d_tiles : cap;
    if (T > cap) return;  // overflowed tile arrays: the builder redoes this step
    const uint32_t num_tiles = (uint32_t)T;
    // longest row-block list
    uint32_t mx = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < R;
         i += (uint64_t)gridDim.x * blockDim.x)
        mx = max(mx, indptr[i + 1] - indptr[i]);
    mx = __reduce_max_sync(kFull, mx);
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(row_max, (unsigned long long)mx);
    // the masks serve only the heavy count variant, which reads them only when row
    // blocks average 8 or more tiles (the same test on the same count)
    if (!masks || (uint64_t)num_tiles < 8ull * (uint64_t)R) return;

    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < num_tiles;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t* b = blocks + t * (16 * WPR);
        uint32_t m = 0;
        if constexpr (WPR == 4) {
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const uint4 v = reinterpret_cast<const uint4*>(b)[r];
                m |= ((v.x | v.y | v.z | v.w) != 0u) ? (1u << r) : 0u;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint4 v = reinterpret_cast<const uint4*>(b)[q];
                m |= (v.x != 0u ? 1u : 0u) << (4 * q);
                m |= (v.y != 0u ? 1u : 0u) << (4 * q + 1);
                m |= (v.z != 0u ? 1u : 0u) << (4 * q + 2);
                m |= (v.w != 0u ? 1u : 0u) << (4 * q + 3);
            }
        }
        rowmask[t] = m;
    }
}
}  // namespace bm

int launch_rowmask(int tile_cols, const uint32_t* blocks, uint32_t cap,
                   const unsigned long long* d_tiles, const uint32_t* indptr, int32_t n_row_blocks,
                   uint32_t* rowmask, unsigned long long* row_max, cudaStream_t s, bool masks)
{
    const uint32_t R = n_row_blocks > 0 ? (uint32_t)n_row_blocks : 0u;
    if (cap || R) {
        const int grid = grid_for((int64_t)(masks ? max(cap, R) : R), 256);
        if (tile_cols == 128)
            bm::k_rowmask<4><<<grid, 256, 0, s>>>(blocks, cap, d_tiles, indptr, R, rowmask, row_max, masks);
        else
            bm::k_rowmask<1><<<grid, 256, 0, s>>>(blocks, cap, d_tiles, indptr, R, rowmask, row_max, masks);
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}
}  // namespace btc200
