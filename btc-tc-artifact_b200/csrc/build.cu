// build.cu -- GPU Bit-BSR builder (restates btc/operations/bcsr_16x128.h:136-241 and
// bcsr_16x32.h:144-249, plus the orientation of convert.h:280-324, as one pipeline).
//
//   k_degree / k_rank_keys / k_rank_scatter   optional descending-degree relabel
//   k_make_keys      orient (max,min), drop self-loops, range-check ids, and emit one
//                    64-bit key per edge: [row block | column block | row%16 | col%C],
//                    compacted with one atomic per CTA
//   radix_sort_u64   stable LSD sort on the (row block, column block) bits only
//   k_seg_count      tile heads per sort tile
//   k_seg_scan       exclusive scan of the head counts -> tile bases, tile total
//   k_fill           tile ids from the head prefix; heads write indices/row_indices;
//                    every edge ORs its bit into its tile (duplicates OR the same bit)
//   k_indptr         indptr[r] = lower_bound(row_indices, r)
//   k_density        tile popcount histogram
#include "common.cuh"

namespace btc200 {

BuildGeom make_geom(int32_t n, int tile_cols)
{
    BuildGeom g{};
    g.n = n;
    g.tile_cols = tile_cols;
    g.log2c = log2_exact(tile_cols);
    g.payload_bits = 4 + g.log2c;
    g.n_row_blocks = (n + 15) / 16;
    g.n_col_blocks = ((int64_t)n + tile_cols - 1) / tile_cols;
    g.cb_bits = bit_length_u64(g.n_col_blocks > 0 ? (uint64_t)(g.n_col_blocks - 1) : 0);
    const uint64_t rb_max = g.n_row_blocks > 0 ? (uint64_t)(g.n_row_blocks - 1) : 0;
    g.t_bits = bit_length_u64(rb_max) + g.cb_bits;
    return g;
}

namespace build_kernels {

constexpr int kThreads = kSortThreads;  // 256
constexpr int kItems = kSortItems;      // 16
constexpr int kWarps = kThreads / kWarp;

__device__ __forceinline__ uint32_t warp_sum(uint32_t v)
{
    return __reduce_add_sync(kFull, v);
}

// ---------------------------------------------------------------------------
// degree relabel
// ---------------------------------------------------------------------------
// Degree count.  On power-law inputs a few hub vertices take a large share of the
// increments, and atomics on one global word serialise; so each CTA keeps a small table
// of counters in shared memory: a vertex takes the free slot its hash points to the first
// time the CTA sees it (compare-and-swap), later increments of it stay in shared memory,
// and the table is added to the global counters once when the CTA ends.  Hubs appear
// often and early, so they own slots in every CTA; a vertex whose slot is taken by
// another counts in global memory as before.  4096 slots (32 KB of keys and counters):
// at R-MAT s22 a CTA's table keeps ~17% of its increments (2048 slots: ~10%) and the
// kernel takes 1.32 ms against 1.48.
constexpr int kDegSlots = 4096;
constexpr uint32_t kDegFree = 0xffffffffu;

__device__ __forceinline__ void degree_add(uint32_t v, uint32_t* __restrict__ keys,
                                           uint32_t* __restrict__ cnt, uint32_t* __restrict__ deg)
{
    const uint32_t slot = (v * 0x9E3779B1u) >> (32 - 12);  // kDegSlots = 2^12
    uint32_t k = keys[slot];
    if (k == kDegFree) {
        const uint32_t prev = atomicCAS(&keys[slot], kDegFree, v);
        k = prev == kDegFree ? v : prev;
    }
    if (k == v) atomicAdd(&cnt[slot], 1u);
    else atomicAdd(&deg[v], 1u);
}

__global__ void __launch_bounds__(256)
k_degree(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
         int64_t m, int32_t n, uint32_t* __restrict__ deg)
{
    static_assert(kDegSlots == 1 << 12, "degree_add hashes to 12 bits");
    __shared__ uint32_t keys[kDegSlots], cnt[kDegSlots];
    for (int i = threadIdx.x; i < kDegSlots; i += blockDim.x) {
        keys[i] = kDegFree;
        cnt[i] = 0;
    }
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = src[i], v = dst[i];
        if (u == v || u < 0 || v < 0 || u >= n || v >= n) continue;
        degree_add((uint32_t)u, keys, cnt, deg);
        degree_add((uint32_t)v, keys, cnt, deg);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kDegSlots; i += blockDim.x)
        if (keys[i] != kDegFree && cnt[i]) atomicAdd(&deg[keys[i]], cnt[i]);
}

// key = ((dmax - deg) << 32) | v ; sorted ascending on bits [32, 32+db) with a stable
// sort over ids given in ascending order, so ties keep ascending id.
__global__ void k_rank_keys(const uint32_t* __restrict__ deg, int32_t n, uint32_t dmax,
                            uint64_t* __restrict__ keys)
{
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)(dmax - deg[v]) << 32) | (uint64_t)v;
}

__global__ void k_rank_scatter(const uint64_t* __restrict__ sorted, int32_t n,
                               int32_t* __restrict__ rank)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        rank[(uint32_t)sorted[i]] = (int32_t)i;
}

// ---------------------------------------------------------------------------
// keys
// ---------------------------------------------------------------------------
// counters[0]: valid (oriented, non-self-loop) edges; counters[1]: out-of-range ids.
template <int LOG2C>
__global__ void __launch_bounds__(kThreads)
k_make_keys(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t m,
            int32_t n, const int32_t* __restrict__ rank, int cb_bits,
            uint64_t* __restrict__ keys, unsigned long long* __restrict__ counters)
{
    constexpr int C = 1 << LOG2C;
    __shared__ uint32_t s_warp[kWarps];
    __shared__ unsigned long long s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t tile = (int64_t)blockIdx.x * (kThreads * kItems);
    const int64_t base = tile + (int64_t)warp * (kItems * kWarp);

    uint64_t key[kItems];
    unsigned vb[kItems];
    uint32_t nvalid = 0, nbad = 0;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const int64_t i = base + it * kWarp + lane;
        bool valid = false, bad = false;
        uint64_t k = 0;
        if (i < m) {
            int32_t u = src[i], v = dst[i];
            bad = (u < 0) | (v < 0) | (u >= n) | (v >= n);
            if (!bad) {
                if (rank) {
                    u = rank[u];
                    v = rank[v];
                }
                valid = u != v;
                const uint32_t r = (uint32_t)max(u, v), c = (uint32_t)min(u, v);
                const uint64_t T = ((uint64_t)(r >> 4) << cb_bits) | (uint64_t)(c >> LOG2C);
                k = (T << (4 + LOG2C)) | ((uint64_t)(r & 15u) << LOG2C) | (uint64_t)(c & (C - 1));
            }
        }
        key[it] = k;
        vb[it] = __ballot_sync(kFull, valid);
        nvalid += __popc(vb[it]);
        nbad += __popc(__ballot_sync(kFull, bad));
    }
    if (lane == 0) s_warp[warp] = nvalid;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t t = s_warp[w];
            s_warp[w] = tot;
            tot += t;
        }
        s_base = tot ? atomicAdd(&counters[0], (unsigned long long)tot) : 0ull;
    }
    if (lane == 0 && nbad) atomicAdd(&counters[1], (unsigned long long)nbad);
    __syncthreads();
    unsigned long long out = s_base + s_warp[warp];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        if (vb[it] >> lane & 1u) keys[out + __popc(vb[it] & lanemask_lt())] = key[it];
        out += __popc(vb[it]);
    }
}

// ---------------------------------------------------------------------------
// segmentation into tiles
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool is_head(const uint64_t* __restrict__ keys, size_t i, uint64_t k,
                                        int payload_bits)
{
    return i == 0 || (keys[i - 1] >> payload_bits) != (k >> payload_bits);
}

__global__ void __launch_bounds__(kThreads)
k_seg_count(const uint64_t* __restrict__ keys, const unsigned long long* __restrict__ d_count,
            int payload_bits, uint32_t* __restrict__ heads_per_tile)
{
    __shared__ uint32_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t n = (size_t)*d_count;
    const size_t base = (size_t)blockIdx.x * (kThreads * kItems) + (size_t)warp * (kItems * kWarp);
    uint32_t h = 0;
#pragma unroll 4
    for (int it = 0; it < kItems; ++it) {
        const size_t i = base + (size_t)it * kWarp + lane;
        bool head = false;
        if (i < n) head = is_head(keys, i, keys[i], payload_bits);
        h += __popc(__ballot_sync(kFull, head));
    }
    if (lane == 0) s_warp[warp] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kWarps; ++w) t += s_warp[w];
        heads_per_tile[blockIdx.x] = t;
    }
}

// Single CTA: exclusive scan of heads_per_tile in place; meta[0] = total tiles.
__global__ void __launch_bounds__(1024)
k_seg_scan(uint32_t* __restrict__ heads_per_tile, uint32_t ntiles,
           unsigned long long* __restrict__ meta)
{
    __shared__ unsigned long long s_warp[32];
    __shared__ unsigned long long s_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long carry = 0;
    for (size_t b = 0; b < ntiles; b += 1024) {
        const size_t i = b + threadIdx.x;
        const unsigned long long v = i < ntiles ? heads_per_tile[i] : 0ull;
        unsigned long long incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long t = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const unsigned long long w = s_warp[lane];
            unsigned long long wi = w;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long t = __shfl_up_sync(kFull, wi, d);
                if (lane >= d) wi += t;
            }
            s_warp[lane] = wi - w;
            if (lane == 31) s_total = wi;
        }
        __syncthreads();
        if (i < ntiles) heads_per_tile[i] = (uint32_t)(carry + s_warp[warp] + incl - v);
        carry += s_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) meta[0] = carry;
}

template <int LOG2C>
__global__ void __launch_bounds__(kThreads)
k_fill(const uint64_t* __restrict__ keys, const unsigned long long* __restrict__ d_count,
       int cb_bits, const uint32_t* __restrict__ tile_base, uint32_t* __restrict__ indices,
       uint32_t* __restrict__ row_indices, uint32_t* __restrict__ blocks)
{
    constexpr int C = 1 << LOG2C;
    constexpr int WPR = C / 32;
    constexpr int TW = 16 * WPR;
    constexpr int P = 4 + LOG2C;
    __shared__ uint32_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t n = (size_t)*d_count;
    const size_t cta0 = (size_t)blockIdx.x * (kThreads * kItems);
    if (cta0 >= n) return;
    const size_t base = cta0 + (size_t)warp * (kItems * kWarp);

    uint64_t key[kItems];
    unsigned hb[kItems];
    uint32_t wh = 0;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const size_t i = base + (size_t)it * kWarp + lane;
        bool head = false;
        key[it] = 0;
        if (i < n) {
            key[it] = keys[i];
            head = is_head(keys, i, key[it], P);
        }
        hb[it] = __ballot_sync(kFull, head);
        wh += __popc(hb[it]);
    }
    if (lane == 0) s_warp[warp] = wh;
    __syncthreads();
    uint32_t before = tile_base[blockIdx.x];
#pragma unroll
    for (int w = 0; w < kWarps; ++w) before += (w < warp) ? s_warp[w] : 0u;

    const uint64_t cb_mask = (1ull << cb_bits) - 1ull;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const size_t i = base + (size_t)it * kWarp + lane;
        const unsigned h = hb[it];
        if (i < n) {
            // heads up to and including this element, minus one
            const uint32_t t = before + __popc(h & lanemask_lt()) + ((h >> lane) & 1u) - 1u;
            const uint64_t k = key[it];
            const uint64_t T = k >> P;
            if ((h >> lane) & 1u) {
                indices[t] = (uint32_t)(T & cb_mask);
                row_indices[t] = (uint32_t)(T >> cb_bits);
            }
            const uint32_t lr = (uint32_t)(k >> LOG2C) & 15u;
            const uint32_t cl = (uint32_t)k & (C - 1);
            atomicOr(&blocks[(size_t)t * TW + lr * WPR + (cl >> 5)], 1u << (cl & 31u));
        }
        before += __popc(h);
    }
}

__global__ void k_indptr(const uint32_t* __restrict__ row_indices, uint32_t num_tiles,
                         int32_t R, uint32_t* __restrict__ indptr)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= R;
         r += (int64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = num_tiles;
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo) >> 1);
            if ((int64_t)row_indices[mid] < r) lo = mid + 1;
            else hi = mid;
        }
        indptr[r] = lo;
    }
}

template <int TW>
__global__ void k_density(const uint32_t* __restrict__ blocks, uint32_t num_tiles,
                          unsigned long long* __restrict__ hist)
{
    constexpr int NB = TW * 32 + 1;
    __shared__ uint32_t s_hist[NB];
    for (int i = threadIdx.x; i < NB; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < num_tiles;
         t += (int64_t)gridDim.x * blockDim.x) {
        uint32_t p = 0;
        const uint4* b = reinterpret_cast<const uint4*>(blocks + (size_t)t * TW);
#pragma unroll
        for (int w = 0; w < TW / 4; ++w) {
            const uint4 q = b[w];
            p += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
        }
        atomicAdd(&s_hist[p], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NB; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], (unsigned long long)s_hist[i]);
}

}  // namespace build_kernels

// ---------------------------------------------------------------------------
// host launchers used by capi.cu
// ---------------------------------------------------------------------------
int grid_for(int64_t work, int threads)
{
    const int64_t cap = (int64_t)device_sm_count() * 16;
    int64_t g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

int launch_degree(const int32_t* src, const int32_t* dst, int64_t m, int32_t n, uint32_t* deg,
                  cudaStream_t s)
{
    if (m > 0) build_kernels::k_degree<<<grid_for(m, 256), 256, 0, s>>>(src, dst, m, n, deg);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_rank_keys(const uint32_t* deg, int32_t n, uint32_t dmax, uint64_t* keys, cudaStream_t s)
{
    if (n > 0) build_kernels::k_rank_keys<<<grid_for(n, 256), 256, 0, s>>>(deg, n, dmax, keys);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_rank_scatter(const uint64_t* sorted, int32_t n, int32_t* rank, cudaStream_t s)
{
    if (n > 0) build_kernels::k_rank_scatter<<<grid_for(n, 256), 256, 0, s>>>(sorted, n, rank);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_make_keys(const BuildGeom& g, const int32_t* src, const int32_t* dst, int64_t m,
                     const int32_t* rank, uint64_t* keys, unsigned long long* counters,
                     cudaStream_t s)
{
    const int64_t tiles = (m + kSortTile - 1) / kSortTile;
    if (tiles > 0) {
        if (g.tile_cols == 128)
            build_kernels::k_make_keys<7><<<(unsigned)tiles, build_kernels::kThreads, 0, s>>>(
                src, dst, m, g.n, rank, g.cb_bits, keys, counters);
        else
            build_kernels::k_make_keys<5><<<(unsigned)tiles, build_kernels::kThreads, 0, s>>>(
                src, dst, m, g.n, rank, g.cb_bits, keys, counters);
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_segment(const BuildGeom& g, const uint64_t* keys, size_t max_n,
                   const unsigned long long* d_count, uint32_t* tile_base,
                   unsigned long long* meta, cudaStream_t s)
{
    const size_t tiles = sort_tiles(max_n);
    if (tiles > 0) {
        build_kernels::k_seg_count<<<(unsigned)tiles, build_kernels::kThreads, 0, s>>>(
            keys, d_count, g.payload_bits, tile_base);
        build_kernels::k_seg_scan<<<1, 1024, 0, s>>>(tile_base, (uint32_t)tiles, meta);
    } else {
        if (cudaMemsetAsync(meta, 0, sizeof(unsigned long long), s) != cudaSuccess) return BTC_E_CUDA;
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_fill(const BuildGeom& g, const uint64_t* keys, size_t max_n,
                const unsigned long long* d_count, const uint32_t* tile_base, uint32_t* indices,
                uint32_t* row_indices, uint32_t* blocks, cudaStream_t s)
{
    const size_t tiles = sort_tiles(max_n);
    if (tiles > 0) {
        if (g.tile_cols == 128)
            build_kernels::k_fill<7><<<(unsigned)tiles, build_kernels::kThreads, 0, s>>>(
                keys, d_count, g.cb_bits, tile_base, indices, row_indices, blocks);
        else
            build_kernels::k_fill<5><<<(unsigned)tiles, build_kernels::kThreads, 0, s>>>(
                keys, d_count, g.cb_bits, tile_base, indices, row_indices, blocks);
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_indptr(const uint32_t* row_indices, uint32_t num_tiles, int32_t R, uint32_t* indptr,
                  cudaStream_t s)
{
    build_kernels::k_indptr<<<grid_for((int64_t)R + 1, 256), 256, 0, s>>>(row_indices, num_tiles, R,
                                                                          indptr);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

int launch_density(int tile_cols, const uint32_t* blocks, uint32_t num_tiles,
                   unsigned long long* hist, cudaStream_t s)
{
    if (num_tiles > 0) {
        if (tile_cols == 128)
            build_kernels::k_density<64><<<grid_for(num_tiles, 256), 256, 0, s>>>(blocks, num_tiles, hist);
        else
            build_kernels::k_density<16><<<grid_for(num_tiles, 256), 256, 0, s>>>(blocks, num_tiles, hist);
    }
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

}  // namespace btc200

namespace btc200 {
namespace build_kernels {
__global__ void k_set_u64(unsigned long long* p, unsigned long long v) { *p = v; }
}  // namespace build_kernels

int launch_set_u64(unsigned long long* p, unsigned long long v, cudaStream_t s)
{
    build_kernels::k_set_u64<<<1, 1, 0, s>>>(p, v);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}
}  // namespace btc200

namespace btc200 {
int launch_tile_scan(uint32_t* per_tile, uint32_t ntiles, unsigned long long* total, cudaStream_t s)
{
    if (ntiles == 0) return cudaMemsetAsync(total, 0, sizeof(unsigned long long), s) == cudaSuccess
                                ? BTC_OK
                                : BTC_E_CUDA;
    build_kernels::k_seg_scan<<<1, 1024, 0, s>>>(per_tile, ntiles, total);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}
}  // namespace btc200
