// preprocess.cu -- btc_preprocess_for_triangle_counting: the reference's
// preprocess_for_triangle_counting (btc/operations/convert.h:600-612 with BTC_REORDER=0)
// on device COO arrays: orient (max,min) (reorder.h:39-46), drop self-loops, sort
// lexicographically, unique (convert.h:280-324), and optionally compact the ids that
// occur to [0, n_used) in ascending order (remap_node_ids_gpu, convert.h:386-425).
// The sort is the engine's radix sort on packed (row, col) keys.
#include <cstdio>

#include "common.cuh"

namespace btc200 {
namespace {

constexpr int kThreads = kSortThreads;
constexpr int kItems = kSortItems;
constexpr int kWarps = kThreads / kWarp;

// valid non-self-loop entries -> key (r << bl) | c, compacted; counters[1] counts
// out-of-range ids.
__global__ void __launch_bounds__(kThreads)
k_pre_keys(const int32_t* __restrict__ rows, const int32_t* __restrict__ cols, int64_t m, int32_t n,
           int bl, uint64_t* __restrict__ keys, unsigned long long* __restrict__ counters)
{
    __shared__ uint32_t s_warp[kWarps];
    __shared__ unsigned long long s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * (kItems * kWarp);
    uint64_t key[kItems];
    unsigned vb[kItems];
    uint32_t nvalid = 0, nbad = 0;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const int64_t i = base + it * kWarp + lane;
        bool valid = false, bad = false;
        uint64_t k = 0;
        if (i < m) {
            const int32_t u = rows[i], v = cols[i];
            bad = (u < 0) | (v < 0) | (u >= n) | (v >= n);
            valid = !bad && u != v;
            k = ((uint64_t)(uint32_t)max(u, v) << bl) | (uint64_t)(uint32_t)min(u, v);
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

__global__ void __launch_bounds__(kThreads)
k_uniq_count(const uint64_t* __restrict__ keys, const unsigned long long* __restrict__ d_count,
             uint32_t* __restrict__ per_tile)
{
    __shared__ uint32_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t n = (size_t)*d_count;
    const size_t base = (size_t)blockIdx.x * kSortTile + (size_t)warp * (kItems * kWarp);
    uint32_t h = 0;
    for (int it = 0; it < kItems; ++it) {
        const size_t i = base + (size_t)it * kWarp + lane;
        const bool head = i < n && (i == 0 || keys[i - 1] != keys[i]);
        h += __popc(__ballot_sync(kFull, head));
    }
    if (lane == 0) s_warp[warp] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kWarps; ++w) t += s_warp[w];
        per_tile[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kThreads)
k_uniq_write(const uint64_t* __restrict__ keys, const unsigned long long* __restrict__ d_count,
             const uint32_t* __restrict__ tile_base, int bl, int32_t* __restrict__ rows,
             int32_t* __restrict__ cols)
{
    __shared__ uint32_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t n = (size_t)*d_count;
    const size_t cta0 = (size_t)blockIdx.x * kSortTile;
    if (cta0 >= n) return;
    const size_t base = cta0 + (size_t)warp * (kItems * kWarp);
    unsigned hb[kItems];
    uint32_t wh = 0;
    for (int it = 0; it < kItems; ++it) {
        const size_t i = base + (size_t)it * kWarp + lane;
        const bool head = i < n && (i == 0 || keys[i - 1] != keys[i]);
        hb[it] = __ballot_sync(kFull, head);
        wh += __popc(hb[it]);
    }
    if (lane == 0) s_warp[warp] = wh;
    __syncthreads();
    uint32_t before = tile_base[blockIdx.x];
    for (int w = 0; w < kWarps; ++w) before += (w < warp) ? s_warp[w] : 0u;
    const uint64_t cmask = (1ull << bl) - 1ull;
    for (int it = 0; it < kItems; ++it) {
        const size_t i = base + (size_t)it * kWarp + lane;
        if ((hb[it] >> lane) & 1u) {
            const uint32_t o = before + __popc(hb[it] & lanemask_lt());
            const uint64_t k = keys[i];
            rows[o] = (int32_t)(k >> bl);
            cols[o] = (int32_t)(k & cmask);
        }
        before += __popc(hb[it]);
    }
}

__global__ void k_mark_used(const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                            int64_t m, uint32_t* __restrict__ used)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        used[rows[i]] = 1u;
        used[cols[i]] = 1u;
    }
}

// per 4096-id tile: number of used ids
__global__ void __launch_bounds__(kThreads)
k_used_count(const uint32_t* __restrict__ used, int32_t n, uint32_t* __restrict__ per_tile)
{
    __shared__ uint32_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t h = 0;
    const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * (kItems * kWarp);
    for (int it = 0; it < kItems; ++it) {
        const int64_t v = base + it * kWarp + lane;
        h += __popc(__ballot_sync(kFull, v < n && used[v]));
    }
    if (lane == 0) s_warp[warp] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kWarps; ++w) t += s_warp[w];
        per_tile[blockIdx.x] = t;
    }
}

// newid[v] = number of used ids below v (in place over `used`)
__global__ void __launch_bounds__(kThreads)
k_used_rank(uint32_t* __restrict__ used, int32_t n, const uint32_t* __restrict__ tile_base)
{
    __shared__ uint32_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * (kItems * kWarp);
    unsigned hb[kItems];
    uint32_t wh = 0;
    for (int it = 0; it < kItems; ++it) {
        const int64_t v = base + it * kWarp + lane;
        hb[it] = __ballot_sync(kFull, v < n && used[v]);
        wh += __popc(hb[it]);
    }
    if (lane == 0) s_warp[warp] = wh;
    __syncthreads();
    uint32_t before = tile_base[blockIdx.x];
    for (int w = 0; w < kWarps; ++w) before += (w < warp) ? s_warp[w] : 0u;
    for (int it = 0; it < kItems; ++it) {
        const int64_t v = base + it * kWarp + lane;
        if (v < n) used[v] = before + __popc(hb[it] & lanemask_lt());
        before += __popc(hb[it]);
    }
}

__global__ void k_apply_map(int32_t* __restrict__ rows, int32_t* __restrict__ cols, int64_t m,
                            const uint32_t* __restrict__ newid)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        rows[i] = (int32_t)newid[rows[i]];
        cols[i] = (int32_t)newid[cols[i]];
    }
}

}  // namespace

// single-CTA exclusive scan of per-tile counts (defined in build.cu's kernels)
int launch_tile_scan(uint32_t* per_tile, uint32_t ntiles, unsigned long long* total, cudaStream_t s);
int grid_for(int64_t work, int threads);

}  // namespace btc200

using namespace btc200;

extern "C" int btc_preprocess_for_triangle_counting(int32_t* d_rows, int32_t* d_cols, int64_t* nnz,
                                                    int32_t* num_rows, int remap)
{
    if (!nnz || !num_rows) return BTC_E_INVAL;
    const int64_t m = *nnz;
    const int32_t n = *num_rows;
    if (m < 0 || n < 0 || (uint64_t)m > (1ull << 32) - (uint64_t)kSortTile) return BTC_E_INVAL;
    if (m == 0) return BTC_OK;
    if (!d_rows || !d_cols) return BTC_E_INVAL;
    const cudaStream_t s = nullptr;
    const int bl = bit_length_u64(n > 0 ? (uint64_t)(n - 1) : 0);
    const size_t tiles = sort_tiles((size_t)m);
    DevBuf k0, k1, scratch, tbase, meta;
    int st = BTC_OK;
    auto cleanup = [&]() {
        k0.release();
        k1.release();
        scratch.release();
        tbase.release();
        meta.release();
    };
#define PRE_TRY(x)                 \
    do {                           \
        st = (x);                  \
        if (st != BTC_OK) {        \
            cleanup();             \
            return st;             \
        }                          \
    } while (0)
    PRE_TRY(k0.reserve(sizeof(uint64_t) * (size_t)m));
    PRE_TRY(k1.reserve(sizeof(uint64_t) * (size_t)m));
    PRE_TRY(scratch.reserve(sizeof(uint32_t) * radix_scratch_words((size_t)m)));
    const size_t id_tiles = sort_tiles((size_t)n);
    PRE_TRY(tbase.reserve(sizeof(uint32_t) * ((tiles > id_tiles ? tiles : id_tiles) + 1)));
    PRE_TRY(meta.reserve(sizeof(unsigned long long) * 4));
    unsigned long long* dm = meta.as<unsigned long long>();
    if (cudaMemset(dm, 0, sizeof(unsigned long long) * 4) != cudaSuccess) PRE_TRY(BTC_E_CUDA);

    k_pre_keys<<<(unsigned)tiles, kThreads, 0, s>>>(d_rows, d_cols, m, n, bl, k0.as<uint64_t>(), dm);
    uint64_t* sorted = radix_sort_u64(k0.as<uint64_t>(), k1.as<uint64_t>(), (size_t)m, dm, 0,
                                      2 * bl, scratch.as<uint32_t>(), s, &st);
    if (st != BTC_OK) PRE_TRY(st);
    k_uniq_count<<<(unsigned)tiles, kThreads, 0, s>>>(sorted, dm, tbase.as<uint32_t>());
    PRE_TRY(launch_tile_scan(tbase.as<uint32_t>(), (uint32_t)tiles, dm + 2, s));
    k_uniq_write<<<(unsigned)tiles, kThreads, 0, s>>>(sorted, dm, tbase.as<uint32_t>(), bl, d_rows,
                                                      d_cols);
    unsigned long long h[4] = {0, 0, 0, 0};
    if (cudaMemcpy(h, dm, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) PRE_TRY(BTC_E_CUDA);
    if (h[1] != 0) PRE_TRY(BTC_E_RANGE);
    const int64_t mu = (int64_t)h[2];
    int32_t n_out = n;
    if (remap && n > 0) {
        DevBuf used;
        if (used.reserve(sizeof(uint32_t) * (size_t)n) != BTC_OK) PRE_TRY(BTC_E_NOMEM);
        cudaMemset(used.ptr, 0, sizeof(uint32_t) * (size_t)n);
        if (mu > 0)
            k_mark_used<<<grid_for(mu, 256), 256, 0, s>>>(d_rows, d_cols, mu, used.as<uint32_t>());
        k_used_count<<<(unsigned)id_tiles, kThreads, 0, s>>>(used.as<uint32_t>(), n,
                                                             tbase.as<uint32_t>());
        st = launch_tile_scan(tbase.as<uint32_t>(), (uint32_t)id_tiles, dm + 3, s);
        if (st == BTC_OK) {
            k_used_rank<<<(unsigned)id_tiles, kThreads, 0, s>>>(used.as<uint32_t>(), n,
                                                                tbase.as<uint32_t>());
            unsigned long long nu = 0;
            if (cudaMemcpy(&nu, dm + 3, sizeof(nu), cudaMemcpyDeviceToHost) != cudaSuccess)
                st = BTC_E_CUDA;
            // the reference skips the remap when every id is used (convert.h:406-409)
            if (st == BTC_OK && (int32_t)nu != n && mu > 0) {
                k_apply_map<<<grid_for(mu, 256), 256, 0, s>>>(d_rows, d_cols, mu, used.as<uint32_t>());
                n_out = (int32_t)nu;
            }
        }
        used.release();
        if (st != BTC_OK) PRE_TRY(st);
    }
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) PRE_TRY(BTC_E_CUDA);
    *nnz = mu;
    *num_rows = n_out;
    cleanup();
    return BTC_OK;
#undef PRE_TRY
}
