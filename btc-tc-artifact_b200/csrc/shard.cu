// shard.cu -- one graph's count split across ranks.
//
// Every rank holds the same Bit-BSR (built from the same input, so the tiles and their
// order agree), counts a contiguous range of sample tiles, and the ranks add their
// counts (one int64 all-reduce).  The ranges come from an estimate of each tile's count
// cost, summed per bucket of kCostBucket consecutive tiles on the device, and cut on
// the host where the running cost crosses r/parts of the total.
//
// Tile cost estimate: the index-list elements of the row blocks J_out under the tile's
// occupied 16-column slices (the search work of the count kernel), plus a quarter of the
// tile's bits (the popcount work), plus 16 (fixed per-tile work).
#include "handle.cuh"

#include <vector>

namespace btc200 {
namespace {

constexpr uint32_t kCostBucket = 256;  // tiles per cost bucket
constexpr int kCostWarps = 8;

template <int C>
__global__ void __launch_bounds__(kCostWarps * 32)
k_tile_cost(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
            const uint32_t* __restrict__ blocks, uint32_t num_tiles, int32_t R,
            unsigned long long* __restrict__ bucket_cost)
{
    constexpr int TW = C / 2, JPT = C / 16;
    __shared__ unsigned long long s_part[kCostWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t t0 = (uint64_t)blockIdx.x * kCostBucket;
    const uint64_t t1 = min(t0 + kCostBucket, (uint64_t)num_tiles);
    unsigned long long acc = 0;
    for (uint64_t t = t0 + warp; t < t1; t += kCostWarps) {
        uint32_t w0 = 0, w1 = 0;
        if constexpr (C == 128) {
            const uint2 v = reinterpret_cast<const uint2*>(blocks + t * TW)[lane];
            w0 = v.x;
            w1 = v.y;
        } else {
            if (lane < 16) w0 = blocks[t * TW + lane];
        }
        // slice j of tile row r: 16x128 lane 2r + (j >= 4) holds it in word (j & 3) / 2,
        // 16x32 lane r holds it in w0
        uint32_t active = 0;
        if constexpr (C == 128) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t sl = ((q < 2 ? w0 : w1) >> (16 * (q & 1))) & 0xFFFFu;
                const unsigned b = __ballot_sync(kFull, sl != 0);
                if (b & 0x55555555u) active |= 1u << q;
                if (b & 0xAAAAAAAAu) active |= 1u << (4 + q);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 2; ++q)
                if (__ballot_sync(kFull, ((w0 >> (16 * q)) & 0xFFFFu) != 0)) active |= 1u << q;
        }
        const uint32_t nnz = __reduce_add_sync(kFull, (unsigned)(__popc(w0) + __popc(w1)));
        uint32_t len = 0;
        if (lane < JPT && ((active >> lane) & 1u)) {
            const uint64_t J = (uint64_t)indices[t] * JPT + lane;
            if (J < (uint64_t)R) len = indptr[J + 1] - indptr[J];
        }
        len = __reduce_add_sync(kFull, len);
        acc += (unsigned long long)len + nnz / 4 + 16;
    }
    if (lane == 0) s_part[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sum = 0;
        for (int w = 0; w < kCostWarps; ++w) sum += s_part[w];
        bucket_cost[blockIdx.x] = sum;
    }
}

}  // namespace
}  // namespace btc200

using namespace btc200;

extern "C" {

int btc_partition_from_costs(const unsigned long long* bucket_cost, uint64_t n_buckets,
                             uint32_t bucket_tiles, uint32_t num_tiles, int parts,
                             uint32_t* bounds)
{
    if (parts < 1 || !bounds || bucket_tiles == 0 || (n_buckets && !bucket_cost)) return BTC_E_INVAL;
    if ((uint64_t)num_tiles > n_buckets * (uint64_t)bucket_tiles) return BTC_E_INVAL;
    unsigned __int128 total = 0;
    for (uint64_t b = 0; b < n_buckets; ++b) total += bucket_cost[b];
    bounds[0] = 0;
    uint64_t b = 0;
    unsigned __int128 run = 0;  // cost of buckets [0, b)
    for (int r = 1; r < parts; ++r) {
        // first bucket boundary whose running cost reaches r/parts of the total
        const unsigned __int128 target = total * (unsigned)r / (unsigned)parts;
        while (b < n_buckets && run + bucket_cost[b] <= target) run += bucket_cost[b++];
        // the cut goes before bucket b, or after it when that is closer to the target
        uint64_t cut = b;
        if (b < n_buckets && (target - run) * 2 > bucket_cost[b]) {
            run += bucket_cost[b++];
            cut = b;
        }
        const uint64_t tile = cut * (uint64_t)bucket_tiles;
        bounds[r] = (uint32_t)(tile < num_tiles ? tile : num_tiles);
        if (bounds[r] < bounds[r - 1]) bounds[r] = bounds[r - 1];
    }
    bounds[parts] = num_tiles;
    return BTC_OK;
}

int btc_partition_tiles(const btc_bitbsr* g, int parts, btc_stream_t stream, uint32_t* bounds)
{
    if (!g || parts < 1 || !bounds) return BTC_E_INVAL;
    BTC_TRY(resolve_build(const_cast<btc_bitbsr*>(g)));
    const uint32_t T = g->num_tiles;
    const uint64_t nb = ((uint64_t)T + kCostBucket - 1) / kCostBucket;
    if (nb == 0) return btc_partition_from_costs(nullptr, 0, kCostBucket, 0, parts, bounds);
    struct Scoped {
        DevBuf b;
        ~Scoped() { b.release(); }
    } tmp;
    DevBuf& cost = tmp.b;
    BTC_TRY(cost.reserve(sizeof(unsigned long long) * nb));
    if (g->tile_cols == 128)
        k_tile_cost<128><<<(unsigned)nb, kCostWarps * 32, 0, stream>>>(
            g->indptr.as<uint32_t>(), g->indices.as<uint32_t>(), g->blocks.as<uint32_t>(), T,
            g->n_row_blocks, cost.as<unsigned long long>());
    else
        k_tile_cost<32><<<(unsigned)nb, kCostWarps * 32, 0, stream>>>(
            g->indptr.as<uint32_t>(), g->indices.as<uint32_t>(), g->blocks.as<uint32_t>(), T,
            g->n_row_blocks, cost.as<unsigned long long>());
    BTC_CUDA_TRY(cudaGetLastError());
    std::vector<unsigned long long> h(nb);
    BTC_CUDA_TRY(cudaMemcpyAsync(h.data(), cost.ptr, sizeof(unsigned long long) * nb,
                                 cudaMemcpyDeviceToHost, stream));
    BTC_CUDA_TRY(cudaStreamSynchronize(stream));
    return btc_partition_from_costs(h.data(), nb, kCostBucket, T, parts, bounds);
}

int btc_count_tiles_async(btc_bitbsr* g, uint32_t tile_begin, uint32_t tile_end, int tau,
                          btc_stream_t stream, unsigned long long* d_out)
{
    if (!g || !d_out) return BTC_E_INVAL;
    BTC_TRY(resolve_build(g));
    if (tile_begin > tile_end || tile_end > g->num_tiles) return BTC_E_INVAL;
    return count_handle(g, tau, stream, d_out, tile_begin, tile_end);
}

}  // extern "C"
