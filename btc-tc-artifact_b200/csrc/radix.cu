// radix.cu -- stable LSD radix sort of 64-bit keys, 8-bit digits, for the Bit-BSR
// builder.  Each pass is three launches:
//   k_radix_hist     per-CTA digit histogram of a 4096-key tile (warp-private bins,
//                    __match_any_sync aggregation), stored digit-major;
//   k_radix_scan     one CTA per digit: exclusive scan over tiles + digit total;
//   k_radix_scatter  stable in-CTA ranking (warp match + per-warp bins), keys staged
//                    in shared memory in digit order, then written out so that
//                    consecutive threads store consecutive addresses of a digit run.
// The key count is read from device memory, so a pass needs no host round trip.
#include "common.cuh"

namespace btc200 {

namespace {

constexpr int kWarps = kSortThreads / kWarp;  // 8

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane)
{
#pragma unroll
    for (int d = 1; d < kWarp; d <<= 1) {
        uint32_t t = __shfl_up_sync(kFull, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

// Exclusive scan of one value per thread over a 256-thread CTA.  `tmp` holds 8 words.
__device__ __forceinline__ uint32_t cta256_excl_scan(uint32_t v, uint32_t* tmp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = warp_incl_scan(v, lane);
    if (lane == 31) tmp[warp] = incl;
    __syncthreads();
    uint32_t off = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) off += (w < warp) ? tmp[w] : 0u;
    __syncthreads();
    return off + incl - v;
}

__global__ void __launch_bounds__(kSortThreads)
k_radix_hist(const uint64_t* __restrict__ keys, const unsigned long long* __restrict__ d_count,
             int shift, uint32_t* __restrict__ hist, uint32_t ntiles)
{
    __shared__ uint32_t s_hist[kWarps][kRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&s_hist[0][0])[i] = 0;
    __syncthreads();
    const size_t n = (size_t)*d_count;
    const size_t base = (size_t)blockIdx.x * kSortTile + (size_t)warp * (kSortItems * kWarp);
#pragma unroll 4
    for (int it = 0; it < kSortItems; ++it) {
        const size_t idx = base + (size_t)it * kWarp + lane;
        const bool ok = idx < n;
        const unsigned active = __ballot_sync(kFull, ok);
        if (ok) {
            const uint32_t d = (uint32_t)(keys[idx] >> shift) & (kRadix - 1);
            const unsigned peers = __match_any_sync(active, d);
            if ((peers & lanemask_lt()) == 0) s_hist[warp][d] += __popc(peers);
        }
    }
    __syncthreads();
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) sum += s_hist[w][threadIdx.x];
    hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = sum;
}

constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads)
k_radix_scan(uint32_t* __restrict__ hist, uint32_t ntiles, uint32_t* __restrict__ totals)
{
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* row = hist + (size_t)blockIdx.x * ntiles;
    uint32_t carry = 0;
    for (size_t base = 0; base < ntiles; base += kScanThreads) {
        const size_t i = base + threadIdx.x;
        const uint32_t v = i < ntiles ? row[i] : 0u;
        const uint32_t incl = warp_incl_scan(v, lane);
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t w = s_warp[lane];
            const uint32_t wi = warp_incl_scan(w, lane);
            s_warp[lane] = wi - w;
            if (lane == 31) s_total = wi;
        }
        __syncthreads();
        if (i < ntiles) row[i] = carry + s_warp[warp] + incl - v;
        carry += s_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(kSortThreads)
k_radix_scatter(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                const unsigned long long* __restrict__ d_count, int shift,
                const uint32_t* __restrict__ hist, const uint32_t* __restrict__ totals,
                uint32_t ntiles)
{
    __shared__ uint64_t s_stage[kSortTile];
    __shared__ uint32_t s_whist[kWarps][kRadix];
    __shared__ uint32_t s_start[kRadix];
    __shared__ uint32_t s_gbase[kRadix];
    __shared__ uint32_t s_tmp[kWarps];

    const size_t n = (size_t)*d_count;
    const size_t tile_base = (size_t)blockIdx.x * kSortTile;
    if (tile_base >= n) return;  // uniform for the CTA

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&s_whist[0][0])[i] = 0;
    __syncthreads();

    uint64_t key[kSortItems];
    uint32_t rank[kSortItems];
    const size_t base = tile_base + (size_t)warp * (kSortItems * kWarp);
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const size_t idx = base + (size_t)it * kWarp + lane;
        const bool ok = idx < n;
        key[it] = ok ? in[idx] : 0ull;
        rank[it] = 0;
        const unsigned active = __ballot_sync(kFull, ok);
        if (ok) {
            const uint32_t d = (uint32_t)(key[it] >> shift) & (kRadix - 1);
            const unsigned peers = __match_any_sync(active, d);
            const uint32_t old = s_whist[warp][d];
            __syncwarp(active);
            if ((peers & lanemask_lt()) == 0) s_whist[warp][d] = old + __popc(peers);
            __syncwarp(active);
            rank[it] = old + __popc(peers & lanemask_lt());
        }
    }
    __syncthreads();

    // thread t owns digit t: warp-major exclusive offsets and the CTA count of the digit
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t v = s_whist[w][d];
        s_whist[w][d] = run;
        run += v;
    }
    const uint32_t start = cta256_excl_scan(run, s_tmp);
    const uint32_t dbase = cta256_excl_scan(totals[d], s_tmp);
    s_start[d] = start;
    s_gbase[d] = dbase + hist[(size_t)d * ntiles + blockIdx.x];
    __syncthreads();

#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const size_t idx = base + (size_t)it * kWarp + lane;
        if (idx < n) {
            const uint32_t dd = (uint32_t)(key[it] >> shift) & (kRadix - 1);
            s_stage[s_start[dd] + s_whist[warp][dd] + rank[it]] = key[it];
        }
    }
    __syncthreads();

    const size_t rem = n - tile_base;
    const int tile_n = rem < (size_t)kSortTile ? (int)rem : kSortTile;
    for (int k = threadIdx.x; k < tile_n; k += kSortThreads) {
        const uint64_t kk = s_stage[k];
        const uint32_t dd = (uint32_t)(kk >> shift) & (kRadix - 1);
        out[(size_t)s_gbase[dd] + (uint32_t)(k - s_start[dd])] = kk;
    }
}

}  // namespace

size_t radix_scratch_words(size_t n) { return (size_t)kRadix * sort_tiles(n) + kRadix; }

uint64_t* radix_sort_u64(uint64_t* keys, uint64_t* alt, size_t max_n,
                         const unsigned long long* d_count, int lo_bit, int hi_bit,
                         uint32_t* scratch, cudaStream_t s, int* status)
{
    *status = BTC_OK;
    const size_t ntiles = sort_tiles(max_n);
    if (ntiles == 0 || hi_bit <= lo_bit) return keys;
    uint32_t* hist = scratch;
    uint32_t* totals = scratch + (size_t)kRadix * ntiles;
    uint64_t* cur = keys;
    uint64_t* other = alt;
    for (int shift = lo_bit; shift < hi_bit; shift += kRadixBits) {
        k_radix_hist<<<(unsigned)ntiles, kSortThreads, 0, s>>>(cur, d_count, shift, hist,
                                                             (uint32_t)ntiles);
        k_radix_scan<<<kRadix, kScanThreads, 0, s>>>(hist, (uint32_t)ntiles, totals);
        k_radix_scatter<<<(unsigned)ntiles, kSortThreads, 0, s>>>(cur, other, d_count, shift, hist,
                                                                totals, (uint32_t)ntiles);
        uint64_t* t = cur;
        cur = other;
        other = t;
    }
    if (cudaGetLastError() != cudaSuccess) *status = BTC_E_CUDA;
    return cur;
}

}  // namespace btc200
