// rowindex.cu -- per-vertex lists of the tiles that hold each tile row (the row-wise count
// kernel's index; no counterpart in the reference).
//
// For vertex u = 16 I + r (row r of row block I) the list holds, in tile order (which is
// column-block order), one entry (K, t) per tile t = (I, K) of row block I whose row r
// has a bit: the column blocks u has lower neighbours in.  All lists sit in one array in
// vertex order; vertex u's list is ent[off[u], off[u+1]).  Entries number at most the
// unique edges (every listed tile row holds at least one edge), so the caller sizes ent
// by the input edge count.  Built from the per-tile row-occupancy masks, when they exist
// (row blocks averaging 8 or more tiles), in three steps:
//   k_ri_totals   one warp per row block: popcount of its tiles' masks
//   scan          exclusive prefix of the totals (per-CTA reduce, one-CTA scan of the
//                 CTA sums, per-CTA down-sweep)
//   k_ri_fill     one warp per row block: per-row counts (16 ballots per 32 tiles), the
//                 rows' list starts, then the entries
#include "common.cuh"

#include <algorithm>

namespace btc200 {

int launch_tile_scan(uint32_t* per_tile, uint32_t ntiles, unsigned long long* total, cudaStream_t s);

namespace ri {

constexpr int kThreads = 256;
constexpr int kScanItems = 16;                       // items per thread in the scan
constexpr uint32_t kScanTile = kThreads * kScanItems;  // 4096 items per CTA

// The index exists only when the masks do: T tiles (device count, bounded by cap) and
// T >= 8 R.
__device__ __forceinline__ bool index_wanted(const unsigned long long* d_tiles, uint32_t cap, uint32_t R,
                                             uint32_t& T)
{
    const unsigned long long t = d_tiles ? *d_tiles : cap;
    if (t > cap) return false;
    T = (uint32_t)t;
    return (uint64_t)T >= 8ull * (uint64_t)R;
}

__global__ void k_ri_totals(const uint32_t* __restrict__ indptr, uint32_t R,
                            const uint32_t* __restrict__ rowmask,
                            const unsigned long long* __restrict__ d_tiles, uint32_t cap,
                            uint32_t* __restrict__ tot)
{
    uint32_t T;
    if (!index_wanted(d_tiles, cap, R, T)) return;
    const int lane = threadIdx.x & 31;
    const uint64_t nw = (uint64_t)gridDim.x * (kThreads / kWarp);
    for (uint64_t I = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / kWarp; I < R; I += nw) {
        const uint32_t a = indptr[I], b = indptr[I + 1];
        uint32_t sum = 0;
        for (uint32_t t = a + lane; t < b; t += kWarp) sum += __popc(rowmask[t]);
        sum = __reduce_add_sync(kFull, sum);
        if (lane == 0) tot[I] = sum;
    }
}

__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    total = 0;
    for (int w = 0; w < kThreads / kWarp; ++w) {
        const uint32_t x = s_warp[w];
        if (w < warp) wbase += x;
        total += x;
    }
    __syncthreads();
    return wbase + incl - v;
}

// CTA c: sum of items [c*kScanTile, (c+1)*kScanTile) -> bsum[c]
__global__ void k_scan_reduce(const uint32_t* __restrict__ v, uint32_t n, uint32_t* __restrict__ bsum)
{
    __shared__ uint32_t s_warp[kThreads / kWarp];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint64_t i = base + (uint64_t)k * kThreads + threadIdx.x;
        if (i < n) sum += v[i];
    }
    uint32_t total;
    cta_exclusive_scan(sum, s_warp, total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// in place: v[i] = bsum[c] + exclusive prefix of v within CTA c (bsum already scanned)
__global__ void k_scan_apply(uint32_t* __restrict__ v, uint32_t n, const uint32_t* __restrict__ bsum)
{
    __shared__ uint32_t s_warp[kThreads / kWarp];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t x[kScanItems], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint64_t i = base + k;
        x[k] = i < n ? v[i] : 0u;
        sum += x[k];
    }
    uint32_t total;
    uint32_t run = bsum[blockIdx.x] + cta_exclusive_scan(sum, s_warp, total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint64_t i = base + k;
        if (i < n) v[i] = run;
        run += x[k];
    }
}

__global__ void k_ri_fill(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                          uint32_t R, const uint32_t* __restrict__ rowmask,
                          const unsigned long long* __restrict__ d_tiles, uint32_t cap,
                          const uint32_t* __restrict__ base_of, const unsigned long long* __restrict__ total,
                          uint32_t* __restrict__ off, uint2* __restrict__ ent, uint64_t ent_cap)
{
    uint32_t T;
    if (!index_wanted(d_tiles, cap, R, T)) return;
    if (*total > ent_cap) return;  // cannot happen: entries <= unique edges <= ent_cap
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const uint64_t nw = (uint64_t)gridDim.x * (kThreads / kWarp);
    for (uint64_t I = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / kWarp; I < R; I += nw) {
        const uint32_t a = indptr[I], b = indptr[I + 1];
        // per-row counts: lane r < 16 holds row r's.  Each lane's 16-bit mask is spread
        // four rows to a word, one row per byte (a nibble times 0x00204081 puts its bit j
        // at bit 8j), and one warp add per word sums four rows over the round's 32 tiles
        // (at most 32 per byte, so no byte carries into the next): 4 adds where one
        // ballot per row took 16.
        uint32_t cnt = 0;
        for (uint32_t t0 = a; t0 < b; t0 += kWarp) {
            const uint32_t m = t0 + lane < b ? rowmask[t0 + lane] : 0u;
            uint32_t q[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                q[k] = __reduce_add_sync(kFull, (((m >> (4 * k)) & 0xFu) * 0x00204081u) & 0x01010101u);
            const uint32_t g = (uint32_t)lane >> 2;  // lane r's word
            const uint32_t w = g == 0 ? q[0] : g == 1 ? q[1] : g == 2 ? q[2] : q[3];
            if (lane < 16) cnt += (w >> (8 * (lane & 3))) & 0xFFu;
        }
        uint32_t incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += y;
        }
        uint32_t start = base_of[I] + incl - cnt;  // lane r: start of row r's list
        if (lane < 16) off[16 * I + lane] = start;
        if (I + 1 == R && lane == 16) off[16 * (uint64_t)R] = start;  // = the entry total
        for (uint32_t t0 = a; t0 < b; t0 += kWarp) {
            const uint32_t t = t0 + lane;
            const uint32_t m = t < b ? rowmask[t] : 0u;
            const uint32_t K = t < b ? indices[t] : 0u;
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const bool has = (m >> r) & 1u;
                const unsigned bl = __ballot_sync(kFull, has);
                const uint32_t br = __shfl_sync(kFull, start, r);
                if (has) ent[br + __popc(bl & lt)] = make_uint2(K, t);
                if (lane == r) start += __popc(bl);
            }
        }
    }
}

}  // namespace ri

// Enqueues the row index of a Bit-BSR whose row masks were just built (see above).
// tot: R + 1 words of scratch; bsum: ri_scan_blocks(R) + 1 words; total: one uint64.
// off: 16 R + 1 words; ent: ent_cap entries.  d_tiles / cap as for launch_rowmask.
uint32_t ri_scan_blocks(uint32_t R) { return (R + ri::kScanTile - 1) / ri::kScanTile; }

int launch_rowindex(const uint32_t* indptr, const uint32_t* indices, int32_t n_row_blocks,
                    const uint32_t* rowmask, const unsigned long long* d_tiles, uint32_t cap,
                    uint32_t* tot, uint32_t* bsum, unsigned long long* total, uint32_t* off,
                    uint2* ent, uint64_t ent_cap, cudaStream_t s)
{
    const uint32_t R = n_row_blocks > 0 ? (uint32_t)n_row_blocks : 0u;
    if (R == 0) return BTC_OK;
    const int wgrid = (int)std::min<uint64_t>((R + 7) / 8, (uint64_t)device_sm_count() * 16);
    ri::k_ri_totals<<<wgrid, ri::kThreads, 0, s>>>(indptr, R, rowmask, d_tiles, cap, tot);
    const uint32_t nb = ri_scan_blocks(R);
    ri::k_scan_reduce<<<nb, ri::kThreads, 0, s>>>(tot, R, bsum);
    BTC_TRY(launch_tile_scan(bsum, nb, total, s));
    ri::k_scan_apply<<<nb, ri::kThreads, 0, s>>>(tot, R, bsum);
    ri::k_ri_fill<<<wgrid, ri::kThreads, 0, s>>>(indptr, indices, R, rowmask, d_tiles, cap, tot, total,
                                                 off, ent, ent_cap);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

}  // namespace btc200
