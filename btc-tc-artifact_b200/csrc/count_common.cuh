// count_common.cuh -- device helpers shared by the count kernels (count.cu, count_rows.cu).
#pragma once

#include "common.cuh"

namespace btc200 {

// global -> shared copies that complete in the background (cp.async, sm_80+); the issuing
// lane waits with cp_async_wait_*, then a __syncwarp publishes the words to the warp.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_pending()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One binary tensor-core MMA: C(16x8, s32) += popc(A(16x128 b1) AND B(128x8 b1)).
__device__ __forceinline__ void mma_b1(int32_t (&c)[4], uint32_t a0, uint32_t a1, uint32_t b0)
{
    asm volatile(
        "mma.sync.aligned.m16n8k128.row.col.s32.b1.b1.s32.and.popc "
        "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
        : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
        : "r"(a0), "r"(a1), "r"(b0));
}

// lower_bound of x in a[0, len)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t len, uint32_t x)
{
    uint32_t lo = 0, hi = len;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Tile geometry of a C-column tile (C = 32 or 128).
template <int C>
struct Cfg {
    static constexpr int WPR = C / 32;       // words per tile row
    static constexpr int TW = 16 * WPR;      // words per tile
    static constexpr int JPT = C / 16;       // 16-row blocks covered by a tile's columns
};

// 16-bit slice j of tile row r.
template <int C>
__device__ __forceinline__ uint32_t slice_of(const uint32_t* S, int r, int j)
{
    constexpr int WPR = Cfg<C>::WPR;
    return (S[r * WPR + ((16 * j) >> 5)] >> ((16 * j) & 31)) & 0xFFFFu;
}

// Adds the warp's partial count to graph g (one atomic per graph change per warp).
// lane 0 keeps the flushed total, so the CTA reduction still sees every unit once.
__device__ __forceinline__ void flush_graph(unsigned long long& acc, unsigned long long& acc_total,
                                            unsigned long long* graph_counts, uint32_t g, int lane)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(kFull, acc, d);
    if (lane == 0 && g != 0xffffffffu) {
        if (acc) atomicAdd(&graph_counts[g], acc);
        acc_total += acc;
    }
    acc = 0;
}

// The graph owning row block I in a batch: the last g with graph_rows[g] <= I.
__device__ __forceinline__ uint32_t graph_of_row_block(const uint32_t* __restrict__ graph_rows,
                                                       uint32_t num_graphs, uint32_t I)
{
    uint32_t lo = 0, hi = num_graphs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (graph_rows[mid] <= I) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Warp-level end of a count launch: per-lane partials -> one uint64 per CTA -> the last
// CTA to finish adds the per-CTA partials and writes the result (no spin-waits: the
// done counter only counts arrivals).  Every thread of the CTA calls it.
template <int kThreadsPerCta>
__device__ __forceinline__ void finish_count(unsigned long long acc, CountScratch scr, bool build_failed,
                                             unsigned long long* s_red, int* s_last)
{
    constexpr int kW = kThreadsPerCta / kWarp;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(kFull, acc, d);
    if (lane == 0) s_red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sum = 0;
        for (int w = 0; w < kW; ++w) sum += s_red[w];
        scr.partials[blockIdx.x] = sum;
        __threadfence();
        const unsigned prev = atomicAdd(scr.done, 1u);
        *s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (*s_last) {
        __threadfence();
        unsigned long long sum = 0;
        for (uint32_t i = threadIdx.x; i < gridDim.x; i += kThreadsPerCta) sum += __ldcg(&scr.partials[i]);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_down_sync(kFull, sum, d);
        if (lane == 0) s_red[warp] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long total = 0;
            for (int w = 0; w < kW; ++w) total += s_red[w];
            if (build_failed) total = ~0ull;
            *scr.result = total;
            if (scr.result2) *scr.result2 = total;
            if (scr.result_host) {
                *reinterpret_cast<volatile unsigned long long*>(scr.result_host) = total;
                __threadfence_system();
            }
            *scr.done = 0u;
            *scr.work = 0ull;
        }
    }
}

// Resident CTAs per SM of the row-wise kernel (count_rows.cu); 0 on error.
int rows_blocks_per_sm(int tile_cols);

// The row-wise count kernel (count_rows.cu), launched by launch_count for heavy graphs.
int launch_count_rows(int tile_cols, const uint32_t* indptr, const uint32_t* indices,
                      const uint32_t* row_indices, const uint32_t* blocks, uint32_t num_tiles,
                      uint32_t tile_begin, uint32_t tile_end, int32_t n_row_blocks, int tau,
                      uint32_t chunk, CountScratch scr, const uint32_t* graph_rows,
                      uint32_t num_graphs, unsigned long long* graph_counts,
                      const uint32_t* rowmask, const uint2* cellpp, uint64_t cell_wpr,
                      const uint32_t* row_off, const uint2* row_ent, const GraphSeg* segs,
                      const unsigned long long* build_meta, bool dense, int grid, cudaStream_t s);

}  // namespace btc200
