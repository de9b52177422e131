// count.cu -- hybrid exact triangle count over a Bit-BSR (16x128 or 16x32 tiles).
//
// Computes what btc/operations/tc_16x128_mma_v5.h:9-211 and tc_16x32_mma_v6.h:9-238
// compute: for every sample tile S = (I, J_L) of L and every 16-row block J_out whose
// rows are a 16-column slice j of S, for every column block K present in both row
// block I and row block J_out,
//      sum over set bits (r, c) of slice j of S of popc(L[I,K][r] & L[J_out,K][c]).
// Integer arithmetic only; per-lane uint64 partials, one uint64 per CTA, and the last
// CTA to finish adds the per-CTA partials (no floating point, no spin-waits).
//
// Work mapping (one warp per sample tile, persistent grid-stride over tiles):
//  * S is loaded once (one 8-byte load per lane for 16x128); its popcount picks the
//    path: > tau -> binary tensor core, else CUDA cores.
//  * The row blocks J_out = J_L*(C/16) + j are consecutive, so their index lists form
//    one contiguous run of indices[]; the warp searches every element of the lists of
//    the slices that have bits (32 at a time, one per lane) in row block I's list,
//    which is staged in shared memory when short.  This replaces the reference's
//    serial two-pointer merge, repeated per slice by all 32 lanes, with one parallel
//    search per tile.
//  * Sparse path: matches of a round are compacted; (match, mask bit) units are spread
//    over the lanes; each unit is one 16-byte AND + 4 popc (16x128) or one word (16x32).
//  * Dense path: per slice, every match feeds mma.sync.m16n8k128.row.col.s32.b1.b1.s32
//    .and.popc twice (16x16 popcount block), masked by the slice's bits.  16x32 tiles
//    pack four matches into the 128-bit k dimension, as tc_16x32_mma_v6.h:72-154 does.
#include "common.cuh"

namespace btc200 {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / kWarp;
constexpr int kACap = 256;  // row-block list entries staged in shared memory per warp

template <int C>
struct Cfg {
    static constexpr int WPR = C / 32;       // words per tile row
    static constexpr int TW = 16 * WPR;      // words per tile
    static constexpr int JPT = C / 16;       // 16-row blocks covered by a tile's columns
    static constexpr int MAXBITS = 16 * C;   // bits per tile
};

template <int C>
struct __align__(16) WarpSmem {
    uint32_t S[Cfg<C>::TW];
    uint32_t alist[kACap];
    uint32_t jptr[Cfg<C>::JPT + 1];
    uint32_t boff[Cfg<C>::JPT + 1];
    uint32_t mpa[kWarp];
    uint32_t mpb[kWarp];
    uint32_t mpre[kWarp + 1];
    uint8_t mj[kWarp];
    uint8_t bits[Cfg<C>::MAXBITS];
};

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

// 16-bit slice j of tile row r.
template <int C>
__device__ __forceinline__ uint32_t slice_of(const uint32_t* S, int r, int j)
{
    constexpr int WPR = Cfg<C>::WPR;
    return (S[r * WPR + ((16 * j) >> 5)] >> ((16 * j) & 31)) & 0xFFFFu;
}

template <int C>
__global__ void __launch_bounds__(kThreads)
k_count(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
        const uint32_t* __restrict__ row_indices, const uint32_t* __restrict__ blocks,
        uint32_t num_tiles, int32_t R, int tau, CountScratch scr)
{
    using K = Cfg<C>;
    constexpr int WPR = K::WPR, TW = K::TW, JPT = K::JPT;
    __shared__ WarpSmem<C> smem_all[kWarps];
    __shared__ unsigned long long s_red[kWarps];
    __shared__ int s_last;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpSmem<C>& s = smem_all[warp];
    const unsigned lt = lanemask_lt();
    const int g = lane >> 2, tg = lane & 3;  // mma fragment coordinates

    unsigned long long acc = 0;

    for (uint64_t t = (uint64_t)blockIdx.x * kWarps + warp; t < num_tiles;
         t += (uint64_t)gridDim.x * kWarps) {
        const uint32_t I = row_indices[t];
        const uint32_t JL = indices[t];

        // ---- sample tile and its slices -------------------------------------
        uint32_t w0 = 0, w1 = 0;
        if constexpr (C == 128) {
            const uint2 v = reinterpret_cast<const uint2*>(blocks + (size_t)t * TW)[lane];
            w0 = v.x;
            w1 = v.y;
            s.S[2 * lane] = w0;
            s.S[2 * lane + 1] = w1;
        } else {
            if (lane < 16) {
                w0 = blocks[(size_t)t * TW + lane];
                s.S[lane] = w0;
            }
        }
        const int nnz = (int)__reduce_add_sync(kFull, (unsigned)(__popc(w0) + __popc(w1)));

        // per-lane slice popcounts, packed 16 bits per slice
        // 16x128: lane = 2r + h holds slices j = 4h + q (q = 0..3) of row r
        // 16x32 : lane = r (< 16) holds slices j = q (q = 0..1) of row r
        uint32_t p[4];
        p[0] = __popc(w0 & 0xFFFFu);
        p[1] = __popc(w0 >> 16);
        p[2] = __popc(w1 & 0xFFFFu);
        p[3] = __popc(w1 >> 16);

        uint32_t active = 0;  // bit j set if slice j has any bit
        if constexpr (C == 128) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const unsigned b = __ballot_sync(kFull, p[q] != 0);
                if (b & 0x55555555u) active |= 1u << q;
                if (b & 0xAAAAAAAAu) active |= 1u << (4 + q);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 2; ++q)
                if (__ballot_sync(kFull, p[q] != 0)) active |= 1u << q;
        }

        const uint32_t startI = indptr[I];
        const uint32_t LA = indptr[I + 1] - startI;
        if (lane <= JPT) {
            const int64_t J = (int64_t)JL * JPT + lane;
            s.jptr[lane] = indptr[J < R ? J : R];
        }
        const bool stageA = LA <= (uint32_t)kACap;
        if (stageA)
            for (uint32_t i = lane; i < LA; i += kWarp) s.alist[i] = indices[startI + i];
        __syncwarp();

        // unit prefix over active slices
        uint32_t upre[JPT + 1];
        upre[0] = 0;
#pragma unroll
        for (int j = 0; j < JPT; ++j)
            upre[j + 1] = upre[j] + (((active >> j) & 1u) ? (s.jptr[j + 1] - s.jptr[j]) : 0u);

        if (nnz <= tau) {
            // ================= sparse path ===================================
            // bit list grouped by slice, then row, then column
            uint32_t excl[4] = {0, 0, 0, 0};
            uint32_t tot[JPT];
            if constexpr (C == 128) {
                unsigned long long x = (unsigned long long)p[0] | ((unsigned long long)p[1] << 16) |
                                       ((unsigned long long)p[2] << 32) |
                                       ((unsigned long long)p[3] << 48);
                const unsigned long long own = x;
#pragma unroll
                for (int d = 2; d < 32; d <<= 1) {
                    const unsigned long long y = __shfl_up_sync(kFull, x, d);
                    if (lane >= d) x += y;
                }
                const unsigned long long e = x - own;
                const unsigned long long t0 = __shfl_sync(kFull, x, 30);
                const unsigned long long t1 = __shfl_sync(kFull, x, 31);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    excl[q] = (uint32_t)(e >> (16 * q)) & 0xFFFFu;
                    tot[q] = (uint32_t)(t0 >> (16 * q)) & 0xFFFFu;
                    tot[4 + q] = (uint32_t)(t1 >> (16 * q)) & 0xFFFFu;
                }
            } else {
                uint32_t x = (lane < 16) ? (p[0] | (p[1] << 16)) : 0u;
                const uint32_t own = x;
#pragma unroll
                for (int d = 1; d < 16; d <<= 1) {
                    const uint32_t y = __shfl_up_sync(kFull, x, d);
                    if (lane >= d) x += y;
                }
                const uint32_t e = x - own;
                const uint32_t t15 = __shfl_sync(kFull, x, 15);
                excl[0] = e & 0xFFFFu;
                excl[1] = e >> 16;
                tot[0] = t15 & 0xFFFFu;
                tot[1] = t15 >> 16;
            }
            uint32_t boff[JPT + 1];
            boff[0] = 0;
#pragma unroll
            for (int j = 0; j < JPT; ++j) boff[j + 1] = boff[j] + tot[j];
            if (lane <= JPT) {
#pragma unroll
                for (int j = 0; j <= JPT; ++j)
                    if (lane == j) s.boff[j] = boff[j];
            }
            // write this lane's slices' bits
            if constexpr (C == 128) {
                const int r = lane >> 1, h = lane & 1;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t sl = ((q < 2 ? w0 : w1) >> (16 * (q & 1))) & 0xFFFFu;
                    uint32_t pos = (h ? boff[4 + q] : boff[q]) + excl[q];
                    while (sl) {
                        const int c = __ffs(sl) - 1;
                        sl &= sl - 1;
                        s.bits[pos++] = (uint8_t)((r << 4) | c);
                    }
                }
            } else if (lane < 16) {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    uint32_t sl = (w0 >> (16 * q)) & 0xFFFFu;
                    uint32_t pos = boff[q] + excl[q];
                    while (sl) {
                        const int c = __ffs(sl) - 1;
                        sl &= sl - 1;
                        s.bits[pos++] = (uint8_t)((lane << 4) | c);
                    }
                }
            }
            __syncwarp();

            const uint32_t W = upre[JPT];
            for (uint32_t ub = 0; ub < W; ub += kWarp) {
                const uint32_t u = ub + lane;
                bool found = false;
                uint32_t pa = 0, pb = 0;
                int jj = 0;
                if (u < W) {
                    uint32_t ustart = 0;
#pragma unroll
                    for (int j = 1; j < JPT; ++j)
                        if (u >= upre[j]) {
                            jj = j;
                            ustart = upre[j];
                        }
                    pb = s.jptr[jj] + (u - ustart);
                    const uint32_t b = indices[pb];
                    uint32_t pos;
                    if (stageA) {
                        pos = lower_bound_u32(s.alist, LA, b);
                        found = pos < LA && s.alist[pos] == b;
                    } else {
                        pos = lower_bound_u32(indices + startI, LA, b);
                        found = pos < LA && indices[startI + pos] == b;
                    }
                    pa = startI + pos;
                }
                const unsigned mb = __ballot_sync(kFull, found);
                if (mb == 0) continue;
                const int nm = __popc(mb);
                uint32_t cnt = 0;
                if (found) {
                    const int k = __popc(mb & lt);
                    s.mpa[k] = pa;
                    s.mpb[k] = pb;
                    s.mj[k] = (uint8_t)jj;
                }
                __syncwarp();
                if (lane < nm) {
                    const int j = s.mj[lane];
                    cnt = s.boff[j + 1] - s.boff[j];
                }
                uint32_t incl = cnt;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t y = __shfl_up_sync(kFull, incl, d);
                    if (lane >= d) incl += y;
                }
                if (lane < nm) s.mpre[lane] = incl - cnt;
                const uint32_t U = __shfl_sync(kFull, incl, 31);
                if (lane == 0) s.mpre[nm] = U;
                __syncwarp();
                for (uint32_t v = lane; v < U; v += kWarp) {
                    // match k: last k with mpre[k] <= v
                    uint32_t lo = 0, hi = (uint32_t)nm;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (s.mpre[mid] <= v) lo = mid;
                        else hi = mid;
                    }
                    const int j = s.mj[lo];
                    const uint32_t code = s.bits[s.boff[j] + (v - s.mpre[lo])];
                    const uint32_t r = code >> 4, c = code & 15u;
                    const uint32_t* A = blocks + (size_t)s.mpa[lo] * TW + r * WPR;
                    const uint32_t* Bq = blocks + (size_t)s.mpb[lo] * TW + c * WPR;
                    if constexpr (C == 128) {
                        const uint4 a = *reinterpret_cast<const uint4*>(A);
                        const uint4 b = *reinterpret_cast<const uint4*>(Bq);
                        acc += (unsigned)(__popc(a.x & b.x) + __popc(a.y & b.y) +
                                          __popc(a.z & b.z) + __popc(a.w & b.w));
                    } else {
                        acc += (unsigned)__popc(A[0] & Bq[0]);
                    }
                }
                __syncwarp();
            }
        } else {
            // ================= dense path: binary tensor core ================
            for (int j = 0; j < JPT; ++j) {
                if (!((active >> j) & 1u)) continue;
                int32_t c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
                const uint32_t jb = s.jptr[j], je = s.jptr[j + 1];
                for (uint32_t ub = jb; ub < je; ub += kWarp) {
                    const uint32_t u = ub + lane;
                    bool found = false;
                    uint32_t pa = 0, pb = 0;
                    if (u < je) {
                        pb = u;
                        const uint32_t b = indices[pb];
                        uint32_t pos;
                        if (stageA) {
                            pos = lower_bound_u32(s.alist, LA, b);
                            found = pos < LA && s.alist[pos] == b;
                        } else {
                            pos = lower_bound_u32(indices + startI, LA, b);
                            found = pos < LA && indices[startI + pos] == b;
                        }
                        pa = startI + pos;
                    }
                    const unsigned mb = __ballot_sync(kFull, found);
                    if (mb == 0) continue;
                    const int nm = __popc(mb);
                    if (found) {
                        const int k = __popc(mb & lt);
                        s.mpa[k] = pa;
                        s.mpb[k] = pb;
                    }
                    __syncwarp();
                    if constexpr (C == 128) {
                        for (int k = 0; k < nm; ++k) {
                            const uint32_t* A = blocks + (size_t)s.mpa[k] * TW;
                            const uint32_t* Bt = blocks + (size_t)s.mpb[k] * TW;
                            const uint32_t a0 = A[g * WPR + tg], a1 = A[(g + 8) * WPR + tg];
                            const uint32_t b0 = Bt[g * WPR + tg], b1 = Bt[(g + 8) * WPR + tg];
                            mma_b1(c0, a0, a1, b0);
                            mma_b1(c1, a0, a1, b1);
                        }
                    } else {
                        for (int k0 = 0; k0 < nm; k0 += 4) {
                            const int k = k0 + tg;
                            uint32_t a0 = 0, a1 = 0, b0 = 0, b1 = 0;
                            if (k < nm) {
                                const uint32_t* A = blocks + (size_t)s.mpa[k] * TW;
                                const uint32_t* Bt = blocks + (size_t)s.mpb[k] * TW;
                                a0 = A[g];
                                a1 = A[g + 8];
                                b0 = Bt[g];
                                b1 = Bt[g + 8];
                            }
                            mma_b1(c0, a0, a1, b0);
                            mma_b1(c1, a0, a1, b1);
                        }
                    }
                    __syncwarp();
                }
                // mask: C[row][col] counts only where slice j of S has bit (row, col)
                const uint32_t sg = slice_of<C>(s.S, g, j), sg8 = slice_of<C>(s.S, g + 8, j);
                const int c = 2 * tg;
                long long part = 0;
                part += ((sg >> c) & 1u) ? c0[0] : 0;
                part += ((sg >> (c + 1)) & 1u) ? c0[1] : 0;
                part += ((sg8 >> c) & 1u) ? c0[2] : 0;
                part += ((sg8 >> (c + 1)) & 1u) ? c0[3] : 0;
                part += ((sg >> (c + 8)) & 1u) ? c1[0] : 0;
                part += ((sg >> (c + 9)) & 1u) ? c1[1] : 0;
                part += ((sg8 >> (c + 8)) & 1u) ? c1[2] : 0;
                part += ((sg8 >> (c + 9)) & 1u) ? c1[3] : 0;
                acc += (unsigned long long)part;
            }
        }
        __syncwarp();
    }

    // ---- int64 block tree + last-CTA reduction ------------------------------
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(kFull, acc, d);
    if (lane == 0) s_red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sum = 0;
        for (int w = 0; w < kWarps; ++w) sum += s_red[w];
        scr.partials[blockIdx.x] = sum;
        __threadfence();
        const unsigned prev = atomicAdd(scr.done, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        unsigned long long sum = 0;
        for (uint32_t i = threadIdx.x; i < gridDim.x; i += kThreads) sum += __ldcg(&scr.partials[i]);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_down_sync(kFull, sum, d);
        if (lane == 0) s_red[warp] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long total = 0;
            for (int w = 0; w < kWarps; ++w) total += s_red[w];
            *scr.result = total;
            if (scr.result2) *scr.result2 = total;
            *scr.done = 0u;
        }
    }
}

}  // namespace

int count_grid_size(int tile_cols)
{
    int per_sm = 0;
    cudaError_t e;
    if (tile_cols == 128)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_count<128>, kThreads, 0);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_count<32>, kThreads, 0);
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    return per_sm * device_sm_count();
}

int launch_count(int tile_cols, const uint32_t* indptr, const uint32_t* indices,
                 const uint32_t* row_indices, const uint32_t* blocks, uint32_t num_tiles,
                 int32_t n_row_blocks, int tau, CountScratch scr, cudaStream_t s)
{
    const int grid = count_grid_size(tile_cols);
    if (tile_cols == 128)
        k_count<128><<<grid, kThreads, 0, s>>>(indptr, indices, row_indices, blocks, num_tiles,
                                               n_row_blocks, tau, scr);
    else
        k_count<32><<<grid, kThreads, 0, s>>>(indptr, indices, row_indices, blocks, num_tiles,
                                              n_row_blocks, tau, scr);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

}  // namespace btc200
