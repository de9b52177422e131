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
// Work mapping (persistent grid; each warp takes runs of consecutive tiles from a
// global queue, so the tiles of one row block usually stay with one warp):
//  * Row block I's column-block list is staged once per row block, as a shared-memory
//    bitmap with per-word prefix counts (membership and rank in O(1)) when its column
//    blocks span at most 8192, else as a sorted list (binary search).
//  * S is loaded once (one 8-byte load per lane for 16x128); its popcount picks the
//    path: > tau -> binary tensor core, else CUDA cores.
//  * The row blocks J_out = J_L*(C/16) + j are consecutive, so their index lists form
//    one contiguous run of indices[]; the warp looks up every element of the lists of
//    the slices that have bits (32 per round, one per lane) in row block I's structure.
//    This replaces the reference's serial two-pointer merge, repeated per slice by all
//    32 lanes, with one parallel search per tile.
//  * Optional per-tile row-occupancy masks (bit r: tile row r has a bit) drop matches
//    whose I tile has no occupied row among S's rows of the slice, or whose J_out tile
//    has none among its columns, and skip units with an empty row on either side before
//    any tile row is read.  On power-law graphs most matches are such empty pairs.
//  * When the Bit-BSR came from the cell-bitmap builder, each slice is searched in the
//    cheaper direction: J_out's list elements looked up in row block I's structure, or
//    the elements of I's list that fall inside J_out's column span looked up in J_out's
//    (row block, column block) cell-bitmap row, ranked with the builder's per-word tile
//    prefix.  On degree-ordered power-law graphs J_out is usually a hub block whose span
//    holds few of I's elements.
//  * Sparse path: matches are appended in slice order (slice j owns entries
//    [mc[j], mc[j+1])).  Each set bit (r, c) of S then adds popc(L[I,K][r] & L[J_out,K][c])
//    over its slice's matches, with the lanes spread over bits (many bits, few matches:
//    stencils) or over the matches of one bit at a time (few bits, many matches:
//    Erdos-Renyi, R-MAT).  One unit is one 16-byte AND + 4 popc (16x128) or one word.
//  * Dense path: per slice, every match feeds mma.sync.m16n8k128.row.col.s32.b1.b1.s32
//    .and.popc twice (16x16 popcount block), masked by the slice's bits.  16x32 tiles
//    pack four matches into the 128-bit k dimension, as tc_16x32_mma_v6.h:72-154 does.
#include "count_common.cuh"

#include <cstddef>
#include <cstdlib>

#include <atomic>

namespace btc200 {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / kWarp;
constexpr int kACap = 256;     // list mode: row-block list entries staged per warp
constexpr int kSmallList = 16; // lists this short are staged as lists, not bitmaps
constexpr int kBmWords = 256;  // bitmap mode: graphs with at most 8192 column blocks
constexpr int kMCap = 64;      // matches buffered per warp before a bit pass
constexpr int kBCap = 512;     // mask-bit codes buffered per warp per bit pass

template <int C>
struct __align__(16) WarpSmem {
    uint32_t S[Cfg<C>::TW];          // sample tile (dense path)
    uint32_t nS[Cfg<C>::TW];         // the next tile's sample words (cp.async prefetch; 8-byte
                                     // copies, so it sits at a 16-byte-aligned offset)
    union {
        uint32_t list[kACap];        // row block I's column blocks (list mode)
        uint32_t bm[kBmWords];       // the same as a bitmap (bitmap mode)
    } a;
    uint16_t apre[kBmWords];         // bitmap mode: list entries below each word
    uint32_t jptr[Cfg<C>::JPT + 1];  // indptr of the row blocks J_out of this tile
    uint32_t upre[Cfg<C>::JPT + 1];  // search-unit prefix over active slices
    uint32_t mc[Cfg<C>::JPT + 1];    // match-list start of each slice
    uint32_t mpa[kMCap];             // matched tile of row block I
    uint32_t mpb[kMCap];             // matched tile of row block J_out
    uint16_t mra[kMCap];             // occupied rows of the matched I tile
    uint16_t mrb[kMCap];             // occupied rows of the matched J_out tile
    uint32_t sstart[Cfg<C>::JPT];    // search list start of slice j (tile index)
    uint8_t sdir[Cfg<C>::JPT];       // 0: J_out's list searched in I; 1: I's list in J_out
    uint16_t rmask[Cfg<C>::JPT];     // rows of S with bits in slice j
    uint16_t cmask[Cfg<C>::JPT];     // columns (rows of J_out tiles) with bits in slice j
    uint16_t bits[kBCap];            // (row << 8) | column of the sample tile's set bits
};
static_assert(offsetof(WarpSmem<128>, nS) % 16 == 0 && offsetof(WarpSmem<32>, nS) % 16 == 0,
              "cp.async destinations must be aligned to the copy size");
static_assert(sizeof(WarpSmem<128>) % 16 == 0 && sizeof(WarpSmem<32>) % 16 == 0,
              "per-warp areas keep the 16-byte alignment of the first one");

// Row block I's column-block list as the search structure of the current tile.
struct ARow {
    uint32_t start;  // indptr[I]
    uint32_t len;    // number of tiles in row block I
    uint32_t last;   // last column block of row block I
    uint32_t base;   // bitmap mode: first column block of the bitmap (multiple of 32)
    uint32_t words;  // bitmap mode: bitmap words in use
    int mode;        // 0: sorted list in shared memory, 1: bitmap, 2: sorted list in HBM
};

// Bits 0, 2, 4, ... 30 of x, packed into bits 0..15.
__device__ __forceinline__ uint32_t compress_even(uint32_t x)
{
    x &= 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
    x = (x | (x >> 4)) & 0x00FF00FFu;
    x = (x | (x >> 8)) & 0x0000FFFFu;
    return x;
}

// Stages row block I's column-block list for lookups.  Called with the warp converged.
// The bitmap spans the row block's own column-block range, so it is used whenever
// that range is at most kBmWords * 32 column blocks wide.
template <int C>
__device__ __forceinline__ ARow stage_row(WarpSmem<C>& s, const uint32_t* __restrict__ indices,
                                          uint32_t start, uint32_t len, int lane)
{
    ARow A;
    A.start = start;
    A.len = len;  // >= 1: a tile of row block I is being counted
    A.base = indices[A.start] & ~31u;
    A.last = indices[A.start + A.len - 1];
    A.words = ((A.last - A.base) >> 5) + 1;
    __syncwarp();  // earlier readers of s.a / s.apre are done
    if (A.len <= (uint32_t)kSmallList) {
        // a short list (meshes: a few tiles per row block) is staged as it is, one element
        // per lane, and searched by bisection: cheaper than building a bitmap per tile run
        A.mode = 0;
        if ((uint32_t)lane < A.len) s.a.list[lane] = indices[A.start + lane];
    } else if (A.words <= (uint32_t)kBmWords) {
        A.mode = 1;
        for (uint32_t w = lane; w < A.words; w += kWarp) s.a.bm[w] = 0u;
        __syncwarp();
        for (uint32_t i = lane; i < A.len; i += kWarp) {
            const uint32_t k = indices[A.start + i] - A.base;
            atomicOr(&s.a.bm[k >> 5], 1u << (k & 31u));
        }
        __syncwarp();
        // per-word exclusive prefix; lane owns words [8*lane, 8*lane + 8)
        uint32_t cnt[8], tot = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t w = 8u * lane + q;
            cnt[q] = w < A.words ? __popc(s.a.bm[w]) : 0u;
            tot += cnt[q];
        }
        uint32_t incl = tot;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += y;
        }
        uint32_t run = incl - tot;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t w = 8u * lane + q;
            if (w < A.words) s.apre[w] = (uint16_t)run;
            run += cnt[q];
        }
    } else if (A.len <= (uint32_t)kACap) {
        A.mode = 0;
        for (uint32_t i = lane; i < A.len; i += kWarp) s.a.list[i] = indices[A.start + i];
    } else {
        A.mode = 2;
    }
    __syncwarp();
    return A;
}

// Is column block b in row block I?  If so, pa = its tile index.
template <int C>
__device__ __forceinline__ bool a_lookup(const WarpSmem<C>& s, const ARow& A,
                                         const uint32_t* __restrict__ indices, uint32_t b,
                                         uint32_t& pa)
{
    if (A.mode == 1) {
        if (b < A.base) return false;
        const uint32_t w = (b - A.base) >> 5;
        if (w >= A.words) return false;
        const uint32_t x = s.a.bm[w];
        const uint32_t bit = 1u << (b & 31u);
        if (!(x & bit)) return false;
        pa = A.start + s.apre[w] + __popc(x & (bit - 1u));
        return true;
    }
    if (A.mode == 0) {
        const uint32_t pos = lower_bound_u32(s.a.list, A.len, b);
        pa = A.start + pos;
        return pos < A.len && s.a.list[pos] == b;
    }
    const uint32_t pos = lower_bound_u32(indices + A.start, A.len, b);
    pa = A.start + pos;
    return pos < A.len && indices[A.start + pos] == b;
}

// Number of elements of row block I's list below column block x.
template <int C>
__device__ __forceinline__ uint32_t a_rank(const WarpSmem<C>& s, const ARow& A,
                                           const uint32_t* __restrict__ indices, uint32_t x)
{
    if (A.mode == 1) {
        if (x <= A.base) return 0;
        const uint32_t w = (x - A.base) >> 5;
        if (w >= A.words) return A.len;
        return s.apre[w] + __popc(s.a.bm[w] & ((1u << ((x - A.base) & 31u)) - 1u));
    }
    if (A.mode == 0) return lower_bound_u32(s.a.list, A.len, x);
    return lower_bound_u32(indices + A.start, A.len, x);
}

// One bit pass: every set bit (r, col) of the sample tile, one per lane, adds
// popc(L[I,K][r] & L[J_out,K][col % 16]) over the buffered matches K of its slice
// j = col / 16, i.e. match-list entries [mc[j], mc[j+1]) clipped to [lo, hi).
template <int C, bool kHeavy>
__device__ __forceinline__ unsigned long long bit_pass(WarpSmem<C>& s, uint32_t w0, uint32_t w1,
                                                       uint32_t e, uint32_t nnz, uint32_t lo,
                                                       uint32_t hi,
                                                       const uint32_t* __restrict__ blocks,
                                                       int lane)
{
    constexpr int WPR = Cfg<C>::WPR, TW = Cfg<C>::TW;
    unsigned long long acc = 0;
    for (uint32_t bb = 0; bb < nnz; bb += kBCap) {
        uint32_t idx = e;
#pragma unroll
        for (int q = 0; q < (C == 128 ? 2 : 1); ++q) {
            uint32_t x = q == 0 ? w0 : w1;
            while (x) {
                const uint32_t b = __ffs(x) - 1;
                x &= x - 1;
                if (idx - bb < (uint32_t)kBCap) {
                    uint32_t r, col;
                    if constexpr (C == 128) {
                        r = lane >> 1;
                        col = 64u * (lane & 1) + 32u * q + b;
                    } else {
                        r = lane;
                        col = b;
                    }
                    s.bits[idx - bb] = (uint16_t)((r << 8) | col);
                }
                ++idx;
            }
        }
        __syncwarp();
        const uint32_t nb = min((uint32_t)kBCap, nnz - bb);
        if (2 * nb <= hi - lo || nb <= 2) {
            // few bits, many matches: one bit at a time, lanes over its slice's matches
            for (uint32_t q = 0; q < nb; ++q) {
                const uint32_t code = s.bits[q];
                const uint32_t r = code >> 8, col = code & 0xFFu;
                const uint32_t j = col >> 4, c = col & 15u;
                const uint32_t k0 = max(s.mc[j], lo), k1 = min(s.mc[j + 1], hi);
                const uint32_t* Ar = blocks + r * WPR;
                const uint32_t* Br = blocks + c * WPR;
#pragma unroll(kHeavy ? 1 : 2)
                for (uint32_t k = k0 + lane; k < k1; k += kWarp) {
                    if (kHeavy && !((s.mra[k - lo] >> r) & (s.mrb[k - lo] >> c) & 1u)) continue;
                    const size_t pa = s.mpa[k - lo], pb = s.mpb[k - lo];
                    if constexpr (C == 128) {
                        const uint4 a = *reinterpret_cast<const uint4*>(Ar + pa * TW);
                        const uint4 b = *reinterpret_cast<const uint4*>(Br + pb * TW);
                        acc += (unsigned)(__popc(a.x & b.x) + __popc(a.y & b.y) +
                                          __popc(a.z & b.z) + __popc(a.w & b.w));
                    } else {
                        acc += (unsigned)__popc(Ar[pa * TW] & Br[pb * TW]);
                    }
                }
            }
        } else {
            // many bits: lanes over bits, each walking its slice's matches
            for (uint32_t q = lane; q < nb; q += kWarp) {
                const uint32_t code = s.bits[q];
                const uint32_t r = code >> 8, col = code & 0xFFu;
                const uint32_t j = col >> 4, c = col & 15u;
                const uint32_t k0 = max(s.mc[j], lo), k1 = min(s.mc[j + 1], hi);
                const uint32_t* Ar = blocks + r * WPR;
                const uint32_t* Br = blocks + c * WPR;
#pragma unroll(kHeavy ? 1 : 2)
                for (uint32_t k = k0; k < k1; ++k) {
                    if (kHeavy && !((s.mra[k - lo] >> r) & (s.mrb[k - lo] >> c) & 1u)) continue;
                    const size_t pa = s.mpa[k - lo], pb = s.mpb[k - lo];
                    if constexpr (C == 128) {
                        const uint4 a = *reinterpret_cast<const uint4*>(Ar + pa * TW);
                        const uint4 b = *reinterpret_cast<const uint4*>(Br + pb * TW);
                        acc += (unsigned)(__popc(a.x & b.x) + __popc(a.y & b.y) +
                                          __popc(a.z & b.z) + __popc(a.w & b.w));
                    } else {
                        acc += (unsigned)__popc(Ar[pa * TW] & Br[pb * TW]);
                    }
                }
            }
        }
        __syncwarp();
    }
    return acc;
}

template <int C, bool kHeavy>
__global__ void __launch_bounds__(kThreads, 4)
k_count(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
        const uint32_t* __restrict__ row_indices, const uint32_t* __restrict__ blocks,
        uint32_t num_tiles, uint32_t tile_begin, uint32_t tile_end, int32_t R, int tau,
        uint32_t chunk, CountScratch scr,
        const uint32_t* __restrict__ graph_rows, uint32_t num_graphs,
        unsigned long long* __restrict__ graph_counts, const uint32_t* __restrict__ rowmask,
        const uint2* __restrict__ cellpp, uint64_t cell_wpr,
        uint32_t chunk_skewed, const unsigned long long* __restrict__ row_max,
        const unsigned long long* __restrict__ build_meta)
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

    // A build enqueued without waiting (build_meta != nullptr): the tile count comes from
    // the device, and a failed build (bad vertex id, tile capacity overflow) counts
    // nothing and leaves 0xFFFFFFFFFFFFFFFF as the result.
    bool build_failed = false;
    if (build_meta) {
        const unsigned long long T = build_meta[kMetaTiles];
        build_failed = (build_meta[kMetaBad] | build_meta[kMetaOverflow]) != 0ull;
        num_tiles = T < num_tiles ? (uint32_t)T : num_tiles;
        if (tile_end > num_tiles) tile_end = num_tiles;
        if (tile_begin > tile_end || build_failed) tile_begin = tile_end;
    }

    // row-occupancy masks exist only when row blocks average 8 or more tiles
    if ((uint64_t)num_tiles < 8ull * (uint64_t)(R > 0 ? R : 0)) rowmask = nullptr;

    unsigned long long acc = 0;
    // Batches (graph_counts != nullptr): the tiles of graph g are row blocks
    // [graph_rows[g], graph_rows[g+1]); acc is flushed to graph_counts[g] whenever the
    // row block moves to another graph, and acc_total keeps what was flushed.
    unsigned long long acc_total = 0;
    uint32_t g_cur = 0xffffffffu;

    // Tile queue over one word.  Grab k is a run of consecutive tiles.  When no row
    // block holds more than four times the mean number of tiles plus 8 (meshes,
    // Erdos-Renyi: tile costs alike), the schedule is guided: `chunk` tiles in the first
    // grid-wide round of grabs, half as many in each later round, down to two tiles.
    // Otherwise (power-law graphs, where a run of tiles can cost many times another) every
    // grab is `chunk_skewed` tiles.  Grab k < (warps in the grid) is warp k's first grab;
    // later grabs are numbered by an atomic on the queue word.  A warp asks for its next
    // grab while it counts the last tile of the current one, so it never holds more than
    // one grab.
    const unsigned long long nwarps = (unsigned long long)gridDim.x * kWarps;
    bool guided = false;
    if (row_max) {
        const uint64_t mx = __ldg(row_max);
        guided = mx * (uint64_t)R <= 4ull * num_tiles + 8ull * (uint64_t)R;
    }
    if (!guided) chunk = chunk_skewed;
    auto grab_range = [&](unsigned long long k, uint32_t& b, uint32_t& e) {
        unsigned long long off = 0;
        uint32_t sz = chunk;
        while (guided && sz > 2 && k >= nwarps) {
            off += nwarps * sz;
            k -= nwarps;
            sz >>= 1;
        }
        off += k * sz;
        const unsigned long long span = tile_end - tile_begin;
        b = tile_begin + (uint32_t)(off < span ? off : span);
        e = tile_begin + (uint32_t)min(off + sz, span);
    };
    // A tile's ids and sample words.
    auto load_ids = [&](uint32_t t, uint32_t& tI, uint32_t& tJL, uint32_t& x0, uint32_t& x1) {
        tI = row_indices[t];
        tJL = indices[t];
        if constexpr (C == 128) {
            const uint2 v = reinterpret_cast<const uint2*>(blocks + (size_t)t * TW)[lane];
            x0 = v.x;
            x1 = v.y;
        } else {
            x0 = lane < 16 ? blocks[(size_t)t * TW + lane] : 0u;
            x1 = 0u;
        }
    };
    // The next tile's ids, and its sample words copied into s.nS in the background (no
    // registers held across the current tile); next_words() reads them back.
    auto load_next = [&](uint32_t t, uint32_t& tI, uint32_t& tJL) {
        tI = row_indices[t];
        tJL = indices[t];
        if constexpr (C == 128) {
            cp_async8(&s.nS[2 * lane], blocks + (size_t)t * TW + 2 * lane);
        } else {
            if (lane < 16) cp_async4(&s.nS[lane], blocks + (size_t)t * TW + lane);
        }
        cp_async_commit();
    };
    auto next_words = [&](uint32_t& x0, uint32_t& x1) {
        cp_async_wait_all();
        __syncwarp();
        if constexpr (C == 128) {
            x0 = s.nS[2 * lane];
            x1 = s.nS[2 * lane + 1];
        } else {
            x0 = lane < 16 ? s.nS[lane] : 0u;
            x1 = 0u;
        }
    };
    // A tile's indptr words: lane j <= JPT holds indptr[J_L*JPT + j] (the row blocks
    // J_out of its slices), lanes 16 and 17 hold indptr[I] and indptr[I + 1].
    auto load_ptrs = [&](uint32_t tI, uint32_t tJL) -> uint32_t {
        if (lane <= JPT) {
            const int64_t J = (int64_t)tJL * JPT + lane;
            return indptr[J < R ? J : R];
        }
        if (lane == 16 || lane == 17) return indptr[tI + (uint32_t)(lane - 16)];
        return 0u;
    };

    uint32_t curI = 0xffffffffu;
    ARow A{0, 0, 0, 0, 0, 0};
    uint32_t t, ce;  // current tile and the end of its grab
    {
        unsigned long long k = 0;
        // the first grab of every warp is its own index (no atomic at launch); the queue
        // word numbers the later grabs
        k = (unsigned long long)blockIdx.x * kWarps + warp;
        grab_range(k, t, ce);
    }
    uint32_t I = 0, JL = 0, w0 = 0, w1 = 0, ptrs = 0;
    if (t < tile_end) {
        load_ids(t, I, JL, w0, w1);
        ptrs = load_ptrs(I, JL);
    }
    while (t < tile_end) {
        // The next tile: inside the grab its ids are loaded now and its indptr words once
        // this tile's search has issued its loads; after the grab's last tile the queue
        // atomic is issued now and read once this tile's search is under way.
        uint32_t tn = t + 1, cen = ce;
        uint32_t nI = 0, nJL = 0, nptrs = 0;
        // 0: next ids loading; 1: and its indptr words; 2: queue atomic in flight;
        // 3: grab resolved, ids loading (indptr words loaded at the top of the next tile)
        int nstate;
        unsigned long long kq = 0;
        if (tn < ce) {
            load_next(tn, nI, nJL);
            nstate = 0;
        } else {
            if (lane == 0) kq = nwarps + atomicAdd(scr.work, 1ull);
            nstate = 2;
        }
        auto next_ready = [&]() {
            if (nstate == 2) {
                grab_range(__shfl_sync(kFull, kq, 0), tn, cen);
                if (tn < tile_end) load_next(tn, nI, nJL);
                nstate = 3;
            } else if (nstate == 0 && !kHeavy) {
                // (heavy tiles are long: holding the next tile's words across one costs
                // more than the load it saves, so the heavy variant loads them at the top)
                nptrs = load_ptrs(nI, nJL);
                nstate = 1;
            }
        };

        // ---- sample tile and its slices -------------------------------------
        const int nnz = (int)__reduce_add_sync(kFull, (unsigned)(__popc(w0) + __popc(w1)));

        // 16x128: lane = 2r + h holds slices j = 4h + q (q = 0..3) of row r
        // 16x32 : lane = r (< 16) holds slices j = q (q = 0..1) of row r
        uint32_t active = 0;  // bit j set if slice j has any bit
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

        if (I != curI) {
            const uint32_t a0 = __shfl_sync(kFull, ptrs, 16), a1 = __shfl_sync(kFull, ptrs, 17);
            A = stage_row<C>(s, indices, a0, a1 - a0, lane);
            curI = I;
            if (graph_counts) {
                const uint32_t lo = graph_of_row_block(graph_rows, num_graphs, I);
                if (lo != g_cur) {
                    flush_graph(acc, acc_total, graph_counts, g_cur, lane);
                    g_cur = lo;
                }
            }
        }
        if (lane <= JPT) s.jptr[lane] = ptrs;
        __syncwarp();

        // unit prefix over active slices (the search's lane -> slice map)
        uint32_t upre[JPT + 1];
        auto compute_upre = [&]() {
            upre[0] = 0;
#pragma unroll
            for (int j = 0; j < JPT; ++j)
                upre[j + 1] = upre[j] + (((active >> j) & 1u) ? (s.jptr[j + 1] - s.jptr[j]) : 0u);
        };

        if (nnz <= tau) {
            // ================= sparse path ===================================
            // Search every element of the active slices' row-block lists in row block
            // I's list (32 per round); matches are appended in slice order, so slice
            // j owns match-list entries [mc[j], mc[j+1]).  Then one lane per set bit.
            const uint32_t mine = (uint32_t)(__popc(w0) + __popc(w1));
            uint32_t e = mine;  // exclusive count of set bits held by lower lanes
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, e, d);
                if (lane >= d) e += y;
            }
            e -= mine;
            const uint32_t* __restrict__ rmask_g = nullptr;
            if constexpr (kHeavy) {
                compute_upre();
                // Tiles with more than one round of list elements take the heavy path:
                // rows and columns of S that carry bits, per slice (to drop matches and
                // units whose tile rows are empty), and the two-direction search plan.
                // Small tiles skip both: a single round costs less than planning it.
                const bool heavy = upre[JPT] > (uint32_t)kWarp;
                rmask_g = heavy ? rowmask : nullptr;
                uint32_t rm[JPT], cm[JPT];
#pragma unroll
                for (int j = 0; j < JPT; ++j) rm[j] = cm[j] = 0xFFFFu;
                if (!heavy) {
                } else if constexpr (C == 128) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const uint32_t sl = ((q < 2 ? w0 : w1) >> (16 * (q & 1))) & 0xFFFFu;
                        const unsigned bl = __ballot_sync(kFull, sl != 0);
                        rm[q] = compress_even(bl);
                        rm[4 + q] = compress_even(bl >> 1);
                        cm[q] = __reduce_or_sync(kFull, (lane & 1) ? 0u : sl);
                        cm[4 + q] = __reduce_or_sync(kFull, (lane & 1) ? sl : 0u);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const uint32_t sl = (w0 >> (16 * q)) & 0xFFFFu;
                        rm[q] = __ballot_sync(kFull, sl != 0) & 0xFFFFu;
                        cm[q] = __reduce_or_sync(kFull, sl);
                    }
                }
                // search plan: lane j < JPT picks slice j's direction and list
                uint32_t len = 0, start = 0, dir = 0;
                if (lane < JPT && ((active >> lane) & 1u)) {
                    const uint32_t jb = s.jptr[lane], je = s.jptr[lane + 1];
                    len = je - jb;
                    start = jb;
                    if (heavy && cellpp && je > jb) {
                        const uint32_t r0 = a_rank<C>(s, A, indices, indices[jb]);
                        const uint32_t r1 = a_rank<C>(s, A, indices, indices[je - 1] + 1);
                        if (r1 - r0 < len) {
                            len = r1 - r0;
                            start = A.start + r0;
                            dir = 1;
                        }
                    }
                    s.sstart[lane] = start;
                    s.sdir[lane] = (uint8_t)dir;
                }
#pragma unroll
                for (int j = 0; j < JPT; ++j) upre[j + 1] = upre[j] + __shfl_sync(kFull, len, j);
                if (lane == 0) {
#pragma unroll
                    for (int j = 0; j < JPT; ++j) {
                        s.rmask[j] = (uint16_t)rm[j];
                        s.cmask[j] = (uint16_t)cm[j];
                    }
                }
            }
            bool searched = false;
            if constexpr (!kHeavy) {
                // When every active slice's list fits in its share of the lanes (meshes:
                // a few column blocks per row block), one round with a fixed lane -> slice
                // map does the search; the ballot order keeps matches grouped by slice.
                constexpr int LPS = kWarp / JPT;  // lanes per slice
                const int jl = lane / LPS, ql = lane % LPS;
                const uint32_t jb = __shfl_sync(kFull, ptrs, jl);
                const uint32_t je = __shfl_sync(kFull, ptrs, jl + 1);
                const uint32_t len = ((active >> jl) & 1u) ? je - jb : 0u;
                if (__all_sync(kFull, len <= (uint32_t)LPS)) {
                    bool found = false;
                    uint32_t pa = 0;
                    const uint32_t pb = jb + (uint32_t)ql;
                    if ((uint32_t)ql < len) found = a_lookup<C>(s, A, indices, indices[pb], pa);
                    const unsigned mb = __ballot_sync(kFull, found);
                    if (found) {
                        const uint32_t k = __popc(mb & lt);
                        s.mpa[k] = pa;
                        s.mpb[k] = pb;
                    }
                    if (lane <= JPT)
                        s.mc[lane] = __popc(mb & (lane == JPT ? kFull : ((1u << (lane * LPS)) - 1u)));
                    next_ready();
                    __syncwarp();
                    if (mb)
                        acc += bit_pass<C, kHeavy>(s, w0, w1, e, (uint32_t)nnz, 0u,
                                                   (uint32_t)__popc(mb), blocks, lane);
                    searched = true;
                } else {
                    compute_upre();
                }
            }
            if (!searched) {
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j <= JPT; ++j) s.upre[j] = upre[j];
            }
            __syncwarp();
            const uint32_t W = upre[JPT];
            uint32_t mc = 0;  // lane j <= JPT: matches so far from slices below j
            uint32_t nm = 0, lo = 0;
            for (uint32_t ub = 0; ub < W; ub += kWarp) {
                const uint32_t u = ub + lane;
                bool found = false;
                uint32_t pa = 0, pb = 0, ra = 0xFFFFu, rb = 0xFFFFu;
                if (u < W) {
                    uint32_t us = 0, jsel = 0;
#pragma unroll
                    for (int j = 1; j < JPT; ++j)
                        if (u >= upre[j]) {
                            us = upre[j];
                            jsel = j;
                        }
                    if constexpr (!kHeavy) {
                        pb = s.jptr[jsel] + (u - us);
                        found = a_lookup<C>(s, A, indices, indices[pb], pa);
                    } else {
                        const uint32_t idx = s.sstart[jsel] + (u - us);
                        if (!s.sdir[jsel]) {
                            pb = idx;
                            found = a_lookup<C>(s, A, indices, indices[pb], pa);
                        } else {
                            pa = idx;
                            const uint32_t a = indices[pa];
                            const uint64_t cw = (uint64_t)(JL * JPT + jsel) * cell_wpr + (a >> 5);
                            const uint2 cp = cellpp[cw];
                            const uint32_t bit = 1u << (a & 31u);
                            found = (cp.x & bit) != 0u;
                            if (found) pb = cp.y + __popc(cp.x & (bit - 1u));
                        }
                        if (found && rmask_g) {
                            ra = rmask_g[pa];
                            rb = rmask_g[pb];
                            found = (ra & s.rmask[jsel]) && (rb & s.cmask[jsel]);
                        }
                    }
                }
                const unsigned mb = __ballot_sync(kFull, found);
                if (found) {
                    const uint32_t k = nm - lo + __popc(mb & lt);
                    s.mpa[k] = pa;
                    s.mpb[k] = pb;
                    if constexpr (kHeavy) {
                        s.mra[k] = (uint16_t)ra;
                        s.mrb[k] = (uint16_t)rb;
                    }
                }
                if (lane <= JPT) {
                    const uint32_t lim = s.upre[lane];
                    const uint32_t below = lim <= ub ? 0u
                                          : (lim - ub >= 32u ? kFull : ((1u << (lim - ub)) - 1u));
                    mc += __popc(mb & below);
                }
                nm += __popc(mb);
                if (nm - lo > (uint32_t)(kMCap - kWarp) || (ub + kWarp >= W && nm > lo)) {
                    next_ready();
                    if (lane <= JPT) s.mc[lane] = mc;
                    __syncwarp();
                    acc += bit_pass<C, kHeavy>(s, w0, w1, e, (uint32_t)nnz, lo, nm, blocks, lane);
                    lo = nm;
                }
            }
            }
        } else {
            // ================= dense path: binary tensor core ================
            next_ready();
            if constexpr (C == 128) {
                s.S[2 * lane] = w0;
                s.S[2 * lane + 1] = w1;
            } else {
                if (lane < 16) s.S[lane] = w0;
            }
            __syncwarp();
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
                        found = a_lookup<C>(s, A, indices, indices[pb], pa);
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
                        // two packed groups' fragments are loaded before their four MMAs
                        for (int k0 = 0; k0 < nm; k0 += 8) {
                            const int k = k0 + tg, k2 = k0 + 4 + tg;
                            uint32_t a0 = 0, a1 = 0, b0 = 0, b1 = 0, e0 = 0, e1 = 0, f0 = 0, f1 = 0;
                            if (k < nm) {
                                const uint32_t* A = blocks + (size_t)s.mpa[k] * TW;
                                const uint32_t* Bt = blocks + (size_t)s.mpb[k] * TW;
                                a0 = A[g];
                                a1 = A[g + 8];
                                b0 = Bt[g];
                                b1 = Bt[g + 8];
                            }
                            if (k2 < nm) {
                                const uint32_t* A = blocks + (size_t)s.mpa[k2] * TW;
                                const uint32_t* Bt = blocks + (size_t)s.mpb[k2] * TW;
                                e0 = A[g];
                                e1 = A[g + 8];
                                f0 = Bt[g];
                                f1 = Bt[g + 8];
                            }
                            mma_b1(c0, a0, a1, b0);
                            mma_b1(c1, a0, a1, b1);
                            if (k0 + 4 < nm) {
                                mma_b1(c0, e0, e1, f0);
                                mma_b1(c1, e0, e1, f1);
                            }
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
        next_ready();
        __syncwarp();
        t = tn;
        ce = cen;
        I = nI;
        JL = nJL;
        if (t < tile_end) next_words(w0, w1);
        ptrs = nstate == 1 ? nptrs : (t < tile_end ? load_ptrs(I, JL) : 0u);
    }

    if (graph_counts) {
        flush_graph(acc, acc_total, graph_counts, g_cur, lane);
        acc = acc_total;
    }

    // ---- int64 block tree + last-CTA reduction ------------------------------
    finish_count<kThreads>(acc, scr, build_failed, s_red, &s_last);
}

}  // namespace

// Resident CTAs per SM of the tile-wise kernel (the same for both variants: 256 threads
// at 64 registers and the same shared memory), cached per device and tile width.
static int tile_blocks_per_sm(int tile_cols)
{
    static std::atomic<int> cache[64][2];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    const int w = tile_cols == 128 ? 0 : 1;
    if (dev >= 0 && dev < 64) {
        const int v = cache[dev][w].load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    int per_sm = 0;
    cudaError_t e;
    if (tile_cols == 128)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_count<128, false>, kThreads, 0);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_count<32, false>, kThreads, 0);
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    if (dev >= 0 && dev < 64) cache[dev][w].store(per_sm, std::memory_order_relaxed);
    return per_sm;
}

// Persistent grid of the count kernels: the larger of the two kernels' resident CTAs
// per SM, times the SMs (the CTAs a count's scratch holds a partial sum for; each
// launch runs at most its own kernel's resident CTAs).
int count_grid_size(int tile_cols)
{
    const int rows = rows_blocks_per_sm(tile_cols);
    const int tile = tile_blocks_per_sm(tile_cols);
    return (rows > tile ? rows : tile) * device_sm_count();
}

int launch_count(int tile_cols, const uint32_t* indptr, const uint32_t* indices,
                 const uint32_t* row_indices, const uint32_t* blocks, uint32_t num_tiles,
                 int32_t n_row_blocks, int tau, CountScratch scr, cudaStream_t s,
                 const uint32_t* graph_rows, uint32_t num_graphs, unsigned long long* graph_counts,
                 const uint32_t* rowmask, const uint2* cellpp,
                 uint64_t cell_wpr, const unsigned long long* row_max, uint32_t tile_begin,
                 uint32_t tile_end, const unsigned long long* build_meta, uint32_t tiles_hint,
                 const uint32_t* row_off, const uint2* row_ent, bool dense_tiles,
                 const GraphSeg* segs)
{
    // build_meta: num_tiles is a capacity bound and the kernel reads the device tile
    // count; the schedule and the variant follow tiles_hint (the previous build's count)
    if (tile_end > num_tiles) tile_end = num_tiles;
    if (tile_begin > tile_end) tile_begin = tile_end;
    const uint32_t span = build_meta ? min(tiles_hint, tile_end - tile_begin) : tile_end - tile_begin;
    const int grid_all = count_grid_size(tile_cols);
    const int grid_tile = tile_blocks_per_sm(tile_cols) * device_sm_count();
    const int grid = grid_tile < grid_all ? grid_tile : grid_all;
    // Guided schedule: the first round of grabs is about half of an even share per warp
    // (2 to 64 tiles; later rounds halve it down to 2: a one-tile grab costs a contended
    // queue atomic per tile).  Fixed schedule: about an eighth of an even share (8 to 64 tiles);
    // a grab of a power-law graph's row block often holds tiles of one long list, which
    // is staged once per grab.
    const uint64_t warps = (uint64_t)grid * kWarps;
    uint64_t chunk = span / (warps * 2), chunk_s = span / (warps * 8);
    chunk = chunk < 2 ? 2 : (chunk > 64 ? 64 : chunk);
    chunk_s = chunk_s < 8 ? 8 : (chunk_s > 64 ? 64 : chunk_s);
    // The occupancy masks and the two-direction search pay off only where row blocks
    // hold many tiles (long lists to search); meshes and stencils (a few tiles per row
    // block) take the light kernel.
    const bool heavy = rowmask != nullptr && n_row_blocks > 0 &&
                       (uint64_t)(build_meta ? tiles_hint : num_tiles) >= 8ull * (uint64_t)n_row_blocks;
    if (!heavy) {
        rowmask = nullptr;
        cellpp = nullptr;
    }
    // Heavy graphs built through the cell bitmap, with a row index, take the row-wise
    // kernel (count_rows.cu); BTC_COUNT_TILEWISE=1 keeps them on this one (a switch for
    // comparing the two).
    static const bool tilewise = [] {
        const char* e = std::getenv("BTC_COUNT_TILEWISE");
        return e && e[0] == '1';
    }();
    // Row-wise kernel: grabs of at most 16 tiles.  Its warps read other row blocks' tile
    // rows at random, so what stays in L2 is what the warps in flight share; smaller
    // grabs keep those warps in fewer row blocks (measured on R-MAT scale 20 / 22 in
    // degree order, 16x128: 5.34 / 23.26 ms at 64 tiles, 2.80 / 21.91 ms at 16, 2.91 /
    // 22.18 ms at 8).  At least half an even share per warp, down to one tile: a graph
    // of few, dense tiles (K_4096: 4224 tiles) keeps every warp busy.
    uint64_t chunk_r = span / (warps * 2);
    const uint32_t chunk_rows = (uint32_t)(chunk_r < 1 ? 1 : (chunk_r > 16 ? 16 : chunk_r));
    if (heavy && cellpp && row_off && row_ent && !tilewise)
        return launch_count_rows(tile_cols, indptr, indices, row_indices, blocks, num_tiles, tile_begin,
                                 tile_end, n_row_blocks, tau, chunk_rows, scr, graph_rows,
                                 num_graphs, graph_counts, rowmask, cellpp, cell_wpr, row_off, row_ent,
                                 segs, build_meta, dense_tiles, grid_all, s);
    // the tile-wise kernel indexes the cell pairs of a single graph only
    if (segs) cellpp = nullptr;
#define BTC_LAUNCH_COUNT(CC, HH)                                                              \
    k_count<CC, HH><<<grid, kThreads, 0, s>>>(indptr, indices, row_indices, blocks, num_tiles, \
                                              tile_begin, tile_end, n_row_blocks, tau,         \
                                              (uint32_t)chunk, scr,                            \
                                              graph_rows, num_graphs, graph_counts, rowmask,   \
                                              cellpp, cell_wpr, (uint32_t)chunk_s,             \
                                              row_max, build_meta)
    if (tile_cols == 128) {
        if (heavy) BTC_LAUNCH_COUNT(128, true);
        else BTC_LAUNCH_COUNT(128, false);
    } else {
        if (heavy) BTC_LAUNCH_COUNT(32, true);
        else BTC_LAUNCH_COUNT(32, false);
    }
#undef BTC_LAUNCH_COUNT
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

}  // namespace btc200
