// count_rows.cu -- the count kernel for graphs whose row blocks hold many tiles (power-law
// graphs in descending-degree order): row-wise matching with flattened work units.
//
// Computes what btc/operations/tc_16x128_mma_v5.h:9-211 and tc_16x32_mma_v6.h:9-238
// compute -- for every set bit (r, c) of every sample tile S = (I, J_L) of L, with c in
// slice j (16 columns: row block J_out = J_L*(C/16) + j, row c % 16 of it), the sum over
// column blocks K of popc(L[I,K][r] & L[J_out,K][c % 16]) -- organised per tile row
// instead of per tile:
//
//  * Vertex u = 16 I + r has its own list of the tiles of row block I whose row r holds a
//    bit (the row index, rowindex.cu), in column-block order.  On degree-ordered power-law
//    graphs a row block lists ~80 tiles but a single row appears in only a few of them.
//    Only entries with K <= J_L can match (J_out's rows are vertices below 128 (J_L + 1),
//    whose lower neighbours lie in column blocks <= J_L), and S itself is u's entry for
//    J_L, so the useful entries run from the list's start up to S.
//  * A sparse tile (popcount <= tau) only records its (J_out, r, 16-bit column mask)
//    groups in a per-warp buffer: a few ballots, no search.  The median tile of these
//    graphs has one bit.
//  * When the buffer fills, the row block changes or the work runs out, each buffered
//    group is resolved to its range of u's list (bisection for S's entry), and the units
//    -- one per list entry -- run as flat rounds over all buffered tiles, two units per
//    lane per round: each unit looks column block K up in J_out's row of the builder's
//    cell bitmap (one 8-byte (word, tile prefix) pair: membership and tile index),
//    checks that tile's row mask against the group's columns and adds popc(row r of I's
//    tile AND row c of J_out's tile) for each column c left.
//  * A dense tile (popcount > tau) runs per slice on the binary tensor core: I's tiles
//    inside J_out's column range that J_out also holds are found 32 at a time by the same
//    cell lookup, and each match feeds mma.sync.m16n8k128.row.col.s32.b1.b1.s32.and.popc
//    twice (16 x 16 popcount block), masked by the slice's bits (16x32 tiles pack four
//    matches into k = 128, as tc_16x32_mma_v6.h:72-154 does).
//  * Tiles come from the same grab queue as the other count kernel; their words arrive
//    by cp.async into a four-tile ring per warp.  Integer arithmetic only; per-lane uint64
//    partials and the last-CTA reduction of count_common.cuh.
//
// Needs the cell bitmap's (word, prefix) pairs (the bitmap builder's); a batch union
// passes the segment of each graph, whose part of the bitmap holds the cells of its rows.  Without the row
// masks and row index at run time (an asynchronous rebuild that left fewer than 8 tiles
// per row block) a group's units are all tiles of row block I up to S, with the mask
// check when masks exist.
#include "count_common.cuh"

#include <atomic>

namespace btc200 {
namespace {

constexpr int kRThreads = 256;
constexpr int kRWarps = kRThreads / kWarp;
constexpr int kGCap = 64;     // buffered (J_out, row, columns) groups per warp
constexpr int kRing = 4;      // tiles whose words are in flight per warp

template <int C>
struct __align__(16) RowSmem {
    uint32_t ring[kRing][Cfg<C>::TW];  // tile words (cp.async destinations; 16-byte aligned)
    uint32_t gJ[kGCap];                // group: J_out
    uint32_t gRC[kGCap];               // group: (r << 16) | column mask
    uint32_t gT[kGCap];                // group: the sample tile
    uint32_t gS[kGCap];                // group: first unit's entry
    uint32_t gPre[kGCap + 1];          // group: unit prefix
    uint32_t mpa[kWarp];               // dense path: matched tiles of I
    uint32_t mpb[kWarp];               // dense path: matched tiles of J_out
};
static_assert(sizeof(RowSmem<128>) % 16 == 0 && sizeof(RowSmem<32>) % 16 == 0,
              "per-warp areas keep the 16-byte alignment of the first one");
static_assert(kGCap == 64, "the group search below takes six steps");

template <int C>
constexpr size_t rows_smem_bytes() { return sizeof(RowSmem<C>) * kRWarps; }

// kMinBlocks: resident CTAs per SM the registers are capped for.  Sparse 16x128 graphs
// take five (48 registers; R-MAT s22 20.85 ms against 21.89 at four: the dependent-load
// chains want every warp they can get), graphs of dense 16x128 tiles four (64 registers:
// K_4096 on the tensor-core path 0.19 ms against 0.23 at five), 16x32 four.
// kSeg: a batch union, whose cells are looked up in each graph's part of the bitmap.
template <int C, int kMinBlocks, bool kSeg>
__global__ void __launch_bounds__(kRThreads, kMinBlocks)
k_count_rows(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
             const uint32_t* __restrict__ row_indices, const uint32_t* __restrict__ blocks,
             uint32_t num_tiles, uint32_t tile_begin, uint32_t tile_end, int32_t R, int tau,
             uint32_t chunk, CountScratch scr, const uint32_t* __restrict__ graph_rows,
             uint32_t num_graphs, unsigned long long* __restrict__ graph_counts,
             const uint32_t* __restrict__ rowmask, const uint2* __restrict__ cellpp,
             uint64_t cell_wpr, const uint32_t* __restrict__ row_off, const uint2* __restrict__ row_ent,
             const GraphSeg* __restrict__ segs, const unsigned long long* __restrict__ build_meta)
{
    using K = Cfg<C>;
    constexpr int WPR = K::WPR, TW = K::TW, JPT = K::JPT;
    extern __shared__ __align__(16) unsigned char rows_smem_raw[];
    __shared__ unsigned long long s_red[kRWarps];
    __shared__ int s_last;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    RowSmem<C>& s = reinterpret_cast<RowSmem<C>*>(rows_smem_raw)[warp];
    const unsigned lt = lanemask_lt();

    // A build enqueued without waiting (build_meta != nullptr): the tile count comes from
    // the device; a failed build counts nothing and leaves 0xFFFFFFFFFFFFFFFF.
    bool build_failed = false;
    if (build_meta) {
        const unsigned long long T = build_meta[kMetaTiles];
        build_failed = (build_meta[kMetaBad] | build_meta[kMetaOverflow]) != 0ull;
        num_tiles = T < num_tiles ? (uint32_t)T : num_tiles;
        if (tile_end > num_tiles) tile_end = num_tiles;
        if (tile_begin > tile_end || build_failed) tile_begin = tile_end;
    }
    // row masks and the row index exist only when row blocks average 8 or more tiles
    const bool have_rm = rowmask != nullptr && (uint64_t)num_tiles >= 8ull * (uint64_t)(R > 0 ? R : 0);
    const bool have_ri = have_rm && row_off != nullptr && row_ent != nullptr;
    auto rmask_of = [&](uint32_t t) -> uint32_t { return have_rm ? __ldg(rowmask + t) : 0xFFFFu; };

    // The (cell word, tile prefix) pair of row block J, column block K, and K's bit in it.
    // A batch union looks the cell up in the part of the bitmap of J's graph (sg, the
    // segment of the row block being counted); a single graph is one segment.
    GraphSeg sg{0u, 0, 0u, 0u, (uint32_t)cell_wpr, 0u, 0ull};
    auto cell = [&](uint32_t J, uint32_t K, uint32_t& bit) -> uint64_t {
        if constexpr (kSeg) {
            const uint32_t k = K - sg.cb_lo;
            bit = 1u << (k & 31u);
            return sg.bm_off + (uint64_t)(J - sg.row_off) * sg.wpr + (k >> 5);
        } else {
            bit = 1u << (K & 31u);
            return (uint64_t)J * cell_wpr + (K >> 5);
        }
    };

    unsigned long long acc = 0, acc_total = 0;
    uint32_t g_cur = 0xffffffffu;
    uint32_t curI = 0xffffffffu, a0 = 0, alen = 0;  // row block I and its tiles [a0, a0 + alen)

    // ---- buffered groups -------------------------------------------------------------
    uint32_t ng = 0;
    auto flush = [&]() {
        if (ng == 0) return;
        __syncwarp();
        // resolve: group g's units are entries [gS, gS + count) -- u's list up to S
        uint32_t ubase = 0;
        for (uint32_t gb = 0; gb < ng; gb += kWarp) {
            const uint32_t g = gb + lane;
            uint32_t cnt = 0, st = 0;
            if (g < ng) {
                const uint32_t tS = s.gT[g];
                if (have_ri) {
                    const uint32_t u = 16u * curI + (s.gRC[g] >> 16);
                    uint32_t lo = row_off[u], hi = row_off[u + 1];
                    st = lo;
                    while (lo < hi) {  // first entry past S
                        const uint32_t mid = (lo + hi) >> 1;
                        if (row_ent[mid].y <= tS) lo = mid + 1;
                        else hi = mid;
                    }
                    cnt = lo - st;
                } else {
                    st = a0;
                    cnt = tS + 1 - a0;
                }
            }
            uint32_t incl = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, incl, d);
                if (lane >= d) incl += y;
            }
            if (g < ng) {
                s.gS[g] = st;
                s.gPre[g] = ubase + incl - cnt;
            }
            ubase += __shfl_sync(kFull, incl, 31);
        }
        // gPre past the last group reads as all-ones, so the six-step search below never
        // leaves [0, ng) for a unit below ubase
        for (uint32_t g = ng + lane; g <= (uint32_t)kGCap; g += kWarp)
            s.gPre[g] = g == ng ? ubase : 0xffffffffu;
        __syncwarp();
        // units: two per lane per round, their loads interleaved
        for (uint32_t ub = 0; ub < ubase; ub += 2 * kWarp) {
            uint32_t uu[2], gg[2];
            bool ok[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                uu[q] = ub + q * kWarp + lane;
                ok[q] = uu[q] < ubase;
                gg[q] = 0;  // last group with gPre <= u (gPre past the groups is all-ones)
            }
#pragma unroll
            for (int step = 32; step > 0; step >>= 1) {
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    if (s.gPre[gg[q] + step] <= uu[q]) gg[q] += step;
            }
#pragma unroll
            for (int q = 0; q < 2; ++q)
                if (!ok[q]) gg[q] = 0;  // past the last unit: any valid group, not used
            uint32_t Kb[2], pa[2], rc[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t e = s.gS[gg[q]] + (uu[q] - s.gPre[gg[q]]);
                rc[q] = s.gRC[gg[q]];
                Kb[q] = 0;
                pa[q] = 0;
                if (ok[q]) {
                    if (have_ri) {
                        const uint2 en = row_ent[e];
                        Kb[q] = en.x;
                        pa[q] = en.y;
                    } else {
                        pa[q] = e;
                        Kb[q] = indices[e];
                        ok[q] = ((rmask_of(e) >> (rc[q] >> 16)) & 1u) != 0u;
                    }
                }
            }
            uint2 cp[2];
            uint32_t bits[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint64_t w = cell(s.gJ[gg[q]], Kb[q], bits[q]);
                cp[q] = ok[q] ? cellpp[w] : make_uint2(0u, 0u);
            }
            uint32_t pb[2], m[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t bit = bits[q];
                pb[q] = cp[q].y + __popc(cp[q].x & (bit - 1u));
                m[q] = (cp[q].x & bit) ? rmask_of(pb[q]) & rc[q] & 0xFFFFu : 0u;
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!m[q]) continue;
                const uint32_t r = rc[q] >> 16;
                const uint32_t* Ar = blocks + (size_t)pa[q] * TW + r * WPR;
                const uint32_t* Bt = blocks + (size_t)pb[q] * TW;
                unsigned part = 0;  // at most 16 x C per unit
                uint32_t mm = m[q];
                if constexpr (C == 128) {
                    const uint4 a = *reinterpret_cast<const uint4*>(Ar);
                    do {
                        const uint32_t c = __ffs(mm) - 1;
                        mm &= mm - 1;
                        const uint4 b = *reinterpret_cast<const uint4*>(Bt + c * WPR);
                        part += __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) +
                                __popc(a.w & b.w);
                    } while (mm);
                } else {
                    const uint32_t a = *Ar;
                    do {
                        const uint32_t c = __ffs(mm) - 1;
                        mm &= mm - 1;
                        part += __popc(a & Bt[c]);
                    } while (mm);
                }
                acc += part;
            }
        }
        ng = 0;
        __syncwarp();
    };

    // ---- dense tile: binary tensor core ------------------------------------------------
    const int fg = lane >> 2, tg = lane & 3;  // mma fragment coordinates
    auto dense = [&](const uint32_t* S, uint32_t JL, uint32_t active) {
        for (int j = 0; j < JPT; ++j) {
            if (!((active >> j) & 1u)) continue;
            const uint32_t J = JL * JPT + j;
            if ((int64_t)J >= (int64_t)R) continue;
            const uint32_t jb = indptr[J], je = indptr[J + 1];
            if (je == jb) continue;
            const uint32_t kmin = indices[jb], kmax = indices[je - 1];
            const uint32_t x = lower_bound_u32(indices + a0, alen, kmin);
            const uint32_t y = lower_bound_u32(indices + a0, alen, kmax + 1u);
            int32_t c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
            for (uint32_t ib = x; ib < y; ib += kWarp) {
                const uint32_t i = ib + lane;
                bool found = false;
                uint32_t pb = 0;
                if (i < y) {
                    const uint32_t Kb = indices[a0 + i];
                    uint32_t bit;
                    const uint2 cp = cellpp[cell(J, Kb, bit)];
                    found = (cp.x & bit) != 0u;
                    pb = cp.y + __popc(cp.x & (bit - 1u));
                }
                const unsigned mb = __ballot_sync(kFull, found);
                if (mb == 0) continue;
                const int nm = __popc(mb);
                if (found) {
                    const int k = __popc(mb & lt);
                    s.mpa[k] = a0 + i;
                    s.mpb[k] = pb;
                }
                __syncwarp();
                if constexpr (C == 128) {
                    for (int k = 0; k < nm; ++k) {
                        const uint32_t* A = blocks + (size_t)s.mpa[k] * TW;
                        const uint32_t* Bt = blocks + (size_t)s.mpb[k] * TW;
                        const uint32_t fa0 = A[fg * WPR + tg], fa1 = A[(fg + 8) * WPR + tg];
                        const uint32_t fb0 = Bt[fg * WPR + tg], fb1 = Bt[(fg + 8) * WPR + tg];
                        mma_b1(c0, fa0, fa1, fb0);
                        mma_b1(c1, fa0, fa1, fb1);
                    }
                } else {
                    // two packed groups' fragments are loaded before their four MMAs (for
                    // 16x128 the same pairing measured slower: registers the sparse path
                    // needs)
                    for (int k0 = 0; k0 < nm; k0 += 8) {
                        const int k = k0 + tg, k2 = k0 + 4 + tg;
                        uint32_t fa0 = 0, fa1 = 0, fb0 = 0, fb1 = 0, ga0 = 0, ga1 = 0, gb0 = 0, gb1 = 0;
                        if (k < nm) {
                            const uint32_t* A = blocks + (size_t)s.mpa[k] * TW;
                            const uint32_t* Bt = blocks + (size_t)s.mpb[k] * TW;
                            fa0 = A[fg];
                            fa1 = A[fg + 8];
                            fb0 = Bt[fg];
                            fb1 = Bt[fg + 8];
                        }
                        if (k2 < nm) {
                            const uint32_t* A = blocks + (size_t)s.mpa[k2] * TW;
                            const uint32_t* Bt = blocks + (size_t)s.mpb[k2] * TW;
                            ga0 = A[fg];
                            ga1 = A[fg + 8];
                            gb0 = Bt[fg];
                            gb1 = Bt[fg + 8];
                        }
                        mma_b1(c0, fa0, fa1, fb0);
                        mma_b1(c1, fa0, fa1, fb1);
                        if (k0 + 4 < nm) {
                            mma_b1(c0, ga0, ga1, gb0);
                            mma_b1(c1, ga0, ga1, gb1);
                        }
                    }
                }
                __syncwarp();
            }
            // mask: C[row][col] counts only where slice j of S has bit (row, col)
            const uint32_t sg = slice_of<C>(S, fg, j), sg8 = slice_of<C>(S, fg + 8, j);
            const int c = 2 * tg;
            long long p = 0;
            p += ((sg >> c) & 1u) ? c0[0] : 0;
            p += ((sg >> (c + 1)) & 1u) ? c0[1] : 0;
            p += ((sg8 >> c) & 1u) ? c0[2] : 0;
            p += ((sg8 >> (c + 1)) & 1u) ? c0[3] : 0;
            p += ((sg >> (c + 8)) & 1u) ? c1[0] : 0;
            p += ((sg >> (c + 9)) & 1u) ? c1[1] : 0;
            p += ((sg8 >> (c + 8)) & 1u) ? c1[2] : 0;
            p += ((sg8 >> (c + 9)) & 1u) ? c1[3] : 0;
            acc += (unsigned long long)p;
        }
    };

    // ---- tile queue: runs of `chunk` consecutive tiles --------------------------------
    const unsigned long long nwarps = (unsigned long long)gridDim.x * kRWarps;
    const unsigned long long span = tile_end - tile_begin;
    auto grab_range = [&](unsigned long long k, uint32_t& b, uint32_t& e) {
        const unsigned long long off = k * chunk;
        b = tile_begin + (uint32_t)(off < span ? off : span);
        e = tile_begin + (uint32_t)(off + chunk < span ? off + chunk : span);
    };
    auto prefetch = [&](uint32_t t, uint32_t gb, uint32_t ge) {
        if (t < ge) {
            uint32_t* dst = s.ring[(t - gb) % kRing];
            if constexpr (C == 128) {
                cp_async8(dst + 2 * lane, blocks + (size_t)t * TW + 2 * lane);
            } else {
                if (lane < 16) cp_async4(dst + lane, blocks + (size_t)t * TW + lane);
            }
        }
        cp_async_commit();  // one group per tile slot, empty past the grab's end
    };

    uint32_t gb, ge;
    grab_range((unsigned long long)blockIdx.x * kRWarps + warp, gb, ge);
    while (gb < ge) {
        // the next grab's number, read when this one ends
        unsigned long long kq = 0;
        if (lane == 0) kq = nwarps + atomicAdd(scr.work, 1ull);
#pragma unroll
        for (int q = 0; q < kRing - 1; ++q) prefetch(gb + q, gb, ge);
        for (uint32_t cb = gb; cb < ge; cb += kWarp) {
            // ids of up to 32 tiles, one per lane
            uint32_t myI = 0, myJL = 0;
            if (cb + lane < ge) {
                myI = row_indices[cb + lane];
                myJL = indices[cb + lane];
            }
            const uint32_t ce = ge - cb < (uint32_t)kWarp ? ge : cb + kWarp;
            for (uint32_t t = cb; t < ce; ++t) {
                prefetch(t + kRing - 1, gb, ge);
                const uint32_t I = __shfl_sync(kFull, myI, t - cb);
                const uint32_t JL = __shfl_sync(kFull, myJL, t - cb);
                if (I != curI) {
                    flush();
                    if (graph_counts) {
                        const uint32_t gI = graph_of_row_block(graph_rows, num_graphs, I);
                        if (gI != g_cur) {
                            flush_graph(acc, acc_total, graph_counts, g_cur, lane);
                            g_cur = gI;
                            if constexpr (kSeg) sg = segs[gI];
                        }
                    }
                    curI = I;
                    a0 = indptr[I];
                    alen = indptr[I + 1] - a0;
                }
                cp_async_wait_pending<kRing - 1>();
                __syncwarp();
                const uint32_t* S = s.ring[(t - gb) % kRing];
                uint32_t w0, w1;
                if constexpr (C == 128) {
                    w0 = S[2 * lane];
                    w1 = S[2 * lane + 1];
                } else {
                    w0 = lane < 16 ? S[lane] : 0u;
                    w1 = 0u;
                }
                const int nnz = (int)__reduce_add_sync(kFull, (unsigned)(__popc(w0) + __popc(w1)));
                // 16x128: lane = 2r + h holds slices j = 4h + q (q = 0..3) of row r
                // 16x32 : lane = r (< 16) holds slices j = q (q = 0..1) of row r
                constexpr int QN = C == 128 ? 4 : 2;
                if (nnz > tau) {
                    uint32_t active = 0;
#pragma unroll
                    for (int q = 0; q < QN; ++q) {
                        const uint32_t sl = ((q < 2 ? w0 : w1) >> (16 * (q & 1))) & 0xFFFFu;
                        const unsigned b = __ballot_sync(kFull, sl != 0);
                        if constexpr (C == 128) {
                            if (b & 0x55555555u) active |= 1u << q;
                            if (b & 0xAAAAAAAAu) active |= 1u << (4 + q);
                        } else {
                            if (b) active |= 1u << q;
                        }
                    }
                    dense(S, JL, active);
                } else {
                    const uint32_t r = C == 128 ? (uint32_t)(lane >> 1) : (uint32_t)lane;
#pragma unroll
                    for (int q = 0; q < QN; ++q) {
                        const uint32_t sl = ((q < 2 ? w0 : w1) >> (16 * (q & 1))) & 0xFFFFu;
                        const unsigned b = __ballot_sync(kFull, sl != 0);
                        if (!b) continue;
                        const uint32_t nb = __popc(b);
                        if (ng + nb > (uint32_t)kGCap) flush();
                        if (sl) {
                            const uint32_t k = ng + __popc(b & lt);
                            const uint32_t j = C == 128 ? 4u * (lane & 1) + q : (uint32_t)q;
                            s.gJ[k] = JL * JPT + j;
                            s.gRC[k] = (r << 16) | sl;
                            s.gT[k] = t;
                        }
                        ng += nb;
                    }
                }
                __syncwarp();  // the ring slot is refilled by the next tile's prefetch
            }
        }
        // buffered groups stay: the next grab often continues the same row block
        cp_async_wait_all();
        grab_range(__shfl_sync(kFull, kq, 0), gb, ge);
    }
    cp_async_wait_all();
    flush();

    if (graph_counts) {
        flush_graph(acc, acc_total, graph_counts, g_cur, lane);
        acc = acc_total;
    }
    finish_count<kRThreads>(acc, scr, build_failed, s_red, &s_last);
}


using RowsKernel = decltype(&k_count_rows<128, 5, false>);

// variant 0: 16x128 sparse, 1: 16x128 dense, 2: 16x32; 3-5: the same for batch unions
RowsKernel rows_kernel(int v)
{
    switch (v) {
    case 0: return k_count_rows<128, 5, false>;
    case 1: return k_count_rows<128, 4, false>;
    case 2: return k_count_rows<32, 4, false>;
    case 3: return k_count_rows<128, 5, true>;
    case 4: return k_count_rows<128, 4, true>;
    default: return k_count_rows<32, 4, true>;
    }
}

int rows_variant(int tile_cols, bool dense, bool seg)
{
    return (seg ? 3 : 0) + (tile_cols == 128 ? (dense ? 1 : 0) : 2);
}

// Resident CTAs per SM of a row-wise kernel variant (dynamic shared memory above 48 KB is
// an opt-in per function, set here once per device); 0 on error.
int rows_variant_blocks_per_sm(int v)
{
    static std::atomic<int> resident[64][6];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    int per_sm = resident[dev][v].load(std::memory_order_acquire);
    if (per_sm > 0) return per_sm;
    const size_t smem = v % 3 == 2 ? rows_smem_bytes<32>() : rows_smem_bytes<128>();
    const RowsKernel k = rows_kernel(v);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kRThreads, smem);
    if (e != cudaSuccess || per_sm < 1) {
        note_cuda_error(e, "k_count_rows launch set-up", __FILE__, __LINE__);
        return 0;
    }
    resident[dev][v].store(per_sm, std::memory_order_release);
    return per_sm;
}

}  // namespace

// Resident CTAs per SM of the row-wise kernel: the most any of its variants for this tile
// width runs (what a count's scratch must hold partial sums for); 0 on error.
int rows_blocks_per_sm(int tile_cols)
{
    int most = 0;
    for (bool seg : {false, true})
        for (bool dense : {false, true}) {
            const int p = rows_variant_blocks_per_sm(rows_variant(tile_cols, dense, seg));
            most = p > most ? p : most;
        }
    return most;
}

int launch_count_rows(int tile_cols, const uint32_t* indptr, const uint32_t* indices,
                      const uint32_t* row_indices, const uint32_t* blocks, uint32_t num_tiles,
                      uint32_t tile_begin, uint32_t tile_end, int32_t n_row_blocks, int tau,
                      uint32_t chunk, CountScratch scr, const uint32_t* graph_rows,
                      uint32_t num_graphs, unsigned long long* graph_counts,
                      const uint32_t* rowmask, const uint2* cellpp, uint64_t cell_wpr,
                      const uint32_t* row_off, const uint2* row_ent, const GraphSeg* segs,
                      const unsigned long long* build_meta, bool dense, int grid, cudaStream_t s)
{
    // the persistent grid is this kernel's resident CTAs, at most `grid` (the CTAs the
    // caller's scratch holds a partial sum for)
    const int v = rows_variant(tile_cols, dense, segs != nullptr);
    const size_t smem = v % 3 == 2 ? rows_smem_bytes<32>() : rows_smem_bytes<128>();
    const int per_sm = rows_variant_blocks_per_sm(v);
    if (per_sm < 1) return BTC_E_CUDA;
    if (per_sm * device_sm_count() < grid) grid = per_sm * device_sm_count();
    rows_kernel(v)<<<grid, kRThreads, smem, s>>>(indptr, indices, row_indices, blocks, num_tiles,
                                                 tile_begin, tile_end, n_row_blocks, tau, chunk, scr,
                                                 graph_rows, num_graphs, graph_counts, rowmask,
                                                 cellpp, cell_wpr, row_off, row_ent, segs, build_meta);
    return cudaGetLastError() == cudaSuccess ? BTC_OK : BTC_E_CUDA;
}

}  // namespace btc200
