/*
 * oracle.c -- CPU restatement of the BTC-TC hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA engine: only tests/, the smoke entry
 * point and bench.py's cpu_baseline leg may load it.  Nothing in the product
 * path calls it, and the product has no CPU fallback.
 *
 * What it restates (paths are within fanna1234/btc-tc-artifact):
 *   orc_lower_csr        btc/operations/convert.h:280-324 (orient to (max,min), drop
 *                        self-loops, lexicographic sort, unique) and the
 *                        OrientLowerTriangular functor, btc/operations/reorder.h:39-46.
 *                        Optional descending-degree relabel first (the engine's
 *                        BTC_ORIENT_DEGREE flag; the reference orients by id only).
 *   orc_tc_merge         btc/operations/triangle_count_cpu.h:59-101
 *                        (merge-based L (.) L L^T on a lower-triangular CSR).
 *   orc_bitbsr_*         btc/operations/bcsr_16x128.h:136-241 and
 *                        btc/operations/bcsr_16x32.h:144-249 (Bit-BSR layout: tiles in
 *                        (row block, column block) order, indptr over row blocks,
 *                        bit (32w+b) of tile row r = word r*W+w, bit b).
 *   orc_bitbsr_count     btc/operations/tc_16x128_mma_v5.h:9-211 and
 *                        btc/operations/tc_16x32_mma_v6.h:9-238 (for every tile S=(I,J_L),
 *                        every 16-row block J_out covered by S's columns, every K
 *                        common to rows I and J_out: sum over mask bits (r,c) of S of
 *                        popc(L[I,K][r] & L[J_out,K][c])).  Accumulates in uint64.
 *   orc_bitbsr_count_range  the same sum over a range of sample tiles (the unit a rank
 *                        of a multi-GPU count takes).
 *
 * Parity pin: counts are pinned against the reference's own CPU path
 * (triangle_count_cpu.h compiled from the reference headers by oracle/ref/Makefile)
 * on every fixture under tests/golden, and against closed forms (K_n, bipartite
 * stencils, the 27-point 64^3 stencil).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* helpers                                                                   */
/* ------------------------------------------------------------------------- */

static int cmp_i32(const void* a, const void* b)
{
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* rank[v] for descending degree, ties by ascending id.  Degrees count every
 * input pair with u != v (duplicates included), so the order is a function of
 * the input multiset alone. */
static void degree_rank(const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                        int32_t* rank)
{
    int64_t* deg = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t e = 0; e < m; ++e) {
        if (src[e] == dst[e]) continue;
        deg[src[e]]++;
        deg[dst[e]]++;
    }
    int64_t maxd = 0;
    for (int32_t v = 0; v < n; ++v) if (deg[v] > maxd) maxd = deg[v];
    /* counting sort by (maxd - deg), stable in id */
    int64_t* cnt = (int64_t*)calloc((size_t)maxd + 2, sizeof(int64_t));
    for (int32_t v = 0; v < n; ++v) cnt[maxd - deg[v] + 1]++;
    for (int64_t k = 1; k <= maxd + 1; ++k) cnt[k] += cnt[k - 1];
    for (int32_t v = 0; v < n; ++v) rank[v] = (int32_t)(cnt[maxd - deg[v]]++);
    free(cnt);
    free(deg);
}

/* ------------------------------------------------------------------------- */
/* lower-triangular extraction                                               */
/* ------------------------------------------------------------------------- */

/* Returns the number of unique lower edges m_L (r > c) and fills rowptr[n+1],
 * col[m_L] (rows sorted, columns ascending and unique).  col must hold m entries.
 * order_mode 0: ids as given; 1: descending-degree relabel.  If rank_out is not
 * NULL it receives the relabel (identity for order_mode 0).  Returns -1 on a
 * vertex id outside [0, n). */
int64_t orc_lower_csr(const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                      int order_mode, int32_t* rowptr, int32_t* col, int32_t* rank_out)
{
    for (int64_t e = 0; e < m; ++e)
        if (src[e] < 0 || src[e] >= n || dst[e] < 0 || dst[e] >= n) return -1;

    int32_t* rank = (int32_t*)malloc(((size_t)n + 1) * sizeof(int32_t));
    if (order_mode == 1) degree_rank(src, dst, m, n, rank);
    else for (int32_t v = 0; v < n; ++v) rank[v] = v;
    if (rank_out) memcpy(rank_out, rank, (size_t)n * sizeof(int32_t));

    int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t e = 0; e < m; ++e) {
        int32_t a = rank[src[e]], b = rank[dst[e]];
        if (a == b) continue;                       /* self-loop */
        int32_t r = a > b ? a : b;                  /* orient to (max, min) */
        cnt[r + 1]++;
    }
    for (int32_t v = 0; v < n; ++v) cnt[v + 1] += cnt[v];
    int64_t* cur = (int64_t*)malloc(((size_t)n + 1) * sizeof(int64_t));
    memcpy(cur, cnt, ((size_t)n + 1) * sizeof(int64_t));
    for (int64_t e = 0; e < m; ++e) {
        int32_t a = rank[src[e]], b = rank[dst[e]];
        if (a == b) continue;
        int32_t r = a > b ? a : b, c = a > b ? b : a;
        col[cur[r]++] = c;
    }
    /* sort + unique within each row, compacting in place */
    int64_t out = 0;
    rowptr[0] = 0;
    for (int32_t r = 0; r < n; ++r) {
        int64_t s = cnt[r], t = cnt[r + 1];
        qsort(col + s, (size_t)(t - s), sizeof(int32_t), cmp_i32);
        for (int64_t i = s; i < t; ++i) {
            if (i > s && col[i] == col[i - 1]) continue;
            col[out++] = col[i];
        }
        rowptr[r + 1] = (int32_t)out;
    }
    free(cur);
    free(cnt);
    free(rank);
    return out;
}

/* ------------------------------------------------------------------------- */
/* merge-based count (triangle_count_cpu.h:59-101)                           */
/* ------------------------------------------------------------------------- */

uint64_t orc_tc_merge(const int32_t* rowptr, const int32_t* col, int32_t n, int threads)
{
    uint64_t total = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 256)
#endif
    for (int32_t r = 0; r < n; ++r) {
        int32_t rs = rowptr[r], re = rowptr[r + 1];
        for (int32_t i = rs; i < re; ++i) {
            int32_t u = col[i];
            int32_t p = rs, q = rowptr[u], qe = rowptr[u + 1];
            while (p < re && q < qe) {
                int32_t a = col[p], b = col[q];
                if (a < b) ++p;
                else if (a > b) ++q;
                else { ++total; ++p; ++q; }
            }
        }
    }
    return total;
}

/* ------------------------------------------------------------------------- */
/* Bit-BSR build (bcsr_16x128.h / bcsr_16x32.h)                              */
/* ------------------------------------------------------------------------- */

/* Number of tiles of the Bit-BSR of a lower CSR with tile width C (32 or 128). */
int64_t orc_bitbsr_num_tiles(const int32_t* rowptr, const int32_t* col, int32_t n, int C)
{
    int32_t R = (n + 15) / 16;
    int32_t ncb = (n + C - 1) / C;
    uint8_t* seen = (uint8_t*)calloc((size_t)ncb + 1, 1);
    int32_t* list = (int32_t*)malloc(((size_t)ncb + 1) * sizeof(int32_t));
    int64_t B = 0;
    for (int32_t I = 0; I < R; ++I) {
        int32_t k = 0;
        for (int32_t r = I * 16; r < I * 16 + 16 && r < n; ++r)
            for (int32_t i = rowptr[r]; i < rowptr[r + 1]; ++i) {
                int32_t cb = col[i] / C;
                if (!seen[cb]) { seen[cb] = 1; list[k++] = cb; }
            }
        B += k;
        for (int32_t t = 0; t < k; ++t) seen[list[t]] = 0;
    }
    free(list);
    free(seen);
    return B;
}

/* Fills indptr[R+1], indices[B], row_indices[B], blocks[B * 16 * C/32] (zeroed
 * here).  Returns B. */
int64_t orc_bitbsr_build(const int32_t* rowptr, const int32_t* col, int32_t n, int C,
                         uint32_t* indptr, uint32_t* indices, uint32_t* row_indices,
                         uint32_t* blocks)
{
    const int WPR = C / 32, TW = 16 * WPR;
    int32_t R = (n + 15) / 16;
    int32_t ncb = (n + C - 1) / C;
    int64_t* slot = (int64_t*)malloc(((size_t)ncb + 1) * sizeof(int64_t));
    for (int32_t k = 0; k <= ncb; ++k) slot[k] = -1;
    int32_t* list = (int32_t*)malloc(((size_t)ncb + 1) * sizeof(int32_t));
    int64_t B = 0;
    indptr[0] = 0;
    for (int32_t I = 0; I < R; ++I) {
        int32_t k = 0;
        for (int32_t r = I * 16; r < I * 16 + 16 && r < n; ++r)
            for (int32_t i = rowptr[r]; i < rowptr[r + 1]; ++i) {
                int32_t cb = col[i] / C;
                if (slot[cb] < 0) { slot[cb] = 0; list[k++] = cb; }
            }
        qsort(list, (size_t)k, sizeof(int32_t), cmp_i32);
        for (int32_t t = 0; t < k; ++t) {
            slot[list[t]] = B + t;
            indices[B + t] = (uint32_t)list[t];
            row_indices[B + t] = (uint32_t)I;
            memset(blocks + (size_t)(B + t) * TW, 0, sizeof(uint32_t) * (size_t)TW);
        }
        for (int32_t r = I * 16; r < I * 16 + 16 && r < n; ++r)
            for (int32_t i = rowptr[r]; i < rowptr[r + 1]; ++i) {
                int32_t c = col[i];
                int64_t t = slot[c / C];
                int pos = (r % 16) * C + (c % C);
                blocks[(size_t)t * TW + pos / 32] |= 1u << (pos % 32);
            }
        for (int32_t t = 0; t < k; ++t) slot[list[t]] = -1;
        B += k;
        indptr[I + 1] = (uint32_t)B;
    }
    free(list);
    free(slot);
    return B;
}

/* Histogram of tile popcounts: hist[p] = #tiles with exactly p bits set,
 * p in [0, 16*C]. */
void orc_bitbsr_density_hist(const uint32_t* blocks, int64_t B, int C, int64_t* hist)
{
    const int TW = 16 * (C / 32);
    memset(hist, 0, sizeof(int64_t) * (size_t)(16 * C + 1));
    for (int64_t t = 0; t < B; ++t) {
        int p = 0;
        for (int w = 0; w < TW; ++w) p += __builtin_popcount(blocks[(size_t)t * TW + w]);
        hist[p]++;
    }
}

/* ------------------------------------------------------------------------- */
/* Bit-BSR count (tc_16x128_mma_v5.h:9-211, tc_16x32_mma_v6.h:9-238)         */
/* ------------------------------------------------------------------------- */

/* Count of the sample tiles [t0, t1) alone; the counts of a partition of [0, B) add
 * up to the whole count (each tile's term of the sum is independent of the others). */
uint64_t orc_bitbsr_count_range(const uint32_t* indptr, const uint32_t* indices,
                                const uint32_t* row_indices, const uint32_t* blocks,
                                int32_t n, int64_t t0, int64_t t1, int C, int threads)
{
    const int WPR = C / 32, TW = 16 * WPR, JPT = C / 16;
    const int32_t R = (n + 15) / 16;
    uint64_t total = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 64)
#endif
    for (int64_t s = t0; s < t1; ++s) {
        const uint32_t I = row_indices[s], JL = indices[s];
        const uint32_t* S = blocks + (size_t)s * TW;
        for (int j = 0; j < JPT; ++j) {
            const int64_t Jout = (int64_t)JL * JPT + j;
            if (Jout >= R) continue;
            /* mask rows: bits [16j, 16j+16) of each tile row of S */
            uint32_t mrow[16];
            int any = 0;
            for (int r = 0; r < 16; ++r) {
                uint32_t w = S[r * WPR + (16 * j) / 32];
                mrow[r] = (w >> ((16 * j) % 32)) & 0xFFFFu;
                any |= mrow[r] != 0;
            }
            if (!any) continue;
            uint32_t pa = indptr[I], ea = indptr[I + 1];
            uint32_t pb = indptr[Jout], eb = indptr[Jout + 1];
            while (pa < ea && pb < eb) {
                uint32_t ka = indices[pa], kb = indices[pb];
                if (ka < kb) { ++pa; continue; }
                if (ka > kb) { ++pb; continue; }
                const uint32_t* A = blocks + (size_t)pa * TW;
                const uint32_t* Bt = blocks + (size_t)pb * TW;
                for (int r = 0; r < 16; ++r) {
                    uint32_t mr = mrow[r];
                    while (mr) {
                        int c = __builtin_ctz(mr);
                        mr &= mr - 1;
                        for (int w = 0; w < WPR; ++w)
                            total += (uint64_t)__builtin_popcount(A[r * WPR + w] & Bt[c * WPR + w]);
                    }
                }
                ++pa;
                ++pb;
            }
        }
    }
    return total;
}

uint64_t orc_bitbsr_count(const uint32_t* indptr, const uint32_t* indices,
                          const uint32_t* row_indices, const uint32_t* blocks,
                          int32_t n, int64_t B, int C, int threads)
{
    return orc_bitbsr_count_range(indptr, indices, row_indices, blocks, n, 0, B, C, threads);
}
