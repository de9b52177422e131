// capi.cu -- the C ABI (include/btc_c.h): handles, build pipeline, count calls and
// the reference-shaped struct surface.  Host code only; kernels live in radix.cu,
// build.cu and count.cu.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "common.cuh"
#include "handle.cuh"

namespace btc200 {

int launch_degree(const int32_t*, const int32_t*, int64_t, int32_t, uint32_t*, cudaStream_t);
int launch_rank_keys(const uint32_t*, int32_t, uint32_t, uint64_t*, cudaStream_t);
int launch_rank_scatter(const uint64_t*, int32_t, int32_t*, cudaStream_t);
int launch_make_keys(const BuildGeom&, const int32_t*, const int32_t*, int64_t, const int32_t*,
                     uint64_t*, unsigned long long*, cudaStream_t);
int launch_segment(const BuildGeom&, const uint64_t*, size_t, const unsigned long long*, uint32_t*,
                   unsigned long long*, cudaStream_t);
int launch_fill(const BuildGeom&, const uint64_t*, size_t, const unsigned long long*,
                const uint32_t*, uint32_t*, uint32_t*, uint32_t*, cudaStream_t);
uint64_t bitmap_words_per_row(const BuildGeom&);
size_t bitmap_chunks(uint64_t W);
int bitmap_mark_and_count(const BuildGeom&, const int32_t*, const int32_t*, int64_t, const int32_t*,
                          uint32_t*, uint32_t*, unsigned long long*, unsigned long long*, cudaStream_t);
int bitmap_emit_and_fill(const BuildGeom&, const int32_t*, const int32_t*, int64_t, const int32_t*,
                         const uint32_t*, const uint32_t*, uint32_t*, uint32_t*, uint32_t*, uint32_t*,
                         uint32_t*, const unsigned long long*, cudaStream_t);
int launch_popcount_sum(int, const uint32_t*, uint64_t, unsigned long long*, cudaStream_t);
int launch_indptr(const uint32_t*, uint32_t, int32_t, uint32_t*, cudaStream_t);
int launch_density(int, const uint32_t*, uint32_t, unsigned long long*, cudaStream_t);
int launch_set_u64(unsigned long long* p, unsigned long long v, cudaStream_t s);

void note_cuda_error(cudaError_t e, const char* what, const char* file, int line)
{
    static const bool verbose = std::getenv("BTC_DEBUG") != nullptr;
    if (verbose)
        std::fprintf(stderr, "[btc] CUDA error %s (%s) at %s:%d: %s\n", cudaGetErrorName(e),
                     cudaGetErrorString(e), file, line, what);
}

int device_sm_count()
{
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}

}  // namespace btc200

using namespace btc200;

// Engine's default dense/sparse switch.  A tile takes the binary tensor-core path
// when its popcount exceeds tau.
int default_tau(int tile_cols) { return tile_cols == 128 ? 512 : 64; }

static constexpr uint64_t kMaxEdges = (1ull << 32) - (uint64_t)kSortTile;

int ensure_count_scratch(btc_bitbsr* g)
{
    const int grid = count_grid_size(128) > count_grid_size(32) ? count_grid_size(128)
                                                                 : count_grid_size(32);
    const size_t need = sizeof(unsigned long long) * (size_t)grid;
    if (g->partials.bytes < need) BTC_TRY(g->partials.reserve(need));
    if (!g->done.ptr) {
        BTC_TRY(g->done.reserve(kCountCtlBytes));
        BTC_CUDA_TRY(cudaMemset(g->done.ptr, 0, kCountCtlBytes));
    }
    if (!g->result.ptr) {
        BTC_TRY(g->result.reserve(sizeof(unsigned long long)));
        BTC_CUDA_TRY(cudaMemset(g->result.ptr, 0, sizeof(unsigned long long)));
    }
    return BTC_OK;
}

static int build_into(btc_bitbsr* g, const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                      int tile_cols, uint32_t flags, cudaStream_t s)
{
    if (n < 0 || m < 0 || (uint64_t)m > kMaxEdges) return BTC_E_INVAL;
    if (m > 0 && (!src || !dst)) return BTC_E_INVAL;
    if (flags & ~(BTC_INPUT_ON_HOST | BTC_ORIENT_DEGREE | BTC_BUILD_RADIX)) return BTC_E_INVAL;
    if (tile_cols == 0) tile_cols = btc_lite_select_tile_cols(m, n, 0);
    if (tile_cols != 32 && tile_cols != 128) return BTC_E_INVAL;
    BTC_CUDA_TRY(cudaGetDevice(&g->device));

    const BuildGeom geom = make_geom(n, tile_cols);
    g->tile_cols = tile_cols;
    g->n = n;
    g->n_row_blocks = geom.n_row_blocks;
    g->input_edges = m;
    g->edges_known = false;
    g->num_edges = 0;

    if (!g->h_meta) {
        void* p = nullptr;
        if (cudaMallocHost(&p, sizeof(unsigned long long) * kMetaSlots) != cudaSuccess) {
            cudaGetLastError();
            return BTC_E_NOMEM;
        }
        g->h_meta = static_cast<unsigned long long*>(p);
    }
    BTC_TRY(g->meta.reserve(sizeof(unsigned long long) * kMetaSlots));
    unsigned long long* meta = g->meta.as<unsigned long long>();
    BTC_CUDA_TRY(cudaMemsetAsync(meta, 0, sizeof(unsigned long long) * kMetaSlots, s));

    // ---- input --------------------------------------------------------------
    const int32_t* d_src = src;
    const int32_t* d_dst = dst;
    if ((flags & BTC_INPUT_ON_HOST) && m > 0) {
        BTC_TRY(g->in_src.reserve(sizeof(int32_t) * (size_t)m));
        BTC_TRY(g->in_dst.reserve(sizeof(int32_t) * (size_t)m));
        BTC_CUDA_TRY(cudaMemcpyAsync(g->in_src.ptr, src, sizeof(int32_t) * (size_t)m,
                                     cudaMemcpyHostToDevice, s));
        BTC_CUDA_TRY(cudaMemcpyAsync(g->in_dst.ptr, dst, sizeof(int32_t) * (size_t)m,
                                     cudaMemcpyHostToDevice, s));
        d_src = g->in_src.as<int32_t>();
        d_dst = g->in_dst.as<int32_t>();
    }

    // The cell bitmap (one bit per (row block, column block)) replaces the sort when it
    // is small next to the edge list; otherwise the radix path sorts tile keys.
    const uint64_t wpr = bitmap_words_per_row(geom);
    const uint64_t bm_words = wpr * (uint64_t)geom.n_row_blocks;
    const uint64_t bm_bytes = 4 * bm_words;
    const bool use_bitmap = !(flags & BTC_BUILD_RADIX) && bm_bytes <= (4ull << 30) &&
                            bm_bytes <= 32ull * (uint64_t)m + (64ull << 20);
    g->used_bitmap = use_bitmap;

    const bool degree = (flags & BTC_ORIENT_DEGREE) && n > 0;
    size_t key_cap = use_bitmap ? 0 : (size_t)m;
    if (degree && (size_t)n > key_cap) key_cap = (size_t)n;
    if (key_cap) {
        BTC_TRY(g->keys0.reserve(sizeof(uint64_t) * key_cap));
        BTC_TRY(g->keys1.reserve(sizeof(uint64_t) * key_cap));
        BTC_TRY(g->sort_scratch.reserve(sizeof(uint32_t) * radix_scratch_words(key_cap)));
    }
    const size_t chunk_slots =
        use_bitmap ? bitmap_chunks(bm_words) : sort_tiles((size_t)m);
    BTC_TRY(g->tile_base.reserve(sizeof(uint32_t) * (chunk_slots + 1)));
    uint64_t* k0 = g->keys0.as<uint64_t>();
    uint64_t* k1 = g->keys1.as<uint64_t>();
    int st = BTC_OK;

    // ---- optional descending-degree relabel ---------------------------------
    const int32_t* rank = nullptr;
    if (degree) {
        BTC_TRY(g->deg.reserve(sizeof(uint32_t) * (size_t)n));
        BTC_TRY(g->rank.reserve(sizeof(int32_t) * (size_t)n));
        BTC_CUDA_TRY(cudaMemsetAsync(g->deg.ptr, 0, sizeof(uint32_t) * (size_t)n, s));
        BTC_TRY(launch_degree(d_src, d_dst, m, n, g->deg.as<uint32_t>(), s));
        int db = bit_length_u64(2ull * (uint64_t)m);  // degrees fit in db bits
        if (db > 32) db = 32;
        const uint32_t dmax = db >= 32 ? 0xffffffffu : ((1u << db) - 1u);
        BTC_TRY(launch_rank_keys(g->deg.as<uint32_t>(), n, dmax, k0, s));
        BTC_TRY(launch_set_u64(meta + kMetaN, (unsigned long long)n, s));
        uint64_t* sorted = radix_sort_u64(k0, k1, (size_t)n, meta + kMetaN, 32, 32 + (db ? db : 1),
                                          g->sort_scratch.as<uint32_t>(), s, &st);
        BTC_TRY(st);
        BTC_TRY(launch_rank_scatter(sorted, n, g->rank.as<int32_t>(), s));
        rank = g->rank.as<int32_t>();
    }

    const size_t TW = (size_t)16 * (tile_cols / 32);
    uint64_t* sorted = nullptr;
    if (use_bitmap) {
        BTC_TRY(g->bitmap.reserve(sizeof(uint32_t) * (bm_words ? bm_words : 1)));
        BTC_TRY(g->prefix.reserve(sizeof(uint32_t) * (bm_words ? bm_words : 1)));
        BTC_TRY(bitmap_mark_and_count(geom, d_src, d_dst, m, rank, g->bitmap.as<uint32_t>(),
                                      g->tile_base.as<uint32_t>(), meta + kMetaBad,
                                      meta + kMetaTiles, s));
    } else {
        // ---- keys, sort, segmentation ---------------------------------------
        BTC_TRY(launch_make_keys(geom, d_src, d_dst, m, rank, k0, meta, s));
        sorted = radix_sort_u64(k0, k1, (size_t)m, meta + kMetaValid, geom.payload_bits,
                                geom.payload_bits + geom.t_bits, g->sort_scratch.as<uint32_t>(), s,
                                &st);
        BTC_TRY(st);
        BTC_TRY(launch_segment(geom, sorted, (size_t)m, meta + kMetaValid,
                               g->tile_base.as<uint32_t>(), meta + kMetaTiles, s));
    }
    BTC_CUDA_TRY(cudaMemcpyAsync(g->h_meta, meta, sizeof(unsigned long long) * 3,
                                 cudaMemcpyDeviceToHost, s));
    BTC_CUDA_TRY(cudaStreamSynchronize(s));
    if (g->h_meta[kMetaBad] != 0) return BTC_E_RANGE;
    const unsigned long long tiles = g->h_meta[kMetaTiles];
    if (tiles > 0xffffffffull) return BTC_E_INVAL;
    g->num_tiles = (uint32_t)tiles;

    // ---- tile arrays ----------------------------------------------------------
    BTC_TRY(g->indptr.reserve(sizeof(uint32_t) * ((size_t)geom.n_row_blocks + 1)));
    BTC_TRY(g->indices.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    BTC_TRY(g->row_indices.reserve(sizeof(uint32_t) * (tiles ? tiles : 1)));
    BTC_TRY(g->blocks.reserve(sizeof(uint32_t) * TW * (tiles ? tiles : 1)));
    BTC_TRY(ensure_count_scratch(g));
    if (tiles)
        BTC_CUDA_TRY(cudaMemsetAsync(g->blocks.ptr, 0, sizeof(uint32_t) * TW * tiles, s));
    if (use_bitmap) {
        BTC_TRY(bitmap_emit_and_fill(geom, d_src, d_dst, m, rank, g->bitmap.as<uint32_t>(),
                                     g->tile_base.as<uint32_t>(), g->prefix.as<uint32_t>(),
                                     g->indices.as<uint32_t>(), g->row_indices.as<uint32_t>(),
                                     g->indptr.as<uint32_t>(), g->blocks.as<uint32_t>(),
                                     meta + kMetaTiles, s));
    } else {
        BTC_TRY(launch_fill(geom, sorted, (size_t)m, meta + kMetaValid, g->tile_base.as<uint32_t>(),
                            g->indices.as<uint32_t>(), g->row_indices.as<uint32_t>(),
                            g->blocks.as<uint32_t>(), s));
        BTC_TRY(launch_indptr(g->row_indices.as<uint32_t>(), g->num_tiles, geom.n_row_blocks,
                              g->indptr.as<uint32_t>(), s));
    }
    BTC_TRY(g->rowmask.reserve(sizeof(uint32_t) * (tiles + 1)));
    BTC_TRY(launch_rowmask(tile_cols, g->blocks.as<uint32_t>(), g->num_tiles,
                           g->indptr.as<uint32_t>(), g->n_row_blocks, g->rowmask.as<uint32_t>(),
                           s));
    return BTC_OK;
}

int count_handle(btc_bitbsr* g, int tau, cudaStream_t s, unsigned long long* d_out2,
                 uint32_t tile_begin, uint32_t tile_end)
{
    if (!g) return BTC_E_INVAL;
    if (tau == BTC_TAU_DEFAULT) tau = default_tau(g->tile_cols);
    if (tau < 0) return BTC_E_INVAL;
    BTC_TRY(ensure_count_scratch(g));
    CountScratch scr{g->partials.as<unsigned long long>(), g->done.as<unsigned int>(),
                     reinterpret_cast<unsigned long long*>(g->done.as<char>() + 8),
                     g->result.as<unsigned long long>(), d_out2};
    return launch_count(g->tile_cols, g->indptr.as<uint32_t>(), g->indices.as<uint32_t>(),
                        g->row_indices.as<uint32_t>(), g->blocks.as<uint32_t>(), g->num_tiles,
                        g->n_row_blocks, tau, scr, s, nullptr, 0, nullptr,
                        g->rowmask.as<uint32_t>(),
                        g->used_bitmap ? g->bitmap.as<uint32_t>() : nullptr,
                        g->used_bitmap ? g->prefix.as<uint32_t>() : nullptr,
                        bitmap_words_per_row(make_geom(g->n, g->tile_cols)),
                        g->rowmask.as<uint32_t>() + g->num_tiles, tile_begin, tile_end);
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int btc_abi_version(void) { return (1 << 16) | 0; }

int btc_default_tau(int tile_cols) { return default_tau(tile_cols); }

const char* btc_strerror(int status)
{
    switch (status) {
    case BTC_OK: return "ok";
    case BTC_E_INVAL: return "invalid argument";
    case BTC_E_NOMEM: return "out of memory";
    case BTC_E_CUDA: return "CUDA error";
    case BTC_E_TIMEOUT: return "device wait timed out";
    case BTC_E_RANGE: return "vertex id out of range";
    default: return "unknown status";
    }
}

int btc_lite_select_tile_cols(int64_t nnz, int32_t num_rows, int mode)
{
    if (mode == 1) return 32;
    if (mode == 2) return 128;
    const float avg = num_rows > 0 ? (float)nnz / (float)num_rows : 0.0f;
    return (avg < 15.0f || num_rows < 50000) ? 32 : 128;
}

int btc_build_bitbsr(const int32_t* src, const int32_t* dst, int64_t m, int32_t n, int tile_cols,
                     uint32_t flags, btc_stream_t stream, btc_bitbsr** out)
{
    if (!out) return BTC_E_INVAL;
    *out = nullptr;
    btc_bitbsr* g = new (std::nothrow) btc_bitbsr();
    if (!g) return BTC_E_NOMEM;
    const int st = build_into(g, src, dst, m, n, tile_cols, flags, stream);
    if (st != BTC_OK) {
        g->release_all();
        delete g;
        return st;
    }
    *out = g;
    return BTC_OK;
}

int btc_rebuild_bitbsr(btc_bitbsr* g, const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                       int tile_cols, uint32_t flags, btc_stream_t stream)
{
    if (!g) return BTC_E_INVAL;
    return build_into(g, src, dst, m, n, tile_cols, flags, stream);
}

int btc_count_async(btc_bitbsr* g, int tau, btc_stream_t stream, unsigned long long* d_out)
{
    return count_handle(g, tau, stream, d_out);
}

int btc_count(btc_bitbsr* g, int tau, btc_stream_t stream, unsigned long long* out_count,
              float* kernel_ms)
{
    if (!g || !out_count) return BTC_E_INVAL;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernel_ms) {
        BTC_CUDA_TRY(cudaEventCreate(&e0));
        BTC_CUDA_TRY(cudaEventCreate(&e1));
        BTC_CUDA_TRY(cudaEventRecord(e0, stream));
    }
    int st = count_handle(g, tau, stream, nullptr);
    if (st == BTC_OK && kernel_ms && cudaEventRecord(e1, stream) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK &&
        cudaMemcpyAsync(g->h_meta + 7, g->result.ptr, sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        st = BTC_E_CUDA;
    if (st == BTC_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK) {
        *out_count = g->h_meta[7];
        if (kernel_ms) cudaEventElapsedTime(kernel_ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return st;
}

int btc_bitbsr_info(const btc_bitbsr* gc, btc_bitbsr_view* v)
{
    if (!gc || !v) return BTC_E_INVAL;
    btc_bitbsr* g = const_cast<btc_bitbsr*>(gc);
    if (!g->edges_known) {
        // unique lower edges = bits set in the tiles (duplicates OR the same bit); the
        // build may have run on any stream, so wait for the device first
        BTC_CUDA_TRY(cudaDeviceSynchronize());
        unsigned long long u = 0;
        unsigned long long* d = g->meta.as<unsigned long long>() + kMetaUniq;
        BTC_TRY(launch_popcount_sum(g->tile_cols, g->blocks.as<uint32_t>(), g->num_tiles, d, nullptr));
        BTC_CUDA_TRY(cudaMemcpy(&u, d, sizeof(u), cudaMemcpyDeviceToHost));
        g->num_edges = (int64_t)u;
        g->edges_known = true;
    }
    std::memset(v, 0, sizeof(*v));
    v->bcsr.indptr = g->indptr.as<uint32_t>();
    v->bcsr.indices = g->indices.as<uint32_t>();
    v->bcsr.blocks = g->blocks.as<uint32_t>();
    v->bcsr.row_indices = g->row_indices.as<uint32_t>();
    v->bcsr.result = g->result.as<unsigned long long>();
    v->bcsr.n = g->n;
    v->bcsr.n_row_blocks = g->n_row_blocks;
    v->bcsr.num_blocks = g->num_tiles;
    v->tile_cols = g->tile_cols;
    v->device = g->device;
    v->num_edges = g->num_edges;
    v->input_edges = g->input_edges;
    v->device_bytes = g->device_bytes();
    return BTC_OK;
}

int btc_density_hist(btc_bitbsr* g, btc_stream_t stream, uint64_t* hist)
{
    if (!g || !hist) return BTC_E_INVAL;
    const size_t nb = (size_t)16 * g->tile_cols + 1;
    DevBuf d;
    BTC_TRY(d.reserve(sizeof(unsigned long long) * nb));
    int st = BTC_OK;
    if (cudaMemsetAsync(d.ptr, 0, sizeof(unsigned long long) * nb, stream) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK)
        st = launch_density(g->tile_cols, g->blocks.as<uint32_t>(), g->num_tiles,
                            d.as<unsigned long long>(), stream);
    if (st == BTC_OK && cudaMemcpyAsync(hist, d.ptr, sizeof(unsigned long long) * nb,
                                        cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        st = BTC_E_CUDA;
    if (st == BTC_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = BTC_E_CUDA;
    d.release();
    return st;
}

void btc_free(btc_bitbsr* g)
{
    if (!g) return;
    g->release_all();
    delete g;
}

// ---------------------------------------------------------------------------
// reference-shaped struct surface
// ---------------------------------------------------------------------------
static int convert_struct(btc_bcsr_device* b, const int32_t* d_rows, const int32_t* d_cols,
                          int64_t nnz, int32_t num_rows, int tile_cols)
{
    if (!b) return BTC_E_INVAL;
    std::memset(b, 0, sizeof(*b));
    btc_bitbsr* g = nullptr;
    const int st = btc_build_bitbsr(d_rows, d_cols, nnz, num_rows, tile_cols, 0, nullptr, &g);
    if (st != BTC_OK) return st;
    // hand the arrays to the struct; it frees them one by one (btc_bcsr_free)
    b->indptr = g->indptr.as<uint32_t>();
    b->indices = g->indices.as<uint32_t>();
    b->blocks = g->blocks.as<uint32_t>();
    b->row_indices = g->row_indices.as<uint32_t>();
    b->result = g->result.as<unsigned long long>();
    b->n = g->n;
    b->n_row_blocks = g->n_row_blocks;
    b->num_blocks = g->num_tiles;
    g->indptr.ptr = g->indices.ptr = g->blocks.ptr = g->row_indices.ptr = g->result.ptr = nullptr;
    g->indptr.bytes = g->indices.bytes = g->blocks.bytes = g->row_indices.bytes = g->result.bytes = 0;
    btc_free(g);
    return BTC_OK;
}

int btc_convert_coo_to_bcsr_16x128_gpu(btc_bcsr_device* b, const int32_t* d_rows,
                                       const int32_t* d_cols, int64_t nnz, int32_t num_rows)
{
    return convert_struct(b, d_rows, d_cols, nnz, num_rows, 128);
}

int btc_convert_coo_to_bcsr_16x32_gpu(btc_bcsr_device* b, const int32_t* d_rows,
                                      const int32_t* d_cols, int64_t nnz, int32_t num_rows)
{
    return convert_struct(b, d_rows, d_cols, nnz, num_rows, 32);
}

void btc_bcsr_free(btc_bcsr_device* b)
{
    if (!b) return;
    if (b->indptr) cudaFree(b->indptr);
    if (b->indices) cudaFree(b->indices);
    if (b->blocks) cudaFree(b->blocks);
    if (b->row_indices) cudaFree(b->row_indices);
    if (b->result) cudaFree(b->result);
    b->indptr = b->indices = b->blocks = b->row_indices = nullptr;
    b->result = nullptr;
}

int btc_bcsr_reset_result(btc_bcsr_device* b)
{
    if (!b || !b->result) return BTC_E_INVAL;
    BTC_CUDA_TRY(cudaMemset(b->result, 0, sizeof(unsigned long long)));
    return BTC_OK;
}

int btc_bcsr_get_result(const btc_bcsr_device* b, unsigned long long* out)
{
    if (!b || !b->result || !out) return BTC_E_INVAL;
    BTC_CUDA_TRY(cudaMemcpy(out, b->result, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return BTC_OK;
}

}  // extern "C"

// Per-device count scratch for the struct surface, whose calls are blocking; a mutex
// serialises them.
namespace {
struct StructScratch {
    std::mutex mu;
    DevBuf partials[64];
    DevBuf done[64];
};
StructScratch& struct_scratch()
{
    static StructScratch s;
    return s;
}
}  // namespace

static int count_struct(btc_bcsr_device* b, int tile_cols, float* kernel_ms,
                        unsigned long long* out)
{
    if (!b || !b->result || !out) return BTC_E_INVAL;
    if (b->num_blocks && (!b->indptr || !b->indices || !b->blocks || !b->row_indices))
        return BTC_E_INVAL;
    int dev = 0;
    BTC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return BTC_E_INVAL;
    StructScratch& ss = struct_scratch();
    std::lock_guard<std::mutex> lock(ss.mu);
    const size_t need = sizeof(unsigned long long) * (size_t)count_grid_size(tile_cols);
    if (ss.partials[dev].bytes < need) BTC_TRY(ss.partials[dev].reserve(need));
    if (!ss.done[dev].ptr) {
        BTC_TRY(ss.done[dev].reserve(kCountCtlBytes));
        BTC_CUDA_TRY(cudaMemset(ss.done[dev].ptr, 0, kCountCtlBytes));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernel_ms) {
        BTC_CUDA_TRY(cudaEventCreate(&e0));
        BTC_CUDA_TRY(cudaEventCreate(&e1));
        BTC_CUDA_TRY(cudaEventRecord(e0, nullptr));
    }
    CountScratch scr{ss.partials[dev].as<unsigned long long>(), ss.done[dev].as<unsigned int>(),
                     reinterpret_cast<unsigned long long*>(ss.done[dev].as<char>() + 8), b->result,
                     nullptr};
    int st = launch_count(tile_cols, b->indptr, b->indices, b->row_indices, b->blocks, b->num_blocks,
                          b->n_row_blocks, default_tau(tile_cols), scr, nullptr);
    if (st == BTC_OK && kernel_ms && cudaEventRecord(e1, nullptr) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK && cudaMemcpy(out, b->result, sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost) != cudaSuccess)
        st = BTC_E_CUDA;
    if (st == BTC_OK && kernel_ms) cudaEventElapsedTime(kernel_ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return st;
}

extern "C" int btc_count_triangles_16x128_adaptive(btc_bcsr_device* b, int threshold_blocks,
                                                   float* kernel_ms, unsigned long long* out)
{
    (void)threshold_blocks;
    return count_struct(b, 128, kernel_ms, out);
}

extern "C" int btc_count_triangles_16x32_adaptive(btc_bcsr_device* b, int threshold_blocks,
                                                  float* kernel_ms, unsigned long long* out)
{
    (void)threshold_blocks;
    return count_struct(b, 32, kernel_ms, out);
}
