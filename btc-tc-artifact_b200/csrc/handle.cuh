// handle.cuh -- the engine's device-resident handle (private to the library).
#pragma once

#include "common.cuh"

// Arguments and buffers of an enqueued build (a cached build graph replays only when
// they are unchanged).
constexpr int kBuildKeyPtrs = 23;
struct BuildGraphKey {
    const void* ptr[kBuildKeyPtrs];
    int64_t m;
    int32_t n;
    int32_t tile_cols;
    uint32_t flags;
    uint32_t cap;
};

struct btc_bitbsr {
    int device = 0;
    int tile_cols = 0;
    int32_t n = 0;
    int32_t n_row_blocks = 0;
    uint32_t num_tiles = 0;
    int64_t input_edges = 0;
    // Bit-BSR arrays (reference layout)
    btc200::DevBuf indptr, indices, row_indices, blocks, result, rowmask;
    // row index of the row-wise count kernel (rowindex.cu): per-vertex list offsets and
    // (column block, tile) entries, plus the scan's scratch
    btc200::DevBuf row_off, row_ent, row_tot, row_bsum;
    // build workspace
    btc200::DevBuf in_src, in_dst, keys0, keys1, sort_scratch, tile_base, meta, deg, rank, bitmap, prefix;
    bool used_bitmap = false;
    bool row_index = false;  // the last build made the row index (its graph can be heavy)
    // count scratch
    btc200::DevBuf partials, done;
    unsigned long long* h_meta = nullptr;  // pinned and mapped, 8 slots
    unsigned long long* d_hmeta = nullptr; // the device's address of h_meta
    bool edges_known = false;
    int64_t num_edges = 0;
    // BTC_BUILD_ASYNC: the build is enqueued and its metadata copy to h_meta is marked
    // by meta_event; num_tiles is the previous build's until resolve_build() has waited.
    bool pending = false;
    uint32_t pending_cap = 0;  // tile capacity the enqueued build ran against
    int failed = 0;  // status of the last build (BTC_OK once resolved without error)
    cudaEvent_t meta_event = nullptr;
    // CUDA graph of a repeated asynchronous rebuild (captured on the second identical call)
    cudaGraphExec_t graph_exec = nullptr;
    BuildGraphKey graph_key{};
    BuildGraphKey last_key{};
    cudaStream_t capture_stream = nullptr;

    template <class F>
    void for_each_buf(F f)
    {
        btc200::DevBuf* all[] = {&indptr, &indices, &row_indices, &blocks, &result, &in_src, &in_dst,
                                 &keys0, &keys1, &sort_scratch, &tile_base, &meta, &deg, &rank,
                                 &bitmap, &prefix, &partials, &done, &rowmask, &row_off, &row_ent,
                                 &row_tot, &row_bsum};
        for (btc200::DevBuf* b : all) f(*b);
    }
    size_t device_bytes() const
    {
        size_t s = 0;
        const_cast<btc_bitbsr*>(this)->for_each_buf([&](btc200::DevBuf& b) { s += b.bytes; });
        return s;
    }
    // every later allocation of this handle is stream-ordered on `s` from `pool` (the
    // handle is then used on `s` only)
    void set_pool(cudaMemPool_t pool, cudaStream_t s)
    {
        for_each_buf([&](btc200::DevBuf& b) {
            b.pool = pool;
            b.stream = s;
        });
    }
    void release_all()
    {
        for_each_buf([](btc200::DevBuf& b) { b.release(); });
        if (h_meta) cudaFreeHost(h_meta);
        h_meta = nullptr;
        d_hmeta = nullptr;
        if (meta_event) cudaEventDestroy(meta_event);
        meta_event = nullptr;
        pending = false;
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
        if (capture_stream) cudaStreamDestroy(capture_stream);
        capture_stream = nullptr;
        graph_key = BuildGraphKey{};
        last_key = BuildGraphKey{};
    }
};

// Waits for an enqueued (BTC_BUILD_ASYNC) build's metadata if one is pending, sets
// num_tiles and returns the build's status (BTC_E_RANGE, BTC_E_CAPACITY or BTC_OK).
int resolve_build(btc_bitbsr* g);


int default_tau(int tile_cols);
int ensure_count_scratch(btc_bitbsr* g);
// Counts tiles [tile_begin, tile_end) (clamped to the tile count) into g->result and,
// when d_out2 is given, *d_out2.
int count_handle(btc_bitbsr* g, int tau, cudaStream_t s, unsigned long long* d_out2,
                 uint32_t tile_begin = 0, uint32_t tile_end = 0xffffffffu, bool to_host = false);
// Allocates the handle's mapped pinned metadata slots (h_meta, d_hmeta) once.
int ensure_host_meta(btc_bitbsr* g);
