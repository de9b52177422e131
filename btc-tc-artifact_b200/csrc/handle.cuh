// handle.cuh -- the engine's device-resident handle (private to the library).
#pragma once

#include "common.cuh"

struct btc_bitbsr {
    int device = 0;
    int tile_cols = 0;
    int32_t n = 0;
    int32_t n_row_blocks = 0;
    uint32_t num_tiles = 0;
    int64_t input_edges = 0;
    // Bit-BSR arrays (reference layout)
    btc200::DevBuf indptr, indices, row_indices, blocks, result, rowmask;
    // build workspace
    btc200::DevBuf in_src, in_dst, keys0, keys1, sort_scratch, tile_base, meta, deg, rank, bitmap, prefix;
    bool used_bitmap = false;
    // count scratch
    btc200::DevBuf partials, done;
    unsigned long long* h_meta = nullptr;  // pinned, 8 slots
    bool edges_known = false;
    int64_t num_edges = 0;

    size_t device_bytes() const
    {
        const btc200::DevBuf* all[] = {&indptr, &indices, &row_indices, &blocks, &result, &in_src, &in_dst,
                               &keys0, &keys1, &sort_scratch, &tile_base, &meta, &deg, &rank,
                               &bitmap, &prefix, &partials, &done, &rowmask};
        size_t s = 0;
        for (const btc200::DevBuf* b : all) s += b->bytes;
        return s;
    }
    void release_all()
    {
        btc200::DevBuf* all[] = {&indptr, &indices, &row_indices, &blocks, &result, &in_src, &in_dst,
                         &keys0, &keys1, &sort_scratch, &tile_base, &meta, &deg, &rank,
                         &bitmap, &prefix, &partials, &done, &rowmask};
        for (btc200::DevBuf* b : all) b->release();
        if (h_meta) cudaFreeHost(h_meta);
        h_meta = nullptr;
    }
};


// meta slots (device uint64): 0 valid edges, 1 out-of-range ids, 2 tiles, 3 unique
// edges, 4 vertex count for the degree sort
enum { kMetaValid = 0, kMetaBad = 1, kMetaTiles = 2, kMetaUniq = 3, kMetaN = 4, kMetaSlots = 8 };

int default_tau(int tile_cols);
int ensure_count_scratch(btc_bitbsr* g);
// Counts tiles [tile_begin, tile_end) (clamped to the tile count) into g->result and,
// when d_out2 is given, *d_out2.
int count_handle(btc_bitbsr* g, int tau, cudaStream_t s, unsigned long long* d_out2,
                 uint32_t tile_begin = 0, uint32_t tile_end = 0xffffffffu);
