// ref_gpu_wrap.cu -- C entry point around the reference's own GPU Bit-BSR build and
// hybrid count, compiled unchanged from its headers for sm_100a.
// TEST INFRASTRUCTURE ONLY: the same-box A/B arm and the Bit-BSR layout pin.
//
// Calls exactly what apps/btc_tc_lite.cu:76-134 calls on a preprocessed COO:
//   convert_coo_to_bcsr_16x128_gpu   btc/operations/bcsr_16x128.h:136-241
//   convert_coo_to_bcsr_16x32_gpu    btc/operations/bcsr_16x32.h:144-249
//   count_triangles_16x128_adaptive  btc/operations/tc_16x128_adaptive.h:12-29 (threshold 2048)
//   count_triangles_16x32_adaptive   btc/operations/tc_16x32_adaptive.h:14-31  (threshold 40000)
// and, for the reorder step of preprocess_for_triangle_counting,
//   reorder_hashorder_gpu            btc/operations/reorder.h:443-587
// The only code here is the adapter from plain host arrays to the template's COO
// member names, event timing around the convert, and copies of the result out.
#include <cstdint>
#include <cstdio>
#include <vector>
#include <algorithm>

#include <thrust/device_vector.h>

#include "btc/operations/bcsr_16x128.h"
#include "btc/operations/bcsr_16x32.h"
#include "btc/operations/tc_16x128_adaptive.h"
#include "btc/operations/tc_16x32_adaptive.h"
#include "btc/operations/reorder.h"

namespace {
struct DevCoo {
    int num_rows = 0;
    int num_cols = 0;
    size_t num_entries = 0;
    thrust::device_vector<int> row_indices;
    thrust::device_vector<int> column_indices;
};

template <class Bcsr>
int export_bcsr(Bcsr& b, int words_per_tile, uint32_t* h_indptr, uint32_t* h_indices,
                uint32_t* h_row_indices, uint32_t* h_blocks, int64_t cap_blocks)
{
    if (!h_indptr) return 0;
    if ((int64_t)b.num_blocks > cap_blocks) return -1;
    cudaMemcpy(h_indptr, b.indptr, sizeof(uint32_t) * (size_t)(b.n_row_blocks + 1),
               cudaMemcpyDeviceToHost);
    if (b.num_blocks) {
        cudaMemcpy(h_indices, b.indices, sizeof(uint32_t) * b.num_blocks, cudaMemcpyDeviceToHost);
        cudaMemcpy(h_row_indices, b.row_indices, sizeof(uint32_t) * b.num_blocks,
                   cudaMemcpyDeviceToHost);
        cudaMemcpy(h_blocks, b.blocks, sizeof(uint32_t) * (size_t)b.num_blocks * words_per_tile,
                   cudaMemcpyDeviceToHost);
    }
    return 0;
}
}  // namespace

// h_rows/h_cols: the preprocessed lower-triangular COO (row > col, unique).
// Returns 0 on success, -1 if the Bit-BSR does not fit the export buffers, -2 on a
// CUDA error.  out_kernel_ms receives `repeat` kernel-only times (the reference's own
// event pair around its launch).
extern "C" int ref_gpu_run(const int* h_rows, const int* h_cols, int64_t nnz, int n,
                           int tile_cols, int warmup, int repeat,
                           unsigned long long* out_count, float* out_convert_ms,
                           float* out_kernel_ms, uint32_t* out_num_blocks,
                           uint32_t* h_indptr, uint32_t* h_indices, uint32_t* h_row_indices,
                           uint32_t* h_blocks, int64_t cap_blocks)
{
    DevCoo coo;
    coo.num_rows = n;
    coo.num_cols = n;
    coo.num_entries = (size_t)nnz;
    coo.row_indices.assign(h_rows, h_rows + nnz);
    coo.column_indices.assign(h_cols, h_cols + nnz);
    cudaDeviceSynchronize();

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    unsigned long long count = 0;
    int rc = 0;
    if (tile_cols == 128) {
        btc::BCSR_16x128_Device d;
        cudaEventRecord(e0);
        btc::convert_coo_to_bcsr_16x128_gpu(d, coo);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(out_convert_ms, e0, e1);
        for (int w = 0; w < warmup; ++w) {
            float t = 0.f;
            btc::count_triangles_16x128_adaptive(d, 2048, &t);
        }
        for (int r = 0; r < repeat; ++r)
            count = btc::count_triangles_16x128_adaptive(d, 2048, &out_kernel_ms[r]);
        *out_num_blocks = d.num_blocks;
        rc = export_bcsr(d, 64, h_indptr, h_indices, h_row_indices, h_blocks, cap_blocks);
        d.free();
    } else {
        btc::BCSR_16x32_Device d;
        cudaEventRecord(e0);
        btc::convert_coo_to_bcsr_16x32_gpu(d, coo);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(out_convert_ms, e0, e1);
        for (int w = 0; w < warmup; ++w) {
            float t = 0.f;
            btc::count_triangles_16x32_adaptive(d, 40000, &t);
        }
        for (int r = 0; r < repeat; ++r)
            count = btc::count_triangles_16x32_adaptive(d, 40000, &out_kernel_ms[r]);
        *out_num_blocks = d.num_blocks;
        rc = export_bcsr(d, 16, h_indptr, h_indices, h_row_indices, h_blocks, cap_blocks);
        d.free();
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *out_count = count;
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) return -2;
    return rc;
}

// The reference's GPU HashOrder on a COO of n vertices (any orientation), in place on
// the host arrays: relabelled and oriented to (max, min) exactly as reorder_hashorder_gpu
// leaves the device COO.  Returns 0, or -2 on a CUDA error.
extern "C" int ref_hashorder_gpu(int* h_rows, int* h_cols, int64_t nnz, int n, int num_hashes,
                                 int num_hops)
{
    DevCoo coo;
    coo.num_rows = n;
    coo.num_cols = n;
    coo.num_entries = (size_t)nnz;
    coo.row_indices.assign(h_rows, h_rows + nnz);
    coo.column_indices.assign(h_cols, h_cols + nnz);
    btc::reorder_hashorder_gpu(coo, num_hashes, num_hops);
    if (cudaDeviceSynchronize() != cudaSuccess) return -2;
    thrust::copy(coo.row_indices.begin(), coo.row_indices.end(), h_rows);
    thrust::copy(coo.column_indices.begin(), coo.column_indices.end(), h_cols);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
