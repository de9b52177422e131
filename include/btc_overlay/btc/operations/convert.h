// btc/operations/convert.h (engine overlay): the conversions and the preprocess of the
// reference's convert.h that its apps call, on the engine.
//
//   convert_csr_to_coo / convert_coo_to_csr   (convert.h:26-45): Thrust, written here
//   preprocess_for_triangle_counting          (convert.h:600-690): orientation to
//       (max, min), self-loop removal, sort, dedup and id compaction by
//       btc_preprocess_for_triangle_counting, then the reorder step BTC_REORDER selects as
//       the reference does -- unset or 9: GPU HashOrder when btc_should_reorder says so
//       (the input's base name is the hint), 8: always, 0: never; BTC_HASHORDER_HASHES /
//       _HOPS (16 / 1 when unset) set the signature.  force_cpu is accepted and ignored
//       (the engine has no CPU path); lower_triangular = false is not supported and
//       prints an error, leaving the COO unchanged.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <string>

#include <cuda_runtime.h>
#include <thrust/binary_search.h>
#include <thrust/copy.h>
#include <thrust/device_ptr.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/sort.h>

#include "btc_compat.hpp"

namespace btc {

// CSR -> COO: every entry's row from the row pointers.
template <typename CSR, typename COO>
void convert_csr_to_coo(COO& coo, const CSR& csr)
{
    coo.resize(csr.num_rows, csr.num_cols, csr.num_entries);
    auto first = thrust::make_counting_iterator<decltype(csr.num_entries)>(0);
    thrust::upper_bound(csr.row_pointers.begin() + 1, csr.row_pointers.end(), first,
                        first + csr.num_entries, coo.row_indices.begin());
    thrust::copy(csr.column_indices.begin(), csr.column_indices.end(), coo.column_indices.begin());
    thrust::copy(csr.values.begin(), csr.values.end(), coo.values.begin());
}

// COO -> CSR: row pointer r is the first entry of row r.  A COO whose rows are not
// sorted (the state a HashOrder relabel leaves it in) is converted from a copy sorted by
// (row, column); the reference's version asserts sorted rows and aborts instead
// (btc/utils/csr_helpers.h:24), so its -v check fails after a reorder while this one works.
template <typename CSR, typename COO>
void convert_coo_to_csr(CSR& csr, const COO& coo)
{
    csr.resize(coo.num_rows, coo.num_cols, coo.num_entries);
    auto first = thrust::make_counting_iterator<decltype(coo.num_rows)>(0);
    if (thrust::is_sorted(coo.row_indices.begin(), coo.row_indices.end())) {
        thrust::lower_bound(coo.row_indices.begin(), coo.row_indices.end(), first,
                            first + coo.num_rows + 1, csr.row_pointers.begin());
        thrust::copy(coo.column_indices.begin(), coo.column_indices.end(), csr.column_indices.begin());
        thrust::copy(coo.values.begin(), coo.values.end(), csr.values.begin());
        return;
    }
    auto rows = coo.row_indices;  // copies in the COO's memory space
    csr.column_indices = coo.column_indices;
    csr.values = coo.values;
    auto cv = thrust::make_zip_iterator(thrust::make_tuple(rows.begin(), csr.values.begin()));
    thrust::stable_sort_by_key(csr.column_indices.begin(), csr.column_indices.end(), cv);
    auto cv2 = thrust::make_zip_iterator(thrust::make_tuple(csr.column_indices.begin(), csr.values.begin()));
    thrust::stable_sort_by_key(rows.begin(), rows.end(), cv2);
    thrust::lower_bound(rows.begin(), rows.end(), first, first + coo.num_rows + 1,
                        csr.row_pointers.begin());
}

namespace compat_detail {
inline int env_int(const char* name, int unset)
{
    const char* v = std::getenv(name);
    return v ? std::atoi(v) : unset;
}
}  // namespace compat_detail

template <typename CooMatrix>
void preprocess_for_triangle_counting(CooMatrix& coo, bool force_cpu = false,
                                      bool lower_triangular = true,
                                      const std::string& input_file = "")
{
    (void)force_cpu;
    if (!lower_triangular) {
        std::printf("preprocess_for_triangle_counting: lower_triangular=false is not supported\n");
        return;
    }
    int64_t nnz = (int64_t)coo.num_entries;
    int32_t rows = (int32_t)coo.num_rows;
    int32_t* r = reinterpret_cast<int32_t*>(thrust::raw_pointer_cast(coo.row_indices.data()));
    int32_t* c = reinterpret_cast<int32_t*>(thrust::raw_pointer_cast(coo.column_indices.data()));
    int st = btc_preprocess_for_triangle_counting(r, c, &nnz, &rows, 1);
    compat_detail::report("preprocess_for_triangle_counting", st);
    if (st != BTC_OK) return;
    coo.resize(rows, rows, (decltype(coo.num_entries))nnz);
    const int mode = compat_detail::env_int("BTC_REORDER", 9);
    if (mode != 8 && mode != 9) return;
    if (mode == 9) {
        int dev = 0, major = 0, minor = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
        const size_t slash = input_file.find_last_of('/');
        std::string base = input_file.substr(slash == std::string::npos ? 0 : slash + 1);
        base = base.substr(0, base.find_last_of('.'));
        if (!btc_should_reorder(rows, nnz, 10 * major + minor, base.c_str())) return;
    }
    r = reinterpret_cast<int32_t*>(thrust::raw_pointer_cast(coo.row_indices.data()));
    c = reinterpret_cast<int32_t*>(thrust::raw_pointer_cast(coo.column_indices.data()));
    st = btc_reorder_hashorder(r, c, nnz, rows, compat_detail::env_int("BTC_HASHORDER_HASHES", 16),
                               compat_detail::env_int("BTC_HASHORDER_HOPS", 1), nullptr, nullptr);
    compat_detail::report("reorder_hashorder_gpu", st);
}

}  // namespace btc
