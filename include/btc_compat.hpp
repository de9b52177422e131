// btc_compat.hpp -- C++ drop-in for the reference's Bit-BSR build + count headers.
//
// A program written against fanna1234/btc-tc-artifact includes
//   btc/operations/bcsr_16x128.h, bcsr_16x32.h        (BCSR_*_Device, convert_*)
//   btc/operations/tc_16x128_adaptive.h, tc_16x32_adaptive.h   (count_triangles_*)
// Including this header instead gives the same names, signatures, field layout and
// call semantics in namespace btc, forwarding to the C ABI of btc_c.h (libbtc_b200.so).
// The COO argument is any type with the reference's CooMatrix members
// (num_rows, num_entries, row_indices, column_indices as device vectors), e.g.
// btc::CooMatrix<int, float, btc::device_memory> (btc/formats/coo.h:10-33).
//
// Error behaviour: the reference printed and returned (bcsr_16x128.h:166-177,
// 228-232); these shims print the engine's status text the same way (stdout) and leave
// the struct zeroed, and the count functions return 0 on failure, so callers see the
// same shape of failure.
#pragma once

#include <cstdint>
#include <cstdio>

#include <thrust/device_vector.h>

#include "btc_c.h"

namespace btc {

// Same field order and types as bcsr_16x128.h:24-51 and bcsr_16x32.h:109-138; the tile
// width is a tag so the two stay distinct types, as in the reference.
template <int TILE_COLS>
struct BcsrDevice {
    uint32_t* indptr = nullptr;
    uint32_t* indices = nullptr;
    uint32_t* blocks = nullptr;
    uint32_t* row_indices = nullptr;
    unsigned long long* result = nullptr;
    int n = 0;
    int n_row_blocks = 0;
    uint32_t num_blocks = 0;

    btc_bcsr_device* c_view() { return reinterpret_cast<btc_bcsr_device*>(this); }
    void free() { btc_bcsr_free(c_view()); }
    void reset_result() { btc_bcsr_reset_result(c_view()); }
    unsigned long long get_result()
    {
        unsigned long long r = 0;
        btc_bcsr_get_result(c_view(), &r);
        return r;
    }
};

using BCSR_16x128_Device = BcsrDevice<128>;
using BCSR_16x32_Device = BcsrDevice<32>;

static_assert(sizeof(BCSR_16x128_Device) == sizeof(btc_bcsr_device), "layout must match btc_c.h");

namespace compat_detail {
inline void report(const char* what, int st)
{
    if (st != BTC_OK) std::printf("%s failed: %s\n", what, btc_strerror(st));
}
template <class COO>
inline const int32_t* rows_of(const COO& coo)
{
    return reinterpret_cast<const int32_t*>(thrust::raw_pointer_cast(coo.row_indices.data()));
}
template <class COO>
inline const int32_t* cols_of(const COO& coo)
{
    return reinterpret_cast<const int32_t*>(thrust::raw_pointer_cast(coo.column_indices.data()));
}
}  // namespace compat_detail

// bcsr_16x128.h:136
template <typename CooMatrixType>
void convert_coo_to_bcsr_16x128_gpu(BCSR_16x128_Device& bcsr, const CooMatrixType& coo)
{
    const int st = btc_convert_coo_to_bcsr_16x128_gpu(
        bcsr.c_view(), compat_detail::rows_of(coo), compat_detail::cols_of(coo),
        (int64_t)coo.num_entries, (int32_t)coo.num_rows);
    compat_detail::report("convert_coo_to_bcsr_16x128_gpu", st);
}

// bcsr_16x32.h:144
template <typename CooMatrixType>
void convert_coo_to_bcsr_16x32_gpu(BCSR_16x32_Device& bcsr, const CooMatrixType& coo)
{
    const int st = btc_convert_coo_to_bcsr_16x32_gpu(
        bcsr.c_view(), compat_detail::rows_of(coo), compat_detail::cols_of(coo),
        (int64_t)coo.num_entries, (int32_t)coo.num_rows);
    compat_detail::report("convert_coo_to_bcsr_16x32_gpu", st);
}

// tc_16x128_adaptive.h:12 and :29
inline unsigned long long count_triangles_16x128_adaptive(BCSR_16x128_Device& d_bcsr,
                                                          int threshold_blocks, float* kernel_ms)
{
    unsigned long long out = 0;
    const int st =
        btc_count_triangles_16x128_adaptive(d_bcsr.c_view(), threshold_blocks, kernel_ms, &out);
    compat_detail::report("count_triangles_16x128_adaptive", st);
    return st == BTC_OK ? out : 0ull;
}
inline unsigned long long count_triangles_16x128_adaptive(BCSR_16x128_Device& d_bcsr,
                                                          int threshold_blocks = 2048)
{
    return count_triangles_16x128_adaptive(d_bcsr, threshold_blocks, nullptr);
}

// tc_16x32_adaptive.h:14 and :29
inline unsigned long long count_triangles_16x32_adaptive(BCSR_16x32_Device& d_bcsr,
                                                         int threshold_blocks, float* kernel_ms)
{
    unsigned long long out = 0;
    const int st =
        btc_count_triangles_16x32_adaptive(d_bcsr.c_view(), threshold_blocks, kernel_ms, &out);
    compat_detail::report("count_triangles_16x32_adaptive", st);
    return st == BTC_OK ? out : 0ull;
}
inline unsigned long long count_triangles_16x32_adaptive(BCSR_16x32_Device& d_bcsr,
                                                         int threshold_blocks = 40000)
{
    return count_triangles_16x32_adaptive(d_bcsr, threshold_blocks, nullptr);
}

// tc_16x128_mma_v5.h:213 / tc_16x32_mma_v6.h:240 (the variants the adaptive calls pick)
inline unsigned long long count_triangles_16x128_v5(BCSR_16x128_Device& d, float* kernel_ms = nullptr)
{
    return count_triangles_16x128_adaptive(d, 0, kernel_ms);
}
inline unsigned long long count_triangles_16x32_v6(BCSR_16x32_Device& d, float* kernel_ms = nullptr)
{
    return count_triangles_16x32_adaptive(d, 0, kernel_ms);
}

}  // namespace btc
