// ref_cpu_wrap.cpp -- C entry point around the reference's own CPU triangle count.
// TEST INFRASTRUCTURE ONLY (the timed CPU baseline and the parity pin).
//
// The counting code is the reference's, included unchanged from
// btc/operations/triangle_count_cpu.h (cpu_tc_intersection_lower_triangular,
// lines 59-101); this file only adapts a plain CSR to the template's member names.
#include <cstdint>
#include <omp.h>

#include "btc/operations/triangle_count_cpu.h"

namespace {
struct HostCsr {
    int num_rows;
    const int* row_pointers;
    const int* column_indices;
};
}  // namespace

extern "C" uint64_t ref_cpu_tc_lower(const int* rowptr, const int* col, int n, int threads)
{
    if (threads > 0) omp_set_num_threads(threads);
    HostCsr csr{n, rowptr, col};
    return (uint64_t)btc::cpu_tc_intersection_lower_triangular(csr);
}

extern "C" int ref_cpu_max_threads(void) { return omp_get_max_threads(); }
