// diag.cu -- the binary tensor-core peak of this GPU (no counterpart in the reference).
//
// The count kernel's dense path runs mma.sync.m16n8k128.row.col.s32.b1.b1.s32.and.popc
// (tcgen05 has no binary kind).  Its utilisation is reported against the throughput of
// that instruction measured here: every warp of a persistent grid issues 8 independent
// accumulator chains of the MMA on register operands, so nothing but the tensor pipe
// limits it.  One MMA is 16 x 8 x 128 = 16,384 binary AND-popcount-accumulates.
#include "common.cuh"

namespace btc200 {
namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256)
k_b1_mma_peak(int iters, uint32_t seed, unsigned long long* sink)
{
    const uint32_t lane = threadIdx.x & 31;
    uint32_t a0 = seed ^ (lane * 0x9E3779B9u), a1 = a0 * 747796405u + 1u, b0 = a1 ^ 0x5bd1e995u;
    int32_t c[kChains][4];
#pragma unroll
    for (int k = 0; k < kChains; ++k) c[k][0] = c[k][1] = c[k][2] = c[k][3] = 0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < kChains; ++k)
            asm volatile(
                "mma.sync.aligned.m16n8k128.row.col.s32.b1.b1.s32.and.popc "
                "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                : "+r"(c[k][0]), "+r"(c[k][1]), "+r"(c[k][2]), "+r"(c[k][3])
                : "r"(a0), "r"(a1), "r"(b0));
        a0 += 1u;  // keep the operands live without a dependence between chains
    }
    long long s = 0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += c[k][0] + c[k][1] + c[k][2] + c[k][3];
    s = __reduce_add_sync(0xffffffffu, (unsigned)s);  // the results are used: the MMAs stay
    if (lane == 0) atomicAdd(sink, (unsigned long long)s);
}

}  // namespace
}  // namespace btc200

using namespace btc200;

extern "C" int btc_b1_mma_peak(btc_stream_t stream, int iters, double* ops_per_s)
{
    if (!ops_per_s || iters < 1) return BTC_E_INVAL;
    const int grid = device_sm_count() * 4;
    DevBuf sink;
    BTC_TRY(sink.reserve(sizeof(unsigned long long)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = BTC_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) st = BTC_E_CUDA;
    if (st == BTC_OK) {
        k_b1_mma_peak<<<grid, 256, 0, stream>>>(iters / 10 + 1, 1u, sink.as<unsigned long long>());
        cudaEventRecord(e0, stream);
        k_b1_mma_peak<<<grid, 256, 0, stream>>>(iters, 2u, sink.as<unsigned long long>());
        cudaEventRecord(e1, stream);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
            st = BTC_E_CUDA;
    }
    if (st == BTC_OK) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double mmas = (double)grid * 8.0 * kChains * (double)iters;
        *ops_per_s = mmas * 16.0 * 8.0 * 128.0 / (ms * 1e-3);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    sink.release();
    return st;
}
