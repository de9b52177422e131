// policy.cu -- tile width and tau per graph class (the engine's autotuned policy; the
// reference's policy is the fixed BTC-Lite rule, apps/btc_tc_lite.cu:45-65, which stays
// available as btc_lite_select_tile_cols).
//
// The rule comes from a sweep on one B200 of 37 graphs over five families (Erdos-Renyi,
// 27- and 7-point stencils, R-MAT in natural and descending-degree order, 8-block SBMs,
// complete graphs) at both tile widths and three taus (btc_b200/tune.py --sweep; table in
// the autotune profile).  Features, all cheap, in this order:
//   * average degree d = 2m/n >= 512 (dense communities, near-cliques): 16x32, whose
//     dense path packs four matches into one k = 128 MMA;
//   * descending-degree order requested (BTC_ORIENT_DEGREE): power-law graphs whose hubs
//     sit in the first column blocks -> 16x128;
//   * id locality L: the share of sampled input edges with |u - v| < 128 over the share
//     uniform ids would give (about 255/n); L >= 16 (banded or clustered ids: stencils)
//     -> 16x128, else (random ids: Erdos-Renyi, natural-order R-MAT, SBM) 16x32.
// tau: 1024 for 16x128 (dense SBM communities near 30% tile density run 2.6-2.9x faster
// on the sparse path than on the b1 MMA path at the reference's 512, while full tiles
// keep the MMA path), 64 for 16x32 (the reference's: its four-match packing wins there).
#include "common.cuh"
#include "handle.cuh"

#include <cstdlib>

namespace btc200 {
namespace pol {

constexpr int kThreads = 256;
constexpr int kGrid = 64;
constexpr uint32_t kSamples = 1u << 16;
constexpr int32_t kNear = 128;  // |u - v| below this counts as local

// Sample i reads edge i * step.  Adds the number of local edges and their expectation
// under uniform ids (per sampled edge: the chance that two uniform ids in [0, n) lie
// closer than kNear, about (2 kNear - 1) / n), scaled by 2^20 to stay integer.  With
// e_off / nv (a batch), an edge's n is its own graph's.
__global__ void k_locality(const int32_t* __restrict__ src, const int32_t* __restrict__ dst, int64_t m,
                           int32_t n, const int64_t* __restrict__ e_off, const int32_t* __restrict__ nv,
                           uint32_t G, int64_t step, unsigned long long* __restrict__ out)
{
    unsigned long long local = 0, expect = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < kSamples;
         i += (uint64_t)gridDim.x * kThreads) {
        const int64_t e = (int64_t)i * step;
        if (e >= m) break;
        int32_t ng = n;
        if (e_off) {
            uint32_t lo = 0, hi = G;  // last g with e_off[g] <= e
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (e_off[mid] <= e) lo = mid;
                else hi = mid;
            }
            ng = nv[lo];
        }
        const int32_t u = src[e], v = dst[e];
        if (u == v || u < 0 || v < 0 || u >= ng || v >= ng) continue;
        local += (u > v ? u - v : v - u) < kNear ? (1ull << 20) : 0ull;
        expect += ng > 2 * kNear ? ((2ull * kNear - 1ull) << 20) / (unsigned long long)ng : (1ull << 20);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        local += __shfl_xor_sync(kFull, local, d);
        expect += __shfl_xor_sync(kFull, expect, d);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], local);
        atomicAdd(&out[1], expect);
    }
}

double locality_host(const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                     const int64_t* e_off, const int32_t* nv, uint32_t G)
{
    const int64_t step = m > (int64_t)kSamples ? m / (int64_t)kSamples : 1;
    double local = 0.0, expect = 0.0;
    uint32_t g = 0;
    for (uint64_t i = 0; i < kSamples; ++i) {
        const int64_t e = (int64_t)i * step;
        if (e >= m) break;
        int32_t ng = n;
        if (e_off) {
            while (g + 1 < G && e_off[g + 1] <= e) ++g;
            ng = nv[g];
        }
        const int32_t u = src[e], v = dst[e];
        if (u == v || u < 0 || v < 0 || u >= ng || v >= ng) continue;
        local += std::abs((int64_t)u - (int64_t)v) < kNear ? 1.0 : 0.0;
        expect += ng > 2 * kNear ? (2.0 * kNear - 1.0) / (double)ng : 1.0;
    }
    return expect > 0.0 ? local / expect : 0.0;
}

}  // namespace pol

// Id locality of an edge list (see above): host arrays are sampled on the host, device
// arrays by one small kernel and one wait on `s` (16 bytes of scratch, allocated here).
// e_off / nv (optional, num_graphs + 1 and num_graphs entries, host or device like
// src/dst): batch layout.
int policy_locality(const int32_t* src, const int32_t* dst, int64_t m, int32_t n, bool on_host,
                    const int64_t* e_off, const int32_t* nv, uint32_t G, cudaStream_t s, double* L)
{
    *L = 0.0;
    if (m <= 0) return BTC_OK;
    if (on_host) {
        *L = pol::locality_host(src, dst, m, n, e_off, nv, G);
        return BTC_OK;
    }
    struct Scratch {
        DevBuf b;
        ~Scratch() { b.release(); }
    } sc;
    BTC_TRY(sc.b.reserve(2 * sizeof(unsigned long long)));
    unsigned long long* d = sc.b.as<unsigned long long>();
    BTC_CUDA_TRY(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), s));
    const int64_t step = m > (int64_t)pol::kSamples ? m / (int64_t)pol::kSamples : 1;
    pol::k_locality<<<pol::kGrid, pol::kThreads, 0, s>>>(src, dst, m, n, e_off, nv, G, step, d);
    BTC_CUDA_TRY(cudaGetLastError());
    unsigned long long h[2] = {0, 0};
    BTC_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
    BTC_CUDA_TRY(cudaStreamSynchronize(s));
    *L = h[1] ? (double)h[0] / (double)h[1] : 0.0;
    return BTC_OK;
}

}  // namespace btc200

using namespace btc200;

extern "C" {

int btc_tile_policy_from_features(int64_t m, int32_t n, uint32_t flags, double locality,
                                  int* tile_cols, int* tau)
{
    if (m < 0 || n < 0 || !tile_cols) return BTC_E_INVAL;
    const double d = n > 0 ? 2.0 * (double)m / (double)n : 0.0;
    int C;
    if (d >= 512.0) C = 32;
    else if (flags & BTC_ORIENT_DEGREE) C = 128;
    else C = locality >= 16.0 ? 128 : 32;
    *tile_cols = C;
    if (tau) *tau = default_tau(C);
    return BTC_OK;
}

int btc_select_tile_policy(const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                           uint32_t flags, btc_stream_t stream, int* tile_cols, int* tau)
{
    if (n < 0 || m < 0 || !tile_cols || (m > 0 && (!src || !dst))) return BTC_E_INVAL;
    double L = 0.0;
    if (!(flags & BTC_ORIENT_DEGREE))
        BTC_TRY(policy_locality(src, dst, m, n, (flags & BTC_INPUT_ON_HOST) != 0, nullptr, nullptr, 0,
                                stream, &L));
    return btc_tile_policy_from_features(m, n, flags, L, tile_cols, tau);
}

}  // extern "C"
