// reorder.cu -- GPU HashOrder vertex reordering (btc_reorder_hashorder) and the
// reference's automatic reorder decision (btc_should_reorder).
//
// Restates reorder_hashorder_gpu (btc/operations/reorder.h:443-587): every vertex gets a
// signature of num_hashes MinHash values over its closed neighbourhood, vertices are
// ordered lexicographically by signature (ties by id), and the COO is relabelled by that
// order and re-oriented to (max, min).  Vertices with similar neighbourhoods end up with
// nearby ids, which packs the Bit-BSR of low-degree graphs into fewer, denser tiles.
//
//   hash j        h_j(v) = (a_j * v + b_j) mod P, P = 2^32 - 5 (reorder.h:411-418); a_j, b_j
//                 drawn in the reference's order from std::mt19937(42) with
//                 uniform_int_distribution(1, 4294967290) (reorder.h:495-506)
//   hop           h'_j(v) = min(h_j(v), min over neighbours u of h_j(u)) (reorder.h:421-441);
//                 the first hop computes h_j(u) from u on the fly (no table gathers), later
//                 hops gather from the previous hop's table
//   order         stable LSD sort of the vertices by h_{H-1}, ..., h_0 (reorder.h:536-549)
//                 with the engine's 64-bit radix sort on keys (h_j << 32 | vertex)
//   relabel       perm[order[i]] = i, applied to both endpoints, then (max, min)
//
// The neighbourhoods come from a symmetric CSR built by counting (degree, scan, scatter);
// neighbour order does not matter to a minimum, so no sort is needed for it.
#include <cctype>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace btc200 {

int grid_for(int64_t work, int threads);
int launch_tile_scan(uint32_t* per_tile, uint32_t ntiles, unsigned long long* total, cudaStream_t s);
int launch_set_u64(unsigned long long* p, unsigned long long v, cudaStream_t s);
int launch_rank_scatter(const uint64_t*, int32_t, int32_t*, cudaStream_t);

namespace ro {

constexpr int kMaxHashes = 64;
constexpr int kChunk = 8;  // hash functions evaluated together per neighbour visit

// (a * v + b) mod (2^32 - 5), exact: 2^32 = 5 (mod P), so the high word folds down as
// five times its value; two folds leave x < 2^32 + 25 < 2P.
__device__ __forceinline__ uint32_t hash_mod(uint32_t a, uint32_t b, uint32_t v)
{
    constexpr uint64_t P = 4294967291ull;
    uint64_t x = (uint64_t)a * v + b;
    x = (x >> 32) * 5ull + (x & 0xffffffffull);
    x = (x >> 32) * 5ull + (x & 0xffffffffull);
    if (x >= P) x -= P;
    return (uint32_t)x;
}

// Both endpoints of every edge: degree counts; flags ids outside [0, n).
__global__ void k_degree2(const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                          int64_t m, int32_t n, uint32_t* __restrict__ deg,
                          unsigned long long* __restrict__ bad)
{
    uint32_t nb = 0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = rows[e], c = cols[e];
        if (r < 0 || r >= n || c < 0 || c >= n) {
            ++nb;
            continue;
        }
        atomicAdd(&deg[r], 1u);
        atomicAdd(&deg[c], 1u);
    }
    nb = __reduce_add_sync(kFull, nb);
    if ((threadIdx.x & 31) == 0 && nb) atomicAdd(bad, (unsigned long long)nb);
}

// Neighbour lists: u's list gets v and v's list gets u for every edge (u, v).
__global__ void k_scatter2(const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                           int64_t m, int32_t n, uint32_t* __restrict__ cursor,
                           int32_t* __restrict__ nbr)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = rows[e], c = cols[e];
        if (r < 0 || r >= n || c < 0 || c >= n) continue;
        nbr[atomicAdd(&cursor[r], 1u)] = c;
        nbr[atomicAdd(&cursor[c], 1u)] = r;
    }
}

// First hop (or, with hops == 0, the plain hashes): hv[j * n + v] for every hash j.
__global__ void k_minhash_first(const uint32_t* __restrict__ start,
                                const uint32_t* __restrict__ deg,
                                const int32_t* __restrict__ nbr, int32_t n, int H, int hops,
                                const uint32_t* __restrict__ ab, uint32_t* __restrict__ hv)
{
    __shared__ uint32_t s_ab[2 * kMaxHashes];
    for (int i = threadIdx.x; i < 2 * H; i += blockDim.x) s_ab[i] = ab[i];
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p0 = start[v], p1 = p0 + (hops > 0 ? deg[v] : 0u);
        for (int j0 = 0; j0 < H; j0 += kChunk) {
            uint32_t h[kChunk];
#pragma unroll
            for (int q = 0; q < kChunk; ++q)
                h[q] = j0 + q < H ? hash_mod(s_ab[2 * (j0 + q)], s_ab[2 * (j0 + q) + 1], (uint32_t)v)
                                  : 0u;
            for (uint32_t p = p0; p < p1; ++p) {
                const uint32_t u = (uint32_t)nbr[p];
#pragma unroll
                for (int q = 0; q < kChunk; ++q)
                    if (j0 + q < H) h[q] = min(h[q], hash_mod(s_ab[2 * (j0 + q)], s_ab[2 * (j0 + q) + 1], u));
            }
#pragma unroll
            for (int q = 0; q < kChunk; ++q)
                if (j0 + q < H) hv[(size_t)(j0 + q) * n + v] = h[q];
        }
    }
}

// A later hop: hout[j][v] = min(hin[j][v], min over neighbours u of hin[j][u]).
__global__ void k_minhash_hop(const uint32_t* __restrict__ start, const uint32_t* __restrict__ deg,
                              const int32_t* __restrict__ nbr, int32_t n, int H,
                              const uint32_t* __restrict__ hin, uint32_t* __restrict__ hout)
{
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t p0 = start[v], p1 = p0 + deg[v];
        for (int j = 0; j < H; ++j) {
            const uint32_t* hj = hin + (size_t)j * n;
            uint32_t h = hj[v];
            for (uint32_t p = p0; p < p1; ++p) h = min(h, hj[nbr[p]]);
            hout[(size_t)j * n + v] = h;
        }
    }
}

// Sort keys for hash j: (h_j(vertex) << 32) | vertex, the vertices taken in the current
// order (the low words of the previous sort, or 0..n-1 for the first pass).
__global__ void k_sig_keys(const uint64_t* __restrict__ prev, int32_t n,
                           const uint32_t* __restrict__ hj, uint64_t* __restrict__ keys)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = prev ? (uint32_t)prev[i] : (uint32_t)i;
        keys[i] = ((uint64_t)hj[v] << 32) | v;
    }
}

// Relabel both endpoints and orient to (max, min) (reorder.h:39-46, 574-584).
__global__ void k_relabel(int32_t* __restrict__ rows, int32_t* __restrict__ cols, int64_t m,
                          const int32_t* __restrict__ perm)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = perm[rows[e]], c = perm[cols[e]];
        rows[e] = r >= c ? r : c;
        cols[e] = r >= c ? c : r;
    }
}

}  // namespace ro

// The reference's hash parameters: for each j, a_j then b_j from one std::mt19937(42)
// through uniform_int_distribution<uint32_t>(1, 4294967290) (reorder.h:495-506).
static void hashorder_params(int H, uint32_t* a, uint32_t* b)
{
    std::mt19937 rng(42);
    std::uniform_int_distribution<uint32_t> dist(1, 4294967290u);
    for (int j = 0; j < H; ++j) {
        a[j] = dist(rng);
        b[j] = dist(rng);
    }
}

}  // namespace btc200

using namespace btc200;

extern "C" int btc_hashorder_params(int num_hashes, uint32_t* a, uint32_t* b)
{
    if (num_hashes < 1 || num_hashes > ro::kMaxHashes || !a || !b) return BTC_E_INVAL;
    hashorder_params(num_hashes, a, b);
    return BTC_OK;
}

extern "C" int btc_reorder_hashorder(int32_t* d_rows, int32_t* d_cols, int64_t nnz, int32_t num_rows,
                                     int num_hashes, int num_hops, int32_t* d_perm,
                                     cudaStream_t stream)
{
    if (nnz < 0 || num_rows < 0 || (nnz > 0 && (!d_rows || !d_cols))) return BTC_E_INVAL;
    if (num_hashes < 1 || num_hashes > ro::kMaxHashes || num_hops < 0 || num_hops > 64)
        return BTC_E_INVAL;
    if ((uint64_t)nnz > 0x7fffffffull) return BTC_E_INVAL;  // 2 * nnz neighbour slots in uint32
    const int32_t n = num_rows;
    if (n == 0) return nnz == 0 ? BTC_OK : BTC_E_RANGE;
    const int H = num_hashes;
    cudaStream_t s = stream;

    // One workspace, carved into 256-byte-aligned pieces, released on every return.
    struct Workspace {
        DevBuf buf;
        ~Workspace() { buf.release(); }
    } ws;
    const size_t nn = (size_t)n, ne = (size_t)(2 * nnz > 0 ? 2 * nnz : 1);
    const size_t sizes[] = {sizeof(uint32_t) * nn,                        // deg
                            sizeof(uint32_t) * nn,                        // start
                            sizeof(uint32_t) * nn,                        // cursor
                            sizeof(int32_t) * ne,                         // nbr
                            sizeof(uint32_t) * nn * H,                    // hv0
                            num_hops > 1 ? sizeof(uint32_t) * nn * H : 0,  // hv1
                            sizeof(uint64_t) * nn,                        // k0
                            sizeof(uint64_t) * nn,                        // k1
                            sizeof(uint32_t) * radix_scratch_words(nn),   // scratch
                            d_perm ? 0 : sizeof(int32_t) * nn,            // perm
                            sizeof(uint32_t) * 2 * (size_t)H,             // ab
                            sizeof(unsigned long long) * 2};              // meta
    constexpr int kParts = (int)(sizeof(sizes) / sizeof(sizes[0]));
    size_t offs[kParts], total = 0;
    for (int i = 0; i < kParts; ++i) {
        offs[i] = total;
        total += (sizes[i] + 255) & ~(size_t)255;
    }
    BTC_TRY(ws.buf.reserve(total));
    char* base = ws.buf.as<char>();
    auto part = [&](int i) { return sizes[i] ? (void*)(base + offs[i]) : nullptr; };
    uint32_t* deg = static_cast<uint32_t*>(part(0));
    uint32_t* start = static_cast<uint32_t*>(part(1));
    uint32_t* cursor = static_cast<uint32_t*>(part(2));
    int32_t* nbr = static_cast<int32_t*>(part(3));
    uint32_t* hv0 = static_cast<uint32_t*>(part(4));
    uint32_t* hv1 = static_cast<uint32_t*>(part(5));
    uint64_t* k0 = static_cast<uint64_t*>(part(6));
    uint64_t* k1 = static_cast<uint64_t*>(part(7));
    uint32_t* scratch = static_cast<uint32_t*>(part(8));
    int32_t* perm = static_cast<int32_t*>(part(9));
    uint32_t* ab = static_cast<uint32_t*>(part(10));
    unsigned long long* d_meta = static_cast<unsigned long long*>(part(11));  // [0] bad ids, [1] n

    std::vector<uint32_t> a(H), b(H), h_ab(2 * (size_t)H);
    hashorder_params(H, a.data(), b.data());
    for (int j = 0; j < H; ++j) {
        h_ab[2 * (size_t)j] = a[j];
        h_ab[2 * (size_t)j + 1] = b[j];
    }
    BTC_CUDA_TRY(cudaMemcpyAsync(ab, h_ab.data(), sizeof(uint32_t) * 2 * (size_t)H,
                                 cudaMemcpyHostToDevice, s));
    BTC_CUDA_TRY(cudaMemsetAsync(d_meta, 0, sizeof(unsigned long long) * 2, s));

    // ---- symmetric neighbour lists -------------------------------------------------
    BTC_CUDA_TRY(cudaMemsetAsync(deg, 0, sizeof(uint32_t) * (size_t)n, s));
    const int eg = grid_for(nnz > 0 ? nnz : 1, 256), vg = grid_for(n, 256);
    if (nnz > 0)
        ro::k_degree2<<<eg, 256, 0, s>>>(d_rows, d_cols, nnz, n, deg, d_meta);
    BTC_CUDA_TRY(cudaMemcpyAsync(start, deg, sizeof(uint32_t) * (size_t)n,
                                 cudaMemcpyDeviceToDevice, s));
    BTC_TRY(launch_tile_scan(start, (uint32_t)n, d_meta + 1, s));
    BTC_CUDA_TRY(cudaMemcpyAsync(cursor, start, sizeof(uint32_t) * (size_t)n,
                                 cudaMemcpyDeviceToDevice, s));
    // An out-of-range id fails the call before anything reaches the caller's arrays
    // (neither d_perm nor the COO is written).
    unsigned long long h_bad = 0;
    BTC_CUDA_TRY(cudaGetLastError());
    BTC_CUDA_TRY(cudaMemcpyAsync(&h_bad, d_meta, sizeof(h_bad), cudaMemcpyDeviceToHost, s));
    BTC_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_bad) return BTC_E_RANGE;
    if (nnz > 0)
        ro::k_scatter2<<<eg, 256, 0, s>>>(d_rows, d_cols, nnz, n, cursor, nbr);

    // ---- signatures ------------------------------------------------------------------
    ro::k_minhash_first<<<vg, 256, 0, s>>>(start, deg, nbr, n, H, num_hops, ab, hv0);
    uint32_t* hin = hv0;
    uint32_t* hout = hv1;
    for (int hop = 1; hop < num_hops; ++hop) {
        ro::k_minhash_hop<<<vg, 256, 0, s>>>(start, deg, nbr, n, H, hin, hout);
        std::swap(hin, hout);
    }
    BTC_CUDA_TRY(cudaGetLastError());

    // ---- lexicographic order: least significant hash first, stable ------------------
    BTC_TRY(launch_set_u64(d_meta + 1, (unsigned long long)n, s));
    const uint64_t* prev = nullptr;
    uint64_t* keys = k0;
    uint64_t* alt = k1;
    for (int j = H - 1; j >= 0; --j) {
        ro::k_sig_keys<<<vg, 256, 0, s>>>(prev, n, hin + (size_t)j * n, keys);
        int st = BTC_OK;
        uint64_t* sorted = radix_sort_u64(keys, alt, (size_t)n, d_meta + 1, 32, 64,
                                          scratch, s, &st);
        BTC_TRY(st);
        // the next pass reads `sorted` and writes the other buffer
        uint64_t* other = sorted == keys ? alt : keys;
        prev = sorted;
        keys = other;
        alt = sorted;
    }

    // ---- relabel -----------------------------------------------------------------------
    int32_t* p = d_perm ? d_perm : perm;
    BTC_TRY(launch_rank_scatter(prev, n, p, s));
    if (nnz > 0) ro::k_relabel<<<eg, 256, 0, s>>>(d_rows, d_cols, nnz, p);
    BTC_CUDA_TRY(cudaGetLastError());
    BTC_CUDA_TRY(cudaStreamSynchronize(s));
    return BTC_OK;
}

// The reference's automatic decision (should_reorder_gpu, convert.h:579-596): devices
// below sm_120 (B200 is sm_100) take the Hopper/Ampere tree (convert.h:510-575), sm_120
// and above the Blackwell tree (convert.h:443-505).  N = vertices after remap, E = COO
// entries; dataset_hint may be null.
extern "C" int btc_should_reorder(int32_t num_rows, int64_t nnz, int sm_version,
                                  const char* dataset_hint)
{
    const double N = (double)num_rows, E = (double)nnz;
    if (num_rows <= 0 || nnz <= 0) return 0;
    std::string name = dataset_hint ? dataset_hint : "";
    std::transform(name.begin(), name.end(), name.begin(), [](unsigned char ch) { return (char)std::tolower(ch); });
    static const char* kStructured[] = {"road", "bcsstk", "bcsstm", "cage", "delaunay", "ga41",
                                        "si41", "struct", "pdb", "cant", "consph", "dawson",
                                        "mac_econ", "mc2depi", "msc", "nemeth", "net50", "pli",
                                        "pwtk", "shyy", "spacestation", "tandem", "torso",
                                        "webbase", "web-notre", "freescale"};
    bool structured = false;
    for (const char* kw : kStructured)
        if (name.find(kw) != std::string::npos) structured = true;
    const double log_n = std::log10(N), log_e = std::log10(E);
    const double avg = 2.0 * E / N;
    if ((structured ? log_e : 0.0) > 2.04) return 0;
    if (sm_version >= 120) {
        if (log_n <= 3.65) return 0;
        if (std::log10(avg) <= 1.84) return (avg > 35.0 && num_rows > 500000) ? 0 : 1;
        return log_n <= 4.96 ? 0 : 1;
    }
    if (num_rows <= 5000) return 0;
    if (avg <= 28.93) return 1;
    if (log_e <= 6.03) return 0;
    return log_n <= (sm_version >= 90 ? 5.95 : 5.80) ? 1 : 0;
}
