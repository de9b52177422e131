// noalloc.cu -- btc_count_bcsr_noalloc: the triangle count for callers that cannot
// allocate device memory.
//
// Every other count entry point keeps its scratch (one partial sum per CTA of the
// persistent count kernel, and the counter the last CTA uses to know it is last) in
// memory obtained from cudaMalloc.  Some callers cannot let a library do that: a serving
// process whose memory pool has already claimed the device's free memory (a fresh
// cudaMalloc then fails), or a latency-bound loop that must not call cudaMalloc/cudaFree
// because they can synchronise the device and take unbounded time.  This entry point
// keeps that scratch in g_noalloc_scratch, a fixed array that is part of the library's
// device image; the caller passes only the Bit-BSR it already holds and a device word
// for the count.
#include <cuda.h>

#include <cstdio>
#include <mutex>

#include "common.cuh"

namespace btc200 {
namespace {

// Slots [0, kNoAllocMaxCtas) hold one partial sum per CTA of the count kernel; slot
// kNoAllocMaxCtas holds the CTA completion counter and the next slot the tile-queue
// head.  (2048 + 2) x 8 bytes = 16,400 bytes, present on every GPU that loads the
// library until the process exits.
constexpr int kNoAllocMaxCtas = 2048;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocMaxCtas + 2];

constexpr int kMaxDevices = 64;
struct ScratchSetup {
    unsigned long long ctx_id = 0;      // context the address belongs to (0: none yet)
    unsigned long long* addr = nullptr;
};
std::mutex g_setup_mu;
ScratchSetup g_setup[kMaxDevices];

// Unique id of the current context (driver API through the runtime's entry-point table,
// so the library needs no link against libcuda); 0 when there is none yet.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_noalloc_scratch on the current device.  In host code the array's
// name is only a host-side handle, so the address comes from cudaGetSymbolAddress, with
// the device current, once per device and context: a device reset (cudaDeviceReset)
// gives the device a new context and the next call looks the address up again.
int scratch_for_current_device(unsigned long long** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BTC_E_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    ScratchSetup& su = g_setup[dev];
    const unsigned long long id = current_context_id();
    if (!su.addr || id == 0 || id != su.ctx_id) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            note_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
            return BTC_E_CUDA;
        }
        su.addr = static_cast<unsigned long long*>(p);
        // the lookup made the context current if there was none; a context whose id
        // cannot be read is looked up again on every call
        su.ctx_id = id ? id : current_context_id();
    }
    *out = su.addr;
    return BTC_OK;
}

}  // namespace
}  // namespace btc200

using namespace btc200;

extern "C" int btc_count_bcsr_noalloc(const btc_bcsr_device* b, int tile_cols, int tau,
                                      btc_stream_t stream, unsigned long long* d_out)
{
    if (!b || (tile_cols != 32 && tile_cols != 128)) return BTC_E_INVAL;
    if (tau == BTC_TAU_DEFAULT) tau = btc_default_tau(tile_cols);
    if (tau < 0) return BTC_E_INVAL;
    unsigned long long* out = d_out ? d_out : b->result;
    if (!out) return BTC_E_INVAL;
    if (b->num_blocks && (!b->indptr || !b->indices || !b->blocks || !b->row_indices))
        return BTC_E_INVAL;

    const int grid = count_grid_size(tile_cols);
    if (grid > kNoAllocMaxCtas) {
        std::fprintf(stderr,
                     "btc_count_bcsr_noalloc: this GPU runs the count with %d CTAs but the "
                     "static scratch holds partial sums for %d\n",
                     grid, kNoAllocMaxCtas);
        return BTC_E_INVAL;
    }
    unsigned long long* scratch = nullptr;
    BTC_TRY(scratch_for_current_device(&scratch));

    // The completion counter and the queue head must start at zero.  The kernel's last
    // CTA puts both back to zero, so this only matters after an interrupted launch.
    BTC_CUDA_TRY(
        cudaMemsetAsync(scratch + kNoAllocMaxCtas, 0, 2 * sizeof(unsigned long long), stream));
    CountScratch scr{scratch, reinterpret_cast<unsigned int*>(scratch + kNoAllocMaxCtas),
                     scratch + kNoAllocMaxCtas + 1, out, nullptr};
    return launch_count(tile_cols, b->indptr, b->indices, b->row_indices, b->blocks, b->num_blocks,
                        b->n_row_blocks, tau, scr, stream);
}
