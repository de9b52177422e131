// server.cu -- continuous-batching triangle-count server (btc_server_*).
//
// Requests (an edge list and a vertex count) are copied into the server on submit and
// queued.  One engine thread owns `slots` batch slots, each with its own stream, batch
// handle, pinned staging buffers and completion event.  Whenever a slot is free and
// requests are waiting, the engine admits requests in arrival order into a batch while
// the batch stays within max_batch_graphs / max_batch_edges and the device memory of all
// slots stays within the HBM budget; it stages the edges, builds the batch and enqueues
// its count on the slot's stream, then returns to the queue.  Requests that arrive while
// a batch is on the GPU therefore go into the next batch, which starts on the other slot
// while the first is still running.  A slot's results are published when its event
// completes; every result carries the request's submit and completion times on the
// server's steady clock.  A request of at least solo_edges edges runs alone on a slot
// through the single-graph path with descending-degree orientation (batching gains
// nothing for it, and degree order keeps its hub rows short) once it reaches the front
// of the queue; a batch being formed passes over such requests and takes the small ones
// behind them.  Solo rebuilds are enqueued without a host wait, so the engine thread
// keeps filling the other slots meanwhile.  One solo launch runs at a time, on whichever
// slot takes it, through one solo handle: a large graph occupies the whole GPU, so two
// at once would gain nothing and would hold both slots while small requests wait.  Every
// device allocation (batch and solo handles, edge copies) is stream-ordered on the
// stream of the slot using it, from a pool the server owns: a handle that grows for a
// larger request frees and allocates without cudaFree's wait for the whole device, so
// one slot's growth never stalls the engine behind another slot's long batch.  With
// slots = 1 and max_batch_graphs = 1 the same server is the plain one-request-at-a-time
// path.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "common.cuh"
#include "handle.cuh"

namespace btc200 {
size_t batch_device_bytes(const btc_batch* b);
btc_bitbsr* bitbsr_new_pooled(cudaMemPool_t pool, cudaStream_t s);
btc_batch* batch_new_pooled(cudaMemPool_t pool, cudaStream_t s);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    int32_t n = 0;
    int64_t m = 0;
    std::vector<int32_t> own_src, own_dst;   // copied on submit
    const int32_t* src = nullptr;            // the edges (owned or borrowed)
    const int32_t* dst = nullptr;
    double submit_s = 0;
};

struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int reserve(size_t need)
    {
        if (need <= bytes && p) return BTC_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const size_t want = need + need / 4 + 4096;
        if (cudaMallocHost(&p, want) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return BTC_E_NOMEM;
        }
        bytes = want;
        return BTC_OK;
    }
    void release()
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr;  // recorded before the slot's first copy
    cudaEvent_t done = nullptr;
    btc_batch* batch = nullptr;
    btc200::DevBuf d_counts, d_src, d_dst;
    PinnedBuf h_src, h_dst, h_counts;
    std::vector<Request> reqs;
    std::vector<int64_t> offsets;
    std::vector<int32_t> nv;
    size_t device_bytes = 0;  // batch handle and edge copies
    bool busy = false;
    bool solo_launch = false; // the slot's current launch runs one request alone
};

}  // namespace

struct btc_server {
    btc_server_config cfg{};
    int device = 0;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request> pending;
    std::vector<btc_server_result> done;
    std::vector<Slot> slots;
    cudaMemPool_t pool = nullptr;  // the slots' device memory (stream-ordered)
    // large requests: one graph, descending-degree order, on whichever slot runs it
    btc_bitbsr* solo = nullptr;
    int solo_slot = -1;        // the slot whose launch holds the solo handle, or -1
    bool solo_async = false;   // its rebuild was enqueued without a wait
    std::thread engine;
    bool stop = false;
    uint64_t next_id = 1;
    btc_server_stats stats{};
    // Host-side allocation-failure injection (tests): the buffer reservations of
    // launch_slot are numbered from 1 in the order the engine thread makes them, and
    // those listed in BTC_SERVER_FAIL_RESERVE (comma-separated) report BTC_E_NOMEM
    // without allocating.  Read once, at btc_server_create.
    std::vector<uint64_t> fail_reserve;
    uint64_t reserve_no = 0;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

size_t slot_budget_in_use(btc_server* s, const Slot* except)
{
    size_t b = s->solo ? s->solo->device_bytes() : 0;
    for (const Slot& sl : s->slots)
        if (&sl != except) b += sl.device_bytes;
    return b;
}

// Device bytes a batch of m edges over `rows` row blocks may need (builder workspace,
// bitmap, tiles at most one per edge), used to admit requests before building.
// Cell-bitmap words of a request's part of a batch (row blocks x column-block words); a
// batch holds at most kBatchWords of them, and a request of more than kSoloWords (a
// large vertex range, however few its edges) runs alone through the single-graph builder,
// which falls back to sorting when a bitmap would be too large.
constexpr int64_t kBatchWords = 1ll << 29;
constexpr int64_t kSoloWords = 1ll << 26;
int64_t cell_words(int32_t n, int tile_cols)
{
    const int64_t rows = ((int64_t)n + 15) / 16;
    const int64_t cbs = ((int64_t)n + tile_cols - 1) / tile_cols;
    return rows * ((cbs + 31) / 32);
}

bool runs_alone(const btc_server* s, const Request& q, int tile_cols)
{
    return q.m >= s->cfg.solo_edges || cell_words(q.n, tile_cols) > kSoloWords;
}

size_t batch_bytes_bound(int64_t m, int64_t rows, int tile_cols)
{
    const size_t tw_bytes = (size_t)2 * tile_cols;  // 16 rows x tile_cols bits
    const size_t m_ = (size_t)m;
    return 8 * m_ + (m_ + 1) * (tw_bytes + 8) + (size_t)rows * 4 + (size_t)rows * 64 + (1 << 20);
}

void publish(btc_server* s, Slot& sl, int status)
{
    const double t = s->now();
    const unsigned long long* c = static_cast<const unsigned long long*>(sl.h_counts.p);
    std::lock_guard<std::mutex> lock(s->mu);
    for (size_t i = 0; i < sl.reqs.size(); ++i) {
        btc_server_result r{};
        r.id = sl.reqs[i].id;
        r.count = status == BTC_OK ? c[i] : 0ull;
        r.status = status;
        r.n = sl.reqs[i].n;
        r.m = sl.reqs[i].m;
        r.submit_s = sl.reqs[i].submit_s;
        r.done_s = t;
        s->done.push_back(r);
    }
    s->stats.batches += 1;
    s->stats.graphs += sl.reqs.size();
    if (status == BTC_OK) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, sl.start, sl.done) != cudaSuccess) cudaGetLastError();
        const bool solo = sl.reqs.size() == 1 && sl.solo_launch;
        (solo ? s->stats.solo_stream_ms : s->stats.batch_stream_ms) += ms;
        s->stats.solo_launches += solo;
    }
    for (const Request& q : sl.reqs) s->stats.edges += (uint64_t)q.m;
    sl.reqs.clear();
    sl.busy = false;
    if (s->solo_slot == (int)(&sl - s->slots.data())) s->solo_slot = -1;
    s->cv.notify_all();
}

// Requests at least this large are copied host-to-device straight from the caller's
// memory (full DMA speed when it is pinned); smaller ones are packed into the slot's
// pinned staging buffer and sent in one copy.
constexpr int64_t kDirectCopyEdges = 1 << 16;

int launch_slot(btc_server* s, Slot& sl)
{
    const int G = (int)sl.reqs.size();
    // small requests first, so they form one contiguous staged run
    std::stable_sort(sl.reqs.begin(), sl.reqs.end(), [](const Request& a, const Request& b) {
        return (a.m >= kDirectCopyEdges) < (b.m >= kDirectCopyEdges);
    });
    sl.offsets.assign(1, 0);
    sl.nv.clear();
    int64_t staged = 0;
    for (const Request& q : sl.reqs) {
        sl.offsets.push_back(sl.offsets.back() + q.m);
        sl.nv.push_back(q.n);
        if (q.m < kDirectCopyEdges) staged += q.m;
    }
    const int64_t m = sl.offsets.back();
    // every reservation is numbered (fail_reserve injects an allocation failure)
    auto reserve = [&](auto& buf, size_t bytes) -> int {
        const uint64_t k = ++s->reserve_no;
        if (std::find(s->fail_reserve.begin(), s->fail_reserve.end(), k) != s->fail_reserve.end())
            return BTC_E_NOMEM;
        return buf.reserve(bytes);
    };
    int st = reserve(sl.h_src, sizeof(int32_t) * (size_t)(staged ? staged : 1));
    if (st == BTC_OK) st = reserve(sl.h_dst, sizeof(int32_t) * (size_t)(staged ? staged : 1));
    if (st == BTC_OK) st = reserve(sl.h_counts, sizeof(unsigned long long) * (size_t)G);
    if (st == BTC_OK) st = reserve(sl.d_counts, sizeof(unsigned long long) * (size_t)G);
    if (st == BTC_OK) st = reserve(sl.d_src, sizeof(int32_t) * (size_t)(m ? m : 1));
    if (st == BTC_OK) st = reserve(sl.d_dst, sizeof(int32_t) * (size_t)(m ? m : 1));
    if (st != BTC_OK) return st;
    if (cudaEventRecord(sl.start, sl.stream) != cudaSuccess) return BTC_E_CUDA;
    int32_t* hs = static_cast<int32_t*>(sl.h_src.p);
    int32_t* hd = static_cast<int32_t*>(sl.h_dst.p);
    int32_t* ds = sl.d_src.as<int32_t>();
    int32_t* dd = sl.d_dst.as<int32_t>();
    for (int i = 0; i < G; ++i) {
        const Request& q = sl.reqs[(size_t)i];
        const size_t off = (size_t)sl.offsets[(size_t)i], bytes = sizeof(int32_t) * (size_t)q.m;
        if (q.m < kDirectCopyEdges) {
            std::memcpy(hs + off, q.src, bytes);
            std::memcpy(hd + off, q.dst, bytes);
        } else if (cudaMemcpyAsync(ds + off, q.src, bytes, cudaMemcpyHostToDevice, sl.stream) !=
                       cudaSuccess ||
                   cudaMemcpyAsync(dd + off, q.dst, bytes, cudaMemcpyHostToDevice, sl.stream) !=
                       cudaSuccess) {
            return BTC_E_CUDA;
        }
    }
    if (staged &&
        (cudaMemcpyAsync(ds, hs, sizeof(int32_t) * (size_t)staged, cudaMemcpyHostToDevice,
                         sl.stream) != cudaSuccess ||
         cudaMemcpyAsync(dd, hd, sizeof(int32_t) * (size_t)staged, cudaMemcpyHostToDevice,
                         sl.stream) != cudaSuccess))
        return BTC_E_CUDA;
    const bool solo = G == 1 && runs_alone(s, sl.reqs[0], s->cfg.tile_cols ? s->cfg.tile_cols : 128);
    sl.solo_launch = solo;
    if (solo) {
        // a large graph gains nothing from batching; descending-degree orientation keeps
        // its hub rows short (the engine's tile policy then picks 16x128)
        // Rebuilds are enqueued without a host wait (BTC_BUILD_ASYNC), so the engine
        // thread goes on filling the other slots; finish_solo checks the build's status.
        // The admission loop handed this slot the solo handle (s->solo_slot); the slot
        // that ran it before has been published, so no stream still uses its buffers, and
        // its allocations now follow this slot's stream.  (The first build into the empty
        // handle waits: there are no arrays to enqueue against yet.)
        if (!s->solo && !(s->solo = btc200::bitbsr_new_pooled(s->pool, sl.stream))) return BTC_E_NOMEM;
        s->solo->set_pool(s->pool, sl.stream);
        st = btc_rebuild_bitbsr(s->solo, ds, dd, m, sl.reqs[0].n, 0,
                                BTC_ORIENT_DEGREE | BTC_BUILD_ASYNC, sl.stream);
        s->solo_async = st == BTC_OK;
        if (st != BTC_OK) return st;
        st = btc_count_async(s->solo, s->cfg.tau, sl.stream, sl.d_counts.as<unsigned long long>());
        if (st != BTC_OK) return st;
    } else {
        if (!sl.batch && !(sl.batch = btc200::batch_new_pooled(s->pool, sl.stream))) return BTC_E_NOMEM;
        st = btc_batch_rebuild(sl.batch, ds, dd, sl.offsets.data(), sl.nv.data(), G,
                               s->cfg.tile_cols, 0, sl.stream);
        if (st != BTC_OK) return st;
        st = btc_batch_count(sl.batch, s->cfg.tau, sl.stream,
                             sl.d_counts.as<unsigned long long>(), nullptr);
        if (st != BTC_OK) return st;
    }
    // device memory held by this slot (read directly: btc_*_info would also count the
    // unique edges, a device pass not needed here)
    sl.device_bytes = (sl.batch ? btc200::batch_device_bytes(sl.batch) : 0) + sl.d_src.bytes +
                      sl.d_dst.bytes;
    if (cudaMemcpyAsync(sl.h_counts.p, sl.d_counts.ptr, sizeof(unsigned long long) * (size_t)G,
                        cudaMemcpyDeviceToHost, sl.stream) != cudaSuccess ||
        cudaEventRecord(sl.done, sl.stream) != cudaSuccess)
        return BTC_E_CUDA;
    const size_t in_use = slot_budget_in_use(s, nullptr);
    std::lock_guard<std::mutex> lock(s->mu);
    s->stats.peak_device_bytes = std::max<uint64_t>(s->stats.peak_device_bytes, in_use);
    return BTC_OK;
}

// Status of a finished slot whose solo graph was rebuilt without a wait: an enqueued
// build that found more tiles than the handle's arrays hold built nothing, so it is
// redone here with a waiting rebuild from the slot's device copy of the edges.
int finish_solo(btc_server* s, Slot& sl, int tau)
{
    if (!sl.solo_launch || !s->solo_async) return BTC_OK;
    s->solo_async = false;
    int st = resolve_build(s->solo);
    if (st != BTC_E_CAPACITY) return st;
    const int64_t m = sl.offsets.back();
    st = btc_rebuild_bitbsr(s->solo, sl.d_src.as<int32_t>(), sl.d_dst.as<int32_t>(), m,
                            sl.reqs[0].n, 0, BTC_ORIENT_DEGREE, sl.stream);
    if (st == BTC_OK)
        st = btc_count_async(s->solo, tau, sl.stream, sl.d_counts.as<unsigned long long>());
    if (st == BTC_OK &&
        (cudaMemcpyAsync(sl.h_counts.p, sl.d_counts.ptr, sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost, sl.stream) != cudaSuccess ||
         cudaStreamSynchronize(sl.stream) != cudaSuccess))
        st = BTC_E_CUDA;
    return st;
}

void engine_loop(btc_server* s)
{
    cudaSetDevice(s->device);
    for (;;) {
        // 1. publish finished slots
        for (Slot& sl : s->slots)
            if (sl.busy && cudaEventQuery(sl.done) == cudaSuccess) publish(s, sl, finish_solo(s, sl, s->cfg.tau));

        // 2. fill a free slot from the queue
        Slot* free_slot = nullptr;
        for (Slot& sl : s->slots)
            if (!sl.busy) {
                free_slot = &sl;
                break;
            }
        bool launched = false;
        if (free_slot) {
            Slot& sl = *free_slot;
            std::vector<btc_server_result> rejected;
            {
                std::unique_lock<std::mutex> lock(s->mu);
                if (s->pending.empty()) {
                    bool any_busy = false;
                    for (const Slot& o : s->slots) any_busy |= o.busy;
                    if (s->stop && !any_busy) return;
                    // idle: wait for a request (or, with work on the GPU, poll again soon)
                    s->cv.wait_for(lock, std::chrono::microseconds(any_busy ? 50 : 2000));
                    continue;
                }
                const size_t others = slot_budget_in_use(s, &sl);
                const size_t budget = s->cfg.hbm_budget_bytes > others
                                          ? (size_t)s->cfg.hbm_budget_bytes - others
                                          : 0;
                sl.offsets.assign(1, 0);
                sl.nv.clear();
                int64_t m = 0, rows = 0, words = 0;
                const int tile = s->cfg.tile_cols ? s->cfg.tile_cols : 128;
                // A batch under way passes over large requests (they run alone when they
                // reach the front), looking at most this many queued requests.
                const size_t max_scan = 4 * (size_t)s->cfg.max_batch_graphs + 64;
                size_t scanned = 0;
                auto it = s->pending.begin();
                while (it != s->pending.end() && (int)sl.reqs.size() < s->cfg.max_batch_graphs &&
                       scanned++ < max_scan) {
                    Request& q = *it;
                    const int64_t qm = q.m;
                    // a large request runs alone (solo path), when the solo handle is free
                    const bool alone = runs_alone(s, q, tile);
                    if (alone && (!sl.reqs.empty() || s->solo_slot >= 0)) {
                        ++it;
                        continue;
                    }
                    const int64_t qr = ((int64_t)q.n + 15) / 16;
                    const size_t need = batch_bytes_bound(m + qm, rows + qr, tile);
                    const int64_t qw = cell_words(q.n, tile);
                    if (!sl.reqs.empty() &&
                        (m + qm > s->cfg.max_batch_edges || need > budget || words + qw > kBatchWords))
                        break;
                    if (sl.reqs.empty() && batch_bytes_bound(qm, qr, tile) > budget &&
                        others == 0) {
                        btc_server_result r{};
                        r.id = q.id;
                        r.status = BTC_E_NOMEM;
                        r.n = q.n;
                        r.m = qm;
                        r.submit_s = q.submit_s;
                        r.done_s = s->now();
                        rejected.push_back(r);
                        it = s->pending.erase(it);
                        continue;
                    }
                    if (sl.reqs.empty() && batch_bytes_bound(qm, qr, tile) > budget) break;
                    m += qm;
                    rows += qr;
                    words += qw;
                    sl.reqs.push_back(std::move(q));
                    sl.offsets.push_back(m);
                    sl.nv.push_back(sl.reqs.back().n);
                    it = s->pending.erase(it);
                    if (alone) {
                        s->solo_slot = (int)(&sl - s->slots.data());
                        break;
                    }
                }
                if (!rejected.empty()) {
                    s->done.insert(s->done.end(), rejected.begin(), rejected.end());
                    s->stats.rejected += rejected.size();
                    s->cv.notify_all();
                }
            }
            if (!sl.reqs.empty()) {
                sl.busy = true;
                const int st = launch_slot(s, sl);
                if (st != BTC_OK) {
                    cudaStreamSynchronize(sl.stream);
                    publish(s, sl, st);
                }
                launched = true;
            }
        }
        if (!launched) {
            // every slot busy, or the next request must wait for memory: wait until any
            // busy slot finishes (polling all of them, so a short batch on one slot is
            // published while a long one still runs on another)
            for (;;) {
                bool any_busy = false, any_done = false;
                for (Slot& sl : s->slots) {
                    if (!sl.busy) continue;
                    any_busy = true;
                    const cudaError_t q = cudaEventQuery(sl.done);
                    if (q == cudaSuccess) any_done = true;
                    else if (q != cudaErrorNotReady) {
                        cudaGetLastError();
                        any_done = true;  // publish reports the slot's failure
                    }
                }
                if (!any_busy || any_done) break;
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
        }
    }
}

}  // namespace

extern "C" {

void btc_server_default_config(btc_server_config* cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->hbm_budget_bytes = 150ull << 30;
    cfg->max_batch_graphs = 4096;
    cfg->max_batch_edges = 256ll << 20;
    cfg->slots = 2;
    cfg->tile_cols = 32;
    cfg->tau = BTC_TAU_DEFAULT;
    cfg->solo_edges = 1ll << 20;
}

int btc_server_create(const btc_server_config* cfg, btc_server** out)
{
    if (!cfg || !out) return BTC_E_INVAL;
    *out = nullptr;
    if (cfg->slots < 1 || cfg->slots > 8 || cfg->max_batch_graphs < 1 || cfg->max_batch_edges < 1 ||
        (cfg->tile_cols != 0 && cfg->tile_cols != 32 && cfg->tile_cols != 128))
        return BTC_E_INVAL;
    btc_server* s = new (std::nothrow) btc_server();
    if (!s) return BTC_E_NOMEM;
    s->cfg = *cfg;
    s->t0 = Clock::now();
    if (const char* f = std::getenv("BTC_SERVER_FAIL_RESERVE")) {
        for (const char* p = f; *p;) {
            char* end = nullptr;
            const unsigned long long k = std::strtoull(p, &end, 10);
            if (end == p) break;
            if (k) s->fail_reserve.push_back(k);
            p = *end == ',' ? end + 1 : end;
        }
    }
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        delete s;
        return BTC_E_CUDA;
    }
    // the slots' device memory: a pool that keeps what is freed for the next request
    // (the HBM budget bounds what the slots hold)
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    uint64_t keep = ~0ull;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
        cudaGetLastError();
        if (s->pool) cudaMemPoolDestroy(s->pool);
        delete s;
        return BTC_E_CUDA;
    }
    s->slots.resize((size_t)cfg->slots);
    for (Slot& sl : s->slots) {
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&sl.start) != cudaSuccess || cudaEventCreate(&sl.done) != cudaSuccess) {
            cudaGetLastError();
            for (Slot& o : s->slots) {
                if (o.stream) cudaStreamDestroy(o.stream);
                if (o.start) cudaEventDestroy(o.start);
                if (o.done) cudaEventDestroy(o.done);
            }
            cudaMemPoolDestroy(s->pool);
            delete s;
            return BTC_E_CUDA;
        }
        for (btc200::DevBuf* d : {&sl.d_counts, &sl.d_src, &sl.d_dst}) {
            d->pool = s->pool;
            d->stream = sl.stream;
        }
    }
    s->engine = std::thread(engine_loop, s);
    *out = s;
    return BTC_OK;
}

int btc_server_submit(btc_server* s, const int32_t* src, const int32_t* dst, int64_t m, int32_t n,
                      uint32_t flags, uint64_t* id_out)
{
    if (!s || m < 0 || n < 0 || (m > 0 && (!src || !dst)) || (flags & ~BTC_SUBMIT_BORROW))
        return BTC_E_INVAL;
    Request q;
    q.n = n;
    q.m = m;
    if (flags & BTC_SUBMIT_BORROW) {
        q.src = src;
        q.dst = dst;
    } else {
        q.own_src.assign(src, src + m);
        q.own_dst.assign(dst, dst + m);
        q.src = q.own_src.data();
        q.dst = q.own_dst.data();
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return BTC_E_INVAL;
    q.id = s->next_id++;
    q.submit_s = s->now();
    if (id_out) *id_out = q.id;
    s->pending.push_back(std::move(q));
    s->cv.notify_all();
    return BTC_OK;
}

int btc_server_poll(btc_server* s, btc_server_result* out, int max_results, int* n_out, int wait_ms)
{
    if (!s || !out || !n_out || max_results < 0) return BTC_E_INVAL;
    std::unique_lock<std::mutex> lock(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv.wait_for(lock, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    const int k = (int)std::min<size_t>(s->done.size(), (size_t)max_results);
    std::copy(s->done.begin(), s->done.begin() + k, out);
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n_out = k;
    return BTC_OK;
}

int btc_server_stats_get(btc_server* s, btc_server_stats* st)
{
    if (!s || !st) return BTC_E_INVAL;
    std::lock_guard<std::mutex> lock(s->mu);
    *st = s->stats;
    st->queued = s->pending.size();
    st->now_s = s->now();
    return BTC_OK;
}

void btc_server_destroy(btc_server* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->engine.joinable()) s->engine.join();
    // the handles' and buffers' frees are ordered on the slot streams: free, then let the
    // streams drain, then drop the streams and the pool
    if (s->solo) btc_free(s->solo);
    for (Slot& sl : s->slots) {
        if (sl.batch) btc_batch_free(sl.batch);
        sl.d_counts.release();
        sl.d_src.release();
        sl.d_dst.release();
        sl.h_src.release();
        sl.h_dst.release();
        sl.h_counts.release();
        if (sl.stream) cudaStreamSynchronize(sl.stream);
    }
    for (Slot& sl : s->slots) {
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.start) cudaEventDestroy(sl.start);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
}

}  // extern "C"
