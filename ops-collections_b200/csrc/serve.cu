// serve.cu -- request server over resident tables (the served pattern):
// requests of uneven sizes arrive over time against resident StaticMap /
// StaticSet tables; the server admits them as launch slots and HBM budget free
// up, so work from many requests overlaps on the device.
//
//  * Arrival times are part of a request: a caller may submit a whole
//    schedule (e.g. Poisson arrivals) ahead of time; a request becomes
//    eligible when its arrival time has passed, and its latency is measured
//    from that arrival to the completion the dispatcher observes.
//  * Admission is FIFO by arrival, bounded by the number of launch slots
//    (streams) and by an HBM budget that counts the registered resident
//    tables plus every slot's staging buffer.  A slot's staging buffer is
//    persistent, sized at creation for a full coalesced lookup batch, and only
//    grows (doubling, from the server's own stream-ordered pool); idle slots
//    give theirs back when the budget is short.
//  * Continuous batching: when a lookup reaches the head, every arrived lookup
//    of the same kind on the same table joins its launch (up to
//    max_batch_keys), skipping requests on other tables and stopping at a
//    write on that table; results are scattered back to each request.
//  * Every request's host buffers are copied in and out on its launch's
//    stream; pinned host memory lets copies overlap other launches.
//  * Per-table arrival order for writes: an Insert / InsertOrAssign launch
//    waits (stream-ordered, cudaStreamWaitEvent) for every launch in flight on
//    the same table, and a lookup waits for the writes in flight on its table,
//    so each request sees exactly the writes that arrived before it; lookups
//    between two writes overlap freely.
//  * Threads: submitters only touch an inbox (one short lock); waiters sleep
//    on a per-server completion condition; the dispatcher owns the queue, the
//    slots and the CUDA calls without holding either lock.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "b2co_host.h"

int b2co_oa_launch_insert(b2co_oa_table* t, void const* pairs, uint64_t n, bool assign,
                          unsigned long long* d_counters, cudaStream_t s);
uint64_t b2co_oa_table_bytes(b2co_oa_table const* t);
void b2co_oa_table_sizes(b2co_oa_table const* t, uint32_t* key_bytes, uint32_t* payload_bytes, uint32_t* pair_bytes);

using namespace b2co;

namespace {

uint64_t now_ns()
{
    return uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(
                        std::chrono::steady_clock::now().time_since_epoch())
                        .count());
}

struct Request {
    b2co_request_info info{};
    b2co_oa_table* table = nullptr;
    void const* host_in = nullptr;
    void* host_out = nullptr;
    void* out_dev = nullptr;  // host_out as the GPU addresses it, when it is pinned (else nullptr)
    uint64_t in_bytes = 0, out_bytes = 0;
    bool taken = false;  // admitted (possibly ahead of the queue's head); popped lazily
    std::atomic<bool> done{false};
    // Two owners: the dispatcher's queue (until it pops the request, which may be
    // long after the request finished, since requests are admitted out of
    // order) and the caller (until its wait returns).  The last one frees it.
    std::atomic<int> refs{2};
};

void unref(Request* r)
{
    if (r->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) delete r;
}

bool is_write(Request const* r) { return r->info.op == B2CO_OP_INSERT || r->info.op == B2CO_OP_INSERT_OR_ASSIGN; }

// Direct results: a lookup launch's results go from the device staging straight
// into the requests' pinned host buffers with SM stores over PCIe (one kernel
// for up to kScatterMax requests) instead of one device-to-host copy per request.
constexpr uint32_t kScatterMax = 32;
struct ScatterEntry {
    void* dst;
    uint64_t off, bytes;
};
struct ScatterList {
    uint32_t count;
    ScatterEntry e[kScatterMax];
};

// Block row y copies entry y; 16-byte stores when both ends and the length
// allow it, 8- or 1-byte stores otherwise.
__global__ void __launch_bounds__(256) k_scatter_out(char const* src, __grid_constant__ const ScatterList L)
{
    for (uint32_t j = blockIdx.y; j < L.count; j += gridDim.y) {
        ScatterEntry const e = L.e[j];
        char const* from = src + e.off;
        char* to = static_cast<char*>(e.dst);
        uint64_t const step = uint64_t(gridDim.x) * blockDim.x;
        uint64_t const t0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
        uintptr_t const al = reinterpret_cast<uintptr_t>(from) | reinterpret_cast<uintptr_t>(to) | e.bytes;
        if ((al & 15) == 0) {
            for (uint64_t i = t0; i < e.bytes / 16; i += step)
                reinterpret_cast<uint4*>(to)[i] = reinterpret_cast<uint4 const*>(from)[i];
        } else if ((al & 7) == 0) {
            for (uint64_t i = t0; i < e.bytes / 8; i += step)
                reinterpret_cast<unsigned long long*>(to)[i] = reinterpret_cast<unsigned long long const*>(from)[i];
        } else {
            for (uint64_t i = t0; i < e.bytes; i += step) to[i] = from[i];
        }
    }
}

// How far past the head the dispatcher looks for lookups to coalesce.
constexpr size_t kCoalesceScan = 4096;
// Staging buffers grow in steps of this many bytes.
constexpr uint64_t kStagingQuantum = 2ull << 20;

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<Request*> reqs;
    char* buf = nullptr;  // persistent staging: [inputs | outputs | 2 counters]
    uint64_t cap = 0;
    unsigned long long* h_counters = nullptr;  // pinned (failed, assigned) of an Insert / IOA launch
    // packed copies: pinned host arenas a coalesced launch's inputs are packed
    // into (one copy in) and its outputs come back to (one copy out)
    char* hin = nullptr;
    char* hout = nullptr;
    uint64_t hin_cap = 0, hout_cap = 0;
    bool packed = false;  // the launch in flight returns its outputs through hout
};

// Host copies spread over a small pool of threads (the caller takes part):
// packing requests' inputs into a launch's pinned arena and scattering its
// outputs back.  Jobs are cut into pieces of at most kPiece bytes.
class CopyPool {
   public:
    static constexpr uint64_t kPiece = 1ull << 20;
    struct Copy {
        void* dst;
        void const* src;
        uint64_t bytes;
    };

    explicit CopyPool(unsigned threads)
    {
        for (unsigned i = 0; i < threads; ++i) workers_.emplace_back([this] { work(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> l(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    size_t threads() const { return workers_.size(); }

    // Runs every copy; returns when all are done.
    void run(std::vector<Copy> const& copies)
    {
        pieces_.clear();
        for (auto const& c : copies)
            for (uint64_t off = 0; off < c.bytes; off += kPiece)
                pieces_.push_back(Copy{static_cast<char*>(c.dst) + off, static_cast<char const*>(c.src) + off,
                                       std::min(kPiece, c.bytes - off)});
        if (pieces_.empty()) return;
        {
            std::lock_guard<std::mutex> l(mu_);
            next_.store(0);
            left_.store(pieces_.size());
            ++epoch_;
        }
        cv_.notify_all();
        drain();
        while (left_.load(std::memory_order_acquire) != 0) std::this_thread::yield();
    }

   private:
    void drain()
    {
        for (;;) {
            size_t const i = next_.fetch_add(1);
            if (i >= pieces_.size()) return;
            std::memcpy(pieces_[i].dst, pieces_[i].src, pieces_[i].bytes);
            left_.fetch_sub(1, std::memory_order_release);
        }
    }
    void work()
    {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&] { return stop_ || epoch_ != seen; });
                if (stop_) return;
                seen = epoch_;
            }
            drain();
        }
    }

    std::vector<std::thread> workers_;
    std::vector<Copy> pieces_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::atomic<size_t> next_{0}, left_{0};
    uint64_t epoch_ = 0;
    bool stop_ = false;
};

enum class Fit { kOk, kWait, kNever, kError };

}  // namespace

struct b2co_server {
    int device = 0;
    uint64_t budget = 0, max_batch_keys = 0;
    // plain mode: every request is its own launch and a table has at most one
    // launch in flight (copy in, kernel, copy out, then the table's next
    // request); the baseline the coalescing server is measured against
    std::atomic<bool> plain{false};
    // packed copies of coalesced launches: the pool and the slots' pinned
    // arenas exist from creation; `pack` switches their use on and off
    std::unique_ptr<CopyPool> packer;
    std::atomic<bool> pack{false};
    std::atomic<bool> direct{false};  // lookups write results straight into pinned host buffers
    std::atomic<uint64_t> packed_launches{0}, direct_launches{0};

    // submission side (in_mu)
    std::mutex in_mu;
    std::condition_variable cv_work;
    std::vector<Request*> inbox;
    std::unordered_map<uint64_t, Request*> all;
    uint64_t next_id = 1, last_arrival = 0;
    bool stop = false;

    // completion side
    std::mutex done_mu;
    std::condition_variable cv_done;

    // accounting, read from any thread (the dispatcher is the only writer of the rest)
    std::atomic<uint64_t> resident{0}, staging{0}, launches{0}, coalesced{0};
    std::atomic<uint64_t> grows{0}, max_launch_ns{0}, max_reserve_ns{0}, max_gap_ns{0}, launch_ns{0}, copies{0};

    // dispatcher-private
    std::deque<Request*> queue;  // in arrival order
    std::vector<Slot> slots;
    cudaMemPool_t pool = nullptr;  // staging buffers; keeps freed memory
    std::thread worker;

    static void raise_max(std::atomic<uint64_t>& m, uint64_t v)
    {
        if (v > m.load(std::memory_order_relaxed)) m.store(v, std::memory_order_relaxed);
    }

    static uint64_t align(uint64_t v) { return (v + 255) & ~uint64_t(255); }

    static uint64_t staging_bytes(std::vector<Request*> const& g)
    {
        uint64_t in = 0, out = 0;
        for (auto* r : g) in += r->in_bytes, out += r->out_bytes;
        return align(in) + align(out) + 256;  // + device counters
    }

    // The free slot for `need` bytes: the smallest buffer that holds it, else the largest.
    Slot* pick_slot(uint64_t need)
    {
        Slot *fit = nullptr, *big = nullptr;
        for (auto& sl : slots) {
            if (sl.busy) continue;
            if (sl.cap >= need && (!fit || sl.cap < fit->cap)) fit = &sl;
            if (!big || sl.cap > big->cap) big = &sl;
        }
        return fit ? fit : big;
    }

    // Streams, events, staging and the pool (the dispatcher has stopped).
    void free_resources()
    {
        for (auto& sl : slots) {
            if (sl.stream) {
                release(sl);
                cudaStreamSynchronize(sl.stream);
                cudaStreamDestroy(sl.stream);
            }
            if (sl.done) cudaEventDestroy(sl.done);
            if (sl.h_counters) cudaFreeHost(sl.h_counters);
            if (sl.hin) cudaFreeHost(sl.hin);
            if (sl.hout) cudaFreeHost(sl.hout);
            sl = Slot{};
        }
        if (pool) cudaMemPoolDestroy(pool);
        pool = nullptr;
    }

    void release(Slot& sl)
    {
        if (!sl.buf) return;
        cudaFreeAsync(sl.buf, sl.stream);
        staging -= sl.cap;
        sl.buf = nullptr;
        sl.cap = 0;
    }

    // Gives a free slot a staging buffer of at least `need` bytes within the
    // budget.  Buffers come from the server's own stream-ordered pool, which
    // keeps what is freed: fresh device memory costs milliseconds of host time
    // (measured up to 19 ms per allocation while copies were in flight),
    // pooled memory does not.  Growth doubles, so a slot regrows rarely.
    Fit reserve(Slot& sl, uint64_t need, bool exact = false)
    {
        if (sl.cap >= need) return Fit::kOk;
        uint64_t const res = resident.load();
        if (res + need > budget) return Fit::kNever;
        auto others = [&] { return staging.load() - sl.cap; };
        uint64_t want = std::max(need, 2 * sl.cap);
        want = (want + kStagingQuantum - 1) / kStagingQuantum * kStagingQuantum;
        if (exact || res + others() + want > budget) want = need;
        for (auto& o : slots) {  // idle slots give their buffers back
            if (res + others() + want <= budget) break;
            if (&o != &sl && !o.busy) release(o);
        }
        if (res + others() + want > budget) return Fit::kWait;  // launches in flight hold the rest
        uint64_t const t0 = now_ns();
        release(sl);
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&sl.buf), want, pool, sl.stream);
        raise_max(max_reserve_ns, now_ns() - t0);
        ++grows;
        if (e != cudaSuccess) {
            cudaGetLastError();
            sl.buf = nullptr;
            return Fit::kError;
        }
        sl.cap = want;
        staging += want;
        return Fit::kOk;
    }

    // Issues one launch (one or more coalesced requests) on a slot's stream.
    int launch(Slot& sl, std::vector<Request*>& g)
    {
        cudaStream_t s = sl.stream;
        Request* h = g.front();
        uint64_t in_total = 0, out_total = 0, n_total = 0;
        for (auto* r : g) in_total += r->in_bytes, out_total += r->out_bytes, n_total += r->info.n;
        char* din = sl.buf;
        char* dout = sl.buf + align(in_total);
        auto* dcnt = reinterpret_cast<unsigned long long*>(dout + align(out_total));
        // lookups whose result buffers are pinned get their results written by
        // the GPU (no copy out); else a coalesced launch may pack its requests
        // into the slot's pinned arena (one copy in and one copy out)
        bool direct_results = !is_write(h) && direct.load(std::memory_order_relaxed);
        for (auto* r : g) direct_results = direct_results && r->out_dev;
        sl.packed = !direct_results && packer && pack.load(std::memory_order_relaxed) && g.size() > 1 &&
                    in_total <= sl.hin_cap && out_total <= sl.hout_cap;
        uint64_t off = 0;
        if (sl.packed) {
            std::vector<CopyPool::Copy> pack;
            for (auto* r : g) {
                pack.push_back(CopyPool::Copy{sl.hin + off, r->host_in, r->in_bytes});
                off += r->in_bytes;
            }
            packer->run(pack);
            B2CO_CUDA(cudaMemcpyAsync(din, sl.hin, in_total, cudaMemcpyHostToDevice, s));
            ++copies;
            ++packed_launches;
        } else {
            for (auto* r : g) {
                B2CO_CUDA(cudaMemcpyAsync(din + off, r->host_in, r->in_bytes, cudaMemcpyHostToDevice, s));
                off += r->in_bytes;
                ++copies;
            }
        }
        int const op = h->info.op;
        bool const writes = is_write(h);
        for (auto& other : slots) {  // per-table arrival order (the copies above still overlap)
            if (&other == &sl || !other.busy || other.reqs.front()->table != h->table) continue;
            if (writes || is_write(other.reqs.front())) B2CO_CUDA(cudaStreamWaitEvent(s, other.done, 0));
        }
        int st = B2CO_OK;
        if (op == B2CO_OP_FIND) {
            st = b2co_oa_find_async(h->table, din, dout, n_total, reinterpret_cast<b2co_stream>(s));
        } else if (op == B2CO_OP_CONTAINS) {
            st = b2co_oa_contains_async(h->table, din, reinterpret_cast<uint8_t*>(dout), n_total,
                                        reinterpret_cast<b2co_stream>(s));
        } else {
            B2CO_CUDA(cudaMemsetAsync(dcnt, 0, 2 * sizeof(unsigned long long), s));
            st = b2co_oa_launch_insert(h->table, din, n_total, op == B2CO_OP_INSERT_OR_ASSIGN, dcnt, s);
            if (!st) {
                B2CO_CUDA(cudaMemcpyAsync(sl.h_counters, dcnt, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                          s));
                ++copies;
            }
        }
        if (st) return st;
        if (direct_results) {
            ScatterList L{};
            uint64_t o = 0;
            size_t done = 0;
            while (done < g.size()) {
                L.count = 0;
                uint64_t most = 0;
                for (; done < g.size() && L.count < kScatterMax; ++done) {
                    Request* r = g[done];
                    L.e[L.count++] = ScatterEntry{r->out_dev, o, r->out_bytes};
                    o += r->out_bytes;
                    most = std::max(most, r->out_bytes);
                }
                uint32_t const gx = uint32_t(std::min<uint64_t>(64, (most + 4095) / 4096 + 1));
                k_scatter_out<<<dim3(gx, L.count), 256, 0, s>>>(dout, L);
                B2CO_CUDA(cudaGetLastError());
            }
            ++direct_launches;
        } else if (sl.packed) {
            if (out_total) {
                B2CO_CUDA(cudaMemcpyAsync(sl.hout, dout, out_total, cudaMemcpyDeviceToHost, s));
                ++copies;
            }
        } else {
            off = 0;
            for (auto* r : g) {
                if (r->out_bytes) {
                    B2CO_CUDA(cudaMemcpyAsync(r->host_out, dout + off, r->out_bytes, cudaMemcpyDeviceToHost, s));
                    ++copies;
                }
                off += r->out_bytes;
            }
        }
        B2CO_CUDA(cudaEventRecord(sl.done, s));
        sl.busy = true;
        sl.reqs = g;
        ++launches;
        coalesced += g.size();
        return B2CO_OK;
    }

    // The launch group headed by the queue's head: for a lookup, every arrived
    // lookup of the same kind on the same table up to max_batch_keys, skipping
    // requests on other tables (independent) and other lookups, stopping at a
    // write on the table (arrival order); a write runs alone.
    std::vector<Request*> group_at_head(uint64_t t) const
    {
        std::vector<Request*> g{queue.front()};
        Request const* h = g[0];
        if (is_write(h)) return g;
        uint64_t keys = h->info.n;
        size_t const scan = std::min<size_t>(queue.size(), kCoalesceScan);
        for (size_t i = 1; i < scan; ++i) {
            Request* r = queue[i];
            if (r->taken) continue;
            if (r->info.arrival_ns > t) break;
            if (r->table != h->table) continue;
            if (is_write(r)) break;
            if (r->info.op != h->info.op) continue;
            if (keys + r->info.n > max_batch_keys) break;
            g.push_back(r);
            keys += r->info.n;
        }
        return g;
    }

    // Publishes finished requests to waiters.
    void finish(std::vector<Request*> const& g, int status, uint64_t t)
    {
        for (auto* r : g) {
            r->info.status = status;
            r->info.done_ns = t;
        }
        {
            std::lock_guard<std::mutex> l(done_mu);
            for (auto* r : g) r->done.store(true, std::memory_order_release);
        }
        cv_done.notify_all();
    }

    // Drops the admitted requests at the queue's head (the queue's reference).
    void pop_taken()
    {
        while (!queue.empty() && queue.front()->taken) {
            Request* r = queue.front();
            queue.pop_front();
            unref(r);
        }
    }

    // Plain mode's admission: the earliest arrived request of each table that
    // has no launch in flight, alone, in arrival order per table (tables run
    // side by side on the slots).
    bool admit_plain()
    {
        bool progress = false;
        uint64_t const t = now_ns();
        pop_taken();
        std::vector<b2co_oa_table const*> blocked;
        for (auto& sl : slots)
            if (sl.busy) blocked.push_back(sl.reqs.front()->table);
        size_t const scan = std::min<size_t>(queue.size(), kCoalesceScan);
        for (size_t i = 0; i < scan; ++i) {
            Request* r = queue[i];
            if (r->taken) continue;
            if (r->info.arrival_ns > t) break;
            if (std::find(blocked.begin(), blocked.end(), r->table) != blocked.end()) continue;
            blocked.push_back(r->table);  // the table's later requests wait for this one
            std::vector<Request*> g{r};
            Slot* sl = pick_slot(staging_bytes(g));
            if (!sl) return progress;
            Fit const fit = reserve(*sl, staging_bytes(g));
            if (fit == Fit::kWait) return progress;
            if (fit != Fit::kOk) {
                r->taken = true;
                finish({r}, fit == Fit::kNever ? B2CO_ENOMEM : B2CO_ECUDA, t);
                progress = true;
                continue;
            }
            r->taken = true;
            r->info.admit_ns = t;
            uint64_t const l0 = now_ns();
            int const st = launch(*sl, g);
            uint64_t const dl = now_ns() - l0;
            raise_max(max_launch_ns, dl);
            launch_ns += dl;
            if (st) {
                cudaStreamSynchronize(sl->stream);
                cudaGetLastError();
                finish(g, st, now_ns());
            }
            progress = true;
        }
        return progress;
    }

    // Admits what the slots and the budget allow; true if anything changed.
    bool admit()
    {
        if (plain.load(std::memory_order_relaxed)) return admit_plain();
        bool progress = false;
        uint64_t const t = now_ns();
        for (;;) {
            pop_taken();
            if (queue.empty() || queue.front()->info.arrival_ns > t) return progress;
            std::vector<Request*> g = group_at_head(t);
            Slot* sl = pick_slot(staging_bytes(g));
            if (!sl) return progress;  // every slot busy
            Fit fit = reserve(*sl, staging_bytes(g));
            if (fit != Fit::kOk && g.size() > 1) {  // try the head alone
                g.resize(1);
                sl = pick_slot(staging_bytes(g));
                fit = reserve(*sl, staging_bytes(g));
            }
            if (fit == Fit::kWait) return progress;  // memory frees up as launches finish
            if (fit != Fit::kOk) {                   // can never fit, or the allocation failed
                g[0]->taken = true;
                finish({g[0]}, fit == Fit::kNever ? B2CO_ENOMEM : B2CO_ECUDA, t);
                progress = true;
                continue;
            }
            for (auto* r : g) {
                r->taken = true;
                r->info.admit_ns = t;
            }
            uint64_t const l0 = now_ns();
            int const st = launch(*sl, g);
            uint64_t const dl = now_ns() - l0;
            raise_max(max_launch_ns, dl);
            launch_ns += dl;
            if (st) {
                cudaStreamSynchronize(sl->stream);  // no kernel ran; let the copies from the caller's buffers finish
                cudaGetLastError();
                finish(g, st, now_ns());
            }
            progress = true;
        }
    }

    // Completes the launches that finished; true if any did.
    bool complete()
    {
        bool progress = false;
        for (auto& sl : slots) {
            if (!sl.busy) continue;
            cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) continue;
            if (q == cudaSuccess && is_write(sl.reqs.front()))
                for (auto* r : sl.reqs) {
                    r->info.failed = sl.h_counters[0];
                    r->info.assigned = sl.h_counters[1];
                }
            if (q == cudaSuccess && sl.packed) {  // the outputs came back packed: hand each request its part
                std::vector<CopyPool::Copy> scatter;
                uint64_t off = 0;
                for (auto* r : sl.reqs) {
                    if (r->out_bytes) scatter.push_back(CopyPool::Copy{r->host_out, sl.hout + off, r->out_bytes});
                    off += r->out_bytes;
                }
                packer->run(scatter);
            }
            sl.busy = false;
            std::vector<Request*> g;
            g.swap(sl.reqs);
            finish(g, q == cudaSuccess ? B2CO_OK : B2CO_ECUDA, now_ns());
            progress = true;
        }
        return progress;
    }

    void run()
    {
        cudaSetDevice(device);
        uint64_t last_poll = 0;
        for (;;) {
            uint64_t const poll = now_ns();
            if (last_poll) raise_max(max_gap_ns, poll - last_poll);
            last_poll = poll;
            bool stopping;
            {
                std::lock_guard<std::mutex> l(in_mu);
                for (auto* r : inbox) queue.push_back(r);
                inbox.clear();
                stopping = stop;
            }
            bool progress = complete();
            progress = admit() || progress;
            bool busy = false;
            for (auto& sl : slots) busy = busy || sl.busy;
            if (stopping && queue.empty() && !busy) break;
            if (progress) continue;
            // Nothing changed: keep polling while work is in flight or due soon
            // (a sleep would add tens of microseconds of timer slack to every
            // latency), else sleep until the head's arrival or a submission.
            uint64_t const head = queue.empty() ? 0 : queue.front()->info.arrival_ns;
            if (busy || (head && head <= now_ns() + 50000)) {
                std::this_thread::yield();
                continue;
            }
            std::unique_lock<std::mutex> l(in_mu);
            auto ready = [this] { return !inbox.empty() || stop; };
            if (head)
                cv_work.wait_until(l, std::chrono::steady_clock::time_point(std::chrono::nanoseconds(head)), ready);
            else
                cv_work.wait(l, ready);
            last_poll = 0;  // an idle sleep is not a polling gap
        }
    }
};

namespace {

// Validates one request and builds it (arrival time and id are set at enqueue).
int make_request(b2co_request_desc const& d, std::unique_ptr<Request>& out)
{
    int const op = d.op;
    if (!d.table || !d.host_in) return fail(B2CO_EINVAL, "null argument");
    if (op < B2CO_OP_FIND || op > B2CO_OP_INSERT_OR_ASSIGN) return fail(B2CO_EINVAL, "unknown request op");
    bool const lookup = op == B2CO_OP_FIND || op == B2CO_OP_CONTAINS;
    if (lookup && !d.host_out) return fail(B2CO_EINVAL, "lookups need an output");
    if (d.n == 0 || d.n > kMaxBatch) return fail(B2CO_ERANGE, "request size out of range");
    uint32_t kb, pb, sb;
    b2co_oa_table_sizes(d.table, &kb, &pb, &sb);
    out.reset(new (std::nothrow) Request);
    if (!out) return fail(B2CO_ENOMEM, "host allocation failed");
    Request& r = *out;
    r.table = d.table;
    r.host_in = d.host_in;
    r.host_out = d.host_out;
    r.info.op = op;
    r.info.n = d.n;
    r.info.arrival_ns = d.arrival_ns;
    r.in_bytes = d.n * (lookup ? kb : sb);
    r.out_bytes = op == B2CO_OP_FIND ? d.n * pb : (op == B2CO_OP_CONTAINS ? d.n : 0);
    if (lookup) {  // a pinned result buffer the GPU can address (checked here, on the submitting thread)
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, d.host_out) == cudaSuccess && pa.type == cudaMemoryTypeHost &&
            pa.devicePointer)
            r.out_dev = pa.devicePointer;
        else
            cudaGetLastError();
    }
    return B2CO_OK;
}

int submit(b2co_server* s, uint64_t count, b2co_request_desc const* descs, uint64_t* ids)
{
    std::vector<std::unique_ptr<Request>> reqs(count);
    for (uint64_t i = 0; i < count; ++i)
        if (int st = make_request(descs[i], reqs[i])) return st;
    {
        std::lock_guard<std::mutex> g(s->in_mu);
        if (s->stop) return fail(B2CO_EINVAL, "the server is shutting down");
        uint64_t const now = now_ns();
        uint64_t last = s->last_arrival;
        for (auto& r : reqs) {
            if (!r->info.arrival_ns) r->info.arrival_ns = now;
            if (r->info.arrival_ns < last) return fail(B2CO_EINVAL, "requests must be submitted in arrival order");
            last = r->info.arrival_ns;
        }
        s->last_arrival = last;
        for (uint64_t i = 0; i < count; ++i) {
            Request* r = reqs[i].release();
            r->info.id = s->next_id++;
            s->inbox.push_back(r);
            s->all[r->info.id] = r;
            ids[i] = r->info.id;
        }
    }
    s->cv_work.notify_one();
    return B2CO_OK;
}

// Waits for one request and releases it; its status.
int wait_one(b2co_server* s, uint64_t id, b2co_request_info* info)
{
    Request* r;
    {
        std::lock_guard<std::mutex> g(s->in_mu);
        auto it = s->all.find(id);
        if (it == s->all.end()) return fail(B2CO_EINVAL, "unknown request id");
        r = it->second;
        s->all.erase(it);
    }
    {
        std::unique_lock<std::mutex> l(s->done_mu);
        s->cv_done.wait(l, [r] { return r->done.load(std::memory_order_acquire); });
    }
    if (info) *info = r->info;
    int st = r->info.status;
    unref(r);  // the dispatcher may still hold it in its queue
    return st == B2CO_OK ? B2CO_OK : fail(st, "request failed");
}

}  // namespace

extern "C" {

uint64_t b2co_server_now_ns(void) { return now_ns(); }

int b2co_server_create(uint32_t max_inflight, uint64_t hbm_budget_bytes, uint64_t max_batch_keys, b2co_server** out)
{
    if (!out) return fail(B2CO_EINVAL, "null output");
    *out = nullptr;
    if (max_inflight == 0 || max_inflight > 256) return fail(B2CO_EINVAL, "max_inflight must be in [1, 256]");
    if (hbm_budget_bytes == 0) return fail(B2CO_EINVAL, "the HBM budget must be positive");
    auto* s = new (std::nothrow) b2co_server;
    if (!s) return fail(B2CO_ENOMEM, "host allocation failed");
    std::unique_ptr<b2co_server> guard(s);
    s->budget = hbm_budget_bytes;
    s->max_batch_keys = max_batch_keys ? max_batch_keys : (1ull << 24);
    s->slots.resize(max_inflight);
    auto setup = [s]() -> int {
        B2CO_CUDA(cudaGetDevice(&s->device));
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = s->device;
        B2CO_CUDA(cudaMemPoolCreate(&s->pool, &props));
        uint64_t keep = ~0ull;
        B2CO_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
        for (auto& sl : s->slots) {
            B2CO_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
            B2CO_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
            B2CO_CUDA(cudaMallocHost(reinterpret_cast<void**>(&sl.h_counters), 2 * sizeof(unsigned long long)));
        }
        // Size every slot for a full coalesced lookup batch of 8-byte keys and
        // 8-byte payloads now, before traffic (at most a quarter of the budget).
        uint64_t per_slot = std::min(2 * b2co_server::align(s->max_batch_keys * 8) + 256,
                                     s->budget / (4 * s->slots.size()) / 256 * 256);
        if (per_slot >= 256)
            for (auto& sl : s->slots)
                if (s->reserve(sl, per_slot, true) != Fit::kOk)
                    return fail(B2CO_ENOMEM, "staging reservation failed");
        for (auto& sl : s->slots) B2CO_CUDA(cudaStreamSynchronize(sl.stream));
        // packed copies: a pinned arena per slot for a coalesced launch of up
        // to 4 Mi keys (16-byte pairs in, 8-byte payloads out) and a pool of
        // host threads that pack and scatter
        uint64_t const keys = std::min<uint64_t>(s->max_batch_keys, 1ull << 22);
        for (auto& sl : s->slots) {
            B2CO_CUDA(cudaMallocHost(reinterpret_cast<void**>(&sl.hin), keys * 16));
            B2CO_CUDA(cudaMallocHost(reinterpret_cast<void**>(&sl.hout), keys * 8));
            sl.hin_cap = keys * 16;
            sl.hout_cap = keys * 8;
        }
        unsigned const hw = std::max(2u, std::thread::hardware_concurrency());
        s->packer.reset(new (std::nothrow) CopyPool(std::min(8u, hw / 2) - 1));
        if (!s->packer) return fail(B2CO_ENOMEM, "host allocation failed");
        return B2CO_OK;
    };
    if (int st = setup()) {
        s->free_resources();
        return st;
    }
    s->worker = std::thread([s] { s->run(); });
    *out = guard.release();
    return B2CO_OK;
}

int b2co_server_set_packing(b2co_server* s, int on)
{
    if (!s) return fail(B2CO_EINVAL, "null server");
    s->pack.store(on != 0);
    return B2CO_OK;
}

int b2co_server_set_direct_results(b2co_server* s, int on)
{
    if (!s) return fail(B2CO_EINVAL, "null server");
    s->direct.store(on != 0);
    return B2CO_OK;
}

int b2co_server_set_plain(b2co_server* s, int plain)
{
    if (!s) return fail(B2CO_EINVAL, "null server");
    s->plain.store(plain != 0);
    return B2CO_OK;
}

int b2co_server_register_table(b2co_server* s, b2co_oa_table* t)
{
    if (!s || !t) return fail(B2CO_EINVAL, "null argument");
    std::lock_guard<std::mutex> g(s->in_mu);
    uint64_t b = b2co_oa_table_bytes(t);
    if (s->resident.load() + s->staging.load() + b > s->budget)
        return fail(B2CO_ENOMEM, "resident table exceeds the HBM budget");
    s->resident += b;
    return B2CO_OK;
}

int b2co_server_submit(b2co_server* s, b2co_oa_table* t, int op, void const* host_in, void* host_out, uint64_t n,
                       uint64_t arrival_ns, uint64_t* request_id)
{
    if (!s || !request_id) return fail(B2CO_EINVAL, "null argument");
    b2co_request_desc d{t, op, 0, host_in, host_out, n, arrival_ns};
    return submit(s, 1, &d, request_id);
}

int b2co_server_submit_many(b2co_server* s, uint64_t count, b2co_request_desc const* requests, uint64_t* ids)
{
    if (!s || (count && (!requests || !ids))) return fail(B2CO_EINVAL, "null argument");
    return count ? submit(s, count, requests, ids) : B2CO_OK;
}

int b2co_server_wait(b2co_server* s, uint64_t id, b2co_request_info* info)
{
    if (!s) return fail(B2CO_EINVAL, "null server");
    return wait_one(s, id, info);
}

int b2co_server_wait_many(b2co_server* s, uint64_t count, uint64_t const* ids, b2co_request_info* infos)
{
    if (!s || (count && !ids)) return fail(B2CO_EINVAL, "null argument");
    int first = B2CO_OK;
    for (uint64_t i = 0; i < count; ++i) {
        int st = wait_one(s, ids[i], infos ? infos + i : nullptr);
        if (st && !first) first = st;
    }
    return first ? fail(first, "a request failed") : B2CO_OK;
}

int b2co_server_stats(b2co_server* s, uint64_t* launches, uint64_t* requests_launched, uint64_t* bytes_in_use)
{
    if (!s) return fail(B2CO_EINVAL, "null server");
    if (launches) *launches = s->launches.load();
    if (requests_launched) *requests_launched = s->coalesced.load();
    if (bytes_in_use) *bytes_in_use = s->resident.load() + s->staging.load();
    return B2CO_OK;
}

int b2co_server_get_stats_ex(b2co_server* s, b2co_server_stats_ex* out)
{
    if (!s || !out) return fail(B2CO_EINVAL, "null argument");
    out->launches = s->launches.load();
    out->requests_launched = s->coalesced.load();
    out->staging_bytes = s->staging.load();
    out->bytes_in_use = s->resident.load() + out->staging_bytes;
    out->staging_grows = s->grows.load();
    out->max_launch_host_ns = s->max_launch_ns.load();
    out->max_reserve_host_ns = s->max_reserve_ns.load();
    out->max_loop_gap_ns = s->max_gap_ns.load();
    out->total_launch_host_ns = s->launch_ns.load();
    out->copies = s->copies.load();
    out->packed_launches = s->packed_launches.load();
    out->direct_launches = s->direct_launches.load();
    return B2CO_OK;
}

int b2co_server_destroy(b2co_server* s)
{
    if (!s) return B2CO_OK;
    {
        std::lock_guard<std::mutex> g(s->in_mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();  // drains every submitted request first
    s->free_resources();
    for (auto& kv : s->all) unref(kv.second);  // never waited for; the drained queue let go of them
    delete s;
    return B2CO_OK;
}

}  // extern "C"
