// server.cu -- the serving loop: continuous batching of single-automaton
// requests with admission by device-memory budget.
//
// One loop thread owns the GPU work; submit/poll/cancel only touch queues
// under a mutex.  Each turn of the loop:
//   * takes newly submitted requests;
//   * requests with n <= 20: whenever one of kSmallSlots mini-batch slots is
//     free, packs up to max_batch of them into pinned 64-byte records, copies
//     them in and runs the batch kernels (per-lane / warp-pooled) on the
//     slot's own stream.  The kernels store each automaton's length and word
//     straight into mapped host memory and then flag it, so every request is
//     delivered as soon as its own search ends -- a mini-batch holding a
//     Cerny search (C_20: 361 levels, ~1 ms in one CTA) does not hold back the
//     other requests in it;
//   * large requests (n >= 21): when the previous level launch batch is done,
//     collects finished slots, admits waiting requests in arrival order while
//     their bitmap + queue fit the arena (the 2^n-bit budget), and launches
//     the next few levels of every admitted request (k_level.cu).  Requests
//     that arrive while others are running are admitted at the next turn and
//     advance together with them: their work overlaps on the device.
//     (n = 17..20 went through level slots too, at a p99 of 7 ms at 32K
//     requests/s: every level of a Cerny C_20 cost one launch shared with all
//     admitted requests.  In the mini-batches a CTA runs it alone.)
// Completion order follows the GPU, not submission order.
#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "runtime.cuh"

using namespace sbfs;

namespace {

struct Request {
    uint64_t id;
    int32_t n;
    uint8_t a[32], b[32];   // zero past n: together the 64-byte record of the batch kernels
    double submit_ms;
};
static_assert(offsetof(Request, b) == offsetof(Request, a) + 32, "a and b form one 64-byte record");

constexpr int kSmallMaxN = 20;
constexpr int kWords = 12;
constexpr int kSmallSlots = 4;   // mini-batches in flight (lanes 0..3; lane 4 runs the level slots)

// One mini-batch of small requests in flight.
struct SmallSlot {
    int lane = 0;                        // handle lane: stream and kernel scratch
    DevBuf d_recs, d_ns;
    HostBuf h_recs, h_ns;                // staging in
    HostBuf h_len, h_words, h_flags;     // mapped: the kernels store results and flags here
    HostBuf h_err;                       // the launch set's device error word, copied back behind it
    int32_t *dl = nullptr;               // device aliases of the mapped buffers
    uint64_t *dw = nullptr;
    unsigned int *df = nullptr;
    std::vector<Request> reqs;
    std::vector<char> delivered;
    size_t left = 0;                     // requests not yet delivered
    unsigned int tag = 0;                // this launch's flag value
    int64_t seq = 0;                     // 1-based launch number of the mini-batch
    int64_t footprint = 0;               // admitted bytes: 2^n / 8 + 64 per request
    cudaEvent_t ev = nullptr;
    bool busy = false;
};

}  // namespace

struct sbfs_server {
    sbfs_server_config cfg{};
    sbfs_handle *h = nullptr;
    std::thread loop;
    std::mutex mu;
    std::condition_variable cv_in, cv_out;
    std::deque<Request> incoming;
    std::deque<sbfs_result> ready;
    std::unordered_set<uint64_t> cancel_req;
    bool stopping = false;
    bool reset_peak = false;
    uint64_t next_id = 1;
    std::chrono::steady_clock::time_point t0;
    // stats (mutex-protected)
    sbfs_server_stats st{};
    // loop-owned
    std::deque<Request> pend_small, pend_big;
    SmallSlot small[kSmallSlots];
    unsigned int next_tag = 1;
    Arena arena;                                   // HBM budget of the admitted large requests
    int64_t small_used = 0, small_peak = 0;        // footprint of the mini-batches in flight
    std::vector<sbfs_result> batch_out;            // results of one poll pass, handed over together
    LevelEngine big;                               // level slots for n >= 21
    std::unordered_map<long long, Request> large;   // admitted, keyed by id
    std::string error;
    // set once a CUDA call of the loop failed: every request still held, and
    // every later one, completes with failed_status (the context may be lost)
    bool failed = false;
    int32_t failed_status = SBFS_ECUDA;
    int64_t batches_launched = 0;
    // host-side fault injection for tests (environment SBFS_SERVER_FAIL_BATCH=k):
    // mini-batch k is reported as failed once its work has completed, as a
    // failed cudaEventQuery would report it; no GPU fault is involved
    int64_t inject_fail_batch = 0;

    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

sbfs_result make_result(const Request &r, int32_t status, int32_t len, const uint64_t *word, double done_ms)
{
    sbfs_result res;
    std::memset(&res, 0, sizeof(res));
    res.id = r.id;
    res.status = status;
    res.len = len;
    res.n = r.n;
    if (word) std::memcpy(res.word, word, sizeof(res.word));
    res.submit_ms = r.submit_ms;
    res.done_ms = done_ms;
    return res;
}

void complete(sbfs_server *s, const Request &r, int32_t status, int32_t len, const uint64_t *word)
{
    const sbfs_result res = make_result(r, status, len, word, s->now_ms());
    std::lock_guard<std::mutex> lock(s->mu);
    s->ready.push_back(res);
    s->st.completed++;
    if (status == SBFS_ECANCELED) s->st.cancelled++;
    s->cv_out.notify_all();
}

// Hands a batch of finished results to the pollers under one lock: a burst of
// thousands of requests finishing together costs one lock and one wake-up,
// not one per request.
void deliver(sbfs_server *s, std::vector<sbfs_result> &batch)
{
    if (batch.empty()) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (const sbfs_result &r : batch) s->ready.push_back(r);
        s->st.completed += (int64_t)batch.size();
    }
    s->cv_out.notify_all();
    batch.clear();
}

enum class Ev { kPending, kDone, kFailed };
Ev event_state(cudaEvent_t ev, cudaError_t *err);
void fail_all(sbfs_server *s, int32_t status, const std::string &why);

// Bytes an n <= 20 request accounts for while its mini-batch is in flight: its
// 2^n-bit visited set (the store the batch kernels keep on chip, or in HBM for
// a hand-off) and its 64-byte record.
int64_t small_footprint(int n)
{
    return (int64_t)(((uint64_t)1 << n) / 8) + 64;
}

bool launch_small(sbfs_server *s, SmallSlot &S)
{
    Lane &L = s->h->lanes[(size_t)S.lane];
    const int cap = s->cfg.max_batch;
    S.reqs.clear();
    // admission by footprint: a request accounts for its 2^n-bit visited set
    // and its record; the mini-batches in flight stay within small_budget_bytes
    int64_t fp = 0;
    while (!s->pend_small.empty() && (int)S.reqs.size() < cap) {
        const int64_t need = small_footprint(s->pend_small.front().n);
        if (s->small_used + fp + need > s->cfg.small_budget_bytes && (fp > 0 || s->small_used > 0)) break;
        fp += need;
        S.reqs.push_back(s->pend_small.front());
        s->pend_small.pop_front();
    }
    const int64_t cnt = (int64_t)S.reqs.size();
    if (!cnt) return false;
    uint8_t *rec = S.h_recs.as<uint8_t>();
    uint8_t *ns = S.h_ns.as<uint8_t>();
    int max_n = 1;
    for (int64_t i = 0; i < cnt; ++i) {
        const Request &r = S.reqs[(size_t)i];
        std::memcpy(rec + i * 64, r.a, 64);
        ns[i] = (uint8_t)r.n;
        max_n = std::max(max_n, r.n);
    }
    S.tag = s->next_tag++;
    if (s->next_tag == 0) s->next_tag = 1;
    cudaStream_t st = L.stream;
    cudaMemcpyAsync(S.d_recs.ptr, rec, (size_t)cnt * 64, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(S.d_ns.ptr, ns, (size_t)cnt, cudaMemcpyHostToDevice, st);
    int launches = 0;
    sbfs_status e = engine_enqueue(s->h, L, S.d_recs.as<uint8_t>(), 32, S.d_ns.as<uint8_t>(), 0, max_n, cnt, S.dl,
                                   S.dw, kWords, &launches, S.df, S.tag);
    if (e != SBFS_OK) {
        s->error = s->h->last_error;
        for (const Request &r : S.reqs) complete(s, r, e, -1, nullptr);
        S.reqs.clear();
        return false;
    }
    // the launch set's error bits come back behind its kernels, before the event
    cudaError_t ce = cudaMemcpyAsync(S.h_err.ptr, &L.counters.as<DevCounters>()->error, sizeof(int),
                                     cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaEventRecord(S.ev, st);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        S.delivered.assign((size_t)cnt, 0);
        S.left = (size_t)cnt;
        S.busy = true;   // fail_all completes this slot's requests
        S.footprint = 0;
        fail_all(s, SBFS_ECUDA, std::string("serving: ") + cudaGetErrorString(ce));
        return true;
    }
    S.delivered.assign((size_t)cnt, 0);
    S.left = (size_t)cnt;
    S.busy = true;
    S.seq = ++s->batches_launched;
    S.footprint = fp;
    s->small_used += fp;
    s->small_peak = std::max(s->small_peak, s->small_used);
    std::lock_guard<std::mutex> lock(s->mu);
    s->st.small_batches++;
    return true;
}

// Delivers the slot's requests whose flags are up; frees the slot once its
// launch sequence has completed.  A launch set that failed (a CUDA error on
// its stream, or error bits in its device error word) completes its requests
// not yet delivered with an error status, never with stale results.
bool poll_small(sbfs_server *s, SmallSlot &S)
{
    bool progress = false;
    const volatile unsigned int *flag = S.h_flags.as<unsigned int>();
    const int32_t *len = S.h_len.as<int32_t>();
    const uint64_t *words = S.h_words.as<uint64_t>();
    cudaError_t err = cudaSuccess;
    Ev ev = event_state(S.ev, &err);   // sampled before the flags: all are up once it is done
    if (ev == Ev::kDone && S.seq == s->inject_fail_batch) {
        ev = Ev::kFailed;
        err = cudaErrorLaunchFailure;
    }
    if (ev == Ev::kFailed) {
        fail_all(s, SBFS_ECUDA, std::string("serving mini-batch: ") + cudaGetErrorString(err));
        return true;
    }
    const bool finished = ev == Ev::kDone;
    int32_t status = SBFS_OK;
    if (finished) {
        const int bits = *(volatile const int *)S.h_err.ptr;
        if (bits) {
            status = (bits & kErrInvalid) ? SBFS_EINVAL : SBFS_ECUDA;
            s->error = (bits & kErrInvalid) ? "serving mini-batch: malformed automaton"
                                            : "serving mini-batch: device error bits set";
        }
    }
    std::vector<sbfs_result> &out = s->batch_out;
    const double now = s->now_ms();
    for (size_t i = 0; i < S.reqs.size() && S.left; ++i) {
        if (S.delivered[i] || (flag[i] != S.tag && !finished)) continue;
        std::atomic_thread_fence(std::memory_order_acquire);
        if (status == SBFS_OK) out.push_back(make_result(S.reqs[i], SBFS_OK, len[i], words + i * kWords, now));
        else out.push_back(make_result(S.reqs[i], status, -1, nullptr, now));
        S.delivered[i] = 1;
        --S.left;
        progress = true;
    }
    deliver(s, out);
    if (finished) {
        S.reqs.clear();
        S.busy = false;
        s->small_used -= S.footprint;
        S.footprint = 0;
        progress = true;
    }
    return progress;
}

// Runs one batch of max_batch automata spanning size classes 0..3 (n = 5, 10,
// 15, 20; seeded maps) through every mini-batch lane and waits for it.  The
// lanes' grow-only work buffers (bucketing arrays, hand-off lists, the CTA-wide
// kernel's queues for n = 20) reach their final size and every kernel is loaded
// before the first request, so the loop never allocates device memory: a
// cudaFree there would wait for the whole device.
cudaError_t prime_small(sbfs_server *s)
{
    const int64_t cnt = s->cfg.max_batch;
    const int sizes[4] = {5, 10, 15, 20};
    for (SmallSlot &S : s->small) {
        Lane &L = s->h->lanes[(size_t)S.lane];
        uint8_t *rec = S.h_recs.as<uint8_t>();
        uint8_t *ns = S.h_ns.as<uint8_t>();
        uint64_t x = 0x9E3779B97F4A7C15ull;
        for (int64_t i = 0; i < cnt; ++i) {
            const int n = sizes[i & 3];
            std::memset(rec + i * 64, 0, 64);
            for (int j = 0; j < n; ++j)
                for (int l = 0; l < 2; ++l) {
                    x += 0x9E3779B97F4A7C15ull;   // splitmix64
                    uint64_t z = x;
                    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
                    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
                    rec[i * 64 + 32 * l + j] = (uint8_t)((z ^ (z >> 31)) % (uint64_t)n);
                }
            ns[i] = (uint8_t)n;
        }
        cudaStream_t st = L.stream;
        cudaError_t e = cudaMemcpyAsync(S.d_recs.ptr, rec, (size_t)cnt * 64, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(S.d_ns.ptr, ns, (size_t)cnt, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
        int launches = 0;
        if (engine_enqueue(s->h, L, S.d_recs.as<uint8_t>(), 32, S.d_ns.as<uint8_t>(), 0, 20, cnt, S.dl, S.dw, kWords,
                           &launches, S.df, ~0u) != SBFS_OK)
            return cudaErrorUnknown;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
        std::memset(S.h_flags.ptr, 0, (size_t)cnt * 4);
    }
    return cudaSuccess;
}

// cudaEventQuery as done / pending / failed: anything but success and
// cudaErrorNotReady is a failure of the work before the event.
Ev event_state(cudaEvent_t ev, cudaError_t *err)
{
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return Ev::kDone;
    cudaGetLastError();
    if (e == cudaErrorNotReady) return Ev::kPending;
    *err = e;
    return Ev::kFailed;
}

// Completes every request the loop holds (mini-batches in flight, admitted and
// waiting large requests, pending small ones) with `status`, and every later
// request too: after a failed CUDA call the loop launches nothing more.
void fail_all(sbfs_server *s, int32_t status, const std::string &why)
{
    if (!s->failed) s->error = why;
    s->failed = true;
    s->failed_status = status;
    for (SmallSlot &S : s->small) {
        if (!S.busy) continue;
        for (size_t i = 0; i < S.reqs.size(); ++i)
            if (!S.delivered[i]) complete(s, S.reqs[i], status, -1, nullptr);
        S.reqs.clear();
        S.left = 0;
        S.busy = false;
        s->small_used -= S.footprint;
        S.footprint = 0;
    }
    for (auto &kv : s->large) complete(s, kv.second, status, -1, nullptr);
    s->large.clear();
    for (const Request &r : s->pend_small) complete(s, r, status, -1, nullptr);
    for (const Request &r : s->pend_big) complete(s, r, status, -1, nullptr);
    s->pend_small.clear();
    s->pend_big.clear();
}

void run_loop(sbfs_server *s)
{
    cudaSetDevice(s->h->device);
    Batch none{};
    std::vector<LevelEngine::Finished> fin;
    while (true) {
        bool progress = false;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            bool small_busy = false;
            for (const SmallSlot &S : s->small) small_busy |= S.busy;
            if (s->incoming.empty() && s->pend_small.empty() && s->pend_big.empty() &&
                !small_busy && s->large.empty()) {
                if (s->stopping) break;
                s->cv_in.wait_for(lock, std::chrono::milliseconds(2));
            }
            while (!s->incoming.empty()) {
                Request r = s->incoming.front();
                s->incoming.pop_front();
                if (s->cancel_req.erase(r.id)) {
                    lock.unlock();
                    complete(s, r, SBFS_ECANCELED, -1, nullptr);
                    lock.lock();
                    continue;
                }
                (r.n <= kSmallMaxN ? s->pend_small : s->pend_big).push_back(r);
                progress = true;
            }
        }
        if (s->failed) {
            // nothing more is launched: what arrives completes with the failure status
            fail_all(s, s->failed_status, s->error);
        }
        // small path
        for (SmallSlot &S : s->small)
            if (S.busy) progress |= poll_small(s, S);
        for (SmallSlot &S : s->small)
            if (!s->failed && !S.busy && !s->pend_small.empty()) progress |= launch_small(s, S);
        // large path
        LevelEngine &E = s->big;
        if (!s->failed && E.launched() && E.ready()) {
            fin.clear();
            const cudaError_t ce = E.collect(fin);
            for (auto &f : fin) {
                auto it = s->large.find(f.tag);
                if (it == s->large.end()) continue;
                complete(s, it->second, f.state == kSlotDone ? SBFS_OK : SBFS_ECUDA, f.len, f.word);
                s->large.erase(it);
            }
            if (ce != cudaSuccess) fail_all(s, SBFS_ECUDA, std::string("serving level slots: ") +
                                                               cudaGetErrorString(ce));
            progress = true;
        }
        if (!s->failed && !E.launched()) {
            while (!s->pend_big.empty()) {
                const Request &r = s->pend_big.front();
                if (E.admit(nullptr, 32, r.n, (long long)r.id, r.a, r.b) < 0) break;
                s->large.emplace((long long)r.id, r);
                s->pend_big.pop_front();
            }
            if (E.in_flight() > 0) {
                const cudaError_t ce = E.launch(s->cfg.max_levels, none, 4 * s->cfg.max_levels);
                if (ce != cudaSuccess) {
                    cudaGetLastError();
                    fail_all(s, SBFS_ECUDA, std::string("serving level launch: ") + cudaGetErrorString(ce));
                } else {
                    std::lock_guard<std::mutex> lock(s->mu);
                    s->st.level_launches += s->cfg.max_levels;
                }
                progress = true;
            }
        }
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (s->reset_peak) {
                s->arena.reset_peak();
                s->small_peak = s->small_used;
                s->reset_peak = false;
            }
            s->st.pending = (int64_t)(s->incoming.size() + s->pend_small.size() + s->pend_big.size());
            size_t small_left = 0;
            for (const SmallSlot &S : s->small) small_left += S.busy ? S.left : 0;
            s->st.in_flight = (int64_t)(small_left + s->large.size());
            s->st.arena_used = (int64_t)s->arena.used();
            s->st.arena_peak = (int64_t)s->arena.peak();
            s->st.arena_capacity = (int64_t)s->arena.capacity();
            s->st.small_used = s->small_used;
            s->st.small_peak = s->small_peak;
            s->st.small_capacity = s->cfg.small_budget_bytes;
        }
        if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

bool valid(const uint8_t *a, const uint8_t *b, int32_t n)
{
    if (!a || !b || n < 1 || n > SBFS_MAX_N) return false;
    for (int i = 0; i < n; ++i)
        if (a[i] >= n || b[i] >= n) return false;
    return true;
}

}  // namespace

extern "C" {

sbfs_status sbfs_server_config_default(sbfs_server_config *cfg)
{
    if (!cfg) return SBFS_EINVAL;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->device = -1;
    return SBFS_OK;
}

sbfs_status sbfs_server_start(const sbfs_server_config *cfg, sbfs_server **out)
{
    if (!out) return SBFS_EINVAL;
    *out = nullptr;
    sbfs_server *s = new (std::nothrow) sbfs_server();
    if (!s) return SBFS_ENOMEM;
    if (cfg) s->cfg = *cfg;
    else sbfs_server_config_default(&s->cfg);
    if (s->cfg.max_batch <= 0) s->cfg.max_batch = 8192;
    if (s->cfg.max_levels <= 0) s->cfg.max_levels = 16;
    if (s->cfg.queue_capacity <= 0) s->cfg.queue_capacity = 1 << 20;
    if (s->cfg.arena_bytes <= 0) s->cfg.arena_bytes = (int64_t)16 << 30;
    if (s->cfg.small_budget_bytes <= 0) s->cfg.small_budget_bytes = (int64_t)1 << 30;
    if (const char *inj = std::getenv("SBFS_SERVER_FAIL_BATCH")) s->inject_fail_batch = std::atoll(inj);
    sbfs_config hc;
    sbfs_config_default(&hc);
    hc.device = s->cfg.device;
    // small batches, then the level slots: stream priority in that order
    hc.streams = kSmallSlots + 1;
    sbfs_status st = sbfs_create(&hc, &s->h);
    if (st) {
        delete s;
        return st;
    }
    const size_t mb = (size_t)s->cfg.max_batch;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < kSmallSlots && e == cudaSuccess; ++i) {
        SmallSlot &S = s->small[i];
        S.lane = i;
        if ((e = S.d_recs.reserve(mb * 64)) || (e = S.d_ns.reserve(mb)) || (e = S.h_recs.reserve(mb * 64)) ||
            (e = S.h_ns.reserve(mb)) || (e = S.h_len.reserve(mb * 4)) || (e = S.h_words.reserve(mb * kWords * 8)) ||
            (e = S.h_flags.reserve(mb * 4)) || (e = S.h_err.reserve(sizeof(int))) ||
            (e = cudaHostGetDevicePointer((void **)&S.dl, S.h_len.ptr, 0)) ||
            (e = cudaHostGetDevicePointer((void **)&S.dw, S.h_words.ptr, 0)) ||
            (e = cudaHostGetDevicePointer((void **)&S.df, S.h_flags.ptr, 0)) ||
            (e = cudaEventCreateWithFlags(&S.ev, cudaEventDisableTiming)))
            break;
        std::memset(S.h_flags.ptr, 0, mb * 4);
    }
    if (e == cudaSuccess && (e = s->arena.reserve((size_t)s->cfg.arena_bytes)) == cudaSuccess)
        e = s->big.init(s->h->sm_count, 0, s->h->lanes[kSmallSlots].stream, &s->arena);
    if (e == cudaSuccess) e = prime_small(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        s->big.destroy();
        s->arena.release();
        for (SmallSlot &S : s->small) {
            if (S.ev) cudaEventDestroy(S.ev);
            for (DevBuf *d : {&S.d_recs, &S.d_ns}) d->release();
            for (HostBuf *b : {&S.h_recs, &S.h_ns, &S.h_len, &S.h_words, &S.h_flags, &S.h_err}) b->release();
        }
        sbfs_destroy(s->h);
        delete s;
        return e == cudaErrorMemoryAllocation ? SBFS_ENOMEM : SBFS_ECUDA;
    }
    s->t0 = std::chrono::steady_clock::now();
    s->loop = std::thread(run_loop, s);
    *out = s;
    return SBFS_OK;
}

sbfs_status sbfs_server_submit(sbfs_server *s, const uint8_t *a, const uint8_t *b, int32_t n, uint64_t *out_id)
{
    if (!s) return SBFS_EINVAL;
    if (!valid(a, b, n)) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->st.rejected++;
        return SBFS_EINVAL;
    }
    Request r;
    std::memset(&r, 0, sizeof(r));
    r.n = n;
    std::memcpy(r.a, a, (size_t)n);
    std::memcpy(r.b, b, (size_t)n);
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stopping) return SBFS_ESTOPPED;
        if (s->st.pending >= s->cfg.queue_capacity || (int64_t)s->incoming.size() >= s->cfg.queue_capacity) {
            s->st.rejected++;
            return SBFS_EBUSY;
        }
        r.id = s->next_id++;
        r.submit_ms = s->now_ms();
        s->incoming.push_back(r);
        s->st.submitted++;
    }
    s->cv_in.notify_one();
    if (out_id) *out_id = r.id;
    return SBFS_OK;
}

sbfs_status sbfs_server_submit_many(sbfs_server *s, const uint8_t *maps, int32_t lstride, const uint8_t *ns,
                                    int64_t count, uint64_t *out_ids)
{
    if (!s || count < 0 || lstride < 1 || lstride > 32 || (count > 0 && (!maps || !ns || !out_ids)))
        return SBFS_EINVAL;
    for (int64_t i = 0; i < count; ++i) {
        const uint8_t *rec = maps + (size_t)i * 2 * (size_t)lstride;
        if (ns[i] > lstride || !valid(rec, rec + lstride, ns[i])) {
            std::lock_guard<std::mutex> lock(s->mu);
            s->st.rejected += count;
            return SBFS_EINVAL;
        }
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stopping) return SBFS_ESTOPPED;
        if (s->st.pending + count > s->cfg.queue_capacity ||
            (int64_t)s->incoming.size() + count > s->cfg.queue_capacity) {
            s->st.rejected += count;
            return SBFS_EBUSY;
        }
        const double now = s->now_ms();
        for (int64_t i = 0; i < count; ++i) {
            const uint8_t *rec = maps + (size_t)i * 2 * (size_t)lstride;
            Request r;
            std::memset(&r, 0, sizeof(r));
            r.n = ns[i];
            std::memcpy(r.a, rec, (size_t)r.n);
            std::memcpy(r.b, rec + lstride, (size_t)r.n);
            r.id = s->next_id++;
            r.submit_ms = now;
            s->incoming.push_back(r);
            out_ids[i] = r.id;
        }
        s->st.submitted += count;
    }
    s->cv_in.notify_one();
    return SBFS_OK;
}

sbfs_status sbfs_server_poll(sbfs_server *s, sbfs_result *out, int32_t max, int32_t *got, int32_t timeout_ms)
{
    if (!s || !got || (max > 0 && !out)) return SBFS_EINVAL;
    *got = 0;
    std::unique_lock<std::mutex> lock(s->mu);
    if (s->ready.empty() && timeout_ms > 0)
        s->cv_out.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return !s->ready.empty(); });
    while (*got < max && !s->ready.empty()) {
        out[(*got)++] = s->ready.front();
        s->ready.pop_front();
    }
    return SBFS_OK;
}

sbfs_status sbfs_server_cancel(sbfs_server *s, uint64_t id)
{
    if (!s) return SBFS_EINVAL;
    std::lock_guard<std::mutex> lock(s->mu);
    for (const Request &r : s->incoming)
        if (r.id == id) {
            s->cancel_req.insert(id);
            return SBFS_OK;
        }
    return SBFS_ENOTFOUND;
}

sbfs_status sbfs_server_stats_get(sbfs_server *s, sbfs_server_stats *out)
{
    if (!s || !out) return SBFS_EINVAL;
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->st;
    out->now_ms = s->now_ms();
    return SBFS_OK;
}

sbfs_status sbfs_server_reset_peak(sbfs_server *s)
{
    if (!s) return SBFS_EINVAL;
    std::lock_guard<std::mutex> lock(s->mu);
    s->reset_peak = true;   // the loop thread owns the arena
    return SBFS_OK;
}

sbfs_status sbfs_server_stop(sbfs_server *s)
{
    if (!s) return SBFS_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
    }
    s->cv_in.notify_all();
    if (s->loop.joinable()) s->loop.join();
    cudaSetDevice(s->h->device);
    for (size_t i = 1; i < s->h->lanes.size(); ++i) cudaStreamSynchronize(s->h->lanes[i].stream);
    cudaStreamSynchronize(s->h->lanes[0].stream);
    s->big.destroy();
    s->arena.release();
    for (SmallSlot &S : s->small) {
        if (S.ev) cudaEventDestroy(S.ev);
        for (DevBuf *d : {&S.d_recs, &S.d_ns}) d->release();
        for (HostBuf *b : {&S.h_recs, &S.h_ns, &S.h_len, &S.h_words, &S.h_flags, &S.h_err}) b->release();
    }
    sbfs_destroy(s->h);
    delete s;
    return SBFS_OK;
}

}  // extern "C"
