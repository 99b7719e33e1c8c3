// server.cu -- the serving loop: continuous batching of single-automaton
// requests with admission by device-memory budget.
//
// One loop thread owns the GPU work; submit/poll/cancel only touch queues
// under a mutex.  Each turn of the loop:
//   * takes newly submitted requests;
//   * small requests (n <= 16): when the previous mini-batch is done, packs up
//     to max_batch of them into pinned 64-byte records, copies them in, runs
//     the batch kernels (per-lane / warp-pooled) on its own stream and copies
//     lengths and words back; a mini-batch completes in one launch sequence;
//   * large requests (n >= 17): when the previous level launch batch is done,
//     collects finished slots, admits waiting requests in arrival order while
//     their bitmap + queue fit the arena (the 2^n-bit budget), and launches
//     the next few levels of every admitted request (k_level.cu).  Requests
//     that arrive while others are running are admitted at the next turn and
//     advance together with them: their work overlaps on the device.
// Completion order follows the GPU, not submission order.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <unordered_set>

#include "runtime.cuh"

using namespace sbfs;

namespace {

struct Request {
    uint64_t id;
    int32_t n;
    uint8_t a[32], b[32];
    double submit_ms;
};

constexpr int kSmallMaxN = 16;
constexpr int kWords = 12;

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
    std::deque<Request> pend_small, pend_large;
    std::vector<Request> small_batch;
    bool small_busy = false;
    cudaEvent_t small_ev = nullptr;
    DevBuf d_recs, d_ns, d_len, d_words;
    HostBuf h_recs, h_ns, h_len, h_words;
    LevelEngine level;
    std::unordered_map<long long, Request> large;   // admitted, keyed by id
    std::string error;

    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

void complete(sbfs_server *s, const Request &r, int32_t status, int32_t len, const uint64_t *word)
{
    sbfs_result res;
    std::memset(&res, 0, sizeof(res));
    res.id = r.id;
    res.status = status;
    res.len = len;
    res.n = r.n;
    if (word) std::memcpy(res.word, word, sizeof(res.word));
    res.submit_ms = r.submit_ms;
    res.done_ms = s->now_ms();
    std::lock_guard<std::mutex> lock(s->mu);
    s->ready.push_back(res);
    s->st.completed++;
    if (status == SBFS_ECANCELED) s->st.cancelled++;
    s->cv_out.notify_all();
}

bool launch_small(sbfs_server *s)
{
    Lane &L = s->h->lanes[0];
    const int cap = s->cfg.max_batch;
    s->small_batch.clear();
    while (!s->pend_small.empty() && (int)s->small_batch.size() < cap) {
        s->small_batch.push_back(s->pend_small.front());
        s->pend_small.pop_front();
    }
    const int64_t cnt = (int64_t)s->small_batch.size();
    if (!cnt) return false;
    uint8_t *rec = s->h_recs.as<uint8_t>();
    uint8_t *ns = s->h_ns.as<uint8_t>();
    int max_n = 1;
    for (int64_t i = 0; i < cnt; ++i) {
        const Request &r = s->small_batch[(size_t)i];
        std::memset(rec + i * 64, 0, 64);
        std::memcpy(rec + i * 64, r.a, (size_t)r.n);
        std::memcpy(rec + i * 64 + 32, r.b, (size_t)r.n);
        ns[i] = (uint8_t)r.n;
        max_n = std::max(max_n, r.n);
    }
    cudaStream_t st = L.stream;
    cudaMemcpyAsync(s->d_recs.ptr, rec, (size_t)cnt * 64, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->d_ns.ptr, ns, (size_t)cnt, cudaMemcpyHostToDevice, st);
    int launches = 0;
    sbfs_status e = engine_enqueue(s->h, L, s->d_recs.as<uint8_t>(), 32, s->d_ns.as<uint8_t>(), 0, max_n, cnt,
                                   s->d_len.as<int32_t>(), s->d_words.as<uint64_t>(), kWords, &launches);
    if (e != SBFS_OK) {
        s->error = s->h->last_error;
        for (const Request &r : s->small_batch) complete(s, r, e, -1, nullptr);
        s->small_batch.clear();
        return false;
    }
    cudaMemcpyAsync(s->h_len.ptr, s->d_len.ptr, (size_t)cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s->h_words.ptr, s->d_words.ptr, (size_t)cnt * kWords * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                    st);
    cudaEventRecord(s->small_ev, st);
    s->small_busy = true;
    std::lock_guard<std::mutex> lock(s->mu);
    s->st.small_batches++;
    return true;
}

void finish_small(sbfs_server *s)
{
    const int32_t *len = s->h_len.as<int32_t>();
    const uint64_t *words = s->h_words.as<uint64_t>();
    for (size_t i = 0; i < s->small_batch.size(); ++i)
        complete(s, s->small_batch[i], SBFS_OK, len[i], words + i * kWords);
    s->small_batch.clear();
    s->small_busy = false;
}

bool event_done(cudaEvent_t ev)
{
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        return false;
    }
    return true;
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
            if (s->incoming.empty() && s->pend_small.empty() && s->pend_large.empty() && !s->small_busy &&
                s->large.empty()) {
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
                (r.n <= kSmallMaxN ? s->pend_small : s->pend_large).push_back(r);
                progress = true;
            }
        }
        // small path
        if (s->small_busy && event_done(s->small_ev)) {
            finish_small(s);
            progress = true;
        }
        if (!s->small_busy && !s->pend_small.empty()) progress |= launch_small(s);
        // large path
        if (s->level.launched() && s->level.ready()) {
            fin.clear();
            s->level.collect(fin);
            for (auto &f : fin) {
                auto it = s->large.find(f.tag);
                if (it == s->large.end()) continue;
                complete(s, it->second, f.state == kSlotDone ? SBFS_OK : SBFS_ECUDA, f.len, f.word);
                s->large.erase(it);
            }
            progress = true;
        }
        if (!s->level.launched()) {
            while (!s->pend_large.empty()) {
                const Request &r = s->pend_large.front();
                if (s->level.admit(nullptr, 32, r.n, (long long)r.id, r.a, r.b) < 0) break;
                s->large.emplace((long long)r.id, r);
                s->pend_large.pop_front();
            }
            if (s->level.in_flight() > 0) {
                s->level.launch(s->cfg.max_levels, none, 4 * s->cfg.max_levels);
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.level_launches += s->cfg.max_levels;
                progress = true;
            }
        }
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (s->reset_peak) {
                s->level.reset_peak();
                s->reset_peak = false;
            }
            s->st.pending = (int64_t)(s->incoming.size() + s->pend_small.size() + s->pend_large.size());
            s->st.in_flight = (int64_t)(s->small_batch.size() + s->large.size());
            s->st.arena_used = (int64_t)s->level.arena_used();
            s->st.arena_peak = (int64_t)s->level.arena_peak();
            s->st.arena_capacity = (int64_t)s->level.arena_capacity();
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
    sbfs_config hc;
    sbfs_config_default(&hc);
    hc.device = s->cfg.device;
    hc.streams = 2;
    sbfs_status st = sbfs_create(&hc, &s->h);
    if (st) {
        delete s;
        return st;
    }
    const size_t mb = (size_t)s->cfg.max_batch;
    cudaError_t e = cudaSuccess;
    if ((e = s->d_recs.reserve(mb * 64)) || (e = s->d_ns.reserve(mb)) || (e = s->d_len.reserve(mb * 4)) ||
        (e = s->d_words.reserve(mb * kWords * 8)) || (e = s->h_recs.reserve(mb * 64)) || (e = s->h_ns.reserve(mb)) ||
        (e = s->h_len.reserve(mb * 4)) || (e = s->h_words.reserve(mb * kWords * 8)) ||
        (e = cudaEventCreateWithFlags(&s->small_ev, cudaEventDisableTiming)) ||
        (e = s->level.init(s->h->sm_count, (size_t)s->cfg.arena_bytes, s->h->lanes[1].stream))) {
        cudaGetLastError();
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
    if (s->h->lanes.size() > 1) cudaStreamSynchronize(s->h->lanes[1].stream);
    s->level.destroy();
    if (s->small_ev) cudaEventDestroy(s->small_ev);
    for (DevBuf *d : {&s->d_recs, &s->d_ns, &s->d_len, &s->d_words}) d->release();
    for (HostBuf *b : {&s->h_recs, &s->h_ns, &s->h_len, &s->h_words}) b->release();
    sbfs_destroy(s->h);
    delete s;
    return SBFS_OK;
}

}  // extern "C"
