// copy_pool.hpp -- host threads that split the copies between a caller's
// pageable buffers and the handle's pinned staging.
//
// Pageable memory cannot be read by the copy engine, so records and results of
// a caller that did not pin its buffers pass through pinned staging, and that
// host-side copy sets the end-to-end time: one thread copies about 11 GB/s,
// while four to sixteen threads copy 55-80 GB/s (measured on the B200 hosts),
// more than the PCIe link carries in one direction.  The pool cuts each copy
// into slices for its workers; the thread that waits for a group of copies
// runs queued slices itself instead of sleeping.
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

namespace sbfs {

class CopyPool {
public:
    // Copies submitted under one group; wait() returns once all of them are done.
    struct Group {
        std::atomic<long> left{0};
    };

    // Starts up to `workers` threads; fewer if the system refuses more (the
    // waiting thread does the rest of the work, so none is needed).
    explicit CopyPool(int workers)
    {
        try {
            for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { loop(); });
        } catch (...) {
        }
    }

    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : threads_) t.join();
    }

    CopyPool(const CopyPool &) = delete;
    CopyPool &operator=(const CopyPool &) = delete;

    // Worker count for this host: half its hardware threads, at most eight
    // (the copy rate stops growing well before that).
    static int default_workers()
    {
        const unsigned hw = std::thread::hardware_concurrency();
        return (int)std::min(8u, hw / 2);
    }

    // Queues the copy of n bytes from src to dst, in slices of at least
    // kMinSlice bytes (one per worker and the waiting thread at most).
    void copy(void *dst, const void *src, size_t n, Group &g)
    {
        if (n == 0) return;
        const size_t most = threads_.size() + 1;
        const size_t parts = std::max<size_t>(1, std::min(most, n / kMinSlice));
        if (parts == 1 || threads_.empty()) {
            std::memcpy(dst, src, n);
            return;
        }
        // slices on 64-byte boundaries (cache lines), the last one takes the rest;
        // a slice that cannot be queued (no memory) is copied here instead
        const size_t per = ((n / parts) + 63) & ~size_t(63);
        size_t a = 0;
        try {
            std::lock_guard<std::mutex> lk(mu_);
            for (size_t p = 0; p < parts && a < n; ++p) {
                const size_t len = p + 1 == parts ? n - a : std::min(per, n - a);
                Task t;
                t.dst = static_cast<char *>(dst) + a;
                t.src = static_cast<const char *>(src) + a;
                t.n = len;
                t.g = &g;
                tasks_.push_back(t);
                g.left.fetch_add(1, std::memory_order_relaxed);
                a += len;
            }
        } catch (...) {
        }
        cv_.notify_all();
        if (a < n) std::memcpy(static_cast<char *>(dst) + a, static_cast<const char *>(src) + a, n - a);
    }

    // Runs f(begin, end) over [0, n) in parts of at least `grain` items, on the
    // workers and this thread; returns when every part is done.
    template <class F>
    void parallel_for(size_t n, size_t grain, F &&f)
    {
        if (n == 0) return;
        const size_t parts = std::max<size_t>(1, std::min(threads_.size() + 1, n / std::max<size_t>(grain, 1)));
        if (parts == 1) {
            f(size_t(0), n);
            return;
        }
        using Fn = typename std::remove_reference<F>::type;
        void (*call)(void *, size_t, size_t) = [](void *ctx, size_t a, size_t b) { (*static_cast<Fn *>(ctx))(a, b); };
        Group g;
        size_t p = 0;
        try {
            std::lock_guard<std::mutex> lk(mu_);
            for (; p < parts; ++p) {
                Task t;
                t.call = call;
                t.ctx = const_cast<void *>(static_cast<const void *>(&f));
                t.a = n * p / parts;
                t.b = n * (p + 1) / parts;
                t.g = &g;
                tasks_.push_back(t);
                g.left.fetch_add(1, std::memory_order_relaxed);
            }
        } catch (...) {
        }
        cv_.notify_all();
        if (p < parts) f(n * p / parts, n);   // parts that could not be queued
        wait(g);
    }

    // Waits for a group when it goes out of scope, early returns included, so
    // that no queued slice outlives the group it counts down (null: nothing).
    struct Scope {
        CopyPool *pool;
        Group &g;
        ~Scope()
        {
            if (pool) pool->wait(g);
        }
    };

    // Returns once every copy of the group is done, running queued slices
    // (of any group) on this thread meanwhile.
    void wait(Group &g)
    {
        while (g.left.load(std::memory_order_acquire) > 0) {
            Task t;
            if (try_pop(t))
                run(t);
            else
                std::this_thread::yield();
        }
    }

private:
    static constexpr size_t kMinSlice = 256u << 10;

    // a slice of a copy, or (call set) a part [a, b) of a parallel_for
    struct Task {
        char *dst = nullptr;
        const char *src = nullptr;
        size_t n = 0;
        Group *g = nullptr;
        void (*call)(void *, size_t, size_t) = nullptr;
        void *ctx = nullptr;
        size_t a = 0, b = 0;
    };

    static void run(const Task &t)
    {
        if (t.call)
            t.call(t.ctx, t.a, t.b);
        else
            std::memcpy(t.dst, t.src, t.n);
        t.g->left.fetch_sub(1, std::memory_order_acq_rel);
    }

    bool try_pop(Task &t)
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (tasks_.empty()) return false;
        t = tasks_.front();
        tasks_.pop_front();
        return true;
    }

    void loop()
    {
        while (true) {
            Task t;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return stop_ || !tasks_.empty(); });
                if (tasks_.empty()) return;   // stop_ with nothing left
                t = tasks_.front();
                tasks_.pop_front();
            }
            run(t);
        }
    }

    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Task> tasks_;
    std::vector<std::thread> threads_;
    bool stop_ = false;
};

}  // namespace sbfs
