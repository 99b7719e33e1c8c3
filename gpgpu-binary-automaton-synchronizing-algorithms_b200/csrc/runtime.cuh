// runtime.cuh -- host-side engine behind the C ABI: handle state, device
// buffers, per-class launch planning.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "classes.cuh"
#include "common.cuh"
#include "copy_pool.hpp"
#include "level.cuh"
#include "sbfs.h"

namespace sbfs {

// Counters one launch sequence reads and writes on the device.
struct DevCounters {
    unsigned long long ticket[kNumClasses + 1];   // per-class work tickets (last one spare)
    unsigned long long first_violation;
    unsigned long long expanded;
    // per-lane kernels of classes 0 and 1: automata appended to the class's
    // escalation list, and claims on it
    unsigned long long escal_count[2];
    unsigned long long escal_claim[2];
    // classes 0..3 (pooled warps, hash-set warps): automata handed to the
    // CTA-wide kernel, as {offset 0, count} work ranges, and that kernel's tickets
    unsigned long long heavy_range[4][2];
    unsigned long long heavy_ticket[4];
    // class 3's sorted hand-offs as two work ranges (n = top, n < top) and the
    // second launch's tickets
    unsigned long long heavy_split[4][4];
    unsigned long long heavy_ticket2[4];
    int error;
    int pad;
    unsigned long long synchronizing;             // lengths >= 0 written by this job
};

// Grow-only device allocation.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t want);
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Grow-only pinned host allocation.
struct HostBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t want);
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// The streamed host path (uniform n <= 14 on the per-lane kernels): records go
// in chunk by chunk on the handle's copy-in stream while one kernel runs, and
// each chunk's results come back on copy_out as soon as the kernel flags it.
struct Streamer {
    cudaStream_t copy_out = nullptr;
    cudaEvent_t ev_in0 = nullptr, ev_kdone = nullptr;
    DevBuf flags;        // chunk_ready[nch] | chunk_done[nch]
    DevBuf escal_out;    // EscalResult per escalation slot
    HostBuf h_flags;     // host_flag[nch] | zeros[nch] | ones[nch] (mapped)
    HostBuf h_escal;     // escal_out copied back
    std::vector<cudaEvent_t> ev_out;   // chunk c's results are in pinned staging (pageable callers)
};

// Parameters of the one-automaton-per-lane kernel (classes 0 and 1).
struct LaneShape {
    int nmax;       // 8 or 12
    int warps;      // warps per CTA
    int ring;       // on-chip frontier ring entries per lane (power of two)
    int refill_k;   // idle lanes that trigger a refill pass
    int tail_k;     // at most this many searching lanes after the last refill: hand them to the warp
    int ctas;       // grid size (persistent)
};

// Parameters of the large-n kernels (classes 3 and 4).
struct CtaShape {
    int threads;    // threads per CTA
    int ctas;       // grid size (persistent)
};

// One stream with everything one in-flight chunk needs.
struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_k0 = nullptr, ev_k1 = nullptr, ev_done = nullptr;
    cudaEvent_t ev_in = nullptr;               // this lane's records have arrived (host path)
    // a mixed batch's size classes 0..2 run on these, beside class 3 on `stream`
    // (their tails -- a Cerny C_16 or C_20 each -- then overlap instead of adding up)
    cudaStream_t aux[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[3] = {nullptr, nullptr, nullptr};
    DevBuf spill_c[3];                         // queue spill of a pooled class, one per class
    DevBuf heavy[4], heavy_queue[4];           // a class's long searches and their CTA queues
    DevBuf maps, ns, len, words, spill, order, counters, ranges, cta_queue, hbm_bitmap, hbm_queue,
        escal, tickets;
    LevelEngine level;                         // device-resident slots for n > 20
    bool level_ready = false;
    unsigned long long level_expanded = 0;     // subsets the level slots expanded for the current job
    HostBuf h_counters;                        // pinned copy of DevCounters
    HostBuf h_maps, h_ns, h_len, h_words;      // pinned staging for pageable callers
    // chunk bookkeeping
    bool busy = false;
    int64_t begin = 0, count = 0;
    bool staged_out = false;
    int32_t *user_len = nullptr;
    uint64_t *user_words = nullptr;
    int32_t word_stride = 0;
    // CUDA graphs of launch sequences already seen on this lane, keyed by their
    // pointers and sizes; `sig` is the lane's buffer addresses at capture time
    struct Graph {
        cudaGraphExec_t exec;
        uint64_t sig;
        int launches;
    };
    std::map<std::string, Graph> graphs;
    std::set<std::string> seen;
    uint64_t signature() const
    {
        uint64_t x = 1469598103934665603ull;
        for (const DevBuf *d : {&maps, &ns, &len, &words, &spill, &order, &counters, &ranges, &cta_queue, &escal,
                                &tickets, &spill_c[0], &spill_c[1], &spill_c[2], &heavy[0], &heavy[1], &heavy[2],
                                &heavy[3], &heavy_queue[0], &heavy_queue[1], &heavy_queue[2], &heavy_queue[3]})
            x = (x ^ reinterpret_cast<uint64_t>(d->ptr)) * 1099511628211ull;
        for (const HostBuf *b : {&h_counters, &h_maps, &h_ns, &h_len, &h_words})
            x = (x ^ reinterpret_cast<uint64_t>(b->ptr)) * 1099511628211ull;
        return x;
    }
    void drop_graphs()
    {
        for (auto &g : graphs) cudaGraphExecDestroy(g.second.exec);
        graphs.clear();
        seen.clear();
    }
};

struct Plan {
    LaneShape lane[2];
    // a uniform batch of n = 13 (in class 2, whose kernels take 13..16) on the
    // per-lane kernel k_lane<13> instead of the class's warp-per-automaton
    // kernel; 0 = off
    LaneShape lane13;
    int use_lane13;
    LaneShape lane14;    // the same for a uniform batch of n = 14
    int use_lane14;
    PoolShape pool[3];
    CtaShape cta;
    CtaShape hbm;
    int use_pool[2];     // classes 0, 1: 1 = warp-pooled kernel instead of one automaton per lane
    int class3_level;    // class 3: 1 = bitmaps in HBM (level slots) instead of shared memory (k_cta)
    // classes 2 and 3 (class 3 in shared memory): hash-set warps first, k_cta for
    // their hand-offs, with 1 = 2048 or 2 = 4096 hash slots per warp; 0 = the
    // pooled kernel (class 2) or k_cta alone (class 3)
    int class2_hash;
    int class3_hash;
    int tuned;           // 1 when the autotuner (or its cache) chose the shapes
};

}  // namespace sbfs

struct sbfs_handle;

namespace sbfs {
// With done_flag, d_len / d_words may be mapped host memory: every automaton's
// result is stored there and then flagged (done_flag[i] = done_tag) as soon as
// it is known, before the launch sequence as a whole completes.
sbfs_status engine_enqueue(sbfs_handle *h, Lane &L, const uint8_t *d_maps, int32_t lstride, const uint8_t *d_ns,
                           int32_t n_uniform, int32_t max_n, int64_t count, int32_t *d_len, uint64_t *d_words,
                           int32_t word_stride, int *launches, unsigned int *done_flag = nullptr,
                           unsigned int done_tag = 0);
}  // namespace sbfs

struct sbfs_handle {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    sbfs_config cfg{};
    std::string last_error;
    std::mutex mu;
    std::vector<sbfs::Lane> lanes;
    // host path: every chunk's records go host->device on this one stream, in
    // chunk order, so the first chunk's kernels start after one chunk's copy
    // rather than after all lanes' copies have shared the link
    cudaStream_t copy_in = nullptr;
    sbfs::Streamer streamer;
    sbfs::Plan plan{};
    bool plan_ready = false;
    // last sbfs_solve_batch_device call: lane 0's buffers are in use until ev_device
    cudaEvent_t ev_device = nullptr;
    bool device_pending = false;
    int64_t device_count = 0;
    int device_launches = 0;
    cudaEvent_t ev_dk0 = nullptr, ev_dk1 = nullptr;
    // host-side fault injection for tests (environment SBFS_TEST_SKIP_CHUNK_READY=c
    // at sbfs_create): the next streamed call never sets chunk c's ready flag,
    // so the kernel's bounded wait for it runs out; then the hook is cleared
    int64_t skip_ready_chunk = -1;
    // host threads for the staging copies of pageable callers (created on first use)
    std::unique_ptr<sbfs::CopyPool> pool;
    sbfs::CopyPool &copy_pool()
    {
        if (!pool) pool.reset(new (std::nothrow) sbfs::CopyPool(sbfs::CopyPool::default_workers()));
        if (!pool) {
            static sbfs::CopyPool inline_only(0);   // no memory for a pool: copy on the calling thread
            return inline_only;
        }
        return *pool;
    }
};
