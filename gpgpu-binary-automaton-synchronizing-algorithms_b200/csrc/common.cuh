// common.cuh -- shared definitions of the sbfs CUDA kernels and host code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sbfs.h"

namespace sbfs {

constexpr unsigned kFull = 0xFFFFFFFFu;

// Length codes written to out_len besides real lengths.
constexpr int32_t kLenNonSync = -1;   // queue emptied without a singleton
constexpr int32_t kLenInvalid = -2;   // malformed record (state >= n); host turns into EINVAL

// Device error bits (one int per launch set, read back by the host).
constexpr int kErrInvalid = 1;        // malformed automaton seen
constexpr int kErrCapacity = 2;       // a queue or frontier exceeded its reserved space
constexpr int kErrWait = 4;           // a bounded wait for streamed input ran out
constexpr int kErrBounds = 8;         // a checked build's index check failed (the access was skipped)

// Checked builds (-DSBFS_CHECKED, libsbfs_checked.so): an index that comes
// from data (an image, a queue position, a list slot) is checked before the
// access; a failed check records kErrBounds in the launch's error word, which
// the host reports as SBFS_ECUDA, and the access is skipped -- no fault, no
// trap.  In the regular build the check compiles to nothing.
#ifdef SBFS_CHECKED
#define SBFS_CHECK(cond, err) ((cond) || (atomicOr((err), kErrBounds), false))
#else
#define SBFS_CHECK(cond, err) true
#endif

// Everything a BFS kernel needs to know about the batch.
struct Batch {
    const uint8_t *maps;        // records, 2*lstride bytes each
    int32_t lstride;
    const uint8_t *ns;          // per-automaton n or nullptr
    int32_t n_uniform;
    const int32_t *order;       // indices of the automata this launch handles, or nullptr = 0..count-1
    int64_t count;              // entries in order (or automata when order == nullptr)
    // When set, range_dev[0] is an offset into order and range_dev[1] the count
    // (a size class produced on the device by the bucketing kernels).
    const unsigned long long *range_dev;
    int32_t *out_len;           // nullable (pure Verify)
    uint64_t *out_words;        // nullable
    int32_t word_stride;
    int32_t slack;
    unsigned long long *first_violation;   // atomicMin target, starts at ULLONG_MAX
    unsigned long long *expanded;          // stats counter (nullable)
    int *error;                            // error bits
    // Per-automaton completion (serving): after an automaton's length and
    // word are stored, done_flag[k] = done_tag (nonzero, new per launch).
    // out_len / out_words may then be mapped host memory the host reads as
    // soon as the flag appears.  nullptr = no flags.
    unsigned int *done_flag;
    unsigned int done_tag;
};

__device__ __forceinline__ int automaton_n(const Batch &b, int64_t k)
{
    return b.ns ? (int)b.ns[k] : b.n_uniform;
}

// Resolves the launch's work list: count and the base of the order array.
__device__ __forceinline__ void resolve_work(const Batch &b, int64_t &count, const int32_t *&order)
{
    if (b.range_dev) {
        order = b.order + b.range_dev[0];
        count = (int64_t)b.range_dev[1];
    } else {
        order = b.order;
        count = b.count;
    }
}

__device__ __forceinline__ int64_t automaton_at(const int32_t *order, int64_t pos)
{
    return order ? (int64_t)order[pos] : pos;
}

__device__ __forceinline__ int cerny_bound(int n, int slack)
{
    return (n - 1) * (n - 1) - slack;
}

__device__ __forceinline__ bool is_singleton(uint32_t s)
{
    return (s & (s - 1u)) == 0u;
}

// Called once the automaton's length and word are stored.
__device__ __forceinline__ void publish_result(const Batch &b, int64_t k)
{
    if (b.done_flag) {
        __threadfence_system();
        *(volatile unsigned int *)(b.done_flag + k) = b.done_tag;
    }
}

__device__ __forceinline__ void record_result(const Batch &b, int64_t k, int n, int32_t len)
{
    if (b.out_len) b.out_len[k] = len;
    if (len > cerny_bound(n, b.slack))
        atomicMin(b.first_violation, (unsigned long long)k);
}

// Host-side launch helpers implemented in the kernel translation units.
struct PoolShape {
    int nmax;          // size class bound: 8, 12 or 16
    int slots;         // automata in flight per warp
    int warps;         // warps per CTA
    int queue_smem;    // on-chip queue entries per automaton
    int ctas;          // grid size (persistent)
    int grab = 16;     // automata a warp claims per work-ticket atomic
};

size_t pool_smem_bytes(const PoolShape &s);
size_t pool_spill_words(const PoolShape &s);   // uint32 spill words for the whole grid
// Optional hand-off of long searches: a slot that reaches level_cap levels is
// abandoned and its automaton appended to list (count = entries appended), to
// be solved by a kernel with more threads per automaton.  list == nullptr = off.
struct PoolHeavy {
    int level_cap;
    int32_t *list;
    unsigned long long *count;
};
cudaError_t launch_pool(const PoolShape &s, const Batch &b, uint32_t *spill,
                        unsigned long long *ticket, cudaStream_t st, const PoolHeavy &heavy = PoolHeavy{0, nullptr,
                                                                                                        nullptr});
int pool_max_ctas_per_sm(const PoolShape &s);

size_t lane_smem_bytes(int nmax, int warps, int ring);
int lane_max_ctas_per_sm(int nmax, int warps, int ring);
// Streaming form of the per-lane kernel (host path, uniform batch in
// order): records arrive chunk by chunk while the kernel runs, and results
// leave chunk by chunk.  All pointers null = everything resident, no tracking.
struct EscalResult {
    int64_t k;          // automaton
    int32_t len;
    int32_t pad;
    uint64_t word[3];   // n <= 13: at most 144 letters
};
struct LaneStream {
    const unsigned int *chunk_ready;   // nonzero once chunk c's records are on the device
    unsigned int *chunk_done;          // lane outcomes recorded per chunk (starts at 0)
    unsigned int *host_flag;           // mapped host memory: 1 once chunk c's outcomes are all written
    int64_t chunk;                     // automata per chunk after the first (whole 128-byte lines of records)
    EscalResult *escal_out;            // by escalation slot: results the whole-warp search writes
    int wait_polls;                    // bounded wait for a chunk's records: polls before giving up
    // automata in chunk 0, at most `chunk`: a short first copy lets the kernel
    // start sooner (whole 128-byte lines of records too)
    int64_t first;

    __host__ __device__ int64_t chunk_of(int64_t k) const { return k < first ? 0 : 1 + (k - first) / chunk; }
    __host__ __device__ int64_t chunk_begin(int64_t c) const { return c == 0 ? 0 : first + (c - 1) * chunk; }
    // chunks of a batch of `count` automata, and the size of chunk c
    __host__ __device__ int64_t chunks(int64_t count) const
    {
        return count <= first ? 1 : 1 + (count - first + chunk - 1) / chunk;
    }
    __host__ __device__ int64_t chunk_size(int64_t c, int64_t count) const
    {
        const int64_t a = chunk_begin(c), e = chunk_begin(c + 1);
        return (e < count ? e : count) - a;
    }
};

// Stores the first *count escalated results into device-accessible (e.g.
// mapped host) len / words (either may be null).
cudaError_t launch_escal_patch(const EscalResult *r, const unsigned long long *count, int32_t *len, uint64_t *words,
                               int ws, int sm_count, cudaStream_t st);

// escal_list holds escal_capacity entries (>= the automata of the launch), all
// -1; escal_count and escal_claim start at 0.
// tail_k: once the batch is handed out, lanes of a warp with at most tail_k
// lanes still searching give their automata to the whole-warp search (0 = off).
cudaError_t launch_lane(int nmax, int warps, int ring, int refill_k, int tail_k, int ctas, const Batch &b,
                        int32_t *escal_list, unsigned long long escal_capacity, unsigned long long *escal_count,
                        unsigned long long *escal_claim, unsigned long long *ticket, const LaneStream &ls,
                        cudaStream_t st);

}  // namespace sbfs
