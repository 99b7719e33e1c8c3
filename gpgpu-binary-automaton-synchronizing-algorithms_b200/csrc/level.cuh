// level.cuh -- device-resident BFS slots for large automata (n <= 28) and the
// host engine that admits automata into them, launches levels and collects
// results.  Used by the batch path for n > 20 and by the serving loop.
#pragma once

#include <cstdint>
#include <map>
#include <vector>

#include <cuda_runtime.h>

#include "common.cuh"

namespace sbfs {

constexpr int kMaxLevelSlots = 256;
constexpr int kLevelTable = 4 * 256;          // byte tables, entry = a-image << 32 | b-image
constexpr int kLevelWordU64 = 12;             // 768 bits >= (28-1)^2
constexpr uint64_t kLevelSubsetMask = 0x0FFFFFFFull;

constexpr int kSlotFree = 0, kSlotInit = 1, kSlotRun = 2, kSlotDone = 3, kSlotFail = 4;

struct LevelSlot {
    // written by the host at admission
    const uint8_t *rec;          // device record: a[j] = rec[j], b[j] = rec[lstride + j]
    uint32_t *bitmap;            // 2^n bits, 16-byte aligned
    uint64_t *queue;             // cap entries
    unsigned long long cap;
    long long tag;               // caller's index (batch position or request id)
    int32_t n;
    int32_t lstride;
    int32_t state;               // kSlot*
    int32_t overflow;
    uint8_t a[32], b[32];        // copy of the maps, filled by the host for convenience
    // device-managed
    unsigned long long lvl_start, lvl_end, tail, level, found;
    int32_t result_len;
    int32_t pad;
    uint64_t word[kLevelWordU64];
};

// Control block.  Fields a launch reads at its start are double-buffered by
// launch parity: launch t reads [t & 1] and its last CTA writes [(t+1) & 1],
// so a CTA that starts late never sees the next level's values.
struct LevelCtl {
    unsigned int done_ctas;
    int nslots;                  // slot entries in use (highest index + 1), host-written per launch batch
    int n_init[2];               // freshly admitted slots to set up (host writes the batch's first parity)
    int running;
    unsigned int finished;       // slots that reached Done/Fail (monotone)
    unsigned int launches;
    int prefix_n[2];             // slots the prefix below was computed for
    unsigned long long total[2]; // items in the current levels of running slots
    unsigned long long expanded;
    unsigned long long prefix[2][kMaxLevelSlots + 1];
    int init_list[kMaxLevelSlots];
};

int level_max_ctas_per_sm();
cudaError_t launch_level(int ctas, int parity, LevelSlot *slots, uint64_t *tables, LevelCtl *ctl, const Batch &out,
                         cudaStream_t st);
cudaError_t launch_level_narrow(int parity, int max_levels, unsigned long long narrow, LevelSlot *slots,
                                uint64_t *tables, LevelCtl *ctl, const Batch &out, cudaStream_t st);

// Level totals at or below this are expanded by one cluster of CTAs looping
// over levels (k_level_narrow).  Raising it to 32768 or 65536 made C_28 slower
// (12.78 and 13.86 ms against 12.51): eight SMs take longer over those levels
// than the whole grid's launch costs.
constexpr unsigned long long kNarrowLevel = 16384;

// First-fit allocator over one device buffer (host-side bookkeeping only).
class Arena {
public:
    cudaError_t reserve(size_t bytes);
    void release();
    // returns offset or SIZE_MAX when nothing fits
    size_t alloc(size_t bytes);
    void free(size_t off);
    size_t capacity() const { return cap_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }
    void reset_peak() { peak_ = used_; }
    char *base() const { return base_; }

private:
    char *base_ = nullptr;
    size_t cap_ = 0, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;   // offset -> size
    std::map<size_t, size_t> busy_;
};

// Host engine of one set of level slots on one stream.
class LevelEngine {
public:
    // with `shared`, slots are carved from that arena (reserved by its owner,
    // possibly shared with other engines) and arena_bytes is ignored
    cudaError_t init(int sm_count, size_t arena_bytes, cudaStream_t st, Arena *shared = nullptr);
    void destroy();
    // bytes an automaton with n states needs (bitmap + full-size queue), 256-aligned
    static size_t footprint(int n);
    // admit one automaton whose record is at d_rec (device); returns slot or -1 (no slot/memory)
    int admit(const uint8_t *d_rec, int lstride, int n, long long tag, const uint8_t *host_a,
              const uint8_t *host_b);
    // upload admissions, launch `levels` level kernels -- or, when the current
    // levels are narrow and nothing awaits set-up, one launch of an 8-CTA
    // cluster that runs up to `narrow_levels` narrow levels -- then copy slot
    // states back
    // (async); results go to `out` when out.out_len is set (batch mode)
    cudaError_t launch(int levels, const Batch &out, int narrow_levels = 0);
    // wait for the last launch and collect finished slots (frees their memory)
    struct Finished {
        long long tag;
        int32_t len;
        int state;
        uint64_t word[kLevelWordU64];
    };
    cudaError_t collect(std::vector<Finished> &done);
    // true when the last launch has completed (collect will not block)
    bool ready() const
    {
        if (!launched_) return true;
        const cudaError_t e = cudaEventQuery(ev_);
        if (e == cudaErrorNotReady) {
            cudaGetLastError();
            return false;
        }
        return true;
    }
    bool launched() const { return launched_; }
    // subsets in the levels the next launch expands (as of the last collect)
    unsigned long long level_total() const { return h_ctl_ ? h_ctl_->total[parity_ & 1] : 0ull; }
    void reset_peak() { arena().reset_peak(); }
    int in_flight() const { return in_flight_; }
    size_t arena_used() const { return arena().used(); }
    size_t arena_peak() const { return arena().peak(); }
    size_t arena_capacity() const { return arena().capacity(); }
    unsigned long long expanded() const { return expanded_; }
    int launches() const { return launches_; }
    cudaStream_t stream() const { return st_; }

private:
    cudaStream_t st_ = nullptr;
    cudaEvent_t ev_ = nullptr;
    int ctas_ = 0;
    LevelSlot *d_slots_ = nullptr;
    uint64_t *d_tables_ = nullptr;
    LevelCtl *d_ctl_ = nullptr;
    LevelSlot *h_slots_ = nullptr;   // pinned mirror
    LevelCtl *h_ctl_ = nullptr;      // pinned mirror
    int *h_init_ = nullptr;          // pinned: nslots, n_init, init_list[]
    Arena own_;
    Arena *shared_ = nullptr;
    Arena &arena() { return shared_ ? *shared_ : own_; }
    const Arena &arena() const { return shared_ ? *shared_ : own_; }
    std::vector<size_t> slot_off_;   // arena offset per slot (SIZE_MAX = free)
    std::vector<int> pending_init_;
    int nslots_ = 0;
    int in_flight_ = 0;
    unsigned long long parity_ = 0;   // launches issued so far (their parity selects the control buffers)
    bool launched_ = false;
    unsigned long long expanded_ = 0;
    int launches_ = 0;
};

}  // namespace sbfs
