// level_host.cu -- host engine of the device-resident level slots (k_level.cu):
// a first-fit arena for bitmaps and queues, admission into free slots, level
// launches and collection of finished automata.
#include <climits>
#include <cstring>

#include "level.cuh"

namespace sbfs {

cudaError_t Arena::reserve(size_t bytes)
{
    if (bytes <= cap_ && base_) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&base_, bytes);
    if (e != cudaSuccess) {
        base_ = nullptr;
        cudaGetLastError();
        return e;
    }
    cap_ = bytes;
    used_ = peak_ = 0;
    free_.clear();
    busy_.clear();
    free_[0] = bytes;
    return cudaSuccess;
}

void Arena::release()
{
    if (base_) cudaFree(base_);
    base_ = nullptr;
    cap_ = used_ = peak_ = 0;
    free_.clear();
    busy_.clear();
}

size_t Arena::alloc(size_t bytes)
{
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second >= bytes) {
            const size_t off = it->first, rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[off + bytes] = rest;
            busy_[off] = bytes;
            used_ += bytes;
            if (used_ > peak_) peak_ = used_;
            return off;
        }
    }
    return SIZE_MAX;
}

void Arena::free(size_t off)
{
    auto it = busy_.find(off);
    if (it == busy_.end()) return;
    size_t start = off, size = it->second;
    used_ -= size;
    busy_.erase(it);
    auto next = free_.lower_bound(start);
    if (next != free_.end() && next->first == start + size) {
        size += next->second;
        next = free_.erase(next);
    }
    if (next != free_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == start) {
            start = prev->first;
            size += prev->second;
            free_.erase(prev);
        }
    }
    free_[start] = size;
}

size_t LevelEngine::footprint(int n)
{
    const size_t bitmap = n >= 7 ? ((size_t)1 << n) / 8 : 16;
    const size_t queue = ((size_t)1 << n) * sizeof(uint64_t);
    return ((bitmap + 255) & ~size_t(255)) + ((queue + 255) & ~size_t(255));
}

cudaError_t LevelEngine::init(int sm_count, size_t arena_bytes, cudaStream_t st, Arena *shared)
{
    st_ = st;
    shared_ = shared;
    cudaError_t e;
    const int per_sm = level_max_ctas_per_sm();
    ctas_ = (per_sm > 0 ? per_sm : 1) * sm_count;
    if ((e = cudaMalloc(&d_slots_, sizeof(LevelSlot) * kMaxLevelSlots)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&d_tables_, sizeof(uint64_t) * kLevelTable * kMaxLevelSlots)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&d_ctl_, sizeof(LevelCtl))) != cudaSuccess) return e;
    if ((e = cudaHostAlloc(&h_slots_, sizeof(LevelSlot) * kMaxLevelSlots, cudaHostAllocDefault)) != cudaSuccess)
        return e;
    if ((e = cudaHostAlloc(&h_ctl_, sizeof(LevelCtl), cudaHostAllocDefault)) != cudaSuccess) return e;
    if ((e = cudaHostAlloc(&h_init_, sizeof(int) * (2 + kMaxLevelSlots), cudaHostAllocDefault)) != cudaSuccess)
        return e;
    if ((e = cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming)) != cudaSuccess) return e;
    std::memset(h_slots_, 0, sizeof(LevelSlot) * kMaxLevelSlots);
    std::memset(h_ctl_, 0, sizeof(LevelCtl));
    if ((e = cudaMemcpyAsync(d_slots_, h_slots_, sizeof(LevelSlot) * kMaxLevelSlots, cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(d_ctl_, h_ctl_, sizeof(LevelCtl), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    slot_off_.assign(kMaxLevelSlots, SIZE_MAX);
    nslots_ = 0;
    in_flight_ = 0;
    parity_ = 0;
    return shared_ ? cudaSuccess : own_.reserve(arena_bytes);
}

void LevelEngine::destroy()
{
    if (st_) cudaStreamSynchronize(st_);
    if (d_slots_) cudaFree(d_slots_);
    if (d_tables_) cudaFree(d_tables_);
    if (d_ctl_) cudaFree(d_ctl_);
    if (h_slots_) cudaFreeHost(h_slots_);
    if (h_ctl_) cudaFreeHost(h_ctl_);
    if (h_init_) cudaFreeHost(h_init_);
    if (ev_) cudaEventDestroy(ev_);
    own_.release();
    d_slots_ = nullptr;
    d_tables_ = nullptr;
    d_ctl_ = nullptr;
    h_slots_ = nullptr;
    h_ctl_ = nullptr;
    h_init_ = nullptr;
    ev_ = nullptr;
}

int LevelEngine::admit(const uint8_t *d_rec, int lstride, int n, long long tag, const uint8_t *host_a,
                       const uint8_t *host_b)
{
    int s = -1;
    for (int i = 0; i < kMaxLevelSlots; ++i)
        if (slot_off_[i] == SIZE_MAX) {
            s = i;
            break;
        }
    if (s < 0) return -1;
    const size_t fp = footprint(n);
    const size_t off = arena().alloc(fp);
    if (off == SIZE_MAX) return -1;
    slot_off_[s] = off;
    LevelSlot &sl = h_slots_[s];
    std::memset(&sl, 0, sizeof(sl));
    const size_t bitmap = ((n >= 7 ? ((size_t)1 << n) / 8 : 16) + 255) & ~size_t(255);
    sl.rec = d_rec;
    sl.bitmap = reinterpret_cast<uint32_t *>(arena().base() + off);
    sl.queue = reinterpret_cast<uint64_t *>(arena().base() + off + bitmap);
    sl.cap = (unsigned long long)1 << n;
    sl.tag = tag;
    sl.n = n;
    sl.lstride = lstride;
    sl.state = kSlotInit;
    for (int j = 0; j < n && j < 32; ++j) {
        sl.a[j] = host_a ? host_a[j] : 0;
        sl.b[j] = host_b ? host_b[j] : 0;
    }
    sl.found = ~0ull;
    pending_init_.push_back(s);
    if (s + 1 > nslots_) nslots_ = s + 1;
    ++in_flight_;
    return s;
}

cudaError_t LevelEngine::launch(int levels, const Batch &out, int narrow_levels)
{
    cudaError_t e;
    // the last copied control block holds the totals the next launch will read
    const bool narrow = narrow_levels > 0 && pending_init_.empty() && launches_ > 0 &&
                        h_ctl_->total[parity_ & 1] <= kNarrowLevel;
    // admissions: descriptors of the new slots, then the control block's init list
    for (int s : pending_init_) {
        if ((e = cudaMemcpyAsync(d_slots_ + s, h_slots_ + s, sizeof(LevelSlot), cudaMemcpyHostToDevice, st_)) !=
            cudaSuccess)
            return e;
    }
    // nslots, this launch parity's n_init and init_list are host-owned
    const int par = (int)(parity_ & 1);
    h_init_[0] = nslots_;
    h_init_[1] = (int)pending_init_.size();
    for (size_t i = 0; i < pending_init_.size(); ++i) h_init_[2 + i] = pending_init_[i];
    const int n_init = (int)pending_init_.size();
    pending_init_.clear();
    if ((e = cudaMemcpyAsync(&d_ctl_->nslots, h_init_, sizeof(int), cudaMemcpyHostToDevice, st_)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(&d_ctl_->n_init[par], h_init_ + 1, sizeof(int), cudaMemcpyHostToDevice, st_)) !=
        cudaSuccess)
        return e;
    if (n_init && (e = cudaMemcpyAsync(d_ctl_->init_list, h_init_ + 2, sizeof(int) * n_init,
                                       cudaMemcpyHostToDevice, st_)) != cudaSuccess)
        return e;
    if (narrow) {
        if ((e = launch_level_narrow((int)(parity_ & 1), narrow_levels, kNarrowLevel, d_slots_, d_tables_, d_ctl_, out,
                                     st_)) != cudaSuccess)
            return e;
        ++parity_;
        ++launches_;
    } else {
        for (int i = 0; i < levels; ++i) {
            if ((e = launch_level(ctas_, (int)(parity_ & 1), d_slots_, d_tables_, d_ctl_, out, st_)) != cudaSuccess)
                return e;
            ++parity_;
            ++launches_;
        }
    }
    if ((e = cudaMemcpyAsync(h_slots_, d_slots_, sizeof(LevelSlot) * (size_t)nslots_, cudaMemcpyDeviceToHost,
                             st_)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(h_ctl_, d_ctl_, sizeof(LevelCtl), cudaMemcpyDeviceToHost, st_)) != cudaSuccess)
        return e;
    if ((e = cudaEventRecord(ev_, st_)) != cudaSuccess) return e;
    launched_ = true;
    return cudaSuccess;
}

cudaError_t LevelEngine::collect(std::vector<Finished> &done)
{
    if (!launched_) return cudaSuccess;
    cudaError_t e = cudaEventSynchronize(ev_);
    if (e != cudaSuccess) return e;
    launched_ = false;
    expanded_ = h_ctl_->expanded;
    for (int s = 0; s < nslots_; ++s) {
        LevelSlot &sl = h_slots_[s];
        if (slot_off_[s] == SIZE_MAX) continue;
        if (sl.state == kSlotDone || sl.state == kSlotFail) {
            Finished f;
            f.tag = sl.tag;
            f.len = sl.result_len;
            f.state = sl.state;
            std::memcpy(f.word, sl.word, sizeof(f.word));
            done.push_back(f);
            arena().free(slot_off_[s]);
            slot_off_[s] = SIZE_MAX;
            sl.state = kSlotFree;   // the device copy stays Done, which the kernel ignores
            --in_flight_;
        }
    }
    while (nslots_ > 0 && slot_off_[nslots_ - 1] == SIZE_MAX) --nslots_;
    return cudaGetLastError();
}

}  // namespace sbfs
