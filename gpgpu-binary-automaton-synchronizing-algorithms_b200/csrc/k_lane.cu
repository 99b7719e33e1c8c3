// k_lane.cu -- power-set BFS with one automaton per lane (n <= 14).
//
// Each lane runs the sequential BFS of GPGPU/CPU/SlimCPU4bits.cs:214-306 on its
// own automaton: pop subsets, look up both images in its nibble table
// (entry = a-image << 16 | b-image, SlimCPU4bits.cs:122-206), test-and-set them
// in its visited bitmap, append the new ones, advance the level when the
// current level is used up (SlimCPUUntweaked.cs:126-130,160-164), stop at the
// first singleton generated (:151-155).  All 32 lanes of a warp do this in
// lockstep on 32 different automata.
//
// Shared memory is lane-interleaved: element e of lane l's bitmap, table and
// queue lives at [e][l], so every lane-private access of a warp touches 32
// different banks.  The queue is a ring of R entries holding only the live
// frontier (current level remainder + next level); with words requested each
// entry carries the letters of the word that reaches it (bit NMAX + d =
// letter d, 1 = b), so a word needs no parent pointers or retained history.
//
// Each iteration a lane takes up to kStep (4) subsets of its current level and
// looks up their eight images: more independent work per step hides the
// shared-memory latencies that one warp's dependent chain exposes at 7 warps
// per SM (2 -> 4 subsets: 0.64 -> 0.56 ms per 10^6 automata at n = 12; 6 and 8
// were slower again).  A singleton among them ends the search (no singleton
// is visited before the first one is generated, so it needs no bitmap test).
// Otherwise the eight images are test-and-set with shared-memory atomicOr, issued
// back to back and kept in program order by the hardware for a repeated
// address, and the fresh ones are appended in queue order (first subset's a, b,
// then the second's), as the sequential loop would.
//
// Two rare cases leave the per-lane search: a frontier wider than R, and (with
// words) a word longer than 32 - NMAX letters.  Such an automaton is abandoned
// and appended to the launch's escalation list.  So is, once the batch is
// handed out, the work of a warp with at most `tail_k` lanes still searching.
// A warp that has no lane work left (no new automata, every lane idle) owns
// its whole shared-memory region again and takes escalated automata from that
// list one at a time, solving each with all 32 lanes: a level-synchronous
// search over a linear queue that holds every subset at most once (2^n
// entries, so it cannot overflow), with parent pointers for the word, the
// nibble table in registers read by warp shuffles, and a linear bitmap updated
// with shared-memory atomics.  Claims never wait (see claim_escalated): every
// escalated automaton is solved in the launch that escalated it.
//
// Lanes that finish wait until `refill_k` lanes of the warp are idle; then the
// warp writes their results and loads new automata for all of them in one
// pass, so the per-automaton set-up (record load, table build, bitmap clear)
// runs with many lanes active instead of one.
//
// Instances: NMAX = 8 and 12 for size classes 0 and 1; 13 and 14 for uniform
// batches of that n (a fourth nibble chunk, 1 or 2 KB of bitmap per lane, and
// words of up to (NMAX - 1)^2 = 144 or 169 letters -- three 64-bit words -- in
// the whole-warp search).
#include "common.cuh"

namespace sbfs {
namespace {

constexpr int kActive = 0, kDone = 1, kEscalate = 2, kIdle = 3, kHeld = 4;
constexpr int kStep = 4;   // subsets a lane expands per step (their 2 * kStep images are tested together)
// At n = 13 and 14 fewer warps fit on an SM (four, two), and six subsets per
// step hide more of each warp's latency: 2^21 automata at n = 14 4.83 -> 4.64 ms,
// the n = 13 streamed kernel 2.19 -> 2.09 ms (eight: no better than six)
constexpr int kStepWide = 6;

__host__ __device__ constexpr int low_bit4(int v)
{
    return (v & 1) ? 0 : (v & 2) ? 1 : (v & 4) ? 2 : 3;
}

template <int NMAX>
struct LaneGeom {
    static constexpr int kBitmapWords = (1 << NMAX) / 32;
    static constexpr int kChunks = (NMAX + 3) / 4;
    static constexpr int kTable = kChunks * 16;
    static constexpr uint32_t kMask = (1u << NMAX) - 1u;
    static constexpr int kWordMax = 32 - NMAX;   // letters an entry can carry
    static constexpr int kWordU64 = ((NMAX - 1) * (NMAX - 1) + 63) / 64;   // words of the whole-warp search
};

template <int NMAX>
__device__ __forceinline__ uint32_t lane_image(const uint32_t *tb, uint32_t x)
{
    uint32_t t = tb[(x & 15u) * 32];
    if (LaneGeom<NMAX>::kChunks > 1) t |= tb[(16 + ((x >> 4) & 15u)) * 32];
    if (LaneGeom<NMAX>::kChunks > 2) t |= tb[(32 + ((x >> 8) & 15u)) * 32];
    if (LaneGeom<NMAX>::kChunks > 3) t |= tb[(48 + ((x >> 12) & 15u)) * 32];
    return t;
}

// Nibble-table entry v of chunk c (a-image << 16 | b-image of the states
// 4c + i for the set bits i of v), read from the record.
template <int NMAX>
__device__ __forceinline__ uint32_t table_entry(const uint8_t *rec, int lstride, int n, int c, int v)
{
    uint32_t t = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int st = 4 * c + i;
        if (((v >> i) & 1) && st < n)
            t |= (1u << (__ldg(rec + st) + 16)) | (1u << __ldg(rec + lstride + st));
    }
    return t;
}

// Claims the next escalated automaton of the launch for a warp with no lane
// work left, or returns -1.  A claim is one atomicAdd on the claim counter and
// one atomicCAS on the claimed slot, raced against the slot's writer (which
// stores with atomicCAS too): if the slot is still empty the claimer marks it
// abandoned (-2) and stops, and the writer, finding it abandoned, keeps the
// automaton and solves it itself once it runs out of lane work.  Nothing ever
// waits for another warp.
__device__ int64_t claim_escalated(int32_t *list, unsigned long long capacity, unsigned long long *claim,
                                   unsigned long long &slot)
{
    slot = atomicAdd(claim, 1ull);
    if (slot >= capacity) return -1;
    const int32_t prev = atomicCAS(list + slot, -1, -2);
    return prev >= 0 ? (int64_t)prev : -1;
}

// Waits (bounded: `polls` polls about 0.2 us apart) until the streamed records
// of chunk c are on the device; false when the wait ran out.
__device__ bool wait_chunk(const unsigned int *ready, int64_t c, int polls)
{
    for (int it = 0; it < polls; ++it) {
        if (*(volatile const unsigned int *)(ready + c)) {
            __threadfence();
            return true;
        }
        __nanosleep(200);
    }
    return false;
}

// One automaton (n <= NMAX) solved by the whole warp inside its region of
// `region_words` shared words (>= 2^NMAX / 32 + 2^NMAX).  Queue entry:
// subset | parent index << NMAX | letter << 2*NMAX (letter 1 = b).
template <int NMAX, bool WORDS, bool STREAM>
__device__ void warp_solve(const Batch &b, int64_t k, uint32_t *region, int lane, unsigned long long &expanded,
                           const LaneStream &ls, unsigned long long slot)
{
    using G = LaneGeom<NMAX>;
    constexpr int BW = G::kBitmapWords;
    uint32_t *bm = region;        // linear bitmap
    uint32_t *q = region + BW;    // linear queue, 2^NMAX entries
    const int n = automaton_n(b, k);
    const uint8_t *rec = b.maps + (size_t)k * 2u * (size_t)b.lstride;
    // chunks 0 and 1 in lanes 0-15 / 16-31 of t01, chunk 2 (and 3) likewise in t23
    const uint32_t t01 = table_entry<NMAX>(rec, b.lstride, n, lane >> 4, lane & 15);
    const uint32_t t23 = G::kChunks > 3   ? table_entry<NMAX>(rec, b.lstride, n, 2 + (lane >> 4), lane & 15)
                         : G::kChunks > 2 ? table_entry<NMAX>(rec, b.lstride, n, 2, lane & 15)
                                          : 0u;
    for (int w = lane; w < BW; w += 32) bm[w] = 0u;
    __syncwarp();
    const uint32_t full = (1u << n) - 1u;
    if (lane == 0) {
        bm[full >> 5] = 1u << (full & 31u);
        q[0] = full;
    }
    __syncwarp();
    // n = 1: the visited root is the only singleton (see the per-lane set-up)
    uint32_t head = 0, lvl_end = n > 1 ? 1u : 0u, tail = lvl_end, level = 0;
    int32_t len = kLenNonSync;
    uint32_t found = 0, found_letter = 0;
    while (true) {
        const uint32_t idx = head + (uint32_t)lane;
        const bool has = idx < lvl_end;
        const uint32_t x = has ? (q[idx] & G::kMask) : 0u;
        uint32_t t = __shfl_sync(kFull, t01, (int)(x & 15u)) | __shfl_sync(kFull, t01, 16 + (int)((x >> 4) & 15u));
        if (G::kChunks > 2) t |= __shfl_sync(kFull, t23, (int)((x >> 8) & 15u));
        if (G::kChunks > 3) t |= __shfl_sync(kFull, t23, 16 + (int)((x >> 12) & 15u));
        const uint32_t ya = t >> 16, yb = t & 0xFFFFu;
        expanded += has ? 1u : 0u;
        const bool sa = has && is_singleton(ya), sb = has && is_singleton(yb);
        const unsigned smask = __ballot_sync(kFull, sa || sb);
        if (smask) {
            // the first singleton in queue order (lowest lane, a before b)
            const int fl = __ffs(smask) - 1;
            found = head + (uint32_t)fl;
            found_letter = (uint32_t)__shfl_sync(kFull, sa ? 0 : 1, fl);
            len = (int32_t)level + 1;
            break;
        }
        bool fa = false, fb = false;
        if (has && SBFS_CHECK((ya >> 5) < (uint32_t)BW && (yb >> 5) < (uint32_t)BW, b.error)) {
            fa = !(atomicOr(&bm[ya >> 5], 1u << (ya & 31u)) & (1u << (ya & 31u)));
            fb = !(atomicOr(&bm[yb >> 5], 1u << (yb & 31u)) & (1u << (yb & 31u)));
        }
        const unsigned ma = __ballot_sync(kFull, fa), mb = __ballot_sync(kFull, fb);
        const unsigned lt = (1u << lane) - 1u;
        uint32_t pos = tail + (uint32_t)(__popc(ma & lt) + __popc(mb & lt));
        const uint32_t par = idx << NMAX;
        // every subset enters the queue at most once: 2^NMAX entries never overflow
        if (fa && SBFS_CHECK(pos < (1u << NMAX), b.error)) q[pos] = ya | par;
        pos += fa ? 1u : 0u;
        if (fb && SBFS_CHECK(pos < (1u << NMAX), b.error)) q[pos] = yb | par | (1u << (2 * NMAX));
        tail += (uint32_t)(__popc(ma) + __popc(mb));
        head = min(head + 32u, lvl_end);
        __syncwarp();
        if (head == lvl_end) {
            if (tail == lvl_end) break;   // no new subset: not synchronizing
            lvl_end = tail;
            ++level;
        }
    }
    if (lane == 0) {
        record_result(b, k, n, len);
        // at most (NMAX - 1)^2 letters: 2 words at n = 12, 3 at n = 13
        static_assert(G::kWordU64 <= 3, "words of at most 192 letters");
        uint64_t w0 = 0, w1 = 0, w2 = 0;
        if (WORDS) {
            // letters from the root: entry at depth d + 1 holds letter d
            if (len > 0) {
                auto set = [&](uint32_t d) {
                    if (d < 64) w0 |= 1ull << d;
                    else if (d < 128) w1 |= 1ull << (d - 64);
                    else if (G::kWordU64 > 2) w2 |= 1ull << (d - 128);
                };
                if (found_letter) set(level);
                uint32_t i = found;
                for (int d = (int)level - 1; d >= 0; --d) {
                    const uint32_t e = q[i];
                    if ((e >> (2 * NMAX)) & 1u) set((uint32_t)d);
                    i = (e >> NMAX) & G::kMask;
                }
            }
            uint64_t *w = b.out_words + (size_t)k * (size_t)b.word_stride;
            w[0] = w0;
            if (b.word_stride > 1) w[1] = w1;
            if (G::kWordU64 > 2) {
                if (b.word_stride > 2) w[2] = w2;
                for (int c = 3; c < b.word_stride; ++c) w[c] = 0ull;
            } else {
                for (int c = 2; c < b.word_stride; ++c) w[c] = 0ull;
            }
        }
        if (STREAM && ls.escal_out) {
            // streamed batches: the host patches escalated automata from here
            EscalResult r;
            r.k = k;
            r.len = len;
            r.pad = 0;
            r.word[0] = w0;
            r.word[1] = w1;
            r.word[2] = w2;
            ls.escal_out[slot] = r;
        }
        publish_result(b, k);
    }
    __syncwarp();
}

template <int NMAX, bool WORDS, bool STREAM>
__global__ void __launch_bounds__(256) k_lane(Batch b, int ring, int refill_k, int tail_k, int32_t *escal_list,
                                              unsigned long long escal_capacity, unsigned long long *escal_count,
                                              unsigned long long *escal_claim, unsigned long long *ticket,
                                              LaneStream ls)
{
    using G = LaneGeom<NMAX>;
    constexpr int BW = G::kBitmapWords;
    constexpr int T = G::kTable;
    extern __shared__ __align__(16) uint32_t smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    uint32_t *base = smem + (size_t)warp * (BW + T + ring) * 32;
    uint32_t *bm = base + lane;                  // bm[w * 32]
    uint32_t *tb = base + BW * 32 + lane;        // tb[e * 32]
    uint32_t *rq = base + (BW + T) * 32 + lane;  // rq[i * 32]
    const uint32_t rmask = (uint32_t)ring - 1u;

    int64_t count;
    const int32_t *order;
    resolve_work(b, count, order);

    int state = kIdle;
    int64_t k = -1;
    int n = 0;
    uint32_t head = 0, tail = 0, lvl_end = 0, level = 0;
    int32_t res_len = kLenNonSync;
    uint32_t res_word = 0;
    bool more = true;
    unsigned long long expanded = 0;
    unsigned long long hslot = 0;   // escalation slot of a held automaton
    int64_t ready_upto = -1;        // streamed chunks known to be on the device

    while (true) {
        // ---- phase: finish waiting lanes, load new automata -----------------
        // no new automata: once at most `tail_k` lanes still search, the warp
        // hands their automata to the whole-warp search instead of finishing
        // them at a few lanes' pace (the launch's tail)
        if (!more && tail_k > 0) {
            const unsigned active = __ballot_sync(kFull, state == kActive);
            if (state == kActive && __popc(active) <= tail_k) state = kEscalate;
        }
        const unsigned not_active = __ballot_sync(kFull, state != kActive);
        if (not_active == kFull ||
            (__popc(not_active) >= refill_k && (more || __any_sync(kFull, state == kDone || state == kEscalate)))) {
            const bool outcome = state == kDone || state == kEscalate;
            if (state == kDone) {
                record_result(b, k, n, res_len);
                if (WORDS) {
                    uint64_t *w = b.out_words + (size_t)k * (size_t)b.word_stride;
                    w[0] = res_len > 0 ? (uint64_t)res_word : 0ull;
                    for (int c = 1; c < b.word_stride; ++c) w[c] = 0ull;
                }
                publish_result(b, k);
            }
            const unsigned esc = __ballot_sync(kFull, state == kEscalate);
            if (esc) {
                unsigned long long pos = 0;
                const int leader = __ffs(esc) - 1;
                if (lane == leader) pos = atomicAdd(escal_count, (unsigned long long)__popc(esc));
                pos = __shfl_sync(kFull, pos, leader);
                if (state == kEscalate) {
                    // a slot a drained warp already gave up on: solve this one ourselves later
                    const unsigned long long slot = pos + __popc(esc & ((1u << lane) - 1u));
                    const int32_t prev = SBFS_CHECK(slot < escal_capacity, b.error)
                                             ? atomicCAS(escal_list + slot, -1, (int32_t)k)
                                             : -2;
                    state = prev == -1 ? kIdle : kHeld;
                    hslot = slot;
                }
            }
            if (STREAM) {
                // streamed batch: count outcomes per chunk; whoever completes a
                // chunk tells the host its lengths and words can be copied out
                const unsigned om = __ballot_sync(kFull, outcome);
                if (outcome) {
                    __threadfence();   // this lane's results before its count
                    const int64_t c = ls.chunk_of(k);
                    const unsigned grp = __match_any_sync(om, (unsigned long long)c);
                    if (lane == __ffs(grp) - 1) {
                        const unsigned add = (unsigned)__popc(grp);
                        const unsigned old = atomicAdd(ls.chunk_done + c, add);
                        const int64_t size = ls.chunk_size(c, count);
                        if ((int64_t)(old + add) == size) {
                            __threadfence_system();
                            *(volatile unsigned int *)(ls.host_flag + c) = 1u;
                        }
                    }
                }
            }
            if (state != kActive && state != kHeld) state = kIdle;
            const unsigned idle = __ballot_sync(kFull, state == kIdle);
            if (more && idle) {
                unsigned long long got = 0;
                const int leader = __ffs(idle) - 1;
                if (lane == leader) got = atomicAdd(ticket, (unsigned long long)__popc(idle));
                got = __shfl_sync(kFull, got, leader);
                if (got + __popc(idle) >= (unsigned long long)count) more = false;
                if (STREAM && got < (unsigned long long)count) {
                    // streamed batch: the records handed out must have arrived
                    const int64_t last = (int64_t)min(got + (unsigned long long)__popc(idle),
                                                      (unsigned long long)count) - 1;
                    const int64_t c_last = ls.chunk_of(last);
                    if (c_last > ready_upto) {
                        bool ok = true;
                        if (lane == 0) ok = wait_chunk(ls.chunk_ready, c_last, ls.wait_polls);
                        ok = __shfl_sync(kFull, ok, 0);
                        if (!ok && lane == 0) atomicOr(b.error, kErrWait);
                        ready_upto = c_last;
                        __syncwarp();
                    }
                }
                if (state == kIdle) {
                    const unsigned long long pos = got + __popc(idle & ((1u << lane) - 1u));
                    if (pos < (unsigned long long)count) {
                        k = automaton_at(order, (int64_t)pos);
                        n = automaton_n(b, k);
                        state = kActive;
                    }
                }
                // every lane that just received an automaton sets it up
                if (state == kActive && (idle & (1u << lane))) {
                    bool bad = (n < 1 || n > NMAX || n > b.lstride);
                    const uint8_t *rec = b.maps + (size_t)k * 2u * (size_t)b.lstride;
                    uint32_t aw[G::kChunks] = {}, bw[G::kChunks] = {};
                    if (!bad) {
                        if ((b.lstride & 3) == 0) {
                            const uint32_t *ra = reinterpret_cast<const uint32_t *>(rec);
                            const uint32_t *rb = reinterpret_cast<const uint32_t *>(rec + b.lstride);
#pragma unroll
                            for (int c = 0; c < G::kChunks; ++c) {
                                aw[c] = 4 * c < n ? __ldg(ra + c) : 0u;
                                bw[c] = 4 * c < n ? __ldg(rb + c) : 0u;
                            }
                        } else {
#pragma unroll
                            for (int c = 0; c < G::kChunks; ++c) {
#pragma unroll
                                for (int j = 0; j < 4; ++j) {
                                    if (4 * c + j < n) {
                                        aw[c] |= (uint32_t)__ldg(rec + 4 * c + j) << (8 * j);
                                        bw[c] |= (uint32_t)__ldg(rec + b.lstride + 4 * c + j) << (8 * j);
                                    }
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int c = 0; c < G::kChunks; ++c) {
                        uint32_t s[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int st = 4 * c + j;
                            const uint32_t av = (aw[c] >> (8 * j)) & 0xFFu, bv = (bw[c] >> (8 * j)) & 0xFFu;
                            const bool in = !bad && st < n;
                            if (in && (av >= (uint32_t)n || bv >= (uint32_t)n)) bad = true;
                            s[j] = in ? ((1u << ((av & 15u) + 16)) | (1u << (bv & 15u))) : 0u;
                        }
                        // table[c*16 + v] = OR of s[j] over the set bits j of v
                        uint32_t t[16];
                        t[0] = 0u;
#pragma unroll
                        for (int v = 1; v < 16; ++v) t[v] = t[v & (v - 1)] | s[low_bit4(v)];
#pragma unroll
                        for (int v = 0; v < 16; ++v) tb[(c * 16 + v) * 32] = t[v];
                    }
                    if (bad) {
                        // written (and counted) at the next refill pass
                        atomicOr(b.error, kErrInvalid);
                        state = kDone;
                        res_len = kLenInvalid;
                        res_word = 0;
                    } else if (n == 1) {
                        // the root is the only singleton and it is visited, so the
                        // search never generates a new one: not synchronizing, as in
                        // GPGPU/CPU/SlimCPUUntweaked.cs:149-157 (and the singleton-first
                        // test below, which relies on no singleton being visited, is
                        // never reached)
                        state = kDone;
                        res_len = kLenNonSync;
                        res_word = 0;
                    } else {
#pragma unroll 16
                        for (int w = 0; w < BW; ++w) bm[w * 32] = 0u;
                        const uint32_t full = (1u << n) - 1u;
                        bm[(full >> 5) * 32] = 1u << (full & 31u);
                        rq[0] = full;
                        head = 0;
                        tail = 1;
                        lvl_end = 1;
                        level = 0;
                    }
                }
            }
            if (__ballot_sync(kFull, state == kActive) == 0u) {
                // no lane is searching: the region is free for whole-warp searches,
                // first of the automata this warp kept
                for (unsigned held = __ballot_sync(kFull, state == kHeld); held; held &= held - 1u) {
                    const int64_t e = __shfl_sync(kFull, k, __ffs(held) - 1);
                    const unsigned long long slot = __shfl_sync(kFull, hslot, __ffs(held) - 1);
                    warp_solve<NMAX, WORDS, STREAM>(b, e, base, lane, expanded, ls, slot);
                }
                if (state == kHeld) state = kIdle;
                if (!more) {
                    // an outcome decided during set-up (n = 1, a malformed record) is
                    // written by the next refill pass: take that pass before leaving
                    if (__any_sync(kFull, state == kDone || state == kEscalate)) continue;
                    // no new automata either: solve escalated ones while any can be claimed
                    while (true) {
                        int64_t e = -1;
                        unsigned long long slot = 0;
                        if (lane == 0) e = claim_escalated(escal_list, escal_capacity, escal_claim, slot);
                        e = __shfl_sync(kFull, e, 0);
                        slot = __shfl_sync(kFull, slot, 0);
                        if (e < 0) break;
                        warp_solve<NMAX, WORDS, STREAM>(b, e, base, lane, expanded, ls, slot);
                    }
                    break;
                }
                continue;
            }
        }

        // ---- up to kStep expansions per active lane ----------------------------
        if (state == kActive) {
            // a lane with fewer than kStep subsets left in the level expands its
            // first one again in the spare places: those copies' images are
            // already visited by the time they are tested
            constexpr int P = NMAX >= 13 ? kStepWide : kStep;
            const uint32_t take = min(lvl_end - head, (uint32_t)P);
            uint32_t e[P];
#pragma unroll
            for (int i = 0; i < P; ++i)
                e[i] = (i == 0 || (uint32_t)i < take) ? rq[((head + (uint32_t)i) & rmask) * 32] : e[0];
            head += take;
            expanded += take;
            uint32_t y[2 * P], hi[2 * P];
            // entries carry the word that reaches them: the parent's letters,
            // plus letter `level` = b for the b-images (an entry holds 32 - NMAX
            // letters; at level >= 32 - NMAX a fresh image escalates instead)
            const uint32_t lb = (WORDS && level < (uint32_t)G::kWordMax) ? 1u << (level + NMAX) : 0u;
#pragma unroll
            for (int i = 0; i < P; ++i) {
                const uint32_t t = lane_image<NMAX>(tb, e[i] & G::kMask);
                y[2 * i] = t >> 16;
                y[2 * i + 1] = t & 0xFFFFu;
                hi[2 * i] = WORDS ? (e[i] & ~G::kMask) : 0u;
                hi[2 * i + 1] = WORDS ? ((e[i] & ~G::kMask) | lb) : 0u;
            }
            // no singleton is ever visited (the search stops at the first one), so
            // a singleton image ends the search without a bitmap test
            int sc = -1;
#pragma unroll
            for (int c = 2 * P - 1; c >= 0; --c)
                if (is_singleton(y[c])) sc = c;
            if (sc >= 0) {
                state = kDone;
                res_len = (int32_t)level + 1;
                uint32_t es = e[0];
#pragma unroll
                for (int i = 1; i < P; ++i)
                    if ((sc >> 1) == i) es = e[i];
                res_word = WORDS ? ((es >> NMAX) | ((uint32_t)(sc & 1) << level)) : 0u;
            } else {
                // test-and-set in queue order: a subset met twice in this step is
                // fresh only the first time (same-address atomics keep program order)
                uint32_t old[2 * P];
#pragma unroll
                for (int c = 0; c < 2 * P; ++c)
                    old[c] = SBFS_CHECK((y[c] >> 5) < (uint32_t)BW, b.error)
                                 ? atomicOr(&bm[(y[c] >> 5) * 32], 1u << (y[c] & 31u))
                                 : ~0u;
                bool any = false;
#pragma unroll
                for (int c = 0; c < 2 * P; ++c) {
                    if (!(old[c] & (1u << (y[c] & 31u)))) {
                        rq[(tail & rmask) * 32] = y[c] | hi[c];
                        ++tail;
                        any = true;
                    }
                }
                // more live entries than ring slots (the oldest were overwritten), or
                // a word longer than an entry carries: the whole-warp search takes over
                if (tail - head > (uint32_t)ring || (WORDS && any && level >= (uint32_t)G::kWordMax)) {
                    state = kEscalate;
                } else if (head == lvl_end) {
                    if (tail == lvl_end) {
                        state = kDone;
                        res_len = kLenNonSync;
                    } else {
                        lvl_end = tail;
                        ++level;
                    }
                }
            }
        }
    }
    for (int o = 16; o; o >>= 1) expanded += __shfl_down_sync(kFull, expanded, o);
    if (lane == 0 && b.expanded) atomicAdd(b.expanded, expanded);
}

template <int NMAX>
size_t smem_for(int warps, int ring)
{
    using G = LaneGeom<NMAX>;
    return (size_t)warps * (G::kBitmapWords + G::kTable + ring) * 32 * sizeof(uint32_t);
}

template <int NMAX, bool WORDS>
cudaError_t launch_t(int warps, int ring, int refill_k, int tail_k, int ctas, const Batch &b, int32_t *escal_list,
                     unsigned long long escal_capacity, unsigned long long *escal_count,
                     unsigned long long *escal_claim, unsigned long long *ticket, const LaneStream &ls,
                     cudaStream_t st)
{
    using G = LaneGeom<NMAX>;
    // the warp-cooperative search needs the bitmap and 2^NMAX queue entries in one region
    if ((size_t)G::kBitmapWords + ((size_t)1 << NMAX) > (size_t)(G::kBitmapWords + G::kTable + ring) * 32)
        return cudaErrorInvalidValue;
    const size_t smem = smem_for<NMAX>(warps, ring);
    // the streamed form's bookkeeping is compiled out of the resident-batch kernel
    auto kernel = ls.chunk_done ? k_lane<NMAX, WORDS, true> : k_lane<NMAX, WORDS, false>;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kernel<<<ctas, warps * 32, smem, st>>>(b, ring, refill_k, tail_k, escal_list, escal_capacity, escal_count,
                                           escal_claim, ticket, ls);
    return cudaGetLastError();
}

}  // namespace

size_t lane_smem_bytes(int nmax, int warps, int ring)
{
    return nmax <= 8    ? smem_for<8>(warps, ring)
           : nmax <= 12 ? smem_for<12>(warps, ring)
           : nmax == 13 ? smem_for<13>(warps, ring)
                        : smem_for<14>(warps, ring);
}

int lane_max_ctas_per_sm(int nmax, int warps, int ring)
{
    if (nmax > 14) return 0;
    const void *k = nmax <= 8    ? (const void *)k_lane<8, true, false>
                    : nmax <= 12 ? (const void *)k_lane<12, true, false>
                    : nmax == 13 ? (const void *)k_lane<13, true, false>
                                 : (const void *)k_lane<14, true, false>;
    const size_t smem = lane_smem_bytes(nmax, warps, ring);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, warps * 32, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return blocks;
}

// Streamed batches: after the chunk copies, the escalated automata's results
// (solved late, after their chunk may already have been copied) are stored
// straight into the host's mapped output.
__global__ void k_escal_patch(const EscalResult *r, const unsigned long long *count, int32_t *len, uint64_t *words,
                              int ws)
{
    const int64_t n = (int64_t)*count;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const EscalResult e = r[i];
        if (len) len[e.k] = e.len;
        if (words) {
            uint64_t *w = words + (size_t)e.k * (size_t)ws;
            for (int j = 0; j < ws; ++j) w[j] = j < 3 ? e.word[j] : 0ull;
        }
    }
}

cudaError_t launch_escal_patch(const EscalResult *r, const unsigned long long *count, int32_t *len, uint64_t *words,
                               int ws, int sm_count, cudaStream_t st)
{
    k_escal_patch<<<2 * sm_count, 256, 0, st>>>(r, count, len, words, ws);
    return cudaGetLastError();
}

cudaError_t launch_lane(int nmax, int warps, int ring, int refill_k, int tail_k, int ctas, const Batch &b,
                        int32_t *escal_list, unsigned long long escal_capacity, unsigned long long *escal_count,
                        unsigned long long *escal_claim, unsigned long long *ticket, const LaneStream &ls,
                        cudaStream_t st)
{
    if ((ring & (ring - 1)) || ring < 8 || warps < 1 || warps > 8 || ctas < 1 || refill_k < 1 || refill_k > 32 ||
        tail_k < 0 || tail_k > 32)
        return cudaErrorInvalidValue;
    if (ls.chunk_done && (ls.chunk < 1 || ls.first < 1 || ls.first > ls.chunk || b.order || b.range_dev))
        return cudaErrorInvalidValue;
    const bool words = b.out_words != nullptr;
    if (nmax <= 8)
        return words ? launch_t<8, true>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                         escal_count, escal_claim, ticket, ls, st)
                     : launch_t<8, false>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                          escal_count, escal_claim, ticket, ls, st);
    if (nmax <= 12)
        return words ? launch_t<12, true>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                          escal_count, escal_claim, ticket, ls, st)
                     : launch_t<12, false>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                           escal_count, escal_claim, ticket, ls, st);
    if (nmax == 13)
        return words ? launch_t<13, true>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                          escal_count, escal_claim, ticket, ls, st)
                     : launch_t<13, false>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                           escal_count, escal_claim, ticket, ls, st);
    if (nmax == 14)
        return words ? launch_t<14, true>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                          escal_count, escal_claim, ticket, ls, st)
                     : launch_t<14, false>(warps, ring, refill_k, tail_k, ctas, b, escal_list, escal_capacity,
                                           escal_count, escal_claim, ticket, ls, st);
    return cudaErrorInvalidValue;
}

}  // namespace sbfs
