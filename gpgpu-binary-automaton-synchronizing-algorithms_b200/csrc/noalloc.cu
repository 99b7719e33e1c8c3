// noalloc.cu -- sbfs_solve_small_noalloc: the n <= 12 solver without any
// device allocation.
//
// Some callers cannot call cudaMalloc: a plugin inside a host process whose
// framework has already reserved the device memory budget (so a new
// allocation fails or evicts someone else's cache), or a latency-critical loop
// where cudaMalloc/cudaFree would synchronise the device and stall other
// streams.  For them this entry point runs the warp-pooled kernel (k_pool.cu)
// with all of its working memory -- the per-slot queue spill area and the
// work/result counters -- in one file-scope __device__ array of fixed size,
// kScratchBytes (16 MiB).  The caller passes only its inputs and outputs, in
// device memory.  Nothing here calls cudaMalloc, cudaFree or any allocating
// library routine.
//
// Limits and contract:
//  * 1 <= n <= 12 (the scratch is sized for 12-state automata: a slot's queue
//    never exceeds 2^12 entries); larger n is rejected with SBFS_EINVAL.
//  * The launch shape is fixed so that the spill area fits the array, which
//    makes this path slower than sbfs_solve_batch_device.
//  * Every call uses the same array; calls that overlap on the GPU race with
//    each other.  Serialise them (one stream, or events between streams).
//  * Every call looks up the array's device address on the current device
//    with cudaGetSymbolAddress (no allocation), so a new context after a
//    device reset gets the array's new address.  The first call on a device
//    may load the library's device code there; make it before any stream
//    capture begins.
//  * d_len is required: a malformed record (a state index >= n) is reported
//    only through its length, -2.

#include "common.cuh"

namespace sbfs {
namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;
constexpr size_t kHeaderBytes = 256;

struct NoAllocHeader {
    unsigned long long ticket;
    unsigned long long first_violation;
    unsigned long long expanded;
    int error;
};
static_assert(sizeof(NoAllocHeader) <= kHeaderBytes, "header");

// The working memory of every call (header, then the queue spill area).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Pooled-kernel shape: 4 automata per warp, 2 warps per CTA, 256 queue
// entries on chip; each slot spills at most 2^12 - 256 entries (15 KiB).
constexpr int kNmax = 12, kSlots = 4, kWarps = 2, kQueueSmem = 256;
constexpr size_t kSpillPerSlot = (size_t(1) << kNmax) - kQueueSmem;
constexpr int kCtas = (int)((kScratchBytes - kHeaderBytes) / (kSpillPerSlot * 4 * kSlots * kWarps));

__global__ void finalize(const NoAllocHeader *hdr, int64_t *out)
{
    *out = hdr->first_violation == ~0ull ? -1ll : (int64_t)hdr->first_violation;
}

// Device address of g_scratch in the current device's context.  In host code
// the name g_scratch is a host-side stand-in, not a device address; it is
// looked up on every call, so a context created after a device reset is
// served at the array's new address.
cudaError_t scratch_address(unsigned char **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char *>(p);
    return cudaSuccess;
}

}  // namespace
}  // namespace sbfs

extern "C" sbfs_status sbfs_solve_small_noalloc(const uint8_t *d_maps, int32_t lstride, int32_t n, int64_t count,
                                                int32_t *d_len, uint64_t *d_words, int32_t word_stride,
                                                int64_t *d_first_violation, void *stream)
{
    using namespace sbfs;
    if (n < 1 || n > kNmax) return SBFS_EINVAL;   // beyond what the static scratch holds
    if (lstride < n || lstride > 32 || count < 0 || (count > 0 && !d_maps) || !d_first_violation ||
        (count > 0 && !d_len))
        return SBFS_EINVAL;
    if (d_words && word_stride < 1) return SBFS_EINVAL;
    unsigned char *scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) {
        cudaGetLastError();
        return SBFS_ECUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NoAllocHeader *hdr = reinterpret_cast<NoAllocHeader *>(scratch);
    uint32_t *spill = reinterpret_cast<uint32_t *>(scratch + kHeaderBytes);
    // the array keeps the previous call's contents: reset the counters
    if (cudaMemsetAsync(hdr, 0, sizeof(NoAllocHeader), st) != cudaSuccess ||
        cudaMemsetAsync(&hdr->first_violation, 0xFF, sizeof(unsigned long long), st) != cudaSuccess) {
        cudaGetLastError();
        return SBFS_ECUDA;
    }
    Batch b{};
    b.maps = d_maps;
    b.lstride = lstride;
    b.ns = nullptr;
    b.n_uniform = n;
    b.order = nullptr;
    b.count = count;
    b.range_dev = nullptr;
    b.out_len = d_len;
    b.out_words = d_words;
    b.word_stride = d_words ? word_stride : 0;
    b.slack = 0;
    b.first_violation = &hdr->first_violation;
    b.expanded = &hdr->expanded;
    b.error = &hdr->error;
    PoolShape s{kNmax, kSlots, kWarps, kQueueSmem, kCtas};
    if (count > 0 && launch_pool(s, b, spill, &hdr->ticket, st) != cudaSuccess) {
        cudaGetLastError();
        return SBFS_ECUDA;
    }
    finalize<<<1, 1, 0, st>>>(hdr, d_first_violation);
    if (cudaGetLastError() != cudaSuccess) return SBFS_ECUDA;
    return SBFS_OK;
}
