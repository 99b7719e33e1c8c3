// dotnet_random.cu -- host-side generator of the reference's exact input
// batches.
//
// The reference draws its automata with .NET Framework's System.Random
// (SharedDefinitions/Problem.cs:32-58): FillArrayOfProblems seeds a master
// Random(seed) and gives each automaton its own Random(master.Next()), which
// draws A[i] then B[i] with Next(0, n) for i = 0..n-1.  System.Random is Knuth's
// subtractive generator (seeded through a 55-entry additive table, lag 21 in
// the .NET variant); this file restates that published algorithm so that the
// batches of GPGPU/Program.cs:94 (seed 1234567 + count) and of
// AlgorithmCorrectnessTestProject/IntegrityTest.cs:71-79 can be regenerated
// bit for bit.  Host code only.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "sbfs.h"

namespace {

// C# int arithmetic is unchecked: a difference that leaves the int32 range
// wraps (two's complement).  Seeds above 161803398 make the table's first
// entry negative and the stirring loop overflows, so the wrap is part of the
// generator's definition.
inline int32_t wrap_sub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }

class DotnetRandom {
public:
    explicit DotnetRandom(int32_t seed)
    {
        const int32_t kBig = 2147483647, kSeed = 161803398;
        const int32_t sub = seed == INT32_MIN ? kBig : (seed < 0 ? -seed : seed);
        int32_t mj = kSeed - sub;
        table_[55] = mj;
        int32_t mk = 1;
        for (int i = 1; i < 55; ++i) {
            const int ii = (21 * i) % 55;
            table_[ii] = mk;
            mk = wrap_sub(mj, mk);
            if (mk < 0) mk += kBig;
            mj = table_[ii];
        }
        for (int k = 1; k < 5; ++k)
            for (int i = 1; i < 56; ++i) {
                table_[i] = wrap_sub(table_[i], table_[1 + (i + 30) % 55]);
                if (table_[i] < 0) table_[i] += kBig;
            }
        next_ = 0;
        nextp_ = 21;
    }

    int32_t sample_int()
    {
        const int32_t kBig = 2147483647;
        if (++next_ >= 56) next_ = 1;
        if (++nextp_ >= 56) nextp_ = 1;
        int32_t r = wrap_sub(table_[next_], table_[nextp_]);
        if (r == kBig) --r;
        if (r < 0) r += kBig;
        table_[next_] = r;
        return r;
    }

    // Next(): [0, 2^31 - 1)
    int32_t next() { return sample_int(); }

    // Next(min, max) for ranges that fit in int32: (int)(Sample() * range) + min
    int32_t next(int32_t lo, int32_t hi)
    {
        const double sample = sample_int() * (1.0 / 2147483647.0);
        return (int32_t)(sample * (double)((int64_t)hi - lo)) + lo;
    }

private:
    int32_t table_[56] = {};
    int next_ = 0, nextp_ = 0;
};

}  // namespace

extern "C" {

// Problem.FillArrayOfProblems(problems, count, n, seed) into records of
// 2*lstride bytes (a[j] = rec[j], b[j] = rec[lstride + j]); bytes past n are 0.
SBFS_API sbfs_status sbfs_generate_reference_batch(int64_t count, int32_t n, int32_t seed, uint8_t *maps,
                                                   int32_t lstride)
{
    if (count < 0 || n < 1 || n > SBFS_MAX_N || lstride < n || lstride > 32 || (count > 0 && !maps))
        return SBFS_EINVAL;
    // the master stream is sequential and cheap; the per-automaton generators
    // (a 55-entry table each) are independent and run on all host threads
    std::vector<int32_t> seeds((size_t)count);
    DotnetRandom master(seed);
    for (int64_t p = 0; p < count; ++p) seeds[(size_t)p] = master.next();   // Problem.cs:37
    auto fill = [&](int64_t lo, int64_t hi) {
        for (int64_t p = lo; p < hi; ++p) {
            DotnetRandom r(seeds[(size_t)p]);
            uint8_t *rec = maps + (size_t)p * 2 * (size_t)lstride;
            std::memset(rec, 0, 2 * (size_t)lstride);
            for (int i = 0; i < n; ++i) {   // Problem.cs:52-56: A[i] then B[i]
                rec[i] = (uint8_t)r.next(0, n);
                rec[lstride + i] = (uint8_t)r.next(0, n);
            }
        }
    };
    const int64_t per = 1 << 14;
    const int threads = (int)std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()),
                                               std::max<int64_t>(1, (count + per - 1) / per));
    if (threads <= 1) {
        fill(0, count);
    } else {
        std::vector<std::thread> pool;
        const int64_t step = (count + threads - 1) / threads;
        for (int t = 0; t < threads; ++t) {
            const int64_t lo = t * step, hi = std::min(count, lo + step);
            if (lo < hi) pool.emplace_back(fill, lo, hi);
        }
        for (auto &th : pool) th.join();
    }
    return SBFS_OK;
}

// First `count` values of new Random(seed).Next(); for pinning the generator.
SBFS_API sbfs_status sbfs_dotnet_random_next(int32_t seed, int32_t count, int32_t *out)
{
    if (count < 0 || (count > 0 && !out)) return SBFS_EINVAL;
    DotnetRandom r(seed);
    for (int32_t i = 0; i < count; ++i) out[i] = r.next();
    return SBFS_OK;
}

}  // extern "C"
