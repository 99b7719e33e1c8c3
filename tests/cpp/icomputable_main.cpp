// Drives include/sbfs_icomputable.hpp (the C++ mirror of IComputable) the way
// the reference harness drives a solver (GPGPU/Program.cs:94-129).
//
//   icomputable_main cpu                 host-only checks, no device needed
//   icomputable_main gpu <n> <seed> <count>
//       Compute over FillArrayOfProblems(count, n, seed) followed by the
//       worst case C_n; prints one length per line (-1 = not synchronizing)
//       after replaying every word and checking Cerny's bound.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "sbfs_icomputable.hpp"

static int fail(const char *what)
{
    std::fprintf(stderr, "FAIL: %s\n", what);
    return 1;
}

static int run_cpu()
{
    using sbfs::Problem;
    std::printf("%s\n", Problem::GenerateWorstCase(5).ToString().c_str());
    for (const Problem &p : Problem::FillArrayOfProblems(3, 13, 12456)) std::printf("%s\n", p.ToString().c_str());
    // Verify.cs checks on hand-made results
    Problem c3 = Problem::GenerateWorstCase(3);
    sbfs::ComputationResult r;
    r.isSynchronizable = true;
    r.shortestSynchronizingWord = {false, true, true, false};   // a b b a: {0,1,2} -> {1,2} -> {2,0} -> {0,1} -> {1}
    r.shortestSynchronizingWordLength = 4;
    if (!sbfs::VerifyValidityOfSynchronizingWord(c3, r)) return fail("a b b a synchronises C_3");
    if (!sbfs::VerifyCernyConjecture(c3, r)) return fail("length 4 <= 4");
    r.shortestSynchronizingWord = {true};
    if (sbfs::VerifyValidityOfSynchronizingWord(c3, r)) return fail("b alone does not synchronise C_3");
    r.shortestSynchronizingWord.assign(5, false);
    if (sbfs::VerifyCernyConjecture(c3, r)) return fail("length 5 > 4");
    try {
        Problem::GenerateWorstCase(2);
        return fail("GenerateWorstCase(2) must throw");
    } catch (const std::invalid_argument &) {
    }
    try {
        Problem::FillArrayOfProblems(1, 29, 1);
        return fail("n = 29 must be refused");
    } catch (const std::invalid_argument &) {
    }
    std::printf("cpu ok\n");
    return 0;
}

static int run_gpu(int n, int seed, int count)
{
    std::vector<sbfs::Problem> problems = sbfs::Problem::FillArrayOfProblems(count, n, seed);
    problems.push_back(sbfs::Problem::GenerateWorstCase(n));
    sbfs::SlimGPUNative solver;
    std::vector<sbfs::ComputationResult> results;
    const int total = (int)problems.size();
    if (solver.Compute(problems, 0, &results, 0, total, solver.GetBestParallelism()) != -1)
        return fail("no automaton exceeds (n-1)^2");
    if ((int)results.size() != total) return fail("one result per automaton");
    for (int i = 0; i < total; ++i) {
        const sbfs::ComputationResult &r = results[(size_t)i];
        if (!sbfs::VerifyValidityOfSynchronizingWord(problems[(size_t)i], r)) return fail("word does not replay");
        if (!sbfs::VerifyCernyConjecture(problems[(size_t)i], r)) return fail("Cerny bound");
        if (r.isSynchronizable && (int)r.shortestSynchronizingWord.size() != r.shortestSynchronizingWordLength)
            return fail("word length");
        std::printf("%d\n", r.isSynchronizable ? r.shortestSynchronizingWordLength : -1);
    }
    if (results.back().shortestSynchronizingWordLength != (n - 1) * (n - 1)) return fail("C_n has (n-1)^2");
    if (solver.Verify(problems, 0, total, 1) != -1) return fail("Verify");
    // offsets: results written from index 5 of a longer vector, problems read from index 1
    std::vector<sbfs::ComputationResult> shifted(5);
    if (solver.Compute(problems, 1, &shifted, 5, total - 1, 1) != -1) return fail("offset Compute");
    for (int i = 1; i < total; ++i)
        if (shifted[(size_t)(4 + i)].shortestSynchronizingWordLength != results[(size_t)i].shortestSynchronizingWordLength)
            return fail("offset results");
    return 0;
}

int main(int argc, char **argv)
{
    try {
        if (argc >= 2 && !std::strcmp(argv[1], "cpu")) return run_cpu();
        if (argc >= 5 && !std::strcmp(argv[1], "gpu"))
            return run_gpu(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]));
    } catch (const std::exception &e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 2;
    }
    std::fprintf(stderr, "usage: %s cpu | gpu <n> <seed> <count>\n", argv[0]);
    return 64;
}
