// sbfs_icomputable.hpp -- header-only C++ mirror of the reference's solver
// contract over the C ABI of sbfs.h.
//
//   Problem            SharedDefinitions/Problem.cs:7-11
//   ComputationResult  GPGPU/Shared/ComputationResult.cs:9-20 (fields the path fills)
//   IComputable        GPGPU/Interfaces/IComputable.cs:11-20
//   SlimGPUNative      IComputable on libsbfs, in place of GPGPU/GPU/SlimGPUQueue.cs
//
// Compute writes results[resultsWritingIndex + i] and returns
// resultsWritingIndex + j for the first automaton j whose shortest word is
// longer than (n-1)^2, else -1.  Verify returns problemsReadingIndex + j.
// Failures of the library are thrown as sbfs::Error (the C ABI itself never
// throws).
#pragma once

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "sbfs.h"

namespace sbfs {

struct Problem {
    std::vector<int> stateTransitioningMatrixA;
    std::vector<int> stateTransitioningMatrixB;
    int size = 0;

    // Problem.GenerateWorstCase (Problem.cs:13-29): A sends 0 to 1, B is the cycle.
    static Problem GenerateWorstCase(int n)
    {
        if (n < 3) throw std::invalid_argument("wrong number!");
        Problem p;
        p.size = n;
        for (int i = 0; i < n; ++i) {
            p.stateTransitioningMatrixA.push_back(i == 0 ? 1 : i);
            p.stateTransitioningMatrixB.push_back(i + 1 == n ? 0 : i + 1);
        }
        return p;
    }

    // Problem.FillArrayOfProblems (Problem.cs:32-39): `count` automata of n
    // states from .NET System.Random(seed), bit for bit (sbfs_generate_reference_batch).
    static std::vector<Problem> FillArrayOfProblems(int count, int n, int seed)
    {
        const int lstride = 32;
        std::vector<uint8_t> recs((size_t)std::max(count, 0) * 2 * lstride);
        const sbfs_status st = sbfs_generate_reference_batch(count, n, seed, recs.data(), lstride);
        if (st != SBFS_OK) throw std::invalid_argument(sbfs_status_string(st));
        std::vector<Problem> out((size_t)count);
        for (int i = 0; i < count; ++i) {
            Problem &p = out[(size_t)i];
            p.size = n;
            p.stateTransitioningMatrixA.assign(recs.begin() + (size_t)i * 2 * lstride,
                                               recs.begin() + (size_t)i * 2 * lstride + n);
            p.stateTransitioningMatrixB.assign(recs.begin() + (size_t)i * 2 * lstride + lstride,
                                               recs.begin() + (size_t)i * 2 * lstride + lstride + n);
        }
        return out;
    }

    // Problem.ToString (Problem.cs:60-79): "[[a0,a1,..],[b0,b1,..]]"
    std::string ToString() const
    {
        std::string s = "[[";
        for (int i = 0; i < size; ++i) s += std::to_string(stateTransitioningMatrixA[i]) + (i + 1 < size ? "," : "");
        s += "],[";
        for (int i = 0; i < size; ++i) s += std::to_string(stateTransitioningMatrixB[i]) + (i + 1 < size ? "," : "");
        return s + "]]";
    }
};

struct ComputationResult {
    bool isSynchronizable = false;
    std::vector<bool> shortestSynchronizingWord;   // true = letter b, index 0 applied first
    int shortestSynchronizingWordLength = 0;
    int size = 0;
    std::string algorithmName;
};

class IComputable {
public:
    virtual ~IComputable() = default;
    virtual int Compute(const std::vector<Problem> &problemsToSolve, int problemsReadingIndex,
                        std::vector<ComputationResult> *computationResults, int resultsWritingIndex,
                        int problemCount, int degreeOfParallelism) = 0;
    virtual int Verify(const std::vector<Problem> &problemsToSolve, int problemsReadingIndex, int problemCount,
                       int degreeOfParallelism) = 0;
    virtual int GetBestParallelism() = 0;
};

class Error : public std::runtime_error {
public:
    Error(sbfs_status s, const std::string &m) : std::runtime_error(m), status(s) {}
    sbfs_status status;
};

class SlimGPUNative : public IComputable {
public:
    explicit SlimGPUNative(const sbfs_config *cfg = nullptr)
    {
        sbfs_config c;
        sbfs_config_default(&c);
        if (cfg) c = *cfg;
        check(sbfs_create(&c, &h_), nullptr);
    }
    ~SlimGPUNative() override { sbfs_destroy(h_); }
    SlimGPUNative(const SlimGPUNative &) = delete;
    SlimGPUNative &operator=(const SlimGPUNative &) = delete;

    int GetBestParallelism() override { return sbfs_best_parallelism(h_); }

    int Compute(const std::vector<Problem> &problemsToSolve, int problemsReadingIndex,
                std::vector<ComputationResult> *computationResults, int resultsWritingIndex, int problemCount,
                int /*degreeOfParallelism*/) override
    {
        if (problemCount == 0) return -1;
        const int lstride = 32;
        std::vector<uint8_t> maps((size_t)problemCount * 2 * lstride, 0), ns((size_t)problemCount);
        int max_n = 1;
        for (int i = 0; i < problemCount; ++i) {
            const Problem &p = problemsToSolve.at((size_t)problemsReadingIndex + i);
            if (p.size < 1 || p.size > SBFS_MAX_N) throw Error(SBFS_EINVAL, "problem size out of range");
            ns[i] = (uint8_t)p.size;
            max_n = std::max(max_n, p.size);
            for (int j = 0; j < p.size; ++j) {
                maps[(size_t)i * 2 * lstride + j] = (uint8_t)p.stateTransitioningMatrixA[j];
                maps[(size_t)i * 2 * lstride + lstride + j] = (uint8_t)p.stateTransitioningMatrixB[j];
            }
        }
        int64_t violation = -1;
        sbfs_stats st;
        if (!computationResults) {
            check(sbfs_verify_batch(h_, maps.data(), lstride, ns.data(), 0, problemCount, nullptr, &violation, &st),
                  h_);
            return violation < 0 ? -1 : problemsReadingIndex + (int)violation;
        }
        const int ws = sbfs_word_stride(max_n);
        std::vector<int32_t> len((size_t)problemCount);
        std::vector<uint64_t> words((size_t)problemCount * ws);
        check(sbfs_solve_batch(h_, maps.data(), lstride, ns.data(), 0, problemCount, len.data(), words.data(), ws,
                               &violation, &st),
              h_);
        if (computationResults->size() < (size_t)resultsWritingIndex + problemCount)
            computationResults->resize((size_t)resultsWritingIndex + problemCount);
        for (int i = 0; i < problemCount; ++i) {
            ComputationResult r;
            r.size = ns[i];
            r.algorithmName = "SlimGPUNative";
            r.isSynchronizable = len[i] >= 0;
            if (len[i] >= 0) {
                r.shortestSynchronizingWordLength = len[i];
                r.shortestSynchronizingWord.resize((size_t)len[i]);
                for (int k = 0; k < len[i] && k < 64 * ws; ++k)
                    r.shortestSynchronizingWord[k] = (words[(size_t)i * ws + k / 64] >> (k % 64)) & 1ull;
            }
            (*computationResults)[(size_t)resultsWritingIndex + i] = std::move(r);
        }
        return violation < 0 ? -1 : resultsWritingIndex + (int)violation;
    }

    int Verify(const std::vector<Problem> &problemsToSolve, int problemsReadingIndex, int problemCount,
               int degreeOfParallelism) override
    {
        return Compute(problemsToSolve, problemsReadingIndex, nullptr, -1, problemCount, degreeOfParallelism);
    }

    sbfs_handle *handle() const { return h_; }

private:
    static void check(sbfs_status s, sbfs_handle *h)
    {
        if (s != SBFS_OK) throw Error(s, std::string(sbfs_status_string(s)) + ": " + sbfs_last_error(h));
    }
    sbfs_handle *h_ = nullptr;
};

// Verify.VerifyValidityOfSynchronizingWord (GPGPU/Result veryfier/Verify.cs:12-54):
// replays the word from every state and requires one end state.
inline bool VerifyValidityOfSynchronizingWord(const Problem &p, const ComputationResult &r)
{
    if (!r.isSynchronizable) return true;
    int end = -1;
    for (int s = 0; s < p.size; ++s) {
        int q = s;
        for (bool isB : r.shortestSynchronizingWord)
            q = isB ? p.stateTransitioningMatrixB[q] : p.stateTransitioningMatrixA[q];
        if (end >= 0 && q != end) return false;
        end = q;
    }
    return true;
}

// Verify.VerifyCernyConjecture (Verify.cs:60-62)
inline bool VerifyCernyConjecture(const Problem &p, const ComputationResult &r)
{
    return !r.isSynchronizable || (int)r.shortestSynchronizingWord.size() <= (p.size - 1) * (p.size - 1);
}

}  // namespace sbfs
