/*
 * sbfs_oracle.c -- CPU restatement of the reference's power-set BFS.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path and the
 * timed CPU baseline; nothing in the product library links or calls it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU legs load liboracle.so.
 *
 * Pinning: the Cerny family C_n has shortest synchronizing word length exactly
 * (n-1)^2 (the reference's known-answer tests, AlgorithmCorrectnessTestProject/
 * SimpleAutomataTests.cs:14-35 and IntegrityTest.cs:44-62); tests/test_oracle.py
 * checks that for n = 3..20 and cross-checks random automata against an
 * independent word-enumeration search for small n.
 *
 * Entry points (all plain C, caller-owned buffers):
 *   orc_solve      SlimCPUUntweaked semantics (GPGPU/CPU/SlimCPUUntweaked.cs:51-223):
 *                  stamped visited array, level bump rule, letter a before b,
 *                  singleton detected on generation; plus the parent-pointer word
 *                  of GPGPU/CPU/CPU.cs:196-235,262-269 when words are requested.
 *   orc_verify4    SlimCPU4bits13 semantics (GPGPU/CPU/SlimCPU4bits.cs:54-345):
 *                  combined nibble table with letter a in the high n bits, the
 *                  reference's timed Verify mode (lengths optional).
 *   orc_replay     Verify.VerifyValidityOfSynchronizingWord and
 *                  VerifyCernyConjecture (GPGPU/Result veryfier/Verify.cs:12-62).
 *   orc_fill_array_of_problems
 *                  Problem.FillArrayOfProblems (SharedDefinitions/Problem.cs:32-58)
 *                  with .NET Framework's System.Random, so that the CPU baseline
 *                  builds the reference's own batches without the product library.
 *
 * Automaton record layout (shared with the CUDA library): record i occupies
 * 2*lstride bytes at maps + i*2*lstride; a[j] = rec[j], b[j] = rec[lstride + j].
 * Lengths: -1 = not synchronizing, else the shortest word length.
 * Words: bit k of word (u64 array, word_stride u64 per automaton, LSB first)
 * is 1 when letter k is b (CPU.cs:262-269 uses true = b); letter 0 acts first.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2

/* Stamps (the reference's uint isDiscovered[2^n], SlimCPUUntweaked.cs:66-67,103)
 * are used up to this n; above it a bitmap cleared by walking the queue keeps
 * per-thread memory bounded.  Both are the same set-membership store. */
#define ORC_STAMP_MAX_N 20

typedef struct {
    uint32_t *queue;    /* subsets in BFS order (SlimCPUUntweaked.cs:69)          */
    uint32_t *parent;   /* (parent queue index << 1) | letter-is-b (CPU.cs:203-205) */
    uint32_t *stamp;    /* n <= ORC_STAMP_MAX_N                                    */
    uint64_t *bits;     /* n >  ORC_STAMP_MAX_N                                    */
    uint32_t stamp_id;
    int cap_n;          /* largest n the buffers are sized for                     */
} orc_ws;

static void ws_free(orc_ws *w)
{
    free(w->queue); free(w->parent); free(w->stamp); free(w->bits);
    memset(w, 0, sizeof(*w));
}

static int ws_reserve(orc_ws *w, int n, int want_parent)
{
    if (n <= w->cap_n && (!want_parent || w->parent)) return ORC_OK;
    int cap = n > w->cap_n ? n : w->cap_n;
    ws_free(w);
    size_t count = (size_t)1 << cap;
    w->queue = (uint32_t *)malloc(count * sizeof(uint32_t));
    if (want_parent) w->parent = (uint32_t *)malloc(count * sizeof(uint32_t));
    /* smaller automata in the same slice keep using stamps */
    size_t stamps = (size_t)1 << (cap < ORC_STAMP_MAX_N ? cap : ORC_STAMP_MAX_N);
    w->stamp = (uint32_t *)calloc(stamps, sizeof(uint32_t));
    if (cap > ORC_STAMP_MAX_N) {
        size_t words = count / 64 ? count / 64 : 1;
        w->bits = (uint64_t *)calloc(words, sizeof(uint64_t));
    }
    if (!w->queue || (want_parent && !w->parent) || !w->stamp || (cap > ORC_STAMP_MAX_N && !w->bits)) {
        ws_free(w);
        return ORC_ENOMEM;
    }
    w->cap_n = cap;
    w->stamp_id = 0;
    return ORC_OK;
}

/*
 * One automaton, SlimCPUUntweaked.cs:103-184 generalised to 32-bit masks.
 * Returns the length (>= 1) or -1 when the queue empties without a singleton.
 * *expanded receives the number of dequeued subsets.
 */
static int32_t bfs_one(orc_ws *w, int n, const uint8_t *a, const uint8_t *b,
                       uint64_t *word, int word_stride, int64_t *expanded)
{
    const uint32_t full = (n >= 32) ? 0xFFFFFFFFu : ((1u << n) - 1u);
    uint32_t pa[32], pb[32];
    for (int i = 0; i < n; ++i) {           /* SlimCPUUntweaked.cs:107-111 */
        pa[i] = 1u << a[i];
        pb[i] = 1u << b[i];
    }
    const int use_stamp = (n <= ORC_STAMP_MAX_N);
    uint32_t id = 0;
    if (use_stamp) {
        if (++w->stamp_id == 0) {           /* wrap: clear once every 2^32 automata */
            memset(w->stamp, 0, ((size_t)1 << ORC_STAMP_MAX_N) * sizeof(uint32_t));
            w->stamp_id = 1;
        }
        id = w->stamp_id;
        w->stamp[full] = id;                /* SlimCPUUntweaked.cs:103 */
    } else {
        w->bits[full >> 6] |= 1ull << (full & 63);
    }
#define SEEN(x) (use_stamp ? (w->stamp[(x)] == id) : ((w->bits[(x) >> 6] >> ((x) & 63)) & 1ull))
#define MARK(x) do { if (use_stamp) w->stamp[(x)] = id; else w->bits[(x) >> 6] |= 1ull << ((x) & 63); } while (0)

    uint32_t *queue = w->queue, *parent = word ? w->parent : NULL;
    uint32_t rd = 0, wr = 1;
    queue[0] = full;
    uint32_t dist = 1;                      /* currentNextDistance, :114 */
    uint32_t until_bump = 0xFFFFFFFFu;      /* verticesUntilBump, :115 (u32 here) */
    int seeking = 1, found = 0;             /* seekingFirstNext, discoveredSingleton */
    uint32_t found_parent = 0, found_letter = 0;
    int64_t pops = 0;

    while (rd < wr) {                        /* :119 */
        uint32_t v = queue[rd++];
        ++pops;
        if (--until_bump == 0) {             /* :126-130 */
            ++dist;
            seeking = 1;
        }
        uint32_t ia = 0, ib = 0;             /* :139-147, iterating the set bits */
        for (uint32_t m = v; m; m &= m - 1) {
            int i = __builtin_ctz(m);
            ia |= pa[i];
            ib |= pb[i];
        }
        const uint32_t img[2] = {ia, ib};
        for (uint32_t x = 0; x < 2; ++x) {   /* a first (:149-165), then b (:167-183) */
            uint32_t s = img[x];
            if (!SEEN(s)) {
                if ((s & (s - 1)) == 0) {    /* singleton on generation, :151-155 */
                    found = 1;
                    found_parent = rd - 1;
                    found_letter = x;
                    break;
                }
                MARK(s);
                if (parent) parent[wr] = ((rd - 1) << 1) | x;
                queue[wr++] = s;
                if (seeking) {               /* :160-164 */
                    seeking = 0;
                    until_bump = wr - rd;
                }
            }
        }
        if (found) break;
    }
    if (!use_stamp) {                        /* clear the bitmap by walking the queue */
        for (uint32_t k = 0; k < wr; ++k) w->bits[queue[k] >> 6] = 0;
    }
#undef SEEN
#undef MARK
    *expanded += pops;
    if (!found) return -1;

    if (word) {                              /* CPU.cs:262-269, true = b */
        memset(word, 0, (size_t)word_stride * sizeof(uint64_t));
        if ((int64_t)dist <= (int64_t)word_stride * 64) {
            uint32_t idx = found_parent;
            word[(dist - 1) >> 6] |= (uint64_t)found_letter << ((dist - 1) & 63);
            for (int32_t d = (int32_t)dist - 2; d >= 0; --d) {
                uint32_t p = parent[idx];
                word[d >> 6] |= (uint64_t)(p & 1u) << (d & 63);
                idx = p >> 1;
            }
        }
    }
    return (int32_t)dist;
}

typedef struct {
    const uint8_t *maps;
    int lstride;
    const uint8_t *ns;
    int n_uniform;
    int64_t begin, end;
    int32_t *out_len;
    uint64_t *out_words;
    int word_stride;
    int slack;
    int64_t first_violation;
    int64_t expanded;
    int status;
} orc_job;

static inline int cerny_bound(int n, int slack)
{
    return (n - 1) * (n - 1) - slack;
}

static void *solve_slice(void *arg)
{
    orc_job *j = (orc_job *)arg;
    orc_ws w;
    memset(&w, 0, sizeof(w));
    j->first_violation = -1;
    j->expanded = 0;
    j->status = ORC_OK;
    for (int64_t i = j->begin; i < j->end; ++i) {
        const uint8_t *rec = j->maps + (size_t)i * 2 * (size_t)j->lstride;
        int n = j->ns ? j->ns[i] : j->n_uniform;
        if (n < 1 || n > 28 || n > j->lstride) { j->status = ORC_EINVAL; break; }
        for (int k = 0; k < n; ++k)
            if (rec[k] >= n || rec[j->lstride + k] >= n) { j->status = ORC_EINVAL; break; }
        if (j->status) break;
        int st = ws_reserve(&w, n, j->out_words != NULL);
        if (st) { j->status = st; break; }
        uint64_t *word = j->out_words ? j->out_words + (size_t)i * (size_t)j->word_stride : NULL;
        int32_t len = bfs_one(&w, n, rec, rec + j->lstride, word, j->word_stride, &j->expanded);
        if (j->out_len) j->out_len[i] = len;
        if (len > cerny_bound(n, j->slack) && j->first_violation < 0) j->first_violation = i;
    }
    ws_free(&w);
    return NULL;
}

static int run_sliced(orc_job *proto, int64_t count, int threads, void *(*fn)(void *),
                      int64_t *out_first_violation, int64_t *out_expanded)
{
    if (count < 0) return ORC_EINVAL;
    if (threads < 1) threads = 1;
    if (threads > count) threads = count > 0 ? (int)count : 1;
    /* contiguous slices as Parallel.For does (SlimCPUUntweaked.cs:33-47) */
    int64_t part = (count + threads - 1) / threads;
    orc_job *jobs = (orc_job *)calloc((size_t)threads, sizeof(orc_job));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!jobs || !tid) { free(jobs); free(tid); return ORC_ENOMEM; }
    for (int t = 0; t < threads; ++t) {
        jobs[t] = *proto;
        jobs[t].begin = (int64_t)t * part < count ? (int64_t)t * part : count;
        jobs[t].end = (int64_t)(t + 1) * part < count ? (int64_t)(t + 1) * part : count;
    }
    for (int t = 1; t < threads; ++t) pthread_create(&tid[t], NULL, fn, &jobs[t]);
    fn(&jobs[0]);
    for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
    int status = ORC_OK;
    int64_t fv = -1, ex = 0;
    for (int t = 0; t < threads; ++t) {
        if (jobs[t].status && !status) status = jobs[t].status;
        if (jobs[t].first_violation >= 0 && (fv < 0 || jobs[t].first_violation < fv))
            fv = jobs[t].first_violation;
        ex += jobs[t].expanded;
    }
    free(jobs);
    free(tid);
    if (out_first_violation) *out_first_violation = fv;
    if (out_expanded) *out_expanded = ex;
    return status;
}

/*
 * SlimCPUUntweaked.Compute (SlimCPUUntweaked.cs:19-49) over records [0, count).
 * ns may be NULL (all automata have n_uniform states).  out_words may be NULL.
 * slack lowers the Cerny bound used for violation reporting (0 = (n-1)^2).
 * out_first_violation: smallest index with length > bound, or -1.
 */
int orc_solve(const uint8_t *maps, int lstride, const uint8_t *ns, int n_uniform,
              int64_t count, int32_t *out_len, uint64_t *out_words, int word_stride,
              int slack, int threads, int64_t *out_first_violation, int64_t *out_expanded)
{
    if (!maps || lstride < 1 || lstride > 32 || (out_words && word_stride < 1)) return ORC_EINVAL;
    orc_job proto;
    memset(&proto, 0, sizeof(proto));
    proto.maps = maps; proto.lstride = lstride; proto.ns = ns; proto.n_uniform = n_uniform;
    proto.out_len = out_len; proto.out_words = out_words; proto.word_stride = word_stride;
    proto.slack = slack;
    return run_sliced(&proto, count, threads, solve_slice, out_first_violation, out_expanded);
}

/* ---------------------------------------------------------------------------
 * SlimCPU4bits13 (SlimCPU4bits.cs:54-345): one combined table over 4-bit
 * chunks of the subset, entry = (a-image << n) | b-image, so both images come
 * from ceil(n/4) lookups.  The reference fixes n = 12 (:63); here n <= 16 is a
 * parameter.  Lengths are written only when out_len != NULL (the reference's
 * timed build defines ignoreOutputArray, :3,312-314).
 * ------------------------------------------------------------------------- */
static void *verify4_slice(void *arg)
{
    orc_job *j = (orc_job *)arg;
    const int n = j->n_uniform;
    const uint32_t power = 1u << n;
    const uint32_t full = power - 1u;
    const uint32_t maskN = full;
    const int chunks = (n + 3) / 4;
    uint32_t *stamp = (uint32_t *)calloc(power, sizeof(uint32_t));
    uint16_t *queue = (uint16_t *)malloc(power * sizeof(uint16_t));
    j->first_violation = -1;
    j->expanded = 0;
    j->status = ORC_OK;
    if (!stamp || !queue) { free(stamp); free(queue); j->status = ORC_ENOMEM; return NULL; }
    uint32_t table[4 * 16];
    uint32_t id = 0;
    int64_t pops = 0;
    for (int64_t i = j->begin; i < j->end; ++i) {
        const uint8_t *a = j->maps + (size_t)i * 2 * (size_t)j->lstride;
        const uint8_t *b = a + j->lstride;
        ++id;                                              /* localProblemId */
        stamp[full] = id;                                  /* :118 */
        /* table build, :122-206: tra[c][v] = OR over set bits k of v of pre[4c+k] */
        for (int c = 0; c < chunks; ++c) {
            table[c * 16] = 0;
            for (int v = 1; v < 16; ++v) {
                int k = __builtin_ctz(v);
                int st = 4 * c + k;
                uint32_t pre = st < n ? ((power << a[st]) | (1u << b[st])) : 0u;
                table[c * 16 + v] = table[c * 16 + (v & (v - 1))] | pre;
            }
        }
        uint32_t rd = 0, wr = 1;
        queue[0] = (uint16_t)full;
        uint32_t dist = 1, until_bump = 0xFFFFFFFFu;
        int seeking = 1, found = 0;
        while (rd < wr) {                                   /* :214-306 */
            uint32_t v = queue[rd++];
            ++pops;
            if (--until_bump == 0) { ++dist; seeking = 1; }
            uint32_t t = table[v & 15];                     /* :252-264 */
            if (chunks > 1) t |= table[16 + ((v >> 4) & 15)];
            if (chunks > 2) t |= table[32 + ((v >> 8) & 15)];
            if (chunks > 3) t |= table[48 + ((v >> 12) & 15)];
            const uint32_t img[2] = {t >> n, t & maskN};    /* :266-267 */
            for (int x = 0; x < 2; ++x) {
                uint32_t s = img[x];
                if (stamp[s] != id) {
                    if ((s & (s - 1)) == 0) { found = 1; break; }
                    stamp[s] = id;
                    queue[wr++] = (uint16_t)s;
                    if (seeking) { seeking = 0; until_bump = wr - rd; }
                }
            }
            if (found) break;
        }
        int32_t len = found ? (int32_t)dist : -1;
        if (j->out_len) j->out_len[i] = len;
        if (len > cerny_bound(n, j->slack) && j->first_violation < 0) j->first_violation = i;
    }
    j->expanded = pops;
    free(stamp);
    free(queue);
    return NULL;
}

int orc_verify4(const uint8_t *maps, int lstride, int n, int64_t count, int32_t *out_len,
                int slack, int threads, int64_t *out_first_violation, int64_t *out_expanded)
{
    if (!maps || n < 2 || n > 16 || lstride < n || lstride > 32) return ORC_EINVAL;
    for (int64_t i = 0; i < count; ++i) {
        const uint8_t *rec = maps + (size_t)i * 2 * (size_t)lstride;
        for (int k = 0; k < n; ++k)
            if (rec[k] >= n || rec[lstride + k] >= n) return ORC_EINVAL;
    }
    orc_job proto;
    memset(&proto, 0, sizeof(proto));
    proto.maps = maps; proto.lstride = lstride; proto.n_uniform = n;
    proto.out_len = out_len; proto.slack = slack;
    return run_sliced(&proto, count, threads, verify4_slice, out_first_violation, out_expanded);
}

/* ---------------------------------------------------------------------------
 * Verify.cs:12-62.  For each automaton with len >= 0: replay the word from every
 * state and require one distinct end state; also require len <= (n-1)^2.
 * out_ok[i] bit 0 = word replays to a singleton, bit 1 = Cerny bound holds.
 * Non-synchronizing entries (len < 0) get both bits (Verify.cs:17-18,61).
 * Returns the number of entries failing either check.
 * ------------------------------------------------------------------------- */
int64_t orc_replay(const uint8_t *maps, int lstride, const uint8_t *ns, int n_uniform,
                   int64_t count, const int32_t *len, const uint64_t *words, int word_stride,
                   uint8_t *out_ok)
{
    int64_t bad = 0;
    for (int64_t i = 0; i < count; ++i) {
        const uint8_t *a = maps + (size_t)i * 2 * (size_t)lstride;
        const uint8_t *b = a + lstride;
        int n = ns ? ns[i] : n_uniform;
        uint8_t ok = 3;
        if (len[i] >= 0) {
            const uint64_t *w = words + (size_t)i * (size_t)word_stride;
            if ((int64_t)len[i] > (int64_t)word_stride * 64) {
                ok &= (uint8_t)~1u;
            } else {
                uint32_t end_set = 0;
                for (int s = 0; s < n; ++s) {
                    int q = s;
                    for (int32_t k = 0; k < len[i]; ++k)
                        q = ((w[k >> 6] >> (k & 63)) & 1ull) ? b[q] : a[q];
                    end_set |= 1u << q;
                }
                if (end_set & (end_set - 1)) ok &= (uint8_t)~1u;
            }
            if (len[i] > (n - 1) * (n - 1)) ok &= (uint8_t)~2u;
        }
        if (out_ok) out_ok[i] = ok;
        if (ok != 3) ++bad;
    }
    return bad;
}

/* ---------------------------------------------------------------------------
 * .NET Framework System.Random: Knuth's subtractive generator (TAOCP vol. 2,
 * 3.6), as .NET seeds it: a 55-entry table filled at stride 21 from
 * 161803398 - |seed|, stirred four times, outputs taken as differences at lags
 * 55 and 34 modulo 2^31 - 1.  C# int arithmetic is unchecked, so differences
 * wrap in two's complement (seeds above 161803398 make that happen).
 * ------------------------------------------------------------------------- */
typedef struct {
    int32_t t[56];
    int inext, inextp;
} orc_dotnet_random;

static inline int32_t orc_wrap_sub(int32_t a, int32_t b)
{
    return (int32_t)((uint32_t)a - (uint32_t)b);
}

static void orc_random_seed(orc_dotnet_random *r, int32_t seed)
{
    const int32_t big = 2147483647, mseed = 161803398;
    const int32_t sub = seed == INT32_MIN ? big : (seed < 0 ? -seed : seed);
    int32_t mj = orc_wrap_sub(mseed, sub), mk = 1;
    memset(r->t, 0, sizeof(r->t));
    r->t[55] = mj;
    for (int i = 1; i < 55; ++i) {
        const int ii = (21 * i) % 55;
        r->t[ii] = mk;
        mk = orc_wrap_sub(mj, mk);
        if (mk < 0) mk += big;
        mj = r->t[ii];
    }
    for (int pass = 0; pass < 4; ++pass)
        for (int i = 1; i < 56; ++i) {
            r->t[i] = orc_wrap_sub(r->t[i], r->t[1 + (i + 30) % 55]);
            if (r->t[i] < 0) r->t[i] += big;
        }
    r->inext = 0;
    r->inextp = 21;
}

static int32_t orc_random_next(orc_dotnet_random *r)   /* Random.Next(): [0, 2^31 - 1) */
{
    const int32_t big = 2147483647;
    if (++r->inext >= 56) r->inext = 1;
    if (++r->inextp >= 56) r->inextp = 1;
    int32_t v = orc_wrap_sub(r->t[r->inext], r->t[r->inextp]);
    if (v == big) --v;
    if (v < 0) v += big;
    r->t[r->inext] = v;
    return v;
}

static int32_t orc_random_range(orc_dotnet_random *r, int32_t lo, int32_t hi)   /* Random.Next(lo, hi) */
{
    const double sample = orc_random_next(r) * (1.0 / 2147483647.0);
    return (int32_t)(sample * (double)((int64_t)hi - lo)) + lo;
}

typedef struct {
    const int32_t *seeds;
    uint8_t *maps;
    int n, lstride;
    int64_t begin, end;
} orc_fill_job;

static void *orc_fill_slice(void *arg)
{
    orc_fill_job *j = (orc_fill_job *)arg;
    orc_dotnet_random r;
    for (int64_t p = j->begin; p < j->end; ++p) {
        uint8_t *rec = j->maps + (size_t)p * 2 * (size_t)j->lstride;
        orc_random_seed(&r, j->seeds[p]);                 /* GenerateProblem(n, seed), Problem.cs:41-58 */
        memset(rec, 0, 2 * (size_t)j->lstride);
        for (int i = 0; i < j->n; ++i) {                  /* A[i] then B[i], Problem.cs:52-56 */
            rec[i] = (uint8_t)orc_random_range(&r, 0, j->n);
            rec[j->lstride + i] = (uint8_t)orc_random_range(&r, 0, j->n);
        }
    }
    return NULL;
}

/* FillArrayOfProblems(problems, count, n, seed) (Problem.cs:32-39) into records
 * of 2*lstride bytes, bytes past n zero; the per-automaton generators run on
 * `threads` threads (the master stream is sequential). */
int orc_fill_array_of_problems(int64_t count, int n, int32_t seed, uint8_t *maps, int lstride, int threads)
{
    if (count < 0 || n < 1 || n > 28 || lstride < n || lstride > 32 || (count > 0 && !maps)) return ORC_EINVAL;
    if (count == 0) return ORC_OK;
    int32_t *seeds = (int32_t *)malloc((size_t)count * sizeof(int32_t));
    if (!seeds) return ORC_ENOMEM;
    orc_dotnet_random master;
    orc_random_seed(&master, seed);
    for (int64_t p = 0; p < count; ++p) seeds[p] = orc_random_next(&master);   /* Problem.cs:37 */
    if (threads < 1) threads = 1;
    if (threads > count) threads = (int)count;
    orc_fill_job *jobs = (orc_fill_job *)calloc((size_t)threads, sizeof(orc_fill_job));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!jobs || !tid) { free(jobs); free(tid); free(seeds); return ORC_ENOMEM; }
    const int64_t part = (count + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        jobs[t].seeds = seeds; jobs[t].maps = maps; jobs[t].n = n; jobs[t].lstride = lstride;
        jobs[t].begin = (int64_t)t * part < count ? (int64_t)t * part : count;
        jobs[t].end = (int64_t)(t + 1) * part < count ? (int64_t)(t + 1) * part : count;
    }
    for (int t = 1; t < threads; ++t) pthread_create(&tid[t], NULL, orc_fill_slice, &jobs[t]);
    orc_fill_slice(&jobs[0]);
    for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
    free(jobs); free(tid); free(seeds);
    return ORC_OK;
}

/* The first count values of new System.Random(seed).Next(). */
int orc_dotnet_random_next(int32_t seed, int32_t count, int32_t *out)
{
    if (count < 0 || (count > 0 && !out)) return ORC_EINVAL;
    orc_dotnet_random r;
    orc_random_seed(&r, seed);
    for (int32_t i = 0; i < count; ++i) out[i] = orc_random_next(&r);
    return ORC_OK;
}
