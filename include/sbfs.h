/*
 * sbfs.h -- C ABI of libsbfs.so, the B200 engine for exact shortest
 * synchronizing words of binary automata (power-set BFS).
 *
 * This ABI is the native side of the reference's solver plugin contract,
 * IComputable (GPGPU/Interfaces/IComputable.cs:11-20):
 *
 *   int Compute(Problem[] problemsToSolve, int problemsReadingIndex,
 *               ComputationResult[] computationResults, int resultsWritingIndex,
 *               int problemCount, int degreeOfParallelism);     -> sbfs_solve_batch
 *   int Verify(Problem[] problemsToSolve, int problemsReadingIndex,
 *              int problemCount, int degreeOfParallelism);      -> sbfs_verify_batch
 *   int GetBestParallelism();                                    -> sbfs_best_parallelism
 *
 * and replaces the Alea GPU solver GPGPU/GPU/SlimGPUQueue.cs:23-208 (host side:
 * allocate, copy, launch, copy back, Cerny check) and its kernel :210-407.
 *
 * Conventions
 *  - Every call returns an sbfs_status; nothing throws or aborts.
 *  - All host pointers are caller-owned and only read/written during the call
 *    (the serving calls copy what they need before returning).
 *  - One handle owns one CUDA stream set and its device buffers.  Calls on one
 *    handle are serialised by the handle; different handles may be used from
 *    different threads concurrently.
 *
 * Automaton records.  Automaton i occupies 2*lstride bytes at
 * maps + i*2*lstride: a[j] = rec[j] and b[j] = rec[lstride + j] for j < n
 * (Problem.stateTransitioningMatrixA/B, SharedDefinitions/Problem.cs:7-11).
 * lstride = 32 is the general 64-byte record; lstride = n packs a uniform
 * batch tightly.  n is per automaton (ns != NULL) or uniform (ns == NULL,
 * n_uniform).  1 <= n <= 28 and n <= lstride.
 *
 * Results.  out_len[i] = shortest synchronizing word length, or -1 when the
 * automaton is not synchronizing (ComputationResult.isSynchronizable /
 * shortestSynchronizingWordLength, GPGPU/Shared/ComputationResult.cs:9-20).
 * Words: word_stride uint64 per automaton, bit k (LSB first across the
 * uint64s) = 1 when letter k is b; letter 0 is applied first (the bool[] word
 * of GPGPU/CPU/CPU.cs:262-269, true = b).  Unused bits are zero.  A word longer
 * than 64*word_stride is not stored (its bits are zero) but the length is.
 * out_first_violation = smallest batch index whose length exceeds
 * (n-1)^2 - slack (the Cerny check of every IComputable.Compute), else -1.
 */
#ifndef SBFS_H
#define SBFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define SBFS_API __declspec(dllexport)
#else
#define SBFS_API __attribute__((visibility("default")))
#endif

#define SBFS_MAX_N 28
#define SBFS_ABI_VERSION 2

typedef enum sbfs_status {
    SBFS_OK = 0,
    SBFS_EINVAL = 1,     /* bad argument or malformed automaton (state >= n)    */
    SBFS_ENOMEM = 2,     /* device or pinned host allocation failed             */
    SBFS_ETIMEOUT = 3,   /* a bounded wait ran out                              */
    SBFS_ECUDA = 4,      /* a CUDA runtime call failed (see sbfs_last_error)    */
    SBFS_EBUSY = 5,      /* admission refused for now / queue full              */
    SBFS_ENOTFOUND = 6,  /* unknown request id                                  */
    SBFS_ECANCELED = 7,  /* request cancelled before completion                 */
    SBFS_ESTOPPED = 8    /* server stopped                                      */
} sbfs_status;

typedef struct sbfs_handle sbfs_handle;

typedef struct sbfs_config {
    int32_t device;            /* CUDA device ordinal; -1 = current device              */
    int32_t slack;             /* violation when len > (n-1)^2 - slack; 0 = Cerny bound */
    int32_t use_graph;         /* 1 = replay batches of an already-seen shape from CUDA graphs */
    int32_t autotune;          /* 1 = measure kernel shapes on first use and cache them */
    int32_t slots_per_warp;    /* small-n kernel: automata in flight per warp; 0 = auto */
    int32_t warps_per_cta;     /* small-n kernel: warps per CTA; 0 = auto               */
    int32_t queue_smem;        /* small-n kernel: on-chip queue entries per automaton; 0 = auto */
    int32_t chunk;             /* host path: 0 = auto -- a uniform batch of n <= 14 with at least
                                  2^18 automata runs as one kernel while its records stream in
                                  and its results stream out in 2^17-automaton pieces; other
                                  batches in chunks of 2^18 over the streams.  > 0 = chunks of
                                  this many automata over the streams, never streamed      */
    int32_t small_kernel;      /* n <= 16: 0 = auto (per lane up to n = 12 and for uniform batches of
                                  n = 13 or 14, hash-set warps for 13..16), 1 = one automaton per
                                  lane (n <= 12), 2 = warp-pooled (n <= 16) */
    int32_t lane_ring;         /* per-lane kernel: on-chip frontier entries (power of 2); 0 = auto */
    int32_t lane_refill;       /* per-lane kernel: idle lanes that trigger a refill; 0 = auto */
    int32_t lane_warps;        /* per-lane kernel: warps per CTA; 0 = auto              */
    int32_t lane_tail;         /* per-lane kernel: after the last automaton is handed out, a warp with at most
                                  this many lanes still searching gives them to the whole-warp search;
                                  0 = auto, -1 = never                                     */
    int32_t streams;           /* streams the host path rotates chunks over; 0 = 4      */
    int64_t level_arena_bytes; /* HBM budget of the n > 20 level slots; 0 = half of free memory, <= 64 GiB */
    const char *tune_cache;    /* autotuner cache file, or NULL for in-memory only      */
    int32_t wait_polls;        /* device-side bounded waits (the streamed host path's wait for a
                                  chunk of records): polls of about 0.2 us before the kernel gives
                                  up and the call returns SBFS_ETIMEOUT; 0 = 2^24 (ABI version 2) */
} sbfs_config;

typedef struct sbfs_stats {
    int64_t automata;          /* automata solved by the call                           */
    int64_t expanded;          /* subsets dequeued and expanded (sum over automata)     */
    int64_t synchronizing;     /* automata with a synchronizing word                    */
    int64_t h2d_bytes;         /* bytes copied host -> device                           */
    int64_t d2h_bytes;         /* bytes copied device -> host                           */
    int32_t launches;          /* kernels launched                                      */
    int32_t classes;           /* size classes used (small / cta / hbm)                 */
    double kernel_ms;          /* device time of the BFS kernels (CUDA events)          */
    double total_ms;           /* wall time of the call                                 */
    int64_t escalated;         /* automata the per-lane search handed to a whole warp   */
} sbfs_stats;

SBFS_API int32_t sbfs_abi_version(void);
SBFS_API sbfs_status sbfs_config_default(sbfs_config *cfg);
SBFS_API sbfs_status sbfs_create(const sbfs_config *cfg, sbfs_handle **out);
SBFS_API sbfs_status sbfs_destroy(sbfs_handle *h);
/* Message of the last failure on this handle ("" when none); h may be NULL
 * for failures of sbfs_create.  Valid until the next call on the handle. */
SBFS_API const char *sbfs_last_error(const sbfs_handle *h);
SBFS_API const char *sbfs_status_string(sbfs_status s);

/* IComputable.GetBestParallelism (IComputable.cs:19): the number of CUDA
 * streams the batched path overlaps (SlimGPUQueue.cs:19 returns 1). */
SBFS_API int32_t sbfs_best_parallelism(const sbfs_handle *h);

/*
 * IComputable.Compute (IComputable.cs:14) on host buffers.  Copies records in,
 * solves every automaton, copies lengths (and words when out_words != NULL)
 * out.  out_len may be NULL only together with out_words == NULL (then this is
 * Verify).  word_stride is ignored when out_words == NULL.
 */
SBFS_API sbfs_status sbfs_solve_batch(sbfs_handle *h, const uint8_t *maps, int32_t lstride,
                                      const uint8_t *ns, int32_t n_uniform, int64_t count,
                                      int32_t *out_len, uint64_t *out_words, int32_t word_stride,
                                      int64_t *out_first_violation, sbfs_stats *stats);

/* IComputable.Verify (IComputable.cs:17): lengths only, no words; out_len may be
 * NULL.  Returns the first violation through out_first_violation. */
SBFS_API sbfs_status sbfs_verify_batch(sbfs_handle *h, const uint8_t *maps, int32_t lstride,
                                       const uint8_t *ns, int32_t n_uniform, int64_t count,
                                       int32_t *out_len, int64_t *out_first_violation,
                                       sbfs_stats *stats);

/* The plain form: one automaton per kernel launch, same kernel body, used as
 * the per-automaton comparison point.  count automata are solved one by one. */
SBFS_API sbfs_status sbfs_solve_plain(sbfs_handle *h, const uint8_t *maps, int32_t lstride,
                                      const uint8_t *ns, int32_t n_uniform, int64_t count,
                                      int32_t *out_len, uint64_t *out_words, int32_t word_stride,
                                      int64_t *out_first_violation, sbfs_stats *stats);

/*
 * Device-buffer form of sbfs_solve_batch: maps, ns, len and words are device
 * memory and the work is enqueued on `stream` (a cudaStream_t; NULL = the
 * handle's first stream).  *d_first_violation is an int64 in device memory
 * (-1 = none).  max_n bounds the sizes in d_ns (0 = 28); it sizes the
 * large-n buffers without reading d_ns back.  The call returns once the work
 * is enqueued; sbfs_device_wait reports its errors and statistics.
 */
SBFS_API sbfs_status sbfs_solve_batch_device(sbfs_handle *h, const uint8_t *d_maps, int32_t lstride,
                                             const uint8_t *d_ns, int32_t n_uniform, int32_t max_n,
                                             int64_t count, int32_t *d_len, uint64_t *d_words,
                                             int32_t word_stride, int64_t *d_first_violation,
                                             void *stream);

/* Waits for the last sbfs_solve_batch_device call of this handle and reports
 * its status (SBFS_EINVAL for a malformed automaton) and statistics. */
SBFS_API sbfs_status sbfs_device_wait(sbfs_handle *h, sbfs_stats *stats);

/* Pinned host memory for callers that want the copy-overlapped path without
 * their own CUDA dependency (the C# shim uses it for its staging arrays). */
SBFS_API sbfs_status sbfs_host_alloc(size_t bytes, void **out);
SBFS_API sbfs_status sbfs_host_free(void *p);

/*
 * Allocation-free solve for callers that must not allocate device memory: a
 * plugin inside a process whose framework already owns the device memory
 * budget (a new cudaMalloc would fail or evict its cache), or a tight serving
 * loop where cudaMalloc/cudaFree would synchronise the device.  This entry
 * point has no counterpart in the reference.  It takes no handle: it solves
 * count automata with 1 <= n <= 12 states (d_maps, d_len, d_words and
 * *d_first_violation are caller-owned device memory) on the current device,
 * enqueued on `stream` (a cudaStream_t; NULL = the default stream), and keeps
 * all of its working memory in one fixed 16 MiB array inside the library.
 * n > 12 returns SBFS_EINVAL.  Every call shares that array, so calls that
 * overlap on the GPU race; serialise them.  Every call looks the array up
 * in the current context (cudaGetSymbolAddress, which allocates nothing); the
 * first call on a device may load the library's device code, so make it
 * before any stream capture.  d_len is required (SBFS_EINVAL without it): a
 * malformed record is reported only as length -2 there.  Words and lengths
 * follow the conventions above; it is slower than sbfs_solve_batch_device.
 */
SBFS_API sbfs_status sbfs_solve_small_noalloc(const uint8_t *d_maps, int32_t lstride, int32_t n,
                                              int64_t count, int32_t *d_len, uint64_t *d_words,
                                              int32_t word_stride, int64_t *d_first_violation,
                                              void *stream);

/* JSON description of the kernel plan the handle uses (kernel and shape per
 * size class), written to buf (NUL-terminated, truncated to len).  Returns
 * the full length needed. */
SBFS_API int32_t sbfs_describe_plan(sbfs_handle *h, char *buf, int32_t len);

/* ---------------------------------------------------------------------------
 * Serving: a request loop on its own thread.  Requests (one automaton each)
 * are admitted as they arrive: automata with n <= 20 are gathered into
 * mini-batches (several in flight) and solved by the batch kernels, which
 * deliver each result as soon as its own search ends; automata with n >= 21
 * are admitted into device-resident BFS slots while their 2^n-bit bitmap and
 * queue fit the arena budget, and advance a few levels per launch alongside
 * every other admitted request, so a request that arrives while others run is
 * taken in as soon as memory frees up.  No reference counterpart (the reference solves fixed
 * batches only, GPGPU/Program.cs:76-111).
 * ------------------------------------------------------------------------- */
typedef struct sbfs_server sbfs_server;

typedef struct sbfs_server_config {
    int32_t device;            /* CUDA device; -1 = current                                 */
    int32_t max_batch;         /* small requests per mini-batch; 0 = 8192                   */
    int32_t max_levels;        /* levels per launch batch of the large path; 0 = 16         */
    int32_t queue_capacity;    /* pending requests before submit returns SBFS_EBUSY; 0 = 1<<20 */
    int64_t arena_bytes;       /* HBM budget for admitted large requests; 0 = 16 GiB        */
    int64_t small_budget_bytes; /* n <= 20: bytes the mini-batches in flight may account for,
                                   2^n / 8 + 64 per request (its visited set and record);
                                   0 = 1 GiB (ABI version 2)                               */
} sbfs_server_config;

typedef struct sbfs_result {
    uint64_t id;
    int32_t status;            /* SBFS_OK or SBFS_ECANCELED                                 */
    int32_t len;               /* -1 = not synchronizing                                    */
    int32_t n;
    int32_t pad;
    uint64_t word[12];         /* letters as in sbfs_solve_batch (768 bits)                 */
    double submit_ms;          /* server clock at submission                                */
    double done_ms;            /* server clock when the result became available             */
} sbfs_result;

typedef struct sbfs_server_stats {
    int64_t submitted, completed, rejected, cancelled;
    int64_t pending;           /* submitted, not yet on the GPU                             */
    int64_t in_flight;         /* on the GPU                                                */
    int64_t small_batches, level_launches;
    int64_t arena_used, arena_peak, arena_capacity;  /* bytes held by admitted large requests */
    double now_ms;
    int64_t small_used, small_peak, small_capacity;  /* footprint of the n <= 20 requests in flight */
} sbfs_server_stats;

SBFS_API sbfs_status sbfs_server_config_default(sbfs_server_config *cfg);
SBFS_API sbfs_status sbfs_server_start(const sbfs_server_config *cfg, sbfs_server **out);
/* Copies the automaton (a[0..n), b[0..n)); returns its id.  SBFS_EINVAL for a
 * malformed automaton, SBFS_EBUSY when the pending queue is full. */
SBFS_API sbfs_status sbfs_server_submit(sbfs_server *s, const uint8_t *a, const uint8_t *b, int32_t n,
                                        uint64_t *out_id);
/* count automata in one call, as records of 2*lstride bytes (a = rec[0..n),
 * b = rec[lstride..lstride+n), n = ns[i]; 1 <= lstride <= 32), taken under one
 * lock: out_ids[i] receives request i's id.  Every request is checked first;
 * the call admits all of them or none (SBFS_EINVAL naming no request when one
 * is malformed, SBFS_EBUSY when they do not all fit the pending queue).  For
 * clients whose requests arrive in bursts: one call instead of count. */
SBFS_API sbfs_status sbfs_server_submit_many(sbfs_server *s, const uint8_t *maps, int32_t lstride,
                                             const uint8_t *ns, int64_t count, uint64_t *out_ids);
/* Up to max finished results; waits up to timeout_ms for the first one. */
SBFS_API sbfs_status sbfs_server_poll(sbfs_server *s, sbfs_result *out, int32_t max, int32_t *got,
                                      int32_t timeout_ms);
/* Cancels a pending request (its result comes back with SBFS_ECANCELED);
 * SBFS_ENOTFOUND when it is unknown or already on the GPU. */
SBFS_API sbfs_status sbfs_server_cancel(sbfs_server *s, uint64_t id);
SBFS_API sbfs_status sbfs_server_stats_get(sbfs_server *s, sbfs_server_stats *out);
SBFS_API sbfs_status sbfs_server_reset_peak(sbfs_server *s);
/* Finishes everything submitted, then stops the loop and frees the server. */
SBFS_API sbfs_status sbfs_server_stop(sbfs_server *s);

/* uint64 per automaton needed for words of automata with at most max_n states:
 * ceil((max_n-1)^2 / 64), at least 1. */
SBFS_API int32_t sbfs_word_stride(int32_t max_n);

/* ---------------------------------------------------------------------------
 * The reference's input batches, bit for bit (host code, no GPU).  The
 * reference draws automata with .NET Framework's System.Random (Knuth's
 * subtractive generator): Problem.FillArrayOfProblems(problems, count, n, seed)
 * (SharedDefinitions/Problem.cs:32-58) seeds Random(seed) and builds each
 * automaton from Random(master.Next()), A[i] then B[i] = Next(0, n).  GPGPU's
 * benchmark uses seed 1234567 + count (GPGPU/Program.cs:94).
 * ------------------------------------------------------------------------- */
/* count records of 2*lstride bytes (a = rec[0..n), b = rec[lstride..lstride+n),
 * bytes past n zero); 1 <= n <= lstride <= 32. */
SBFS_API sbfs_status sbfs_generate_reference_batch(int64_t count, int32_t n, int32_t seed, uint8_t *maps,
                                                   int32_t lstride);
/* The first count values of new System.Random(seed).Next(). */
SBFS_API sbfs_status sbfs_dotnet_random_next(int32_t seed, int32_t count, int32_t *out);

#ifdef __cplusplus
}
#endif

#endif /* SBFS_H */
