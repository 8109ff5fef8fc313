/*
 * rabung_census.h -- C ABI of the B200 (sm_100a) power-residue census library
 * (librabung_census.so).
 *
 * For every prime p and every r in {2..9} with r | p-1 the library computes
 * the profile of the r-th power-residue colouring of 1..p-1: M (longest
 * monochromatic run), L (initial run of the residue colour from x = 1), the
 * canonical reflected witness min(s, p-(s+M-1)) over runs of length M, and
 * the Rabung threshold K; optionally the quadratic A4 four-window count.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   - the census worker's per-prime computation behind its line protocol,
 *     src/census/worker32.cu:10-45 (GPU) and src/census/small_cpu.cpp:15-40 (CPU);
 *   - the A4 worker's per-prime count, src/census/moment_worker.cpp:19-52;
 *   - the only in-process C ABI of the reference, baseline_init /
 *     baseline_profile, src/census/engine32/src/baseline_bridge.cu:7,21-27.
 *
 * Conventions: caller-owned buffers; plain pointers and sizes; return 0 on
 * success and a nonzero code on refusal, in which case outputs are invalid
 * as a whole (no partial results, docs/METHODS.md:35 of the reference).
 * One handle per host thread; a handle owns one CUDA stream.
 */
#ifndef RABUNG_CENSUS_H
#define RABUNG_CENSUS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mode flags for cz_census. */
#define CZ_DENSE 1u   /* exhaustive half-interval scan (the dense oracle) */
#define CZ_SPARSE 2u  /* certified rational-anchor filter */
#define CZ_AUTO 3u    /* sparse for p >= sparse_min_p, dense below */
#define CZ_A4 4u      /* also compute the quadratic A4 count */
#define CZ_VERIFY 8u  /* certify every witness run and prefix by direct powers */

/* Return codes. */
#define CZ_OK 0
#define CZ_EINVAL 1   /* bad argument (not prime, out of domain, buffer too small) */
#define CZ_ECUDA 2    /* CUDA error */
#define CZ_EREFUSED 3 /* a device status check failed: the whole request is refused */
#define CZ_ELIMIT 4   /* request exceeds a fixed limit or a caller buffer (nothing written) */
#define CZ_EPENDING 5 /* cz_poll / cz_next_done: the request is not complete yet */

/* One (p, r) profile, 32 bytes.  Records come grouped by prime in input
 * order and, within a prime, by ascending r. */
typedef struct cz_profile {
    uint32_t p, r;
    uint32_t M;        /* longest monochromatic run */
    uint32_t L;        /* initial residue run */
    uint32_t witness;  /* least reflected start of a run of length M */
    uint32_t status;   /* 0 */
    uint64_t K;        /* Rabung threshold */
} cz_profile;

typedef struct cz_config {
    int32_t device;          /* CUDA device ordinal */
    uint32_t sparse_min_p;   /* CZ_AUTO routes p >= this to the anchor filter */
    uint32_t cover_n;        /* cover shape: D ~ 2 sqrt(p/H) / cover_n (2..8) */
    uint32_t q_cap[10];      /* cover window Q per order r (index r), 3..255 */
    uint32_t anchor_bits;    /* anchor length: 32 r^-(t-1) <= 2^-anchor_bits */
    uint32_t screen;         /* 1: bilateral screen after the anchor filter */
    uint32_t sparse_blocks;  /* persistent filter grid (0: 2 per SM) */
    uint32_t use_graph;      /* 1: replay device work through a captured CUDA graph */
    uint32_t cta_per_profile; /* CTAs sharing one profile's rows (L2 working set) */
    uint32_t epoch_rows;     /* filter rows d per threshold epoch (0: 1024; at most 2^20) */
    uint32_t speculate;      /* 1: speculative thresholds floor(log_r p - margin), re-run on a miss */
    uint32_t spec_margin10[10];  /* margin per order r, in tenths */
    uint32_t plane_budget_mb;    /* plane pool per wave; larger batches run as consecutive waves */
    uint32_t dense_steps;        /* dense scan segment: 32 x dense_steps values of x per warp */
    uint32_t anchor_t[10];       /* anchor stages per order r (index r), 2..32; 0: from anchor_bits */
    uint32_t reserved[1];
} cz_config;

typedef struct cz_stats {
    float ms_setup, ms_table, ms_sparse, ms_dense, ms_a4, ms_finalize, ms_device;
    float ms_h2d, ms_d2h;
    uint32_t n_primes, n_dense, n_sparse, n_profiles, n_fallback;
    uint32_t n_respec;              /* primes re-run because a speculative threshold missed */
    float ms_respec;                /* device time of that re-run */
    uint32_t waves;                 /* consecutive waves the batch ran as */
    uint32_t kernels;               /* kernel launches of the call */
    uint64_t words, completions;    /* sparse filter words visited, exact completions */
    uint64_t tests;                 /* plane-window comparisons executed by the filter */
    uint64_t h2d_bytes, d2h_bytes;
    uint64_t staged_bytes;          /* colour-plane bytes the filter copied into shared memory */
} cz_stats;

typedef struct cz_handle cz_handle;

/* Fill *cfg with the defaults. */
int cz_default_config(cz_config *cfg);

/* Open a handle on cfg->device (allocates device tables); NULL cfg = defaults. */
int cz_open(const cz_config *cfg, cz_handle **out);
void cz_close(cz_handle *h);
const char *cz_last_error(const cz_handle *h);

/* Number of profiles (sum over primes of #{r in 2..9 : r | p-1}). */
uint32_t cz_count_profiles(const uint32_t *primes, uint32_t n);

/* Census of n primes (host buffers).  out must hold cz_count_profiles()
 * records; a4_out (may be NULL unless CZ_A4) holds n values (0 for p = 2).
 * stats may be NULL. */
int cz_census(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags,
              cz_profile *out, uint32_t out_cap, uint32_t *a4_out, cz_stats *stats);

/* Re-run the device work of the previous cz_census call on its inputs, which
 * are still resident in device memory (no host transfer, no planning); used
 * to time the device path alone.  Results land in the same device buffers and
 * are checked; stats receives the device times. */
int cz_replay(cz_handle *h, cz_stats *stats);

/* Device memory the colour planes of these primes would take (admission
 * control for serving; no reference counterpart). */
uint64_t cz_plane_bytes(const cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags);

/* Name and SM count of the handle's GPU (keys the autotuner's saved choices;
 * no reference counterpart). */
int cz_device_info(cz_handle *h, char *name, uint32_t len, uint32_t *sms);

/* Free and total device memory of the handle's GPU (no reference counterpart). */
int cz_mem_info(cz_handle *h, uint64_t *free_bytes, uint64_t *total_bytes);

/* Device sieve for interval requests: for each i, the first count[i] primes
 * >= lo[i] (fewer only where 2^32 is reached), written to out from slot
 * sum(count[0..i-1]); found[i] = primes written.  Replaces the reference's
 * bounded host sieve, src/census/prime_sieve.cpp:8-22. */
int cz_sieve(cz_handle *h, const uint32_t *lo, const uint32_t *count, uint32_t n, uint32_t *out,
             uint32_t *found);

/* Quadratic A4 counts only (src/census/moment_worker.cpp:19-52 semantics):
 * x in [1, p-4] with x..x+3 all of one quadratic character; 0 for p = 2. */
int cz_a4(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t *a4_out);

/* Measured integer peaks of this GPU (for the roofline; no reference
 * counterpart): kind 0 = plane-word tests per second (one funnel shift plus
 * one three-input logic op on 32-bit words), kind 1 = 32-bit Montgomery
 * products per second. */
int cz_microbench(cz_handle *h, uint32_t kind, double *per_second);

/* Dense census that allocates no memory (no counterpart in the reference).
 * For callers that cannot call cudaMalloc: plugins inside a host process that
 * owns the device memory budget, and allocator-free services that must not
 * grow their device footprint after start-up.  All device scratch is one fixed
 * 2 MiB array inside the library, held by every GPU that loads the library
 * until the process exits.  Limits: n <= 64 primes, each p < 4,194,304
 * (CZ_ELIMIT beyond them).  primes and out are host arrays as in cz_census
 * (out holds cz_count_profiles() records); stream is a cudaStream_t (NULL for
 * the legacy default stream) on the current device.  The call is synchronous:
 * it returns after that stream has finished.  Every call resolves the array's
 * device address for the current device (also after a cudaDeviceReset).  Calls
 * share the array: calls that overlap on the GPU race. */
int cz_census_dense_noalloc(const uint32_t *primes, uint32_t n, cz_profile *out, uint32_t out_cap,
                            void *stream);

/* Number of primes in [lo, hi) (hi <= 2^33), computed exactly on the host:
 * a segmented sieve for short intervals, else pi(hi-1) - pi(lo-1) by the
 * Lucy-Hedgehog recursion (O(x^(3/4)), ~30 ms at 2^32).  Sizes interval
 * buffers in one pass; replaces the reference's Meissel-Lehmer count,
 * src/census/prime_count.cpp:11-24.  Needs no GPU. */
uint64_t cz_prime_count(uint64_t lo, uint64_t hi);

/* Census of every prime in [lo, hi) (hi <= 2^32): the primes are found by the
 * device sieve, then censused as by cz_census.  primes_out (capacity
 * primes_cap) receives them ascending and *n_primes their count; out
 * (capacity out_cap) the records and *n_profiles their count; a4_out (NULL, or
 * capacity primes_cap) A4 per prime when flags has CZ_A4.  When a capacity is
 * too small the call returns CZ_ELIMIT with the needed counts in *n_primes /
 * *n_profiles (n_profiles 0 if the primes did not fit) and no records.  One
 * call replaces a supervisor's sieve of a block plus the worker round trip
 * (src/census/prime_sieve.cpp:8-22, src/census/worker32.cu:10-45). */
int cz_census_interval(cz_handle *h, uint64_t lo, uint64_t hi, uint32_t flags, uint32_t *primes_out,
                       uint32_t primes_cap, uint32_t *n_primes, cz_profile *out, uint32_t out_cap,
                       uint32_t *n_profiles, uint32_t *a4_out, cz_stats *stats);

/* ---- serving ---------------------------------------------------------------
 * A server keeps every admitted request resident on the GPU until its records
 * are final: the descriptors, per-profile state, colour planes, records and A4
 * of its primes live in device arrays sized when the server opens (colour
 * planes: slots x slot_budget_bytes, capped by free device memory), so a
 * request is admitted as soon as its planes and descriptors fit.  The anchor
 * filter runs as one persistent kernel over the unfinished profiles of all
 * admitted requests; when requests arrive it yields between work items and is
 * relaunched over the old and new profiles together, so an arrival joins the
 * work in flight instead of waiting for a batch to end.  The last CTA to
 * finish a profile certifies and writes its record; a request's records are
 * copied out as soon as its last profile is final.  Primes below the sparse
 * route (small p) and dense re-runs use a second handle between launches;
 * a profile whose speculative threshold missed is re-run there without
 * speculation, as cz_census does (records are unchanged by it).  A request
 * whose colour planes exceed the server's whole plane budget runs on the
 * second handle in waves of at most one slot's planes; a caller's non-prime is
 * refused before any device work.  A refusal reaches only the request that
 * caused it.  Submit and poll may be
 * called from any host thread.  The reference has no serving path; the
 * records equal cz_census's for the same primes. */
typedef struct cz_server cz_server;
int cz_server_open(const cz_config *cfg, uint32_t slots, uint64_t slot_budget_bytes, cz_server **out);
void cz_server_close(cz_server *s);             /* stops the filter at its next work item; drops unpolled work */
/* a request for the `count` consecutive primes from lo (device sieve), or,
 * when primes != NULL, for those `count` primes; flags as for cz_census */
int cz_submit(cz_server *s, uint32_t lo, uint32_t count, const uint32_t *primes, uint32_t flags,
              uint64_t *request_id);
/* the id of a completed request not yet announced; waits up to timeout_ms
 * (negative: until one completes); CZ_EPENDING on timeout */
int cz_next_done(cz_server *s, int32_t timeout_ms, uint64_t *request_id);
/* waits up to timeout_ms for request_id (CZ_EPENDING if still running); then
 * copies its primes (capacity primes_cap), records (capacity out_cap) and A4
 * (capacity primes_cap; any output may be NULL), releases the request and
 * returns its status (CZ_OK, or the refusal; cz_server_last_error says why).
 * CZ_ELIMIT with the needed counts when a capacity is too small (the request
 * is kept). */
int cz_poll(cz_server *s, uint64_t request_id, int32_t timeout_ms, uint32_t *primes_out, uint32_t primes_cap,
            uint32_t *n_primes, cz_profile *out, uint32_t out_cap, uint32_t *n_profiles, uint32_t *a4_out);
/* filter launches so far, requests completed, requests waiting */
int cz_server_info(cz_server *s, uint64_t *batches, uint64_t *completed, uint64_t *waiting);
/* scheduler counters: filter launches, launches that yielded to arrivals or
 * re-runs, requests completed and waiting, primes re-run without speculation
 * (a speculative miss) and on the dense scan (other fallbacks), requests
 * served in waves on the second handle (larger than the plane arena), and the
 * milliseconds spent draining yielded launches (yield flag to kernel end) and
 * in the windows between launches (kernel end to relaunch) */
typedef struct cz_server_counters {
    uint64_t launches, yields, completed, waiting;
    uint64_t respec_primes, fallback_primes, oversize_requests;
    double ms_drain, ms_window;
} cz_server_counters;
int cz_server_stats(cz_server *s, cz_server_counters *out);
const char *cz_server_last_error(cz_server *s);

/* ---- the 33-bit domain -------------------------------------------------------
 * The same census for primes below 2^33 (the reference's 33-bit engine,
 * src/census/math33.hpp:13-37 and reproducibility/gpu_method/source/engine33):
 * identical kernels and planning compiled for 64-bit prime words.  A record
 * carries p in 64 bits; the canonical witness is at most (p-1)/2 < 2^32.
 * Flags, refusal rules and statistics as for cz_census. */
typedef struct cz_profile64 {
    uint64_t p;
    uint32_t r, M, L, witness, status, reserved;
    uint64_t K;
} cz_profile64;

typedef struct cz_handle64 cz_handle64;
int cz_open64(const cz_config *cfg, cz_handle64 **out);
void cz_close64(cz_handle64 *h);
const char *cz_last_error64(const cz_handle64 *h);
/* profiles of n primes (0 when a prime is at or above 2^33) */
uint32_t cz_count_profiles64(const uint64_t *primes, uint32_t n);
int cz_census64(cz_handle64 *h, const uint64_t *primes, uint32_t n, uint32_t flags, cz_profile64 *out,
                uint32_t out_cap, uint32_t *a4_out, cz_stats *stats);

/* Reference-compatible adapter (src/census/engine32/src/baseline_bridge.cu:7,21-27):
 * profile of one prime for the orders in `mask` (bit r-2), M into out[r] and
 * L into prefix[r] (arrays of >= 10).  With full = 0 only the masks the
 * reference serves without `full` are accepted -- 1 {2}, 5 {2,4}, 18 {3,6},
 * 19 {2,3,6}, 23 {2,3,4,6} -- and any other mask returns 2, as there; with
 * full = 1 any mask of admissible orders.  Returns 0, or 2 for a refused mask,
 * a mask naming an order that does not divide p-1, p < 3 or a failed census.
 * Every witness run and prefix is certified by direct powers.  cap is
 * accepted and unused (buffers grow on demand).  One global handle, guarded
 * by a lock. */
void baseline_init(unsigned cap);
int baseline_profile(unsigned p, unsigned mask, unsigned *out, unsigned *prefix, int full);

#ifdef __cplusplus
}
#endif

#endif /* RABUNG_CENSUS_H */
