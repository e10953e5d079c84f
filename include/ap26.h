/* ap26.h -- C ABI of the B200-native AP26 per-K search (libap26.so).
 *
 * The search finds arithmetic progressions of primes first + j*K*23# with at
 * least 10 base-2 strong-probable-prime terms, over the reference's 10-shift
 * candidate set (SHIFT, SHIFT+64, ..., SHIFT+576), and reports each one raw,
 * exactly as the reference's GPU kernel checkn (ibethune/ap26,
 * src/opencl/kernels/checkn.cl:198-202) and CPU search
 * (src/cpu/cpuavx2.cpp:548-552) hand it to ReportSolution.  ReportSolution
 * itself (hash, 9-base validation, split recursion, SOL lines;
 * src/common/AP26.cpp:484-602) runs on the device behind ap26_search_k_sol,
 * ap26_report_batch and the batched and serving forms; ap26_report below is
 * the same step on the host for callers that keep their own, byte-compatible
 * with src/common/AP26.cpp.
 *
 * Conventions: plain pointers and sizes; the caller owns every buffer; every
 * entry point returns an int status (0 = AP26_OK, < 0 = error) and never
 * exits the process; one host thread at a time per context.
 */
#ifndef AP26_H
#define AP26_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define AP26_OK          0
#define AP26_E_ARG      -1   /* bad argument / null pointer                  */
#define AP26_E_CAPACITY -2   /* caller buffer too small; *n_out holds need   */
#define AP26_E_CUDA     -3   /* CUDA runtime error                           */
#define AP26_E_DOMAIN   -4   /* K / SHIFT outside the exact-arithmetic domain */
#define AP26_E_TIMEOUT  -5   /* a bounded device wait gave up                */
#define AP26_E_OVERFLOW -6   /* internal device buffer overflowed            */
#define AP26_E_NOMEM    -7   /* device memory budget exceeded (admission)    */
#define AP26_E_INVALID  -8   /* an AP failed even base-2 re-validation
                                (reference: "Computation error", AP26.cpp:569-574) */
#define AP26_E_NODEV    -9   /* no CUDA device / extension not usable        */

/* Largest K for which the reference's int64 setup arithmetic
 * (src/opencl/AP26.h:112-120) cannot overflow. */
#define AP26_KMAX_SAFE 400000000
/* Largest SHIFT such that every chain term stays below 2^62, the domain of
 * the reference's PrimeQ (src/common/PrimeQ_x86.h:189-195). */
#define AP26_SHIFT_MAX 16000

/* ---- types -------------------------------------------------------------- */
typedef struct ap26_ctx ap26_ctx;

/* Tuning knobs; zero fields take the context's defaults (or autotuned values,
 * see ap26_autotune). */
typedef struct {
  int32_t dense_primes;   /* primes sieved for all 10 words before compaction */
  int32_t warp_queue;     /* per-warp shared-memory queue depth (items)       */
  int32_t block_threads;  /* sieve CTA size (multiple of 32)                  */
  int32_t late_stage;     /* prime index where items move to the late queue   */
  int32_t chunk_tiles;    /* sieve tiles (one n53 start per CTA thread) per
                             launch (default 131072, about a quarter of a K;
                             the autotuner times the sizes the rings hold)    */
  int32_t use_graphs;     /* 1 (default) = every run (set-up, chunks, chain
                             walks, ReportSolution, read-backs) is one CUDA
                             graph launch, captured once per run shape and
                             cached; -1 = plain stream launches               */
  int32_t profile;        /* 1 = time every sieve launch with CUDA events
                             (ap26_stats.sieve_ms; in a graph the events are
                             event-record nodes)                              */
  int32_t cand_ring_log2; /* each of the two candidate rings holds 2^n
                             entries of 16 bytes (default 26; 12..27).  A
                             chunk whose survivors overflow it is redone with
                             4x fewer tiles per launch (at most six times);
                             serving slices use chunks small enough for the
                             densest K                                        */
  int64_t mem_budget;     /* serving: device bytes for admitted units' tables
                             and the fixed serving buffers; 0 = half of the
                             device memory free at the first admission, at
                             most 8 GiB (see ap26_serve_submit)               */
  double wait_timeout_s;  /* limit of each host wait on the device (default
                             3600 s); beyond it the call returns
                             AP26_E_TIMEOUT, and the next call on the context
                             first waits for the abandoned work to finish     */
  int32_t tail_group;     /* primes a queued shift word advances per pass of
                             the tail stages                                  */
  int32_t batch_wave;     /* K-jobs per run of ap26_search_batch (default 512,
                             1..2048): a batch of any size runs as waves of
                             this many, so the report buffer and each device
                             wait stay bounded                                */
} ap26_opts;

/* One raw report: AP length k, difference multiplier K, first term, and the
 * sieve candidate n whose chain produced it (n orders reports the way the
 * reference's AVX2 search meets them; see ap26_sort_aps). */
typedef struct {
  int32_t k;
  int32_t K;
  int64_t first;
  int64_t n;
} ap26_ap;

typedef struct {
  int64_t candidates;   /* sieve survivors after the 7..23 filter; the
                           reference's "total n" (src/opencl/AP26.h:343)     */
  int64_t late_items;   /* shift words that reached the late sieve stage     */
  int64_t prp_tests;    /* base-2 SPRP tests run by the chain walk           */
  int64_t aps;          /* raw reports (k >= 10)                             */
  double device_ms;     /* CUDA-event time of the device work                */
  int32_t error_flags;  /* bit 0: candidate buffer overflow (retried), bit 1:
                           late buffer overflow (retried), bit 2: chain term
                           >= 2^62, bit 3: AP buffer overflow, bit 4: a chain
                           walk reached its 4096-test limit (corrupt data) */
  int32_t launches;     /* kernels launched for this call                    */
  double sieve_ms;      /* summed CUDA-event time of the sieve launches
                           (only with ap26_opts.profile = 1)                 */
  int64_t sieve_cells;  /* (lattice value, shift word) cells sieved          */
  int32_t sieve_launches;
  int32_t reserved;
  int64_t chain_walks;  /* candidates the chain walk took (equals candidates
                           when no candidate buffer overflowed)             */
} ap26_stats;

/* A work item: every searchable K in [kmin, kmax] at one SHIFT. */
typedef struct {
  int64_t id;
  int32_t kmin, kmax, shift, reserved;
} ap26_item;

typedef struct {
  int64_t id;
  int32_t status;       /* AP26_OK or an error code                          */
  int32_t n_aps;        /* raw reports of this item                          */
  int64_t first_ap;     /* index of its first report in the caller's array   */
  int64_t candidates;   /* sieve survivors over all its K                    */
  int32_t ks_searched;  /* K with will_search(K) true                        */
  int32_t result_hash;  /* the reference's result_hash after ReportSolution
                           of all the item's reports, starting from 0
                           (AP26.cpp:556-560), computed on the device        */
  double latency_ms;    /* serving: admission-to-completion wall time        */
} ap26_item_result;

/* ReportSolution (src/common/AP26.cpp:549-602) of one raw report, computed
 * on the device: the report's call and every call its split recursion makes
 * add first%1000 + len to the hash; pieces that pass the 9-base validation
 * (validate_ap26, AP26.cpp:513-543) with len >= 20 are solutions, in the
 * order the reference appends them to SOL-AP26.txt. */
#define AP26_FINAL_MAX_SOL 3
typedef struct {
  int64_t hash_add;     /* sum of first%1000 + len over all those calls      */
  int32_t status;       /* AP26_OK; AP26_E_INVALID: a piece is not even a
                           base-2 AP ("Computation error", AP26.cpp:569-574);
                           AP26_E_DOMAIN: a term outside [0, 2^62)
                           (AP26.cpp:529-533); AP26_E_ARG: k < 0, first <= 23
                           or K outside [1, AP26_KMAX_SAFE]; AP26_E_OVERFLOW:
                           k > 128 or more than AP26_FINAL_MAX_SOL solutions */
  int32_t n_sol;        /* solutions (len >= 20) in sol_len / sol_first       */
  int32_t sol_len[AP26_FINAL_MAX_SOL];
  int32_t reserved;
  int64_t sol_first[AP26_FINAL_MAX_SOL];
} ap26_final;

/* One line of SOL-AP26.txt: "len K first" (AP26.cpp:593). */
typedef struct {
  int32_t len;
  int32_t K;
  int64_t first;
} ap26_sol;

/* ---- library / context --------------------------------------------------- */
int ap26_version(void);
const char *ap26_strerror(int code);
/* Text of the last CUDA error / timeout seen by ctx ("" if none). */
const char *ap26_last_error(const ap26_ctx *ctx);

/* Creates a context on CUDA device `device` (replaces the OpenCL set-up and
 * buffer allocation of src/common/AP26.cpp:834-939). */
int ap26_create(int device, const ap26_opts *opts, ap26_ctx **out);
void ap26_destroy(ap26_ctx *ctx);
int ap26_get_opts(const ap26_ctx *ctx, ap26_opts *out);
/* Changes the options of a live context; the sieve variant is re-picked
 * from (dense_primes, warp_queue, block_threads, late_stage, tail_group),
 * zero fields keep their current values.  AP26_E_ARG if no compiled variant
 * matches, or while serving slices are queued. */
int ap26_set_opts(ap26_ctx *ctx, const ap26_opts *opts);
/* The compiled sieve variants (autotuner search space): fills up to cap
 * entries (dense_primes, warp_queue, block_threads, late_stage, tail_group)
 * and returns the total count. */
int ap26_list_variants(ap26_opts *out, int cap);

/* ---- the per-K search (plain GPU form) -----------------------------------
 * Replaces void SearchAP26(int K, int startSHIFT, int s_local, int compute)
 * (src/opencl/AP26.h:78, called at src/common/AP26.cpp:976) and
 * Search_avx2(K, SHIFT, ITER, K_COUNT, K_DONE) (src/cpu/cpuavx2.h:12).
 * Writes the raw reports of K into out[0..cap), sorted in the reference's
 * AVX2 order; *n_out = count.  The caller feeds them to ap26_report (or its
 * own ReportSolution).  K must satisfy ap26_will_search(K). */
int ap26_search_k(ap26_ctx *ctx, int K, int shift, ap26_ap *out, int cap,
                  int *n_out, ap26_stats *stats);

/* The whole per-K step of the reference's K loop (AP26.cpp:976, SearchAP26
 * followed by ReportSolution of every result) with the reporting done on
 * the device: *result_hash (in [0, 2e9]) is advanced exactly as the
 * reference's ReportSolution calls advance result_hash, and the solutions
 * (9-base valid, len >= 20) are written to sol[0..cap) in the order the
 * reference appends them to SOL-AP26.txt; *n_sol = count.
 * iter is the reference's ITER, the first of the 10 shift words to report:
 * 0 for a whole K; a checkpoint of the reference's CPU build holds 4 or 8
 * (written before its second and third 4-word pass, cpuavx2.cpp:860) with
 * the hash of the words before it, and iter = that ITER continues the K
 * exactly (any 0..9 is accepted).  Errors: AP26_E_INVALID / AP26_E_DOMAIN
 * where the reference exits (then *result_hash is unchanged),
 * AP26_E_CAPACITY (*n_sol holds the need). */
int ap26_search_k_sol(ap26_ctx *ctx, int K, int shift, int iter, int32_t *result_hash,
                      ap26_sol *sol, int cap, int *n_sol, ap26_stats *stats);

/* ap26_search_k_sol with progress at shift-word granularity, from per-word
 * hash sums the device keeps for every K-job: hash_at_word[w] (10 entries,
 * or NULL) is the value *result_hash has after ReportSolution of the reports
 * of shift words iter..w (for w < iter, the value passed in), and
 * sol_word[i] (cap entries, or NULL) is the shift word of the report SOL line
 * i came from.  The reference's CPU build checkpoints between its 4-word
 * passes (src/cpu/cpuavx2.cpp:858-861, write_state at AP26.cpp:360-390)
 * with ITER 4 and 8 and the hash of the words before: those states are
 * (K, 4, hash_at_word[3]) and (K, 8, hash_at_word[7]), and the SOL lines
 * written by then are the ones with sol_word < ITER, a prefix of sol. */
int ap26_search_k_sol_words(ap26_ctx *ctx, int K, int shift, int iter, int32_t *result_hash,
                            int32_t *hash_at_word, ap26_sol *sol, int32_t *sol_word, int cap,
                            int *n_sol, ap26_stats *stats);

/* ---- batched persistent form ----------------------------------------------
 * All searchable K of all items in one persistent work-stealing pipeline:
 * sieve tiles of every item share launches, survivors of every K share PRP
 * batches, and each run (set-up, chunks, chain walks, ReportSolution,
 * read-backs) is one CUDA-graph launch (ap26_opts.use_graphs).  A batch of
 * more than ap26_opts.batch_wave K-jobs runs as consecutive runs of that
 * many, so any batch size fits the report buffer and the wait limit.
 * Reports are grouped per item (res[i].first_ap, res[i].n_aps), inside an
 * item by K ascending, inside a K in AVX2 order.  No counterpart in the
 * reference: it replaces the per-K loop of AP26.cpp:957-982 when many
 * workunits run in one process. */
int ap26_search_batch(ap26_ctx *ctx, const ap26_item *items, int n_items,
                      ap26_ap *aps, int64_t ap_cap, int64_t *n_aps,
                      ap26_item_result *res, ap26_stats *stats);

/* ---- serving: continuous batching ------------------------------------------
 * No counterpart in the reference (BOINC hands out one workunit per
 * process).  A unit is every searchable K of an item.
 *
 * ap26_serve_submit admits a unit (its id unique among the units admitted and
 * not yet polled, AP26_E_ARG otherwise) while device memory allows, else
 * returns AP26_E_NOMEM: the unit holds one table per K on the device (the
 * K's sieve bitstrings and lattice order, 36,572 bytes) from admission to
 * completion, in a pool sized from
 * ap26_opts.mem_budget at the first admission, together with its checkpoint
 * slot (at most 1024 units at once).  Admission enqueues the unit's tables
 * and never waits for work already on the device.
 *
 * ap26_serve_step does not block: it takes in every finished slice and keeps
 * two slices queued on the device while admitted units have K left.  A slice
 * is up to 4 K-jobs drawn round-robin from the admitted units (each unit's K
 * in ascending order).  Units submitted while slices run join the next
 * slice that is built.  *active_units = admitted, unfinished units.
 * ap26_serve_wait blocks until the oldest queued slice has finished (or
 * max_wait_s passes: AP26_E_TIMEOUT, nothing lost).
 * ap26_serve_poll returns 1 and one finished unit (raw reports in the
 * reference's AVX2 order per K, result_hash computed on the device), or 0.
 *
 * Each unit keeps its running ReportSolution hash, survivor count and
 * checkpoint on the device; every slice reads its units' slots back in
 * stream order.  ap26_serve_checkpoint returns that checkpoint in the fields
 * of the reference's state file (ap26_write_state): every K below *K has
 * been searched (K from shift word *ITER on) and *result_hash is the
 * reference's result_hash at that point.  ap26_serve_submit_from admits a
 * unit that resumes from such a state; its result_hash then ends where the
 * uninterrupted unit's does, and its reports are those of the rest. */
int ap26_serve_submit(ap26_ctx *ctx, const ap26_item *item);
int ap26_serve_submit_from(ap26_ctx *ctx, const ap26_item *item, int K, int ITER,
                           int32_t result_hash);
int ap26_serve_step(ap26_ctx *ctx, int *active_units);
int ap26_serve_wait(ap26_ctx *ctx, double max_wait_s);
int ap26_serve_poll(ap26_ctx *ctx, ap26_item_result *res, ap26_ap *aps,
                    int64_t ap_cap, int64_t *n_aps);
int ap26_serve_checkpoint(ap26_ctx *ctx, int64_t id, int *kmin, int *kmax, int *shift,
                          int *K, int *ITER, int32_t *result_hash);
/* Device bytes the serving pool accounts for: held now (fixed buffers plus
 * admitted units' tables) and its size. */
int ap26_serve_memory(const ap26_ctx *ctx, int64_t *in_use, int64_t *budget);

/* ---- kernel-level entry points (parity and roofline measurements) -------- */
/* Sieve only, over n53 starts [q_begin, q_end) of K (0 <= q < 137375320):
 * candidate values n (unordered) into cand[0..cap); *n_cand = total.
 * Replaces the sieve kernel (src/opencl/kernels/sieve.cl:12-156). */
int ap26_sieve_range(ap26_ctx *ctx, int K, int shift, int64_t q_begin,
                     int64_t q_end, int64_t *cand, int64_t cap,
                     int64_t *n_cand, ap26_stats *stats);
/* Sieve survivor counts for nK values of K at one SHIFT (counts only), in
 * runs of at most ap26_opts.batch_wave K. */
int ap26_sieve_count(ap26_ctx *ctx, const int32_t *Ks, int nK, int shift,
                     int64_t *counts, ap26_stats *stats);
/* Base-2 strong-PRP verdicts (1 = probable prime) for odd N in (2, 2^63).
 * Replaces strong_prp (src/opencl/kernels/checkn.cl:59-122,
 * src/common/PrimeQ_x86.h:143-182). */
int ap26_sprp_batch(ap26_ctx *ctx, const uint64_t *N, int64_t count,
                    uint8_t *verdict, ap26_stats *stats);
/* strong_prp(a[i], N[i]) verdicts (src/common/PrimeQ_x86.h:143-182) for
 * the validation bases: a[i] in [2, 31] (AP26_E_ARG otherwise); verdict 0
 * for even N, N <= a or N >= 2^63. */
int ap26_sprp_bases(ap26_ctx *ctx, const uint64_t *N, const uint32_t *a, int64_t count,
                    uint8_t *verdict, ap26_stats *stats);
/* ReportSolution of n given raw reports on the device, one ap26_final each
 * (the same values the reference's recursion produces).  If result_hash is
 * not NULL and every report is AP26_OK, *result_hash (in [0, 2e9]) is
 * advanced by all of them; otherwise the first non-OK status is returned
 * and *result_hash is unchanged. */
int ap26_report_batch(ap26_ctx *ctx, const ap26_ap *raw, int64_t n, ap26_final *out,
                      int32_t *result_hash, ap26_stats *stats);
/* Chain walk for given candidates n of K (checkn.cl:128-206): k and first
 * per candidate (first undefined when k < 10). */
int ap26_chain_batch(ap26_ctx *ctx, int K, const int64_t *n, int64_t count,
                     int32_t *k_out, int64_t *first_out, ap26_stats *stats);

/* ---- allocation-free survivor counts --------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory: code under a host framework that owns the device's memory pool,
 * plugin hosts that forbid cudaMalloc/cudaFree (both synchronise the whole
 * device), or callers that must not fail on memory exhaustion mid-run.
 * Same result as ap26_sieve_count, but the caller passes DEVICE buffers it
 * already owns: d_Ks (nK K values) in, d_counts (nK survivor counts) out;
 * a K outside [1, AP26_KMAX_SAFE] gets -1.  The work is enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default) of `device`; counts are
 * valid once that stream reaches this point.
 * - Allocates nothing (no cudaMalloc/cudaFree, no context object): all
 *   scratch -- job descriptors, tables, counters -- lives in one
 *   file-scope device array of AP26_NOALLOC_SCRATCH_BYTES (2,349,440 bytes)
 *   that every GPU loading the library keeps until process exit.  At most
 *   AP26_NOALLOC_MAX_K values of K per call; more returns AP26_E_CAPACITY.
 *   An invalid K costs no sieve time.
 * - A CUDA error already pending in the calling thread when the call starts
 *   is neither returned as this call's own nor cleared: the call launches
 *   nothing and returns AP26_E_CUDA.
 * - The first call on a device sets that device up synchronously (looks up
 *   the array's device address, fills the constant tables), so it must come
 *   before any stream capture.
 * - Every call reuses the same array and clears what must start at zero;
 *   calls whose work overlaps on the GPU (other streams, other threads)
 *   race on it and must be serialised by the caller. */
#define AP26_NOALLOC_MAX_K 64
#define AP26_NOALLOC_SCRATCH_BYTES 2349440
int ap26_sieve_count_noalloc(int device, const int32_t *d_Ks, int nK, int shift,
                             int64_t *d_counts, void *stream);

/* Picks the sieve variant (dense_primes / warp_queue / block_threads /
 * late_stage) by timing every compiled one on 1/64 of K's lattice, then
 * chunk_tiles by timing the whole pipeline over K at each chunk size the
 * candidate rings hold, and stores them in the context.  K must be
 * searchable; not while serving slices are queued (AP26_E_ARG). */
int ap26_autotune(ap26_ctx *ctx, int K, int shift, ap26_opts *chosen);

/* Measured device peaks for the roofline: conflict-free shared-memory load
 * bandwidth (GB/s) and 32-bit integer multiply-add throughput (Tops/s). */
int ap26_probe_peaks(ap26_ctx *ctx, double *smem_gbs, double *int_tops);

/* ---- host services (no GPU) -------------------------------------------------
 * will_search: src/common/AP26.cpp:649-653. */
int ap26_will_search(int K);

/* ReportSolution (src/common/AP26.cpp:549-602): adds first%1000 + len to
 * *result_hash (reduced by 2e9), re-validates with 9 SPRP bases, splits
 * non-APs recursively, and appends "len K first\n" for valid APs with
 * len >= 20 to sol[0..sol_cap) (NUL-terminated, *sol_len updated).
 * Returns AP26_E_INVALID where the reference exits with "Computation
 * error", AP26_E_CAPACITY if sol is too small. */
int ap26_report(int32_t *result_hash, int len, int K, int64_t first,
                char *sol, int sol_cap, int *sol_len);

/* write_hash (AP26.cpp:295-357): 16 hex digits + NUL into out. */
int ap26_hash_hex(int kmin, int kmax, int32_t result_hash, char *out17);

/* Sorts reports of one K into the order the reference AVX2 search meets
 * them (4-word passes, lattice order, word, bit: src/cpu/cpuavx2.cpp:334-820). */
int ap26_sort_aps(ap26_ap *aps, int n, int shift);

/* A/B checkpoint files (AP26.cpp:360-476) in directory dir ("" = cwd).
 * write: alternates A/B as the reference does; read: returns 1 and fills
 * *K, *ITER, *result_hash, *last_trickle if a matching state exists. */
int ap26_write_state(const char *dir, int kmin, int kmax, int shift, int K,
                     int ITER, int32_t result_hash, double last_trickle,
                     int *write_a_next);
int ap26_read_state(const char *dir, int kmin, int kmax, int shift, int *K,
                    int *ITER, int32_t *result_hash, double *last_trickle,
                    int *write_a_next);

#ifdef __cplusplus
}
#endif
#endif /* AP26_H */
