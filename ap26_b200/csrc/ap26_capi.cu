// ap26_capi.cu -- C ABI of libap26.so: context, per-K search, batched
// persistent search, serving loop, kernel-level entry points.
//
// Replaces the reference's GPU host orchestration (ibethune/ap26,
// src/opencl/AP26.h:78-346 SearchAP26, src/common/AP26.cpp:834-939 set-up):
// one H2D of the K-job descriptors, a chunked chain of kernels on one
// stream (optionally replayed from a CUDA graph), one D2H of the raw reports.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/ap26.h"
#include "ap26_kernels.cuh"
#include "ap26_hostcore.h"

namespace ap26 {

// ---- per-job set-up kernel ----------------------------------------------------
// The reference's per-K constants (src/opencl/AP26.h:112-120, int64 split
// multiplications).
__device__ int kmul_mod(int64_t c, int K, int64_t *out) {
  *out = (c * (K % 17835) + ((c * 17835) % MOD) * (K / 17835)) % MOD;
  return 0;
}

// Bit j of prime p's bitstring, B_p[j] = OK_p[((j + SHIFT) * MOD) mod p], with
// OK_p[r] = 0 iff r = (jj * (STEP mod p)) mod p for some jj in [p-23, p]
// (MAKE_OK, src/cpu/cpusse2.cpp:32-36; setok.cl:79-81).  stinv = (STEP mod
// p)^-1 mod p, or 0 when p divides STEP.
__device__ __forceinline__ bool bstr_bit(int p, int stinv, int cm, int sh, int j) {
  const int r = (j + sh) % p * cm % p;
  if (!stinv) return r != 0;
  const int tt = r * stinv % p;
  return tt != 0 && tt < p - 23;
}

__device__ int step_inv(int K, int p) {     // (K * 23# mod p)^(p-2) mod p, or 0
  const int st = (int)(((int64_t)(K % p) * (int)(PRIM23 % p)) % p);
  if (!st) return 0;
  int e = p - 2, base = st, r = 1;
  while (e) { if (e & 1) r = r * base % p; base = base * base % p; e >>= 1; }
  return r;
}

// The sieve bitstrings of one (K, SHIFT), built by all threads of a block:
// the two pair bitstrings (bit j = B_61[j] & B_67[j], then B_71[j] &
// B_73[j]) and one bitstring per prime 4..82 at c_params[g].off.
__device__ void build_table(int K, int shift, uint32_t *tab) {
  for (int t = threadIdx.x; t < TABLE_WORDS; t += blockDim.x) {
    uint32_t word = 0;
    if (t < PAIR1_WORDS + PAIR2_WORDS) {
      const bool first = t < PAIR1_WORDS;
      const int p = first ? 61 : 71, q = first ? 67 : 73;
      const int ip = step_inv(K, p), iq = step_inv(K, q);
      const int cp = (int)(MOD % p), cq = (int)(MOD % q);
      const int j0 = (first ? t : t - PAIR1_WORDS) * 32;
      for (int u = 0; u < 32; u++)
        if (bstr_bit(p, ip, cp, shift % p, j0 + u) && bstr_bit(q, iq, cq, shift % q, j0 + u))
          word |= 1u << u;
    } else {
      int g = PAIR_PRIMES;
      while (g + 1 < NPRIMES && c_params[g + 1].off <= t) g++;
      const int p = c_params[g].p;
      const int stinv = step_inv(K, p), cm = (int)(MOD % p), sh = shift % p;
      const int j0 = (t - c_params[g].off) * 32;
      for (int u = 0; u < 32; u++)
        if (bstr_bit(p, stinv, cm, sh, j0 + u)) word |= 1u << u;
    }
    tab[t] = word;
  }
}

// The sorted lattice order of K, built by all threads of a block with
// ORDER_SMEM bytes of dynamic shared memory: the 12673 n53 starts of an n43
// value, index i = j43*667 + j47*29 + j53, ordered by (k1 / ORDER_BUCKET,
// k2, i) with k1 = (j43*d43 + j47*d47 + j53*d53) mod 4087 and k2 the same
// mod 5183 (d = S * MOD^-1 mod the pair's period): a bitonic sort of
// 16384 packed keys (18 key bits, 14 index bits; padding sorts last).
constexpr int ORDER_N = 16384;
constexpr size_t ORDER_SMEM = sizeof(uint32_t) * ORDER_N;
static_assert((PAIR1_P / ORDER_BUCKET + 1) * PAIR2_P < (1 << 18), "sort key fits 18 bits");

__device__ void build_order(int K, uint16_t *perm) {
  extern __shared__ uint32_t sk[];
  __shared__ int d[6];
  if (threadIdx.x == 0) {
    int64_t S[3];
    kmul_mod(PRES5, K, &S[0]);
    kmul_mod(PRES6, K, &S[1]);
    kmul_mod(PRES7, K, &S[2]);
    for (int x = 0; x < 3; x++) {
      d[x] = (int)(S[x] % PAIR1_P) * PAIR1_PARAM.A % PAIR1_P;
      d[3 + x] = (int)(S[x] % PAIR2_P) * PAIR2_PARAM.A % PAIR2_P;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < ORDER_N; i += blockDim.x) {
    uint32_t v = 0xffffffffu;
    if (i < N53_PER_N43) {
      const int j43 = i / 667, j47 = (i - j43 * 667) / 29, j53 = i - j43 * 667 - j47 * 29;
      const int k1 = (j43 * d[0] + j47 * d[1] + j53 * d[2]) % PAIR1_P;
      const int k2 = (j43 * d[3] + j47 * d[4] + j53 * d[5]) % PAIR2_P;
      v = ((uint32_t)((k1 / ORDER_BUCKET) * PAIR2_P + k2) << 14) | (uint32_t)i;
    }
    sk[i] = v;
  }
  __syncthreads();
  for (int k = 2; k <= ORDER_N; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < ORDER_N; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const uint32_t a = sk[i], b = sk[ixj];
          if ((a > b) == ((i & k) == 0)) { sk[i] = b; sk[ixj] = a; }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < N53_PER_N43; i += blockDim.x) perm[i] = (uint16_t)(sk[i] & 0x3fffu);
  __syncthreads();
}

// Block j: job j (256 threads, ORDER_SMEM dynamic shared memory).  Thread 0
// sets the reference's per-K constants; the block builds the job's
// bitstrings and lattice order in its block at KJob::table unless
// build_tables is 0 (a serving unit builds them once, at admission).
__global__ void setup_jobs_kernel(KJob *jobs, int njobs, uint32_t *tables, int build_tables) {
  const int j = blockIdx.x;
  if (j >= njobs) return;
  KJob &J = jobs[j];
  const int K = J.K;
  if (threadIdx.x == 0) {
    J.STEP = (int64_t)K * PRIM23;
    J.n0 = (N0 * (K % 17835) + ((N0 * 17835) % MOD) * (K / 17835) + N30) % MOD;
    kmul_mod(PRES2, K, &J.S31);
    kmul_mod(PRES3, K, &J.S37);
    kmul_mod(PRES4, K, &J.S41);
    kmul_mod(PRES5, K, &J.S43);
    kmul_mod(PRES6, K, &J.S47);
    kmul_mod(PRES7, K, &J.S53);
    kmul_mod(PRES8, K, &J.S59);
  }
  if (build_tables) {
    uint32_t *blk = tables + (size_t)J.table * JOB_TABLE_WORDS;
    build_table(K, J.shift, blk);
    build_order(K, reinterpret_cast<uint16_t *>(blk + TABLE_WORDS));
  }
}

// Chunk bookkeeping; `ring` selects the candidate ring this chunk fills.
__global__ void chunk_begin_kernel(DevState *st, int ring) {
  st->tile_next = st->chunk_begin;
  unsigned long long e = st->chunk_begin + st->chunk_size;
  st->tile_end = e < st->total_tiles ? e : st->total_tiles;
  st->cand_count[ring] = 0;
  st->chain_next[ring] = 0;
}

__global__ void chunk_end_kernel(DevState *st, long long cand_cap, int ring) {
  unsigned long long c = st->cand_count[ring];
  st->cand_total += c;
  if ((long long)c > cand_cap) st->err_flags |= ERR_CAND_OVERFLOW;
  st->chunk_begin += st->chunk_size;
}

// ---- peak probes: conflict-free LDS.128 stream and dependent-free IMAD chains ----
__global__ void smem_probe_kernel(int iters, unsigned *sink) {
  __shared__ uint4 buf[1024];
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) buf[i] = make_uint4(i, i * 3, i * 5, i * 7);
  __syncthreads();
  uint4 acc = make_uint4(0, 0, 0, 0);
  int idx = threadIdx.x & 1023;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      uint4 v = buf[(idx + u * 128) & 1023];
      acc.x ^= v.x; acc.y ^= v.y; acc.z ^= v.z; acc.w ^= v.w;
    }
    idx = (idx + 32) & 1023;
  }
  if ((acc.x ^ acc.y ^ acc.z ^ acc.w) == 0x12345678u) sink[0] = 1;
}

__global__ void int_probe_kernel(int iters, unsigned *sink) {
  uint32_t a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5,
           a6 = a0 + 6, a7 = a0 + 7;
  const uint32_t m = 0x9E3779B1u, c = blockIdx.x | 1;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      a0 = a0 * m + c; a1 = a1 * m + c; a2 = a2 * m + c; a3 = a3 * m + c;
      a4 = a4 * m + c; a5 = a5 * m + c; a6 = a6 * m + c; a7 = a7 * m + c;
    }
  }
  if ((a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7) == 0x12345678u) sink[0] = 1;
}

// ---- PRP microbenchmark kernel: verdicts of sprp2 over an array ----------------
__global__ void sprp_batch_kernel(const uint64_t *N, long long count, uint8_t *verdict,
                                  unsigned long long *squarings) {
  unsigned sq = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const uint64_t n = N[i];
    verdict[i] = (uint8_t)((n & 1) && n < (1ull << 63) ? sprp2(n, sq) : 0);
  }
  unsigned v = sq;
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(squarings, (unsigned long long)v);
}

// strong_prp(a, N) for explicit (N, a) pairs, a in [2, 31].
__global__ void sprp_bases_kernel(const uint64_t *N, const uint32_t *a, long long count,
                                  uint8_t *verdict) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const uint64_t n = N[i];
    const uint32_t b = a[i];
    unsigned sq = 0;
    bool v = false;
    if ((n & 1) && n > b && n < (1ull << 63)) v = b == 2 ? sprp2(n, sq) : sprp_base(b, n);
    verdict[i] = (uint8_t)v;
  }
}

// Chain walk for explicit candidates (kernel-level parity entry point).
__global__ void chain_explicit_kernel(const KJob *job, const int64_t *n, long long count,
                                      int32_t *k_out, int64_t *first_out, DevState *st) {
  unsigned tests = 0, sq = 0;
  const int64_t S = job->STEP;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    int k = 0;
    int64_t m = n[i] + S * 5;
    while (prp_term(st, m, tests, sq)) { k++; m += S; }
    if (k >= 10) {
      m = n[i] + S * 4;
      while (m > 0 && prp_term(st, m, tests, sq)) { k++; m -= S; }
    }
    k_out[i] = k;
    first_out[i] = m + S;
  }
}

// Argument blocks are only built through these, so no field can be left
// value-initialised (a null counter pointer would fault on the device).
static SieveArgs sieve_args(const KJob *jobs, int njobs, const uint32_t *tables, DevState *st,
                            Cand *cand, long long cand_cap, unsigned long long *job_counts,
                            int count_only, unsigned long long *cand_count) {
  SieveArgs a;
  a.jobs = jobs;
  a.njobs = njobs;
  a.tables = tables;
  a.st = st;
  a.cand = cand;
  a.cand_cap = cand_cap;
  a.job_counts = job_counts;
  a.count_only = count_only;
  a.cand_count = cand_count;
  return a;
}

static ChainArgs chain_args(const KJob *jobs, DevState *st, const Cand *cand, long long cand_cap,
                            APRec *aps, long long ap_cap, const unsigned long long *cand_count,
                            unsigned long long *chain_next) {
  ChainArgs a;
  a.chain_next = chain_next;
  a.jobs = jobs;
  a.st = st;
  a.cand = cand;
  a.cand_cap = cand_cap;
  a.aps = aps;
  a.ap_cap = ap_cap;
  a.cand_count = cand_count;
  return a;
}

// ---- sieve variants (autotuner candidates) --------------------------------------
struct SieveVariant {
  int G, R, SL, QCAP, LCAP, WARPS;
  void (*kernel)(SieveArgs);
  size_t smem() const {
    return sizeof(uint4) * (QCAP + LCAP) * WARPS + (size_t)table_bytes(G);
  }
};

#define AP26_VARIANT(G, R, SL, Q, L, W) \
  SieveVariant{G, R, SL, Q, L, W, sieve_kernel<G, R, SL, Q, L, W>}

// (dense primes, tail group, late stage, queue, late queue, warps per CTA)
static const SieveVariant kVariants[] = {
    AP26_VARIANT(22, 6, 52, 320, 96, 8),   // default
    AP26_VARIANT(22, 6, 52, 320, 96, 12),
    AP26_VARIANT(24, 8, 56, 320, 96, 8),
    AP26_VARIANT(20, 6, 44, 320, 96, 12),
    AP26_VARIANT(20, 4, 44, 320, 96, 8),
    AP26_VARIANT(16, 4, 44, 320, 96, 8),
    AP26_VARIANT(24, 4, 52, 320, 96, 8),
    AP26_VARIANT(28, 4, 52, 320, 96, 8),
    AP26_VARIANT(20, 4, 44, 384, 128, 8),
    AP26_VARIANT(24, 4, 52, 320, 96, 12),
    AP26_VARIANT(20, 4, 44, 320, 96, 4),
    AP26_VARIANT(20, 6, 48, 320, 96, 8),
    AP26_VARIANT(18, 6, 44, 320, 96, 8),
    AP26_VARIANT(22, 4, 52, 320, 96, 8),
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

}  // namespace ap26

using namespace ap26;

// ---- context --------------------------------------------------------------------
// A serving unit's state, kept on the device in the unit's slot: the running
// ReportSolution hash sum, survivor count and K-jobs finished, and the unit's
// checkpoint in the fields of the reference's state file (write_state,
// src/common/AP26.cpp:360-390): every K below K_next is searched, K_next from
// shift word iter on, and result_hash is the reference's result_hash there.
struct UnitState {
  unsigned long long hash_add;   // sum of first%1000 + len over the unit's reports so far
  unsigned long long candidates;
  int32_t ks_done;
  int32_t K_next;
  int32_t iter;
  int32_t result_hash;           // fold(h0, hash_add)
  int32_t h0;                    // result_hash the unit started from
  int32_t kmin, kmax, shift;
};
constexpr int kUnitSlots = 1024;

constexpr long long kMaxIntV = 2000000000;   // MAXINTV, AP26.cpp:88

// result_hash after adding `add` through ReportSolution calls, each of which
// adds first%1000 + len and subtracts MAXINTV when above it (AP26.cpp:556-560):
// for a start in [0, MAXINTV] the value stays in [0, MAXINTV], is congruent
// to the total and is 0 only for a zero total.
__host__ __device__ inline int32_t hash_fold(int32_t h0, unsigned long long add) {
  const unsigned long long total = (unsigned long long)h0 + add;
  if (total == 0) return 0;
  return (int32_t)((total - 1) % (unsigned long long)kMaxIntV + 1);
}

// After a serving slice (one block): each K-job's survivor count and
// ReportSolution hash sums go into its unit's slot (KJob::item holds the
// slot), then every touched slot's checkpoint advances past its finished K.
// A unit's K-jobs run in ascending K and a slice finishes all of its jobs,
// so the checkpoint K is the largest finished K + 1.
__global__ void unit_accumulate_kernel(const KJob *jobs, int njobs,
                                       const unsigned long long *job_counts,
                                       const unsigned long long *job_hash, UnitState *units,
                                       UnitState *snap, const DevState *st) {
  // a slice whose buffers overflowed has incomplete sums: it leaves the
  // units' state as it was (the host fails those units)
  const bool ok = !(st->err_flags & (ERR_CAND_OVERFLOW | ERR_AP_OVERFLOW));
  for (int j = threadIdx.x; ok && j < njobs; j += blockDim.x) {
    UnitState &u = units[jobs[j].item];
    unsigned long long h = 0;
    for (int w = 0; w < WORDS; w++) h += job_hash[j * WORDS + w];
    atomicAdd(&u.hash_add, h);
    atomicAdd(&u.candidates, job_counts[j]);
    atomicAdd(&u.ks_done, 1);
    atomicMax(&u.K_next, jobs[j].K + 1);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < njobs; j += blockDim.x) {
    UnitState &u = units[jobs[j].item];
    u.iter = 0;
    u.result_hash = hash_fold(u.h0, u.hash_add);
  }
  __syncthreads();
  // the slice's copy of each of its units' state, read back in stream order
  for (int j = threadIdx.x; j < njobs; j += blockDim.x) snap[j] = units[jobs[j].item];
}

// Admission of a serving unit: its slot's initial state (first launch only)
// and the sieve bitstrings of up to kAdmitMax of its K, one block per K,
// into the serving pool.  Everything travels as kernel parameters, so
// admission needs no staging buffer and no wait on work already queued.
constexpr int kAdmitMax = 448;
struct AdmitArgs {
  UnitState init;
  int32_t slot, write_init, shift, n;
  int32_t K[kAdmitMax];
  int32_t table[kAdmitMax];
};
static_assert(sizeof(AdmitArgs) <= 4000, "kernel parameters stay below 4 KB");

__global__ void admit_unit_kernel(const AdmitArgs a, UnitState *units, uint32_t *pool) {
  if (a.write_init && blockIdx.x == 0 && threadIdx.x == 0) units[a.slot] = a.init;
  if ((int)blockIdx.x < a.n) {
    uint32_t *blk = pool + (size_t)a.table[blockIdx.x] * JOB_TABLE_WORDS;
    build_table(a.K[blockIdx.x], a.shift, blk);
    build_order(a.K[blockIdx.x], reinterpret_cast<uint16_t *>(blk + TABLE_WORDS));
  }
}

// Device and pinned host buffers of one pipeline run: K-job descriptors and
// (unless a serving pool provides them) their tables, per-job counters and
// per-word hash sums, run state, raw reports and ReportSolution results.
struct JobSet {
  int cap = 0;                        // K-jobs
  long long ap_cap = 0;               // raw reports
  bool own_tables = true;             // tables here, job j's at index j
  KJob *d_jobs = nullptr, *h_jobs = nullptr;
  uint32_t *d_tables = nullptr;
  unsigned long long *d_job_counts = nullptr, *h_job_counts = nullptr;
  unsigned long long *d_job_hash = nullptr, *h_job_hash = nullptr;   // cap * WORDS
  DevState *d_st = nullptr, *h_st = nullptr;
  APRec *d_aps = nullptr, *h_aps = nullptr;
  FinRec *d_fin = nullptr, *h_fin = nullptr;
  cudaEvent_t t0 = nullptr, done = nullptr;   // around the run, on the main stream
  // shape of the run last enqueued into this set
  int njobs = 0;
  int chunk_tiles = 0;
  bool count_only = false;
  unsigned long long nchunks = 0, nprof = 0;
  int launches = 0;
};

// A cached CUDA graph of one whole run shape.
struct GraphEntry {
  long long key[7];
  cudaGraphExec_t exec;
  unsigned long long used;
};
constexpr size_t kMaxGraphs = 8;

struct ServeUnit {
  ap26_item item;
  std::vector<int> ks;           // searchable K of the unit still to search
  std::vector<int> tables;       // its tables in the serving pool, one per K of ks
  int iter0 = 0;                 // first shift word of ks[0] (a resumed unit)
  size_t next_k = 0;             // next K to put on the device
  int done_k = 0;                // host copy of the count, for scheduling
  int slot = -1;                 // its UnitState on the device
  std::vector<ap26_ap> aps;
  int status = AP26_OK;
  std::chrono::steady_clock::time_point t_submit;
  double latency_ms = 0;
  int64_t bytes = 0;             // device bytes it holds while admitted
  UnitState snap;                // its slot as of its last finished slice
};

// A serving slice in flight: its job set and, per job, the unit it serves.
struct Slice {
  JobSet set;
  std::vector<int64_t> unit_ids;   // per job
  UnitState *d_snap = nullptr, *h_snap = nullptr;   // per job: its unit's state after it
  bool busy = false;
  int rc = AP26_OK;
};

struct ap26_ctx {
  int device = 0;
  ap26_opts opts{};
  int variant = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;              // chain walks of the overlapped form
  cudaStream_t copy_stream = nullptr;          // read-backs of finished serving slices
  cudaEvent_t sieve_done[2] = {nullptr, nullptr}, chain_done[2] = {nullptr, nullptr};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int num_sms = 0, sieve_blocks = 0, chain_blocks = 0;
  JobSet main;                                 // every synchronous entry point
  Cand *d_cand[2] = {nullptr, nullptr};        // two candidate rings (overlapped form)
  long long cand_cap = 0;
  // graphs
  std::vector<GraphEntry> graphs;
  unsigned long long graph_clock = 0;
  std::vector<cudaEvent_t> prof_events;        // per-sieve-launch timing pairs
  // serving
  std::deque<ServeUnit> units;
  std::deque<ServeUnit> finished;
  Slice slices[2];
  std::deque<int> inflight;                    // slice indices, oldest first
  uint32_t *d_pool = nullptr;                  // serving units' tables
  int pool_tables = 0;
  std::vector<int> free_tables;
  int64_t bytes_in_use = 0;                    // device bytes held by admitted units
  int64_t serve_budget = 0;                    // pool + fixed serving buffers
  UnitState *d_units = nullptr;                // kUnitSlots serving-unit states
  std::vector<int> free_slots;
  std::string last_error;
  bool pending = false;        // a call timed out with its work still queued
};

// A call that gave up waiting (AP26_E_TIMEOUT) left its work queued, and its
// read-backs still target the pinned host mirrors: the next call that reuses
// them waits for that work first.
static void drain(ap26_ctx *ctx) {
  if (!ctx->pending) return;
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->stream2);
  ctx->pending = false;
}

static int cuda_fail(ap26_ctx *ctx, cudaError_t e, const char *what) {
  if (ctx) ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return AP26_E_CUDA;
}
#define CK(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

constexpr int kChainThreads = 256;   // chain_kernel block size

// Device buffer owned by one call of a kernel-level entry point: freed on
// every return path, the early CUDA-error returns of CK included.
template <typename T>
struct DevBuf {
  T *p = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * n); }
};

extern "C" int ap26_version(void) { return 10100; }

extern "C" const char *ap26_strerror(int code) {
  switch (code) {
    case AP26_OK: return "ok";
    case AP26_E_ARG: return "bad argument";
    case AP26_E_CAPACITY: return "output buffer too small";
    case AP26_E_CUDA: return "CUDA error";
    case AP26_E_DOMAIN: return "K or SHIFT outside the exact-arithmetic domain";
    case AP26_E_TIMEOUT: return "device wait timed out";
    case AP26_E_OVERFLOW: return "internal device buffer overflow";
    case AP26_E_NOMEM: return "device memory budget exceeded";
    case AP26_E_INVALID: return "computation error: AP is not even a base-2 PRP AP";
    case AP26_E_NODEV: return "no usable CUDA device";
    default: return "unknown error";
  }
}

extern "C" const char *ap26_last_error(const ap26_ctx *ctx) {
  return ctx ? ctx->last_error.c_str() : "";
}

// K-jobs per run of ap26_search_batch (ap26_opts.batch_wave): by default
// about 3 minutes of device time and at most a few hundred thousand raw
// reports (the main set holds 2^20); at most 2048 (about 12 minutes).
constexpr int kBatchWave = 512;
constexpr int kMaxBatchWave = 2048;

static int default_opts(ap26_opts *o) {
  if (!o->dense_primes) o->dense_primes = kVariants[0].G;
  if (!o->warp_queue) o->warp_queue = kVariants[0].QCAP;
  if (!o->block_threads) o->block_threads = kVariants[0].WARPS * 32;
  if (!o->late_stage) o->late_stage = kVariants[0].SL;
  if (!o->tail_group) o->tail_group = kVariants[0].R;
  if (!o->chunk_tiles) o->chunk_tiles = 131072;
  if (!o->use_graphs) o->use_graphs = 1;
  if (!o->cand_ring_log2) o->cand_ring_log2 = 26;
  if (!(o->wait_timeout_s > 0)) o->wait_timeout_s = 3600.0;
  if (o->batch_wave <= 0) o->batch_wave = kBatchWave;
  return 0;
}

static int pick_variant(const ap26_opts &o) {
  for (int i = 0; i < kNumVariants; i++) {
    const SieveVariant &v = kVariants[i];
    if (v.G == o.dense_primes && v.QCAP == o.warp_queue && v.WARPS * 32 == o.block_threads &&
        v.SL == o.late_stage && v.R == o.tail_group)
      return i;
  }
  return -1;
}

static void drop_graphs(ap26_ctx *ctx) {
  for (auto &g : ctx->graphs) cudaGraphExecDestroy(g.exec);
  ctx->graphs.clear();
}

static int set_variant(ap26_ctx *ctx, int vi) {
  const SieveVariant &v = kVariants[vi];
  CK(cudaFuncSetAttribute(v.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem()));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.kernel, v.WARPS * 32, v.smem()));
  if (per_sm < 1) per_sm = 1;
  ctx->variant = vi;
  ctx->sieve_blocks = ctx->num_sms * per_sm;
  ctx->opts.dense_primes = v.G;
  ctx->opts.warp_queue = v.QCAP;
  ctx->opts.block_threads = v.WARPS * 32;
  ctx->opts.late_stage = v.SL;
  ctx->opts.tail_group = v.R;
  drop_graphs(ctx);
  return AP26_OK;
}

static void jobset_free(JobSet &S) {
  cudaFree(S.d_jobs); cudaFree(S.d_tables); cudaFree(S.d_job_counts); cudaFree(S.d_job_hash);
  cudaFree(S.d_st); cudaFree(S.d_aps); cudaFree(S.d_fin);
  cudaFreeHost(S.h_jobs); cudaFreeHost(S.h_job_counts); cudaFreeHost(S.h_job_hash);
  cudaFreeHost(S.h_st); cudaFreeHost(S.h_aps); cudaFreeHost(S.h_fin);
  if (S.t0) cudaEventDestroy(S.t0);
  if (S.done) cudaEventDestroy(S.done);
  const long long ap_cap = S.ap_cap;
  const bool own = S.own_tables;
  S = JobSet();
  S.ap_cap = ap_cap;
  S.own_tables = own;
}

// Grows a job set to hold njobs K-jobs (its report capacity is fixed at the
// first allocation).  Cleared first: a failed allocation leaves no freed
// pointers behind for jobset_free to free again.
static int jobset_ensure(ap26_ctx *ctx, JobSet &S, int njobs) {
  if (njobs <= S.cap && S.d_st) return AP26_OK;
  const int cap = std::max(njobs, std::max(64, S.cap * 2));
  if (S.d_st) {
    drain(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    jobset_free(S);
    drop_graphs(ctx);   // graphs hold the old buffers' addresses
  }
  CK(cudaMalloc(&S.d_jobs, sizeof(KJob) * cap));
  if (S.own_tables) CK(cudaMalloc(&S.d_tables, sizeof(uint32_t) * JOB_TABLE_WORDS * (size_t)cap));
  CK(cudaMalloc(&S.d_job_counts, sizeof(unsigned long long) * cap));
  CK(cudaMalloc(&S.d_job_hash, sizeof(unsigned long long) * WORDS * cap));
  CK(cudaMalloc(&S.d_st, sizeof(DevState)));
  CK(cudaMalloc(&S.d_aps, sizeof(APRec) * S.ap_cap));
  CK(cudaMalloc(&S.d_fin, sizeof(FinRec) * S.ap_cap));
  CK(cudaMallocHost(&S.h_jobs, sizeof(KJob) * cap));
  CK(cudaMallocHost(&S.h_job_counts, sizeof(unsigned long long) * cap));
  CK(cudaMallocHost(&S.h_job_hash, sizeof(unsigned long long) * WORDS * cap));
  CK(cudaMallocHost(&S.h_st, sizeof(DevState)));
  CK(cudaMallocHost(&S.h_aps, sizeof(APRec) * S.ap_cap));
  CK(cudaMallocHost(&S.h_fin, sizeof(FinRec) * S.ap_cap));
  CK(cudaEventCreate(&S.t0));
  CK(cudaEventCreate(&S.done));
  S.cap = cap;
  return AP26_OK;
}

static unsigned long long job_hash_total(const JobSet &S, int j) {
  unsigned long long h = 0;
  for (int w = 0; w < WORDS; w++) h += S.h_job_hash[(size_t)j * WORDS + w];
  return h;
}

static int alloc_rings(ap26_ctx *ctx, int log2) {
  ctx->cand_cap = 1ll << log2;
  CK(cudaMalloc(&ctx->d_cand[0], sizeof(Cand) * ctx->cand_cap));
  CK(cudaMalloc(&ctx->d_cand[1], sizeof(Cand) * ctx->cand_cap));
  return AP26_OK;
}

extern "C" int ap26_create(int device, const ap26_opts *opts, ap26_ctx **out) {
  if (!out) return AP26_E_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
    return AP26_E_NODEV;
  ap26_ctx *ctx = new ap26_ctx();
  ctx->device = device;
  if (opts) ctx->opts = *opts;
  default_opts(&ctx->opts);
  ctx->main.ap_cap = 1ll << 20;
  int rc;
#define CKC(call)                                     \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) { rc = cuda_fail(ctx, e_, #call); goto fail; } \
  } while (0)
  {
    CKC(cudaSetDevice(device));
    cudaDeviceProp prop;
    CKC(cudaGetDeviceProperties(&prop, device));
    ctx->num_sms = prop.multiProcessorCount;
    // 16 blocks of 256 threads per SM: 0.3% faster on an 8-K batch than
    // 8 x 128 (1126.5 ms against 1130.1 ms); 4 x 128 was slower
    ctx->chain_blocks = prop.multiProcessorCount * 16;
    CKC(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CKC(cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking));
    CKC(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    CKC(cudaEventCreate(&ctx->ev0));
    CKC(cudaEventCreate(&ctx->ev1));
    for (int r = 0; r < 2; r++) {
      CKC(cudaEventCreateWithFlags(&ctx->sieve_done[r], cudaEventDisableTiming));
      CKC(cudaEventCreateWithFlags(&ctx->chain_done[r], cudaEventDisableTiming));
    }
    // constant tables
    uint16_t trip[NUM_TRIPLES];
    int nt = ap26h_triples(trip);
    if (nt != NUM_TRIPLES) { rc = AP26_E_ARG; goto fail; }
    CKC(cudaMemcpyToSymbol(c_triples, trip, sizeof(trip)));
    PrimeParam params[NPRIMES];
    for (int g = 0; g < NPRIMES; g++) params[g] = make_param(g);
    CKC(cudaMemcpyToSymbol(c_params, params, sizeof(params)));
    // the set-up kernels sort each K's lattice order in 64 KB of shared memory
    CKC(cudaFuncSetAttribute(setup_jobs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ORDER_SMEM));
    CKC(cudaFuncSetAttribute(admit_unit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ORDER_SMEM));
    // buffers
    if (ctx->opts.cand_ring_log2 < 12 || ctx->opts.cand_ring_log2 > 27 ||
        ctx->opts.batch_wave > kMaxBatchWave) {
      rc = AP26_E_ARG;
      goto fail;
    }
    if ((rc = alloc_rings(ctx, ctx->opts.cand_ring_log2)) != AP26_OK) goto fail;
    CKC(cudaMalloc(&ctx->d_units, sizeof(UnitState) * kUnitSlots));
    for (int i = kUnitSlots - 1; i >= 0; i--) ctx->free_slots.push_back(i);
    for (int i = 0; i < 2; i++) {
      ctx->slices[i].set.ap_cap = 1ll << 16;
      ctx->slices[i].set.own_tables = false;
    }
    if ((rc = jobset_ensure(ctx, ctx->main, 64)) != AP26_OK) goto fail;
    int vi = pick_variant(ctx->opts);
    if (vi < 0) { rc = AP26_E_ARG; goto fail; }
    if ((rc = set_variant(ctx, vi)) != AP26_OK) goto fail;
  }
  *out = ctx;
  return AP26_OK;
fail:
  ap26_destroy(ctx);
  return rc;
#undef CKC
}

extern "C" void ap26_destroy(ap26_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  drop_graphs(ctx);
  for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
  jobset_free(ctx->main);
  for (int i = 0; i < 2; i++) {
    jobset_free(ctx->slices[i].set);
    cudaFree(ctx->slices[i].d_snap);
    cudaFreeHost(ctx->slices[i].h_snap);
  }
  cudaFree(ctx->d_units);
  cudaFree(ctx->d_pool);
  cudaFree(ctx->d_cand[0]); cudaFree(ctx->d_cand[1]);
  for (int r = 0; r < 2; r++) {
    if (ctx->sieve_done[r]) cudaEventDestroy(ctx->sieve_done[r]);
    if (ctx->chain_done[r]) cudaEventDestroy(ctx->chain_done[r]);
  }
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

extern "C" int ap26_list_variants(ap26_opts *out, int cap) {
  for (int i = 0; i < kNumVariants && i < cap && out; i++) {
    memset(&out[i], 0, sizeof(ap26_opts));
    out[i].dense_primes = kVariants[i].G;
    out[i].warp_queue = kVariants[i].QCAP;
    out[i].block_threads = kVariants[i].WARPS * 32;
    out[i].late_stage = kVariants[i].SL;
    out[i].tail_group = kVariants[i].R;
  }
  return kNumVariants;
}

static bool serving_idle(const ap26_ctx *ctx) { return ctx->inflight.empty(); }

extern "C" int ap26_set_opts(ap26_ctx *ctx, const ap26_opts *opts) {
  if (!ctx || !opts) return AP26_E_ARG;
  ap26_opts o = ctx->opts;
  if (opts->dense_primes) o.dense_primes = opts->dense_primes;
  if (opts->warp_queue) o.warp_queue = opts->warp_queue;
  if (opts->block_threads) o.block_threads = opts->block_threads;
  if (opts->late_stage) o.late_stage = opts->late_stage;
  if (opts->tail_group) o.tail_group = opts->tail_group;
  if (opts->chunk_tiles) o.chunk_tiles = opts->chunk_tiles;
  if (opts->mem_budget) o.mem_budget = opts->mem_budget;
  if (opts->cand_ring_log2) o.cand_ring_log2 = opts->cand_ring_log2;
  if (opts->wait_timeout_s > 0) o.wait_timeout_s = opts->wait_timeout_s;
  if (opts->use_graphs) o.use_graphs = opts->use_graphs;
  if (opts->batch_wave) o.batch_wave = opts->batch_wave;
  o.profile = opts->profile;
  const int vi = pick_variant(o);
  if (vi < 0 || o.cand_ring_log2 < 12 || o.cand_ring_log2 > 27 || o.chunk_tiles < 1 ||
      o.batch_wave < 1 || o.batch_wave > kMaxBatchWave)
    return AP26_E_ARG;
  if (o.mem_budget != ctx->opts.mem_budget && ctx->d_pool) return AP26_E_ARG;
  if (!serving_idle(ctx)) return AP26_E_ARG;   // slices in flight use the rings
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  if (o.cand_ring_log2 != ctx->opts.cand_ring_log2) {
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream2));
    cudaFree(ctx->d_cand[0]);
    cudaFree(ctx->d_cand[1]);
    ctx->d_cand[0] = ctx->d_cand[1] = nullptr;
    drop_graphs(ctx);
    int rc = alloc_rings(ctx, o.cand_ring_log2);
    if (rc != AP26_OK) return rc;
  }
  ctx->opts = o;
  int rc = set_variant(ctx, vi);
  drop_graphs(ctx);
  return rc;
}

extern "C" int ap26_get_opts(const ap26_ctx *ctx, ap26_opts *out) {
  if (!ctx || !out) return AP26_E_ARG;
  *out = ctx->opts;
  return AP26_OK;
}

static bool k_in_domain(int K, int shift) {
  return K >= 1 && K <= AP26_KMAX_SAFE && shift >= 0 && shift <= AP26_SHIFT_MAX;
}

// Bounded host wait on an event: polls it, gives up after timeout_s.
static int wait_event(ap26_ctx *ctx, cudaEvent_t e, double timeout_s) {
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t q = cudaEventQuery(e);
    if (q == cudaSuccess) return AP26_OK;
    if (q != cudaErrorNotReady) return cuda_fail(ctx, q, "cudaEventQuery");
    double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > timeout_s) {
      ctx->last_error = "device wait exceeded the timeout";
      ctx->pending = true;
      return AP26_E_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 20 : 200));
  }
}

static int ensure_prof_events(ap26_ctx *ctx, unsigned long long n) {
  while ((unsigned long long)ctx->prof_events.size() < 2 * n) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    ctx->prof_events.push_back(e);
  }
  return AP26_OK;
}

// The whole run of S.h_jobs[0..njobs): H2D of the jobs and the run state,
// set-up, per chunk of chunk_tiles tiles chunk_begin -> sieve -> chain ->
// chunk_end (the chain walk of chunk c on the second stream while chunk c+1
// is sieved into the other candidate ring, when overlapped), ReportSolution
// of every raw report, and the read-back of the run state, per-job counts and
// per-word hash sums into the pinned mirrors.  Issued on ctx->stream (and
// stream2); with `capture` the profiling events become event-record nodes of
// the graph being captured.
static cudaError_t emit_run(ap26_ctx *ctx, JobSet &S, const uint32_t *tables, int build_tables,
                            bool two_streams, bool capture) {
  cudaStream_t s = ctx->stream;
  const SieveVariant &V = kVariants[ctx->variant];
  const int njobs = S.njobs;
  cudaError_t e;
#define EM(call) do { if ((e = (call)) != cudaSuccess) return e; } while (0)
  EM(cudaMemcpyAsync(S.d_jobs, S.h_jobs, sizeof(KJob) * njobs, cudaMemcpyHostToDevice, s));
  EM(cudaMemcpyAsync(S.d_st, S.h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
  EM(cudaMemsetAsync(S.d_job_counts, 0, sizeof(unsigned long long) * njobs, s));
  EM(cudaMemsetAsync(S.d_job_hash, 0, sizeof(unsigned long long) * WORDS * njobs, s));
  setup_jobs_kernel<<<njobs, 256, ORDER_SMEM, s>>>(S.d_jobs, njobs, const_cast<uint32_t *>(tables),
                                          build_tables);
  EM(cudaGetLastError());
  // ring r: candidate buffer d_cand[r] and its fill count DevState::cand_count[r]
  SieveArgs sa[2];
  ChainArgs ca[2];
  for (int r = 0; r < 2; r++) {
    sa[r] = sieve_args(S.d_jobs, njobs, tables, S.d_st, ctx->d_cand[r], ctx->cand_cap,
                       S.d_job_counts, S.count_only ? 1 : 0, &S.d_st->cand_count[r]);
    ca[r] = chain_args(S.d_jobs, S.d_st, ctx->d_cand[r], ctx->cand_cap, S.d_aps, S.ap_cap,
                       &S.d_st->cand_count[r], &S.d_st->chain_next[r]);
  }
  const unsigned flag = capture ? cudaEventRecordExternal : cudaEventRecordDefault;
  for (unsigned long long c = 0; c < S.nchunks; c++) {
    const int r = two_streams ? (int)(c & 1) : 0;
    // ring r is free once the chain walk of chunk c-2 has read it
    if (two_streams && c >= 2) EM(cudaStreamWaitEvent(s, ctx->chain_done[r], 0));
    chunk_begin_kernel<<<1, 1, 0, s>>>(S.d_st, r);
    if (c < S.nprof) EM(cudaEventRecordWithFlags(ctx->prof_events[2 * c], s, flag));
    V.kernel<<<ctx->sieve_blocks, V.WARPS * 32, V.smem(), s>>>(sa[r]);
    if (c < S.nprof) EM(cudaEventRecordWithFlags(ctx->prof_events[2 * c + 1], s, flag));
    if (two_streams) {
      chunk_end_kernel<<<1, 1, 0, s>>>(S.d_st, ctx->cand_cap, r);
      EM(cudaEventRecord(ctx->sieve_done[r], s));
      EM(cudaStreamWaitEvent(ctx->stream2, ctx->sieve_done[r], 0));
      chain_kernel<<<ctx->chain_blocks, kChainThreads, 0, ctx->stream2>>>(ca[r]);
      EM(cudaEventRecord(ctx->chain_done[r], ctx->stream2));
    } else {
      if (!S.count_only) chain_kernel<<<ctx->chain_blocks, kChainThreads, 0, s>>>(ca[r]);
      chunk_end_kernel<<<1, 1, 0, s>>>(S.d_st, ctx->cand_cap, r);
    }
    EM(cudaGetLastError());
  }
  if (two_streams) {   // the last chain walks finish before the reports are read
    EM(cudaStreamWaitEvent(s, ctx->chain_done[0], 0));
    if (S.nchunks > 1) EM(cudaStreamWaitEvent(s, ctx->chain_done[1], 0));
  }
  if (!S.count_only) {
    // ReportSolution of every report on the device (AP26.cpp:549-602)
    ReportArgs ra;
    ra.aps = S.d_aps;
    ra.count = &S.d_st->ap_count;
    ra.n = S.ap_cap;
    ra.jobs = S.d_jobs;
    ra.fin = S.d_fin;
    ra.job_hash = S.d_job_hash;
    report_kernel<<<ctx->num_sms * 2, REPORT_WARPS * 32, 0, s>>>(ra);
    EM(cudaGetLastError());
  }
  EM(cudaMemcpyAsync(S.h_st, S.d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  EM(cudaMemcpyAsync(S.h_job_counts, S.d_job_counts, sizeof(unsigned long long) * njobs,
                     cudaMemcpyDeviceToHost, s));
  if (!S.count_only)
    EM(cudaMemcpyAsync(S.h_job_hash, S.d_job_hash, sizeof(unsigned long long) * WORDS * njobs,
                       cudaMemcpyDeviceToHost, s));
#undef EM
  return cudaSuccess;
}

// Captures emit_run into a graph (on failure the stream leaves capture mode
// and the caller runs the work directly).
static cudaError_t capture_run(ap26_ctx *ctx, JobSet &S, const uint32_t *tables,
                               int build_tables, bool two_streams, cudaGraphExec_t *exec) {
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t em = emit_run(ctx, S, tables, build_tables, two_streams, true);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(ctx->stream, &g);
  if (em != cudaSuccess) e = em;
  if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();   // a failed capture leaves no error behind for later calls
  return e;
}

// Enqueues the run of S.h_jobs[0..njobs) and returns without waiting:
// S.done fires once the run state, counts and hash sums are in the pinned
// mirrors.  With opts.use_graphs the run is one CUDA-graph launch, captured
// once per run shape and replayed from the cache.
static int enqueue_jobs(ap26_ctx *ctx, JobSet &S, int njobs, bool count_only, bool overlap,
                        const uint32_t *tables = nullptr, int build_tables = 1,
                        bool record_done = true, int chunk_tiles = 0) {
  if (chunk_tiles <= 0) chunk_tiles = ctx->opts.chunk_tiles;
  int rc;
  if ((rc = jobset_ensure(ctx, S, njobs)) != AP26_OK) return rc;
  if (!tables) tables = S.d_tables;
  // tile prefix; a tile is one start per thread of the variant's CTA
  const SieveVariant &V = kVariants[ctx->variant];
  const int64_t tile_n53 = (int64_t)V.WARPS * 32;
  unsigned long long tiles = 0;
  for (int j = 0; j < njobs; j++) {
    KJob &J = S.h_jobs[j];
    const int64_t span = J.q_end - J.q_begin;
    J.ntiles = (int32_t)((span + tile_n53 - 1) / tile_n53);
    J.tile_begin = (int64_t)tiles;
    if (S.own_tables) J.table = j;
    tiles += (unsigned long long)J.ntiles;
  }
  memset(S.h_st, 0, sizeof(DevState));
  S.h_st->chunk_size = (unsigned long long)chunk_tiles;
  S.chunk_tiles = chunk_tiles;
  S.h_st->total_tiles = tiles;
  S.njobs = njobs;
  S.count_only = count_only;
  S.nchunks = tiles ? (tiles + chunk_tiles - 1) / chunk_tiles : 0;
  const bool two_streams = overlap && !count_only && S.nchunks > 1;
  // sieve launches timed with events: the first kProfChunks chunks at most
  constexpr unsigned long long kProfChunks = 4096;
  S.nprof = (ctx->opts.profile && &S == &ctx->main) ? std::min(S.nchunks, kProfChunks) : 0;
  if ((rc = ensure_prof_events(ctx, S.nprof)) != AP26_OK) return rc;
  S.launches = 1 + (int)S.nchunks * (count_only ? 3 : 4) + (count_only ? 0 : 1);
  CK(cudaEventRecord(S.t0, ctx->stream));
  bool launched = false;
  if (ctx->opts.use_graphs > 0) {
    const long long key[7] = {(long long)(uintptr_t)&S, ctx->variant, njobs,
                              (long long)S.nchunks, chunk_tiles,
                              (count_only ? 1 : 0) | (two_streams ? 2 : 0) | (build_tables ? 4 : 0) |
                                  ((long long)S.nprof << 3),
                              (long long)(uintptr_t)tables};
    GraphEntry *hit = nullptr;
    for (auto &g : ctx->graphs)
      if (!memcmp(g.key, key, sizeof(key))) hit = &g;
    if (!hit) {
      cudaGraphExec_t exec = nullptr;
      if (capture_run(ctx, S, tables, build_tables, two_streams, &exec) == cudaSuccess) {
        if (ctx->graphs.size() >= kMaxGraphs) {   // evict the least recently used
          auto lru = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                      [](const GraphEntry &a, const GraphEntry &b) {
                                        return a.used < b.used;
                                      });
          cudaGraphExecDestroy(lru->exec);
          ctx->graphs.erase(lru);
        }
        GraphEntry g;
        memcpy(g.key, key, sizeof(key));
        g.exec = exec;
        g.used = 0;
        ctx->graphs.push_back(g);
        hit = &ctx->graphs.back();
      }
    }
    if (hit) {
      hit->used = ++ctx->graph_clock;
      CK(cudaGraphLaunch(hit->exec, ctx->stream));
      launched = true;
    }
  }
  if (!launched) CK(emit_run(ctx, S, tables, build_tables, two_streams, false));
  if (record_done) CK(cudaEventRecord(S.done, ctx->stream));
  return AP26_OK;
}

// Reads back the reports of a finished run (S.done has fired) with one copy
// on `cs`, and fills stats.
static int collect_run(ap26_ctx *ctx, JobSet &S, cudaStream_t cs, ap26_stats *stats,
                       long long *n_aps_out) {
  long long n_aps = (long long)std::min<unsigned long long>(S.h_st->ap_count, S.ap_cap);
  if (n_aps > 0) {
    CK(cudaMemcpyAsync(S.h_aps, S.d_aps, sizeof(APRec) * n_aps, cudaMemcpyDeviceToHost, cs));
    if (!S.count_only)
      CK(cudaMemcpyAsync(S.h_fin, S.d_fin, sizeof(FinRec) * n_aps, cudaMemcpyDeviceToHost, cs));
    CK(cudaStreamSynchronize(cs));
  }
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    float ms = 0;
    cudaEventElapsedTime(&ms, S.t0, S.done);
    stats->candidates = (int64_t)S.h_st->cand_total;
    stats->late_items = (int64_t)S.h_st->late_items;
    stats->prp_tests = (int64_t)S.h_st->prp_tests;
    stats->chain_walks = (int64_t)S.h_st->chain_walks;
    stats->aps = (int64_t)S.h_st->ap_count;
    stats->device_ms = ms;
    stats->error_flags = (int32_t)S.h_st->err_flags;
    stats->launches = S.launches;
    int64_t n53 = 0;
    for (int j = 0; j < S.njobs; j++) n53 += S.h_jobs[j].q_end - S.h_jobs[j].q_begin;
    stats->sieve_cells = n53 * J59 * WORDS;
    stats->sieve_launches = (int32_t)S.nchunks;
    if (S.nprof) {
      if (S.nprof < S.nchunks) {
        // only the first nprof chunks were timed; all of them are full
        const int64_t tile_n53 = (int64_t)kVariants[ctx->variant].WARPS * 32;
        stats->sieve_cells = (int64_t)(S.nprof * (unsigned long long)S.chunk_tiles) *
                             tile_n53 * J59 * WORDS;
        stats->sieve_launches = (int32_t)S.nprof;
      }
      double sm = 0;
      for (unsigned long long c = 0; c < S.nprof; c++) {
        float t = 0;
        cudaEventElapsedTime(&t, ctx->prof_events[2 * c], ctx->prof_events[2 * c + 1]);
        sm += t;
      }
      stats->sieve_ms = sm;
    }
    if (S.count_only) {
      // count-only runs have no candidate buffer use: totals come from job counts
      unsigned long long tot = 0;
      for (int j = 0; j < S.njobs; j++) tot += S.h_job_counts[j];
      stats->candidates = (int64_t)tot;
    }
  }
  if (n_aps_out) *n_aps_out = n_aps;
  const unsigned err = S.h_st->err_flags;
  if (err & ERR_CHAIN_LIMIT) {
    ctx->last_error = "a chain walk reached its test limit (corrupt candidate data)";
    return AP26_E_CUDA;
  }
  if (!S.count_only && S.h_st->chain_check != 0) {
    ctx->last_error = "the chain walk did not take each candidate exactly once";
    return AP26_E_CUDA;
  }
  if (err & ERR_DOMAIN) {
    ctx->last_error = "chain term reached 2^62";
    return AP26_E_DOMAIN;
  }
  if (err & (ERR_CAND_OVERFLOW | ERR_AP_OVERFLOW)) {
    ctx->last_error = "device buffer overflow";
    return AP26_E_OVERFLOW;
  }
  return AP26_OK;
}

// Synchronous run on the main job set.
static int run_jobs(ap26_ctx *ctx, int njobs, bool count_only, ap26_stats *stats,
                    long long *n_aps_out, bool overlap = false) {
  int rc;
  drain(ctx);
  if ((rc = enqueue_jobs(ctx, ctx->main, njobs, count_only, overlap)) != AP26_OK) return rc;
  if ((rc = wait_event(ctx, ctx->main.done, ctx->opts.wait_timeout_s)) != AP26_OK) return rc;
  return collect_run(ctx, ctx->main, ctx->stream, stats, n_aps_out);
}

static void fill_job(KJob &J, int K, int shift, int item, int64_t q0, int64_t q1,
                     int word_begin = 0) {
  memset(&J, 0, sizeof(J));
  J.K = K;
  J.shift = shift;
  J.item = item;
  J.q_begin = q0;
  J.q_end = q1;
  J.word_begin = word_begin;
  J.flags = JOB_SORTED;
}

// Runs jobs, retrying with smaller chunks on a candidate-buffer overflow.
static int run_jobs_retry(ap26_ctx *ctx, int njobs, bool count_only, ap26_stats *stats,
                          long long *n_aps, bool overlap = false) {
  const int saved = ctx->opts.chunk_tiles;
  std::vector<KJob> keep(ctx->main.h_jobs, ctx->main.h_jobs + njobs);
  int rc = run_jobs(ctx, njobs, count_only, stats, n_aps, overlap);
  int tries = 0;
  while (rc == AP26_E_OVERFLOW && (ctx->main.h_st->err_flags & ERR_CAND_OVERFLOW) &&
         ctx->opts.chunk_tiles > 64 && tries < 6) {
    ctx->opts.chunk_tiles /= 4;
    memcpy(ctx->main.h_jobs, keep.data(), sizeof(KJob) * njobs);
    rc = run_jobs(ctx, njobs, count_only, stats, n_aps, overlap);
    if (stats) stats->error_flags |= 1;
    tries++;
  }
  ctx->opts.chunk_tiles = saved;
  return rc;
}

static void aprec_to_ap(const JobSet &S, const APRec &r, ap26_ap &a) {
  a.k = r.k;
  a.K = S.h_jobs[r.job].K;
  a.first = r.first;
  a.n = r.n;
}

static_assert(sizeof(FinRec) == sizeof(ap26_final) && FIN_MAX_SOL == AP26_FINAL_MAX_SOL &&
                  offsetof(FinRec, sol_first) == offsetof(ap26_final, sol_first),
              "FinRec mirrors ap26_final");
static_assert(sizeof(APRec) == sizeof(ap26_ap) && offsetof(APRec, first) == offsetof(ap26_ap, first),
              "APRec mirrors ap26_ap (job in place of K)");
static_assert(REP_INVALID == AP26_E_INVALID && REP_DOMAIN == AP26_E_DOMAIN &&
                  REP_ARG == AP26_E_ARG && REP_OVERFLOW == AP26_E_OVERFLOW,
              "report status codes are the public ones");

// A report with its ReportSolution result and AVX2 order key.
struct RepOut {
  ap26_ap ap;
  FinRec fin;
  uint64_t key;
  int word;
};

// Reports of a finished run, job index alongside.
static std::vector<std::pair<int, RepOut>> collect_reports(const JobSet &S, long long n) {
  std::vector<std::pair<int, RepOut>> v((size_t)n);
  for (long long i = 0; i < n; i++) {
    const APRec &r = S.h_aps[i];
    v[i].first = r.job;
    aprec_to_ap(S, r, v[i].second.ap);
    v[i].second.fin = S.h_fin[i];
    const int shift = S.h_jobs[r.job].shift;
    v[i].second.key = ap26h_order_key(v[i].second.ap.K, shift, r.n);
    const int t = (int)((uint64_t)r.n / (uint64_t)MOD) - shift;
    v[i].second.word = std::min(std::max(t >> 6, 0), WORDS - 1);
  }
  return v;
}

// The order ap26_sort_aps gives within one K: order key, first, k.
static bool rep_less(const RepOut &x, const RepOut &y) {
  if (x.ap.K != y.ap.K) return x.ap.K < y.ap.K;
  if (x.key != y.key) return x.key < y.key;
  if (x.ap.first != y.ap.first) return x.ap.first < y.ap.first;
  return x.ap.k < y.ap.k;
}

extern "C" int ap26_search_k(ap26_ctx *ctx, int K, int shift, ap26_ap *out, int cap,
                             int *n_out, ap26_stats *stats) {
  if (!ctx || !n_out || (cap > 0 && !out)) return AP26_E_ARG;
  if (!k_in_domain(K, shift)) return AP26_E_DOMAIN;
  if (!ap26_will_search(K)) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  int rc;
  if ((rc = jobset_ensure(ctx, ctx->main, 1)) != AP26_OK) return rc;
  fill_job(ctx->main.h_jobs[0], K, shift, 0, 0, N53_PER_K);
  long long n = 0;
  rc = run_jobs_retry(ctx, 1, false, stats, &n);
  if (rc != AP26_OK) return rc;
  *n_out = (int)n;
  if (n > cap) return AP26_E_CAPACITY;
  for (long long i = 0; i < n; i++) aprec_to_ap(ctx->main, ctx->main.h_aps[i], out[i]);
  ap26_sort_aps(out, (int)n, shift);
  return AP26_OK;
}

extern "C" int ap26_search_k_sol_words(ap26_ctx *ctx, int K, int shift, int iter,
                                       int32_t *result_hash, int32_t *hash_at_word,
                                       ap26_sol *sol, int32_t *sol_word, int cap, int *n_sol,
                                       ap26_stats *stats) {
  if (!ctx || !result_hash || !n_sol || cap < 0 || (cap > 0 && !sol)) return AP26_E_ARG;
  if (iter < 0 || iter >= WORDS) return AP26_E_ARG;
  if (*result_hash < 0 || *result_hash > kMaxIntV) return AP26_E_ARG;
  if (!k_in_domain(K, shift)) return AP26_E_DOMAIN;
  if (!ap26_will_search(K)) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  int rc;
  if ((rc = jobset_ensure(ctx, ctx->main, 1)) != AP26_OK) return rc;
  fill_job(ctx->main.h_jobs[0], K, shift, 0, 0, N53_PER_K, iter);
  long long n = 0;
  rc = run_jobs_retry(ctx, 1, false, stats, &n);
  if (rc != AP26_OK) return rc;
  auto v = collect_reports(ctx->main, n);
  std::sort(v.begin(), v.end(),
            [](const std::pair<int, RepOut> &x, const std::pair<int, RepOut> &y) {
              return rep_less(x.second, y.second);
            });
  int ns = 0;
  for (const auto &r : v) {
    if (r.second.fin.status != AP26_OK) {
      ctx->last_error = "ReportSolution failed for a report of K=" + std::to_string(K);
      return r.second.fin.status;
    }
    ns += r.second.fin.n_sol;
  }
  *n_sol = ns;
  if (ns > cap) return AP26_E_CAPACITY;
  int o = 0;
  for (const auto &r : v)
    for (int i = 0; i < r.second.fin.n_sol; i++) {
      sol[o].len = r.second.fin.sol_len[i];
      sol[o].K = K;
      sol[o].first = r.second.fin.sol_first[i];
      if (sol_word) sol_word[o] = r.second.word;
      o++;
    }
  // per-word progress: the hash after the reports of words iter..w
  unsigned long long acc = 0;
  for (int w = 0; w < WORDS; w++) {
    acc += ctx->main.h_job_hash[w];
    if (hash_at_word) hash_at_word[w] = w < iter ? *result_hash : hash_fold(*result_hash, acc);
  }
  *result_hash = hash_fold(*result_hash, job_hash_total(ctx->main, 0));
  return AP26_OK;
}

extern "C" int ap26_search_k_sol(ap26_ctx *ctx, int K, int shift, int iter,
                                 int32_t *result_hash, ap26_sol *sol, int cap, int *n_sol,
                                 ap26_stats *stats) {
  return ap26_search_k_sol_words(ctx, K, shift, iter, result_hash, nullptr, sol, nullptr, cap,
                                 n_sol, stats);
}

// ---- batched persistent form ------------------------------------------------------
// Sums the stats of consecutive runs of one call.
static void add_stats(ap26_stats &a, const ap26_stats &b) {
  a.candidates += b.candidates;
  a.late_items += b.late_items;
  a.prp_tests += b.prp_tests;
  a.aps += b.aps;
  a.device_ms += b.device_ms;
  a.error_flags |= b.error_flags;
  a.launches += b.launches;
  a.sieve_ms += b.sieve_ms;
  a.sieve_cells += b.sieve_cells;
  a.sieve_launches += b.sieve_launches;
  a.chain_walks += b.chain_walks;
}

extern "C" int ap26_search_batch(ap26_ctx *ctx, const ap26_item *items, int n_items,
                                 ap26_ap *aps, int64_t ap_cap, int64_t *n_aps,
                                 ap26_item_result *res, ap26_stats *stats) {
  if (!ctx || !items || n_items < 0 || !n_aps || !res) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  std::vector<std::pair<int, int>> jobs;   // (item, K)
  for (int i = 0; i < n_items; i++) {
    const ap26_item &it = items[i];
    if (it.kmax < it.kmin || !k_in_domain(it.kmin, it.shift) || !k_in_domain(it.kmax, it.shift))
      return AP26_E_DOMAIN;
    for (int K = it.kmin; K <= it.kmax; K++)
      if (ap26_will_search(K)) jobs.push_back({i, K});
  }
  // the K-jobs run in waves of at most opts.batch_wave: the report buffer
  // and each device wait stay bounded whatever the batch's size
  std::vector<std::vector<RepOut>> per_item(n_items);
  std::vector<unsigned long long> hash_add(n_items, 0);
  std::vector<int64_t> cand(n_items, 0);
  std::vector<int32_t> nks(n_items, 0);
  if (stats) memset(stats, 0, sizeof(*stats));
  const JobSet &S = ctx->main;
  const size_t wave = (size_t)ctx->opts.batch_wave;
  for (size_t w0 = 0; w0 < jobs.size(); w0 += wave) {
    const int nw = (int)std::min(wave, jobs.size() - w0);
    int rc;
    if ((rc = jobset_ensure(ctx, ctx->main, nw)) != AP26_OK) return rc;
    for (int j = 0; j < nw; j++) {
      const auto &jb = jobs[w0 + j];
      fill_job(ctx->main.h_jobs[j], jb.second, items[jb.first].shift, jb.first, 0, N53_PER_K);
    }
    long long n = 0;
    ap26_stats st;
    rc = run_jobs_retry(ctx, nw, false, stats ? &st : nullptr, &n, true);
    if (rc != AP26_OK) return rc;
    // reports grouped by item here, put in K and AVX2 order below
    for (auto &r : collect_reports(S, n)) per_item[S.h_jobs[r.first].item].push_back(r.second);
    for (int j = 0; j < nw; j++) {
      const int item = S.h_jobs[j].item;
      hash_add[item] += job_hash_total(S, j);
      cand[item] += (int64_t)S.h_job_counts[j];
      nks[item]++;
    }
    if (stats) add_stats(*stats, st);
  }
  int64_t total = 0;
  for (int i = 0; i < n_items; i++) {
    auto &v = per_item[i];
    std::sort(v.begin(), v.end(), rep_less);
    res[i].id = items[i].id;
    res[i].status = AP26_OK;
    for (const auto &r : v)
      if (r.fin.status != AP26_OK) { res[i].status = r.fin.status; break; }
    res[i].n_aps = (int32_t)v.size();
    res[i].first_ap = total;
    res[i].candidates = cand[i];
    res[i].ks_searched = nks[i];
    res[i].result_hash = hash_fold(0, hash_add[i]);
    res[i].latency_ms = 0;
    total += (int64_t)v.size();
  }
  *n_aps = total;
  if (total > ap_cap) return AP26_E_CAPACITY;
  for (int i = 0; i < n_items; i++)
    for (size_t e = 0; e < per_item[i].size(); e++) aps[res[i].first_ap + e] = per_item[i][e].ap;
  return AP26_OK;
}

// ---- serving: continuous batching ----------------------------------------------------
// Device memory a serving context holds.  Fixed: the two slices' job sets
// (descriptors, counters, hash sums, 2^16 reports each) and the unit slots;
// the candidate rings are the context's own and shared with every other
// form.  Per admitted unit: one table (the sieve bitstrings of one K) per
// searchable K still to search.  The pool of tables is allocated at the first
// admission, sized from opts.mem_budget (default: half of the device memory
// free at that moment, at most 8 GiB), so a unit is admitted only while its
// tables fit in memory the device really had.
constexpr int kSliceJobs = 4;          // K-jobs per serving slice

// Survivors per tile of 256 n53 starts: about 69 for a K that no sieve
// prime divides; a sieve prime p dividing K multiplies the density by
// (p-1)/(p-24) (one bad residue instead of 24), and at most four of them
// divide a K <= 4e8 (61*67*71*73*79 > 4e8), so at most 5.44 times: about
// 373.  A serving slice cannot be redone in smaller chunks without finishing
// after slices queued behind it, so its chunks are sized to this bound.
constexpr int kMaxSurvivorsPer256Tile = 400;

static int serve_chunk_tiles(const ap26_ctx *ctx) {
  const int64_t tile_n53 = (int64_t)kVariants[ctx->variant].WARPS * 32;
  const int64_t bound = ctx->cand_cap * 256 / (kMaxSurvivorsPer256Tile * tile_n53);
  return (int)std::max<int64_t>(64, std::min<int64_t>(ctx->opts.chunk_tiles, bound));
}
constexpr int64_t kTableBytes = (int64_t)JOB_TABLE_WORDS * 4;   // bitstrings + lattice order

static int64_t slice_set_bytes() {
  const int64_t jobs = 64;   // jobset_ensure's minimum capacity
  return jobs * ((int64_t)sizeof(KJob) + 8 + 8 * WORDS) + (int64_t)sizeof(DevState) +
         (1ll << 16) * (int64_t)(sizeof(APRec) + sizeof(FinRec));
}

static int serve_pool_init(ap26_ctx *ctx) {
  if (ctx->d_pool) return AP26_OK;
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  int64_t budget = ctx->opts.mem_budget;
  if (budget <= 0) budget = std::min<int64_t>((int64_t)(free_b / 2), (int64_t)8 << 30);
  budget = std::min<int64_t>(budget, (int64_t)free_b);
  const int64_t fixed = 2 * slice_set_bytes() + (int64_t)sizeof(UnitState) * kUnitSlots;
  const int64_t n = (budget - fixed) / kTableBytes;
  if (n < 1) {
    ctx->last_error = "serving memory budget below its fixed buffers";
    return AP26_E_NOMEM;
  }
  CK(cudaMalloc(&ctx->d_pool, (size_t)n * kTableBytes));
  ctx->pool_tables = (int)std::min<int64_t>(n, INT32_MAX);
  ctx->serve_budget = fixed + n * kTableBytes;
  ctx->bytes_in_use = fixed;
  ctx->free_tables.clear();
  for (int i = ctx->pool_tables - 1; i >= 0; i--) ctx->free_tables.push_back(i);
  for (int i = 0; i < 2; i++) {
    int rc = jobset_ensure(ctx, ctx->slices[i].set, kSliceJobs);
    if (rc != AP26_OK) return rc;
    CK(cudaMalloc(&ctx->slices[i].d_snap, sizeof(UnitState) * kSliceJobs));
    CK(cudaMallocHost(&ctx->slices[i].h_snap, sizeof(UnitState) * kSliceJobs));
  }
  return AP26_OK;
}

static int serve_admit(ap26_ctx *ctx, const ap26_item *item, int K_start, int iter,
                       int32_t h0) {
  if (!ctx || !item || item->kmax < item->kmin) return AP26_E_ARG;
  if (!k_in_domain(item->kmin, item->shift) || !k_in_domain(item->kmax, item->shift))
    return AP26_E_DOMAIN;
  if (iter < 0 || iter >= WORDS || h0 < 0 || h0 > kMaxIntV) return AP26_E_ARG;
  if (K_start < item->kmin || K_start > item->kmax + 1) return AP26_E_ARG;
  for (const auto &v : ctx->units)      // slices map their jobs back to units by id
    if (v.item.id == item->id) return AP26_E_ARG;
  for (const auto &v : ctx->finished)
    if (v.item.id == item->id) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  int rc;
  if ((rc = serve_pool_init(ctx)) != AP26_OK) return rc;
  ServeUnit u;
  u.item = *item;
  for (int K = K_start; K <= item->kmax; K++)
    if (ap26_will_search(K)) u.ks.push_back(K);
  u.iter0 = (!u.ks.empty() && u.ks[0] == K_start) ? iter : 0;
  u.bytes = (int64_t)u.ks.size() * kTableBytes;
  if (ctx->free_slots.empty() || u.ks.size() > ctx->free_tables.size()) {
    ctx->last_error = "serving memory budget exceeded";
    return AP26_E_NOMEM;
  }
  for (size_t i = 0; i < u.ks.size(); i++) {
    u.tables.push_back(ctx->free_tables.back());
    ctx->free_tables.pop_back();
  }
  u.slot = ctx->free_slots.back();
  ctx->free_slots.pop_back();
  ctx->bytes_in_use += u.bytes;
  // the unit's checkpoint and tables go to the device now, on the pipeline
  // stream, ahead of every slice that can use them
  UnitState &us = u.snap;
  memset(&us, 0, sizeof(us));
  us.K_next = K_start;
  us.iter = u.iter0;
  us.result_hash = h0;
  us.h0 = h0;
  us.kmin = item->kmin;
  us.kmax = item->kmax;
  us.shift = item->shift;
  size_t i = 0;
  do {
    AdmitArgs a;
    memset(&a, 0, sizeof(a));
    a.init = us;
    a.slot = u.slot;
    a.write_init = i == 0;
    a.shift = item->shift;
    a.n = (int)std::min<size_t>(kAdmitMax, u.ks.size() - i);
    for (int b = 0; b < a.n; b++) {
      a.K[b] = u.ks[i + b];
      a.table[b] = u.tables[i + b];
    }
    admit_unit_kernel<<<std::max(1, a.n), 256, ORDER_SMEM, ctx->stream>>>(a, ctx->d_units,
                                                                          ctx->d_pool);
    CK(cudaGetLastError());
    i += (size_t)a.n;
  } while (i < u.ks.size());
  u.t_submit = std::chrono::steady_clock::now();
  ctx->units.push_back(std::move(u));
  return AP26_OK;
}

extern "C" int ap26_serve_submit(ap26_ctx *ctx, const ap26_item *item) {
  if (!item) return AP26_E_ARG;
  return serve_admit(ctx, item, item->kmin, 0, 0);
}

extern "C" int ap26_serve_submit_from(ap26_ctx *ctx, const ap26_item *item, int K, int ITER,
                                      int32_t result_hash) {
  return serve_admit(ctx, item, K, ITER, result_hash);
}

static ServeUnit *find_unit(ap26_ctx *ctx, int64_t id) {
  for (auto &u : ctx->units)
    if (u.item.id == id) return &u;
  return nullptr;
}

// Folds a finished slice into its units: reports (host), progress.
static int harvest_slice(ap26_ctx *ctx, Slice &sl) {
  JobSet &S = sl.set;
  long long n = 0;
  int rc = sl.rc;
  if (rc == AP26_OK) rc = collect_run(ctx, S, ctx->copy_stream, nullptr, &n);
  std::vector<std::vector<RepOut>> per_job(S.njobs);
  if (rc == AP26_OK)
    for (auto &r : collect_reports(S, n)) per_job[r.first].push_back(r.second);
  for (int j = 0; j < S.njobs; j++) {
    ServeUnit *u = find_unit(ctx, sl.unit_ids[j]);
    if (!u) continue;
    if (rc != AP26_OK) {
      if (u->status == AP26_OK) u->status = rc;
      continue;
    }
    std::sort(per_job[j].begin(), per_job[j].end(), rep_less);
    for (const auto &r : per_job[j]) {
      u->aps.push_back(r.ap);
      if (r.fin.status != AP26_OK && u->status == AP26_OK) u->status = r.fin.status;
    }
    u->done_k++;
    // slices finish in order and this one holds the unit's latest state
    u->snap = sl.h_snap[j];
  }
  sl.busy = false;
  return rc;
}

// Builds and enqueues one slice: up to kSliceJobs K-jobs, one per admitted
// unit per round (round-robin), each unit's K in ascending order.
static int launch_slice(ap26_ctx *ctx, Slice &sl) {
  std::vector<std::pair<ServeUnit *, size_t>> picked;
  bool progress = true;
  while ((int)picked.size() < kSliceJobs && progress) {
    progress = false;
    for (auto &u : ctx->units) {
      if ((int)picked.size() >= kSliceJobs) break;
      if (u.status == AP26_OK && u.next_k < u.ks.size()) {
        picked.push_back({&u, u.next_k++});
        progress = true;
      }
    }
  }
  if (picked.empty()) return AP26_OK;
  JobSet &S = sl.set;
  int rc;
  if ((rc = jobset_ensure(ctx, S, (int)picked.size())) != AP26_OK) return rc;
  sl.unit_ids.clear();
  for (size_t j = 0; j < picked.size(); j++) {
    ServeUnit *u = picked[j].first;
    const size_t i = picked[j].second;
    fill_job(S.h_jobs[j], u->ks[i], u->item.shift, u->slot, 0, N53_PER_K, i == 0 ? u->iter0 : 0);
    S.h_jobs[j].table = u->tables[i];
    sl.unit_ids.push_back(u->item.id);
  }
  sl.busy = true;
  sl.rc = enqueue_jobs(ctx, S, (int)picked.size(), false, true, ctx->d_pool, 0, false,
                       serve_chunk_tiles(ctx));
  if (sl.rc == AP26_OK) {
    // the units' running sums and checkpoints stay on the device; the slice
    // reads back its units' states in stream order, then S.done fires
    unit_accumulate_kernel<<<1, 256, 0, ctx->stream>>>(S.d_jobs, S.njobs, S.d_job_counts,
                                                       S.d_job_hash, ctx->d_units, sl.d_snap,
                                                       S.d_st);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sl.h_snap, sl.d_snap, sizeof(UnitState) * S.njobs,
                          cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(S.done, ctx->stream);
    if (e != cudaSuccess) sl.rc = cuda_fail(ctx, e, "serving slice");
  }
  return sl.rc;
}

static void retire_units(ap26_ctx *ctx) {
  for (auto it = ctx->units.begin(); it != ctx->units.end();) {
    bool in_flight = false;
    for (int i : ctx->inflight)
      for (int64_t id : ctx->slices[i].unit_ids)
        if (id == it->item.id) in_flight = true;
    const bool done = it->done_k == (int)it->ks.size();
    if ((done || it->status != AP26_OK) && !in_flight) {
      it->latency_ms = std::chrono::duration<double, std::milli>(
                           std::chrono::steady_clock::now() - it->t_submit).count();
      for (int t : it->tables) ctx->free_tables.push_back(t);
      it->tables.clear();
      ctx->bytes_in_use -= it->bytes;
      ctx->finished.push_back(std::move(*it));
      it = ctx->units.erase(it);
    } else {
      ++it;
    }
  }
}

// Non-blocking: harvests every finished slice, then keeps two slices in
// flight while admitted units have K left.  Units submitted while slices run
// join the next slice that is built.
extern "C" int ap26_serve_step(ap26_ctx *ctx, int *active_units) {
  if (!ctx) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  int rc = AP26_OK;
  while (!ctx->inflight.empty()) {
    Slice &sl = ctx->slices[ctx->inflight.front()];
    cudaError_t q = cudaEventQuery(sl.set.done);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return cuda_fail(ctx, q, "cudaEventQuery");
    ctx->inflight.pop_front();
    int r = harvest_slice(ctx, sl);
    if (r != AP26_OK && rc == AP26_OK) rc = r;
  }
  while (ctx->inflight.size() < 2) {
    int idx = ctx->slices[0].busy ? 1 : 0;
    if (ctx->slices[idx].busy) break;
    int r = launch_slice(ctx, ctx->slices[idx]);
    if (!ctx->slices[idx].busy) break;   // nothing left to schedule
    ctx->inflight.push_back(idx);
    if (r != AP26_OK && rc == AP26_OK) rc = r;
  }
  retire_units(ctx);
  if (active_units) *active_units = (int)ctx->units.size();
  return rc;
}

// Blocks until the oldest slice in flight has finished (AP26_OK, also when
// none is in flight) or max_wait_s has passed (AP26_E_TIMEOUT, nothing lost).
extern "C" int ap26_serve_wait(ap26_ctx *ctx, double max_wait_s) {
  if (!ctx) return AP26_E_ARG;
  if (ctx->inflight.empty()) return AP26_OK;
  CK(cudaSetDevice(ctx->device));
  int rc = wait_event(ctx, ctx->slices[ctx->inflight.front()].set.done, max_wait_s);
  if (rc == AP26_E_TIMEOUT) ctx->pending = false;   // the slice is still tracked
  return rc;
}

extern "C" int ap26_serve_checkpoint(ap26_ctx *ctx, int64_t id, int *kmin, int *kmax,
                                     int *shift, int *K, int *ITER, int32_t *result_hash) {
  if (!ctx || !K || !ITER || !result_hash) return AP26_E_ARG;
  const ServeUnit *u = find_unit(ctx, id);
  if (!u)
    for (const auto &f : ctx->finished)
      if (f.item.id == id) u = &f;
  if (!u) return AP26_E_ARG;
  // the unit's device slot as its last finished slice read it back
  const UnitState &us = u->snap;
  if (kmin) *kmin = us.kmin;
  if (kmax) *kmax = us.kmax;
  if (shift) *shift = us.shift;
  *K = us.K_next;
  *ITER = us.iter;
  *result_hash = us.result_hash;
  return AP26_OK;
}

extern "C" int ap26_serve_poll(ap26_ctx *ctx, ap26_item_result *res, ap26_ap *aps,
                               int64_t ap_cap, int64_t *n_aps) {
  if (!ctx || !res || !n_aps) return AP26_E_ARG;
  if (ctx->finished.empty()) return 0;
  ServeUnit &u = ctx->finished.front();
  *n_aps = (int64_t)u.aps.size();
  if ((int64_t)u.aps.size() > ap_cap) return AP26_E_CAPACITY;
  // its last slice has finished and read its device slot back
  const UnitState &us = u.snap;
  if (!u.aps.empty()) memcpy(aps, u.aps.data(), sizeof(ap26_ap) * u.aps.size());
  res->id = u.item.id;
  res->status = u.status;
  if (res->status == AP26_OK && us.ks_done != u.done_k) {
    res->status = AP26_E_CUDA;       // the device record disagrees with the schedule
    ctx->last_error = "serving unit state on the device is inconsistent";
  }
  res->n_aps = (int32_t)u.aps.size();
  res->first_ap = 0;
  res->candidates = (int64_t)us.candidates;
  res->ks_searched = (int32_t)u.ks.size();
  res->result_hash = hash_fold(us.h0, us.hash_add);
  res->latency_ms = u.latency_ms;
  ctx->free_slots.push_back(u.slot);
  ctx->finished.pop_front();
  return 1;
}

extern "C" int ap26_serve_memory(const ap26_ctx *ctx, int64_t *in_use, int64_t *budget) {
  if (!ctx) return AP26_E_ARG;
  if (in_use) *in_use = ctx->bytes_in_use;
  if (budget) *budget = ctx->serve_budget;
  return AP26_OK;
}

// ---- kernel-level entry points ---------------------------------------------------------
extern "C" int ap26_sieve_range(ap26_ctx *ctx, int K, int shift, int64_t q_begin, int64_t q_end,
                                int64_t *cand, int64_t cap, int64_t *n_cand, ap26_stats *stats) {
  if (!ctx || !n_cand || q_begin < 0 || q_end > N53_PER_K || q_end < q_begin) return AP26_E_ARG;
  if (!k_in_domain(K, shift)) return AP26_E_DOMAIN;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  JobSet &S = ctx->main;
  int rc;
  if ((rc = jobset_ensure(ctx, S, 1)) != AP26_OK) return rc;
  // set-up and sieve only, in one launch over the whole range, candidates kept
  fill_job(S.h_jobs[0], K, shift, 0, q_begin, q_end);
  const int64_t tile_n53 = (int64_t)kVariants[ctx->variant].WARPS * 32;
  const int64_t tiles = (q_end - q_begin + tile_n53 - 1) / tile_n53;
  KJob &J = S.h_jobs[0];
  J.ntiles = (int32_t)tiles;
  J.tile_begin = 0;
  J.table = 0;
  J.flags = 0;   // natural lattice order: [q_begin, q_end) are the reference's positions
  memset(S.h_st, 0, sizeof(DevState));
  S.h_st->chunk_size = (unsigned long long)std::max<int64_t>(1, tiles);
  S.h_st->total_tiles = (unsigned long long)tiles;
  cudaStream_t s = ctx->stream;
  const SieveVariant &V = kVariants[ctx->variant];
  CK(cudaEventRecord(ctx->ev0, s));
  CK(cudaMemcpyAsync(S.d_jobs, S.h_jobs, sizeof(KJob), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(S.d_st, S.h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(S.d_job_counts, 0, sizeof(unsigned long long), s));
  setup_jobs_kernel<<<1, 256, ORDER_SMEM, s>>>(S.d_jobs, 1, S.d_tables, 1);
  chunk_begin_kernel<<<1, 1, 0, s>>>(S.d_st, 0);
  const SieveArgs sa = sieve_args(S.d_jobs, 1, S.d_tables, S.d_st, ctx->d_cand[0],
                                  ctx->cand_cap, S.d_job_counts, 0, &S.d_st->cand_count[0]);
  V.kernel<<<ctx->sieve_blocks, V.WARPS * 32, V.smem(), s>>>(sa);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(S.h_st, S.d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(ctx->ev1, s));
  rc = wait_event(ctx, ctx->ev1, ctx->opts.wait_timeout_s);
  if (rc != AP26_OK) return rc;
  const long long nc = (long long)S.h_st->cand_count[0];
  *n_cand = nc;
  if (nc > ctx->cand_cap) return AP26_E_OVERFLOW;
  if (nc > cap) return AP26_E_CAPACITY;
  if (nc > 0) {
    std::vector<Cand> tmp(nc);
    CK(cudaMemcpy(tmp.data(), ctx->d_cand[0], sizeof(Cand) * nc, cudaMemcpyDeviceToHost));
    for (long long i = 0; i < nc; i++) cand[i] = tmp[i].n;
  }
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    memset(stats, 0, sizeof(*stats));
    stats->candidates = nc;
    stats->late_items = (int64_t)S.h_st->late_items;
    stats->device_ms = ms;
    stats->error_flags = (int32_t)S.h_st->err_flags;
    stats->launches = 3;
  }
  return AP26_OK;
}

extern "C" int ap26_sieve_count(ap26_ctx *ctx, const int32_t *Ks, int nK, int shift,
                                int64_t *counts, ap26_stats *stats) {
  if (!ctx || !Ks || nK <= 0 || !counts) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  for (int i = 0; i < nK; i++)
    if (!k_in_domain(Ks[i], shift)) return AP26_E_DOMAIN;
  if (stats) memset(stats, 0, sizeof(*stats));
  // waves of at most opts.batch_wave K, as ap26_search_batch
  for (int w0 = 0; w0 < nK; w0 += ctx->opts.batch_wave) {
    const int nw = std::min(ctx->opts.batch_wave, nK - w0);
    int rc;
    if ((rc = jobset_ensure(ctx, ctx->main, nw)) != AP26_OK) return rc;
    for (int i = 0; i < nw; i++) fill_job(ctx->main.h_jobs[i], Ks[w0 + i], shift, i, 0, N53_PER_K);
    ap26_stats st;
    rc = run_jobs(ctx, nw, true, stats ? &st : nullptr, nullptr);
    if (rc != AP26_OK) return rc;
    for (int i = 0; i < nw; i++) counts[w0 + i] = (int64_t)ctx->main.h_job_counts[i];
    if (stats) add_stats(*stats, st);
  }
  return AP26_OK;
}

extern "C" int ap26_sprp_batch(ap26_ctx *ctx, const uint64_t *N, int64_t count, uint8_t *verdict,
                               ap26_stats *stats) {
  if (!ctx || !N || !verdict || count < 0) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  if (count == 0) return AP26_OK;
  DevBuf<uint64_t> dN;
  DevBuf<uint8_t> dV;
  DevBuf<unsigned long long> dsq;
  unsigned long long hsq = 0;
  CK(dN.alloc(count));
  CK(dV.alloc(count));
  CK(dsq.alloc(1));
  cudaStream_t s = ctx->stream;
  CK(cudaMemsetAsync(dsq.p, 0, sizeof(unsigned long long), s));
  CK(cudaMemcpyAsync(dN.p, N, sizeof(uint64_t) * count, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(ctx->ev0, s));
  sprp_batch_kernel<<<ctx->num_sms * 16, 256, 0, s>>>(dN.p, count, dV.p, dsq.p);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev1, s));
  CK(cudaMemcpyAsync(verdict, dV.p, count, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&hsq, dsq.p, sizeof(hsq), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->prp_tests = count;
    stats->device_ms = ms;
    stats->late_items = (int64_t)hsq;   // modular squarings performed
    stats->launches = 1;
  }
  return AP26_OK;
}

extern "C" int ap26_sprp_bases(ap26_ctx *ctx, const uint64_t *N, const uint32_t *a,
                               int64_t count, uint8_t *verdict, ap26_stats *stats) {
  if (!ctx || count < 0 || (count > 0 && (!N || !a || !verdict))) return AP26_E_ARG;
  for (int64_t i = 0; i < count; i++)
    if (a[i] < 2 || a[i] > 31) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  if (count == 0) return AP26_OK;
  DevBuf<uint64_t> dN;
  DevBuf<uint32_t> dA;
  DevBuf<uint8_t> dV;
  CK(dN.alloc(count));
  CK(dA.alloc(count));
  CK(dV.alloc(count));
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(dN.p, N, sizeof(uint64_t) * count, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dA.p, a, sizeof(uint32_t) * count, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(ctx->ev0, s));
  sprp_bases_kernel<<<ctx->num_sms * 16, 256, 0, s>>>(dN.p, dA.p, count, dV.p);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev1, s));
  CK(cudaMemcpyAsync(verdict, dV.p, count, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->prp_tests = count;
    stats->device_ms = ms;
    stats->launches = 1;
  }
  return AP26_OK;
}

extern "C" int ap26_report_batch(ap26_ctx *ctx, const ap26_ap *raw, int64_t n, ap26_final *out,
                                 int32_t *result_hash, ap26_stats *stats) {
  if (!ctx || n < 0 || (n > 0 && (!raw || !out))) return AP26_E_ARG;
  if (result_hash && (*result_hash < 0 || *result_hash > kMaxIntV)) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  if (n == 0) return AP26_OK;
  DevBuf<APRec> dR;
  DevBuf<FinRec> dF;
  CK(dR.alloc(n));
  CK(dF.alloc(n));
  cudaStream_t s = ctx->stream;
  // ap26_ap and APRec share a layout; with jobs == null the job field is K
  CK(cudaMemcpyAsync(dR.p, raw, sizeof(APRec) * n, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(ctx->ev0, s));
  ReportArgs ra;
  ra.aps = dR.p;
  ra.count = nullptr;
  ra.n = n;
  ra.jobs = nullptr;
  ra.fin = dF.p;
  ra.job_hash = nullptr;
  const long long want = (n + REPORT_WARPS - 1) / REPORT_WARPS;
  report_kernel<<<(int)std::min<long long>(want, ctx->num_sms * 8), REPORT_WARPS * 32, 0, s>>>(ra);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev1, s));
  CK(cudaMemcpyAsync(out, dF.p, sizeof(FinRec) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (stats) {
    stats->aps = n;
    stats->device_ms = ms;
    stats->launches = 1;
  }
  unsigned long long add = 0;
  for (int64_t i = 0; i < n; i++) {
    if (out[i].status != AP26_OK) return out[i].status;
    add += (unsigned long long)out[i].hash_add;
  }
  if (result_hash) *result_hash = hash_fold(*result_hash, add);
  return AP26_OK;
}

extern "C" int ap26_chain_batch(ap26_ctx *ctx, int K, const int64_t *n, int64_t count,
                                int32_t *k_out, int64_t *first_out, ap26_stats *stats) {
  if (!ctx || (count > 0 && (!n || !k_out || !first_out)) || count < 0) return AP26_E_ARG;
  if (!k_in_domain(K, 0)) return AP26_E_DOMAIN;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  if (count == 0) return AP26_OK;
  JobSet &S = ctx->main;
  int rc;
  if ((rc = jobset_ensure(ctx, S, 1)) != AP26_OK) return rc;
  fill_job(S.h_jobs[0], K, 0, 0, 0, 0);
  DevBuf<int64_t> dn, df;
  DevBuf<int32_t> dk;
  CK(dn.alloc(count));
  CK(df.alloc(count));
  CK(dk.alloc(count));
  cudaStream_t s = ctx->stream;
  memset(S.h_st, 0, sizeof(DevState));
  CK(cudaMemcpyAsync(S.d_jobs, S.h_jobs, sizeof(KJob), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(S.d_st, S.h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
  setup_jobs_kernel<<<1, 256, ORDER_SMEM, s>>>(S.d_jobs, 1, S.d_tables, 0);
  CK(cudaMemcpyAsync(dn.p, n, sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(ctx->ev0, s));
  chain_explicit_kernel<<<ctx->num_sms * 8, 128, 0, s>>>(S.d_jobs, dn.p, count, dk.p, df.p,
                                                         S.d_st);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev1, s));
  CK(cudaMemcpyAsync(k_out, dk.p, sizeof(int32_t) * count, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(first_out, df.p, sizeof(int64_t) * count, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(S.h_st, S.d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->device_ms = ms;
    stats->error_flags = (int32_t)S.h_st->err_flags;
    stats->launches = 2;
  }
  return (S.h_st->err_flags & ERR_DOMAIN) ? AP26_E_DOMAIN : AP26_OK;
}

extern "C" int ap26_probe_peaks(ap26_ctx *ctx, double *smem_gbs, double *int_tops) {
  if (!ctx) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  DevBuf<unsigned> sink;
  CK(sink.alloc(1));
  cudaStream_t s = ctx->stream;
  const int blocks = ctx->num_sms * 4, threads = 256;
  const int siters = 4096, iiters = 4096;
  float ms = 0;
  for (int rep = 0; rep < 2; rep++) {
    CK(cudaEventRecord(ctx->ev0, s));
    smem_probe_kernel<<<blocks, threads, 0, s>>>(siters, sink.p);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, s));
    CK(cudaEventSynchronize(ctx->ev1));
  }
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (smem_gbs) *smem_gbs = (double)blocks * threads * siters * 8 * 16 / (ms * 1e-3) / 1e9;
  for (int rep = 0; rep < 2; rep++) {
    CK(cudaEventRecord(ctx->ev0, s));
    int_probe_kernel<<<blocks, threads, 0, s>>>(iiters, sink.p);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, s));
    CK(cudaEventSynchronize(ctx->ev1));
  }
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  // one IMAD (a*m + c) per element per step: 8 * 16 per iteration
  if (int_tops) *int_tops = (double)blocks * threads * iiters * 8 * 16 / (ms * 1e-3) / 1e12;
  return AP26_OK;
}

// ---- autotuner -------------------------------------------------------------------------------
// Two stages.  (1) Every compiled sieve variant (dense primes, tail group,
// late stage, queue depth, CTA size) on the same slice of K's lattice, the
// first 1/64 of its starts, count-only in one launch, so only the sieve is
// timed.  (2) For the fastest variant, the whole pipeline (sieve, chain walk
// on the second stream, ReportSolution) over one whole K at each chunk size
// the candidate rings can hold: a chunk is the unit the chain walk overlaps
// and each chunk boundary drains the persistent sieve once.
extern "C" int ap26_autotune(ap26_ctx *ctx, int K, int shift, ap26_opts *chosen) {
  if (!ctx) return AP26_E_ARG;
  if (!k_in_domain(K, shift) || !ap26_will_search(K)) return AP26_E_DOMAIN;
  if (!serving_idle(ctx)) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  int rc;
  if ((rc = jobset_ensure(ctx, ctx->main, 1)) != AP26_OK) return rc;
  const int64_t q1 = N53_PER_K / 64;
  const int saved_chunk = ctx->opts.chunk_tiles;
  ctx->opts.chunk_tiles = 1 << 20;   // the slice in one launch
  double best_ms = 1e30;
  int best_v = ctx->variant;
  for (int vi = 0; vi < kNumVariants; vi++) {
    if ((rc = set_variant(ctx, vi)) != AP26_OK) return rc;
    double t = 0;
    for (int rep = 0; rep < 2; rep++) {
      fill_job(ctx->main.h_jobs[0], K, shift, 0, 0, q1);
      ap26_stats st;
      rc = run_jobs(ctx, 1, true, &st, nullptr);
      if (rc != AP26_OK) { ctx->opts.chunk_tiles = saved_chunk; return rc; }
      if (rep == 1) t = st.device_ms;   // first run warms up
    }
    if (t < best_ms) { best_ms = t; best_v = vi; }
  }
  if ((rc = set_variant(ctx, best_v)) != AP26_OK) return rc;
  // chunk sizes whose worst-case survivors (about 115 per tile) fit a ring
  const int tile_n53 = kVariants[best_v].WARPS * 32;
  int best_chunk = saved_chunk;
  best_ms = 1e30;
  for (int chunk = 32768; chunk <= (1 << 20); chunk *= 2) {
    if ((long long)chunk * 115 * tile_n53 / 256 > ctx->cand_cap) break;
    ctx->opts.chunk_tiles = chunk;
    fill_job(ctx->main.h_jobs[0], K, shift, 0, 0, N53_PER_K);
    ap26_stats st;
    long long n = 0;
    rc = run_jobs(ctx, 1, false, &st, &n, true);
    if (rc == AP26_E_OVERFLOW) break;
    if (rc != AP26_OK) { ctx->opts.chunk_tiles = saved_chunk; return rc; }
    if (st.device_ms < best_ms) { best_ms = st.device_ms; best_chunk = chunk; }
  }
  ctx->opts.chunk_tiles = best_chunk;
  drop_graphs(ctx);
  if (chosen) *chosen = ctx->opts;
  return AP26_OK;
}

// ---- allocation-free survivor counts ----------------------------------------------------
// For callers that may not allocate device memory themselves: code that runs
// under a host framework which owns the device's memory pool, plugin hosts
// that forbid cudaMalloc/cudaFree (both synchronise the device and stall
// work already queued by others), or callers that must not fail on memory
// exhaustion in the middle of a run.  Such a caller passes device buffers it
// already owns for the K list and the counts; every other byte this path
// touches lives in the file-scope array below, which every GPU that loads
// the library holds until the process exits.
namespace ap26 {
struct NoallocScratch {
  DevState st;
  KJob jobs[AP26_NOALLOC_MAX_K];
  unsigned long long counts[AP26_NOALLOC_MAX_K];
  uint32_t tables[AP26_NOALLOC_MAX_K][JOB_TABLE_WORDS];
};
static_assert(sizeof(NoallocScratch) == AP26_NOALLOC_SCRATCH_BYTES,
              "the scratch size stated in ap26.h");
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoallocScratch)];

// Fills the job descriptors and zeroes the counters and state left behind by
// the previous call (the array keeps the last call's contents).  A K outside
// [1, AP26_KMAX_SAFE] gets an empty lattice range, no tiles and a count of
// -1, so it costs the sieve nothing; the tile prefix skips it (find_job takes
// the last job whose first tile is <= the tile, which is never an empty one).
__global__ void noalloc_init_kernel(NoallocScratch *s, const int32_t *Ks, int nK, int shift,
                                    int tile_n53) {
  __shared__ int32_t s_tiles[AP26_NOALLOC_MAX_K];
  const int j = threadIdx.x;
  const int64_t ntiles = (N53_PER_K + tile_n53 - 1) / tile_n53;
  if (j < nK) {
    KJob &J = s->jobs[j];
    const int K = Ks[j];
    const bool ok = K >= 1 && K <= AP26_KMAX_SAFE;
    memset(&J, 0, sizeof(KJob));
    J.K = ok ? K : 1;
    J.shift = shift;
    J.item = ok ? 0 : -1;
    J.q_begin = 0;
    J.q_end = ok ? N53_PER_K : 0;
    J.ntiles = ok ? (int32_t)ntiles : 0;
    J.table = j;
    J.flags = JOB_SORTED;
    s_tiles[j] = J.ntiles;
    s->counts[j] = 0;
  }
  __syncthreads();
  if (j < nK) {
    int64_t begin = 0;
    for (int i = 0; i < j; i++) begin += s_tiles[i];
    s->jobs[j].tile_begin = begin;
  }
  if (j == 0) {
    int64_t total = 0;
    for (int i = 0; i < nK; i++) total += s_tiles[i];
    memset(&s->st, 0, sizeof(DevState));
    s->st.chunk_size = (unsigned long long)total;
    s->st.total_tiles = (unsigned long long)total;
  }
}

__global__ void noalloc_finish_kernel(const NoallocScratch *s, int nK, int64_t *out) {
  const int j = threadIdx.x;
  if (j < nK) out[j] = s->jobs[j].item < 0 ? -1 : (int64_t)s->counts[j];
}

struct NoallocDevice {
  NoallocScratch *ptr = nullptr;
  int sieve_blocks = 0;
  bool ready = false;
};
static NoallocDevice g_noalloc_dev[64];
static std::mutex g_noalloc_mu;

// Once per device, with that device current: the scratch array's device
// address (its host-side name is only a stand-in), the constant tables, and
// the launch shape of the default sieve variant.  Synchronous calls, so the
// first call on a device must come before any stream capture.
static int noalloc_setup(int device, NoallocDevice **out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocDevice &d = g_noalloc_dev[device];
  if (!d.ready) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return AP26_E_CUDA;
    uint16_t trip[NUM_TRIPLES];
    if (ap26h_triples(trip) != NUM_TRIPLES) return AP26_E_ARG;
    PrimeParam params[NPRIMES];
    for (int g = 0; g < NPRIMES; g++) params[g] = make_param(g);
    if (cudaMemcpyToSymbol(c_triples, trip, sizeof(trip)) != cudaSuccess) return AP26_E_CUDA;
    if (cudaMemcpyToSymbol(c_params, params, sizeof(params)) != cudaSuccess) return AP26_E_CUDA;
    if (cudaFuncSetAttribute(setup_jobs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ORDER_SMEM) != cudaSuccess)
      return AP26_E_CUDA;
    const SieveVariant &V = kVariants[0];
    if (cudaFuncSetAttribute(V.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)V.smem()) != cudaSuccess)
      return AP26_E_CUDA;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, V.kernel, V.WARPS * 32,
                                                      V.smem()) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
      return AP26_E_CUDA;
    d.ptr = static_cast<NoallocScratch *>(p);
    d.sieve_blocks = sms * (per_sm > 0 ? per_sm : 1);
    d.ready = true;
  }
  *out = &d;
  return AP26_OK;
}
}  // namespace ap26

// A launch error raised by this entry point's own launches: taken (and so
// cleared) here.  An error already pending before the first launch belongs
// to the caller's earlier work and is left untouched: the call returns
// AP26_E_CUDA without launching anything.
static bool noalloc_launch_failed() {
  if (cudaPeekAtLastError() == cudaSuccess) return false;
  cudaGetLastError();
  return true;
}

extern "C" int ap26_sieve_count_noalloc(int device, const int32_t *d_Ks, int nK, int shift,
                                        int64_t *d_counts, void *stream) {
  if (!d_Ks || !d_counts || nK < 1 || device < 0 || device >= 64) return AP26_E_ARG;
  if (nK > AP26_NOALLOC_MAX_K) return AP26_E_CAPACITY;
  if (shift < 0 || shift > AP26_SHIFT_MAX) return AP26_E_DOMAIN;
  if (cudaPeekAtLastError() != cudaSuccess) return AP26_E_CUDA;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return AP26_E_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return AP26_E_CUDA;
  NoallocDevice *d = nullptr;
  int rc = noalloc_setup(device, &d);
  if (rc == AP26_OK) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const SieveVariant &V = kVariants[0];
    NoallocScratch *S = d->ptr;
    do {
      noalloc_init_kernel<<<1, AP26_NOALLOC_MAX_K, 0, s>>>(S, d_Ks, nK, shift, V.WARPS * 32);
      if (noalloc_launch_failed()) { rc = AP26_E_CUDA; break; }
      setup_jobs_kernel<<<nK, 256, ORDER_SMEM, s>>>(S->jobs, nK, &S->tables[0][0], 1);
      if (noalloc_launch_failed()) { rc = AP26_E_CUDA; break; }
      chunk_begin_kernel<<<1, 1, 0, s>>>(&S->st, 0);
      if (noalloc_launch_failed()) { rc = AP26_E_CUDA; break; }
      const SieveArgs sa = sieve_args(S->jobs, nK, &S->tables[0][0], &S->st, nullptr, 0,
                                      S->counts, 1, &S->st.cand_count[0]);
      V.kernel<<<d->sieve_blocks, V.WARPS * 32, V.smem(), s>>>(sa);
      if (noalloc_launch_failed()) { rc = AP26_E_CUDA; break; }
      noalloc_finish_kernel<<<1, AP26_NOALLOC_MAX_K, 0, s>>>(S, nK, d_counts);
      if (noalloc_launch_failed()) { rc = AP26_E_CUDA; break; }
    } while (0);
  }
  if (prev != device) cudaSetDevice(prev);
  return rc;
}
