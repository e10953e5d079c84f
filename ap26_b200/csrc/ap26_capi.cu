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
// Thread 0: the reference's per-K constants (src/opencl/AP26.h:112-120, int64
// split multiplications).  All threads: the bitstrings
//   B_p[j] = OK_p[((j + SHIFT) * MOD) mod p],
// OK_p[r] = 0 iff r = (jj * (STEP mod p)) mod p for some jj in [p-23, p]
// (MAKE_OK, src/cpu/cpusse2.cpp:32-36; setok.cl:79-81).
__device__ int kmul_mod(int64_t c, int K, int64_t *out) {
  *out = (c * (K % 17835) + ((c * 17835) % MOD) * (K / 17835)) % MOD;
  return 0;
}

__global__ void setup_jobs_kernel(KJob *jobs, int njobs, uint32_t *tables) {
  const int j = blockIdx.x;
  if (j >= njobs) return;
  KJob &J = jobs[j];
  const int K = J.K, shift = J.shift;
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
  uint32_t *tab = tables + (size_t)j * TABLE_WORDS;
  for (int t = threadIdx.x; t < TABLE_WORDS; t += blockDim.x) {
    int g = 0;
    while (g + 1 < NPRIMES && c_params[g + 1].off <= t) g++;
    const int p = c_params[g].p;
    const int st = (int)(((int64_t)(K % p) * (int)(PRIM23 % p)) % p);
    int stinv = 0;
    if (st) {  // st^(p-2) mod p
      int e = p - 2, base = st, r = 1;
      while (e) { if (e & 1) r = r * base % p; base = base * base % p; e >>= 1; }
      stinv = r;
    }
    const int cm = (int)(MOD % p);
    const int sh = shift % p;
    const int j0 = (t - c_params[g].off) * 32;
    uint32_t word = 0;
    for (int u = 0; u < 32; u++) {
      const int x = (j0 + u + sh) % p;
      const int r = x * cm % p;
      bool bad;
      if (st == 0) bad = (r == 0);
      else { const int tt = r * stinv % p; bad = (tt == 0) || (tt >= p - 23); }
      if (!bad) word |= 1u << u;
    }
    tab[t] = word;
  }
}

// Chunk bookkeeping; `ring` selects the candidate ring this chunk fills.
__global__ void chunk_begin_kernel(DevState *st, int ring) {
  st->tile_next = st->chunk_begin;
  unsigned long long e = st->chunk_begin + st->chunk_size;
  st->tile_end = e < st->total_tiles ? e : st->total_tiles;
  st->cand_count[ring] = 0;
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
                            APRec *aps, long long ap_cap, const unsigned long long *cand_count) {
  ChainArgs a;
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
    return sizeof(uint4) * (QCAP + LCAP) * WARPS + 2 * sizeof(uint32_t) * TABLE_WORDS;
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
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

}  // namespace ap26

using namespace ap26;

// ---- context --------------------------------------------------------------------
// A serving unit's running state, kept on the device in the unit's slot:
// the partial ReportSolution hash sum, survivor count and K-jobs finished.
struct UnitState {
  unsigned long long hash_add;
  unsigned long long candidates;
  int32_t ks_done;
  int32_t pad;
};
constexpr int kUnitSlots = 1024;

// After a serving slice: each K-job's survivor count and ReportSolution hash
// sum go into its unit's slot (KJob::item holds the slot).
__global__ void unit_accumulate_kernel(const KJob *jobs, int njobs,
                                       const unsigned long long *job_counts,
                                       const unsigned long long *job_hash, UnitState *units) {
  for (int j = threadIdx.x; j < njobs; j += blockDim.x) {
    UnitState &u = units[jobs[j].item];
    atomicAdd(&u.hash_add, job_hash[j]);
    atomicAdd(&u.candidates, job_counts[j]);
    atomicAdd(&u.ks_done, 1);
  }
}

struct ServeUnit {
  ap26_item item;
  std::vector<int> ks;           // searchable K of the unit
  size_t next_k = 0;             // next K to put on the device
  int inflight = 0;              // K-jobs of this unit in the current slice
  int done_k = 0;                // host copy of the count, for scheduling
  int slot = -1;                 // its UnitState on the device
  std::vector<ap26_ap> aps;
  int status = AP26_OK;
  std::chrono::steady_clock::time_point t_submit;
  double latency_ms = 0;
};

struct ap26_ctx {
  int device = 0;
  ap26_opts opts{};
  int variant = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;              // chain walks of the overlapped form
  cudaEvent_t sieve_done[2] = {nullptr, nullptr}, chain_done[2] = {nullptr, nullptr};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int num_sms = 0, sieve_blocks = 0, chain_blocks = 0;
  // device buffers
  KJob *d_jobs = nullptr;
  uint32_t *d_tables = nullptr;
  unsigned long long *d_job_counts = nullptr;
  int jobs_cap = 0;
  DevState *d_st = nullptr;
  Cand *d_cand[2] = {nullptr, nullptr};   // two candidate rings (overlapped form)
  long long cand_cap = 0;
  APRec *d_aps = nullptr;
  long long ap_cap = 0;
  FinRec *d_fin = nullptr;                   // ReportSolution result per report
  unsigned long long *d_job_hash = nullptr;  // per-job sum of hash contributions
  // pinned host mirrors
  KJob *h_jobs = nullptr;
  DevState *h_st = nullptr;
  APRec *h_aps = nullptr;
  FinRec *h_fin = nullptr;
  unsigned long long *h_job_counts = nullptr, *h_job_hash = nullptr;
  // graphs
  cudaGraphExec_t chunk_graph = nullptr;
  long long graph_key = -1;
  std::vector<cudaEvent_t> prof_events;   // per-sieve-launch timing pairs
  // serving
  std::deque<ServeUnit> units;
  std::deque<ServeUnit> finished;
  int64_t bytes_in_use = 0;     // device bytes held by admitted serving units
  UnitState *d_units = nullptr; // kUnitSlots serving-unit states
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

extern "C" int ap26_version(void) { return 10000; }

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

static int default_opts(ap26_opts *o) {
  if (!o->dense_primes) o->dense_primes = kVariants[0].G;
  if (!o->warp_queue) o->warp_queue = kVariants[0].QCAP;
  if (!o->block_threads) o->block_threads = kVariants[0].WARPS * 32;
  if (!o->late_stage) o->late_stage = kVariants[0].SL;
  if (!o->chunk_tiles) o->chunk_tiles = 32768;
  if (!o->mem_budget) o->mem_budget = (int64_t)8 << 30;
  if (!o->cand_ring_log2) o->cand_ring_log2 = 23;
  if (!(o->wait_timeout_s > 0)) o->wait_timeout_s = 3600.0;
  return 0;
}

static int pick_variant(const ap26_opts &o) {
  for (int i = 0; i < kNumVariants; i++) {
    const SieveVariant &v = kVariants[i];
    if (v.G == o.dense_primes && v.QCAP == o.warp_queue && v.WARPS * 32 == o.block_threads &&
        v.SL == o.late_stage)
      return i;
  }
  return -1;
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
  if (ctx->chunk_graph) {
    cudaGraphExecDestroy(ctx->chunk_graph);
    ctx->chunk_graph = nullptr;
  }
  return AP26_OK;
}

static int ensure_jobs(ap26_ctx *ctx, int njobs) {
  if (njobs <= ctx->jobs_cap) return AP26_OK;
  int cap = std::max(njobs, std::max(64, ctx->jobs_cap * 2));
  const int64_t need = (int64_t)cap * (sizeof(KJob) + TABLE_WORDS * 4 + 8);
  if (cap > 64 && need > ctx->opts.mem_budget) return AP26_E_NOMEM;
  if (ctx->d_jobs) {
    drain(ctx);
    cudaFree(ctx->d_jobs); cudaFree(ctx->d_tables); cudaFree(ctx->d_job_counts);
    cudaFree(ctx->d_job_hash);
    cudaFreeHost(ctx->h_jobs); cudaFreeHost(ctx->h_job_counts); cudaFreeHost(ctx->h_job_hash);
    // cleared first: a failed allocation below must not leave freed pointers
    // for ap26_destroy to free again
    ctx->d_jobs = nullptr; ctx->d_tables = nullptr; ctx->d_job_counts = nullptr;
    ctx->d_job_hash = nullptr;
    ctx->h_jobs = nullptr; ctx->h_job_counts = nullptr; ctx->h_job_hash = nullptr;
    ctx->jobs_cap = 0;
  }
  CK(cudaMalloc(&ctx->d_jobs, sizeof(KJob) * cap));
  CK(cudaMalloc(&ctx->d_tables, sizeof(uint32_t) * TABLE_WORDS * (size_t)cap));
  CK(cudaMalloc(&ctx->d_job_counts, sizeof(unsigned long long) * cap));
  CK(cudaMalloc(&ctx->d_job_hash, sizeof(unsigned long long) * cap));
  CK(cudaMallocHost(&ctx->h_jobs, sizeof(KJob) * cap));
  CK(cudaMallocHost(&ctx->h_job_counts, sizeof(unsigned long long) * cap));
  CK(cudaMallocHost(&ctx->h_job_hash, sizeof(unsigned long long) * cap));
  ctx->jobs_cap = cap;
  if (ctx->chunk_graph) {
    cudaGraphExecDestroy(ctx->chunk_graph);
    ctx->chunk_graph = nullptr;
  }
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
    CKC(cudaEventCreate(&ctx->ev0));
    CKC(cudaEventCreate(&ctx->ev1));
    // constant tables
    uint16_t trip[NUM_TRIPLES];
    int nt = ap26h_triples(trip);
    if (nt != NUM_TRIPLES) { rc = AP26_E_ARG; goto fail; }
    CKC(cudaMemcpyToSymbol(c_triples, trip, sizeof(trip)));
    PrimeParam params[NPRIMES];
    for (int g = 0; g < NPRIMES; g++) params[g] = make_param(g);
    CKC(cudaMemcpyToSymbol(c_params, params, sizeof(params)));
    // buffers
    if (ctx->opts.cand_ring_log2 < 12 || ctx->opts.cand_ring_log2 > 26) {
      rc = AP26_E_ARG;
      goto fail;
    }
    ctx->cand_cap = 1ll << ctx->opts.cand_ring_log2;
    ctx->ap_cap = 1ll << 20;
    CKC(cudaMalloc(&ctx->d_st, sizeof(DevState)));
    CKC(cudaMalloc(&ctx->d_cand[0], sizeof(Cand) * ctx->cand_cap));
    CKC(cudaMalloc(&ctx->d_cand[1], sizeof(Cand) * ctx->cand_cap));
    CKC(cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking));
    for (int r = 0; r < 2; r++) {
      CKC(cudaEventCreateWithFlags(&ctx->sieve_done[r], cudaEventDisableTiming));
      CKC(cudaEventCreateWithFlags(&ctx->chain_done[r], cudaEventDisableTiming));
    }
    CKC(cudaMalloc(&ctx->d_aps, sizeof(APRec) * ctx->ap_cap));
    CKC(cudaMalloc(&ctx->d_units, sizeof(UnitState) * kUnitSlots));
    for (int i = kUnitSlots - 1; i >= 0; i--) ctx->free_slots.push_back(i);
    CKC(cudaMalloc(&ctx->d_fin, sizeof(FinRec) * ctx->ap_cap));
    CKC(cudaMallocHost(&ctx->h_fin, sizeof(FinRec) * ctx->ap_cap));
    CKC(cudaMallocHost(&ctx->h_st, sizeof(DevState)));
    CKC(cudaMallocHost(&ctx->h_aps, sizeof(APRec) * ctx->ap_cap));
    if ((rc = ensure_jobs(ctx, 64)) != AP26_OK) goto fail;
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
  if (ctx->chunk_graph) cudaGraphExecDestroy(ctx->chunk_graph);
  for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
  cudaFree(ctx->d_jobs); cudaFree(ctx->d_tables); cudaFree(ctx->d_job_counts);
  cudaFree(ctx->d_job_hash); cudaFree(ctx->d_fin); cudaFree(ctx->d_units);
  cudaFreeHost(ctx->h_job_hash); cudaFreeHost(ctx->h_fin);
  cudaFree(ctx->d_st); cudaFree(ctx->d_cand[0]); cudaFree(ctx->d_cand[1]); cudaFree(ctx->d_aps);
  for (int r = 0; r < 2; r++) {
    if (ctx->sieve_done[r]) cudaEventDestroy(ctx->sieve_done[r]);
    if (ctx->chain_done[r]) cudaEventDestroy(ctx->chain_done[r]);
  }
  if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
  cudaFreeHost(ctx->h_jobs); cudaFreeHost(ctx->h_job_counts);
  cudaFreeHost(ctx->h_st); cudaFreeHost(ctx->h_aps);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
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
  }
  return kNumVariants;
}

extern "C" int ap26_set_opts(ap26_ctx *ctx, const ap26_opts *opts) {
  if (!ctx || !opts) return AP26_E_ARG;
  ap26_opts o = ctx->opts;
  if (opts->dense_primes) o.dense_primes = opts->dense_primes;
  if (opts->warp_queue) o.warp_queue = opts->warp_queue;
  if (opts->block_threads) o.block_threads = opts->block_threads;
  if (opts->late_stage) o.late_stage = opts->late_stage;
  if (opts->chunk_tiles) o.chunk_tiles = opts->chunk_tiles;
  if (opts->mem_budget) o.mem_budget = opts->mem_budget;
  if (opts->cand_ring_log2) o.cand_ring_log2 = opts->cand_ring_log2;
  if (opts->wait_timeout_s > 0) o.wait_timeout_s = opts->wait_timeout_s;
  o.use_graphs = opts->use_graphs;
  o.profile = opts->profile;
  const int vi = pick_variant(o);
  if (vi < 0 || o.cand_ring_log2 < 12 || o.cand_ring_log2 > 26) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  if (o.cand_ring_log2 != ctx->opts.cand_ring_log2) {
    cudaFree(ctx->d_cand[0]);
    cudaFree(ctx->d_cand[1]);
    ctx->d_cand[0] = ctx->d_cand[1] = nullptr;
    ctx->cand_cap = 1ll << o.cand_ring_log2;
    CK(cudaMalloc(&ctx->d_cand[0], sizeof(Cand) * ctx->cand_cap));
    CK(cudaMalloc(&ctx->d_cand[1], sizeof(Cand) * ctx->cand_cap));
  }
  const int64_t keep_budget = o.mem_budget;
  ctx->opts = o;
  int rc = set_variant(ctx, vi);
  ctx->opts.mem_budget = keep_budget;
  if (ctx->chunk_graph) { cudaGraphExecDestroy(ctx->chunk_graph); ctx->chunk_graph = nullptr; }
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

// Bounded host wait on the stream: polls an event, gives up after timeout_s.
static int wait_stream(ap26_ctx *ctx, double timeout_s) {
  cudaEvent_t e = ctx->ev1;
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

// Enqueues the chunked pipeline for ctx->h_jobs[0..njobs) (K, shift, q range
// and item filled by the caller).  count_only: survivors are counted, no
// chain walk.  Returns after the D2H of state, counts and reports.
static int run_jobs(ap26_ctx *ctx, int njobs, bool count_only, ap26_stats *stats,
                    long long *n_aps_out, bool overlap = false) {
  int rc;
  drain(ctx);
  if ((rc = ensure_jobs(ctx, njobs)) != AP26_OK) return rc;
  // tile prefix; a tile is one start per thread of the variant's CTA
  const SieveVariant &V = kVariants[ctx->variant];
  const int64_t tile_n53 = (int64_t)V.WARPS * 32;
  unsigned long long tiles = 0;
  for (int j = 0; j < njobs; j++) {
    KJob &J = ctx->h_jobs[j];
    const int64_t span = J.q_end - J.q_begin;
    J.ntiles = (int32_t)((span + tile_n53 - 1) / tile_n53);
    J.tile_begin = (int64_t)tiles;
    tiles += (unsigned long long)J.ntiles;
  }
  memset(ctx->h_st, 0, sizeof(DevState));
  ctx->h_st->chunk_size = (unsigned long long)ctx->opts.chunk_tiles;
  ctx->h_st->total_tiles = tiles;
  cudaStream_t s = ctx->stream;
  CK(cudaEventRecord(ctx->ev0, s));
  CK(cudaMemcpyAsync(ctx->d_jobs, ctx->h_jobs, sizeof(KJob) * njobs, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->d_st, ctx->h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(ctx->d_job_counts, 0, sizeof(unsigned long long) * njobs, s));
  CK(cudaMemsetAsync(ctx->d_job_hash, 0, sizeof(unsigned long long) * njobs, s));
  setup_jobs_kernel<<<njobs, 256, 0, s>>>(ctx->d_jobs, njobs, ctx->d_tables);
  CK(cudaGetLastError());
  int launches = 1;
  // ring r: candidate buffer d_cand[r] and its fill count DevState::cand_count[r]
  SieveArgs sa[2];
  ChainArgs ca[2];
  for (int r = 0; r < 2; r++) {
    sa[r] = sieve_args(ctx->d_jobs, njobs, ctx->d_tables, ctx->d_st, ctx->d_cand[r],
                       ctx->cand_cap, ctx->d_job_counts, count_only ? 1 : 0,
                       &ctx->d_st->cand_count[r]);
    ca[r] = chain_args(ctx->d_jobs, ctx->d_st, ctx->d_cand[r], ctx->cand_cap, ctx->d_aps,
                       ctx->ap_cap, &ctx->d_st->cand_count[r]);
  }
  const unsigned long long nchunks =
      tiles ? (tiles + ctx->opts.chunk_tiles - 1) / ctx->opts.chunk_tiles : 0;
  // Overlapped form: the chain walk of chunk c runs on a second stream while
  // the sieve of chunk c+1 fills the other ring.
  const bool two_streams = overlap && !count_only && nchunks > 1;
  const bool use_graph = ctx->opts.use_graphs != 0 && !two_streams;
  const long long key = ((long long)ctx->variant << 40) | ((long long)(count_only ? 1 : 0) << 32) |
                        (long long)njobs;
  if (use_graph && (ctx->chunk_graph == nullptr || ctx->graph_key != key)) {
    if (ctx->chunk_graph) { cudaGraphExecDestroy(ctx->chunk_graph); ctx->chunk_graph = nullptr; }
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    chunk_begin_kernel<<<1, 1, 0, cs>>>(ctx->d_st, 0);
    V.kernel<<<ctx->sieve_blocks, V.WARPS * 32, V.smem(), cs>>>(sa[0]);
    if (!count_only) chain_kernel<<<ctx->chain_blocks, kChainThreads, 0, cs>>>(ca[0]);
    chunk_end_kernel<<<1, 1, 0, cs>>>(ctx->d_st, ctx->cand_cap, 0);
    cudaError_t ce = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&ctx->chunk_graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaGraphInstantiate");
    ctx->graph_key = key;
  }
  const bool prof = ctx->opts.profile != 0;
  // sieve launches timed with events: the first kProfChunks chunks at most
  constexpr unsigned long long kProfChunks = 4096;
  const unsigned long long nprof = prof ? std::min(nchunks, kProfChunks) : 0;
  if ((unsigned long long)ctx->prof_events.size() < 2 * nprof) {
    for (size_t i = ctx->prof_events.size(); i < 2 * nprof; i++) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      ctx->prof_events.push_back(e);
    }
  }
  for (unsigned long long c = 0; c < nchunks; c++) {
    const int r = two_streams ? (int)(c & 1) : 0;
    if (use_graph && !prof) {
      CK(cudaGraphLaunch(ctx->chunk_graph, s));
    } else {
      // ring r is free once the chain walk of chunk c-2 has read it
      if (two_streams && c >= 2) CK(cudaStreamWaitEvent(s, ctx->chain_done[r], 0));
      chunk_begin_kernel<<<1, 1, 0, s>>>(ctx->d_st, r);
      if (c < nprof) CK(cudaEventRecord(ctx->prof_events[2 * c], s));
      V.kernel<<<ctx->sieve_blocks, V.WARPS * 32, V.smem(), s>>>(sa[r]);
      if (c < nprof) CK(cudaEventRecord(ctx->prof_events[2 * c + 1], s));
      if (two_streams) {
        chunk_end_kernel<<<1, 1, 0, s>>>(ctx->d_st, ctx->cand_cap, r);
        CK(cudaEventRecord(ctx->sieve_done[r], s));
        CK(cudaStreamWaitEvent(ctx->stream2, ctx->sieve_done[r], 0));
        chain_kernel<<<ctx->chain_blocks, kChainThreads, 0, ctx->stream2>>>(ca[r]);
        CK(cudaEventRecord(ctx->chain_done[r], ctx->stream2));
      } else {
        if (!count_only) chain_kernel<<<ctx->chain_blocks, kChainThreads, 0, s>>>(ca[r]);
        chunk_end_kernel<<<1, 1, 0, s>>>(ctx->d_st, ctx->cand_cap, r);
      }
      CK(cudaGetLastError());
    }
    launches += count_only ? 3 : 4;
  }
  if (two_streams) {   // the last chain walks must finish before the read-back
    CK(cudaStreamWaitEvent(s, ctx->chain_done[0], 0));
    CK(cudaStreamWaitEvent(s, ctx->chain_done[1], 0));
  }
  if (!count_only) {
    // ReportSolution of every report on the device (AP26.cpp:549-602)
    ReportArgs ra;
    ra.aps = ctx->d_aps;
    ra.count = &ctx->d_st->ap_count;
    ra.n = ctx->ap_cap;
    ra.jobs = ctx->d_jobs;
    ra.fin = ctx->d_fin;
    ra.job_hash = ctx->d_job_hash;
    report_kernel<<<ctx->num_sms * 2, REPORT_WARPS * 32, 0, s>>>(ra);
    CK(cudaGetLastError());
    launches++;
  }
  CK(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ctx->h_job_counts, ctx->d_job_counts, sizeof(unsigned long long) * njobs,
                     cudaMemcpyDeviceToHost, s));
  if (!count_only)
    CK(cudaMemcpyAsync(ctx->h_job_hash, ctx->d_job_hash, sizeof(unsigned long long) * njobs,
                       cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(ctx->ev1, s));
  if ((rc = wait_stream(ctx, ctx->opts.wait_timeout_s)) != AP26_OK) return rc;
  long long n_aps = (long long)std::min<unsigned long long>(ctx->h_st->ap_count, ctx->ap_cap);
  if (n_aps > 0) {
    CK(cudaMemcpyAsync(ctx->h_aps, ctx->d_aps, sizeof(APRec) * n_aps, cudaMemcpyDeviceToHost, s));
    if (!count_only)
      CK(cudaMemcpyAsync(ctx->h_fin, ctx->d_fin, sizeof(FinRec) * n_aps, cudaMemcpyDeviceToHost,
                         s));
    CK(cudaStreamSynchronize(s));
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->candidates = (int64_t)ctx->h_st->cand_total;
    stats->late_items = (int64_t)ctx->h_st->late_items;
    stats->prp_tests = (int64_t)ctx->h_st->prp_tests;
    stats->aps = (int64_t)ctx->h_st->ap_count;
    stats->device_ms = ms;
    stats->error_flags = (int32_t)ctx->h_st->err_flags;
    stats->launches = launches;
    int64_t n53 = 0;
    for (int j = 0; j < njobs; j++) n53 += ctx->h_jobs[j].q_end - ctx->h_jobs[j].q_begin;
    stats->sieve_cells = n53 * J59 * WORDS;
    stats->sieve_launches = (int32_t)nchunks;
    if (prof) {
      if (nprof < nchunks) {
        // only the first nprof chunks were timed; all of them are full
        stats->sieve_cells = (int64_t)(nprof * (unsigned long long)ctx->opts.chunk_tiles) *
                             tile_n53 * J59 * WORDS;
        stats->sieve_launches = (int32_t)nprof;
      }
      double sm = 0;
      for (unsigned long long c = 0; c < nprof; c++) {
        float t = 0;
        cudaEventElapsedTime(&t, ctx->prof_events[2 * c], ctx->prof_events[2 * c + 1]);
        sm += t;
      }
      stats->sieve_ms = sm;
    }
  }
  if (count_only) {
    // count-only runs have no candidate buffer use: totals come from job counts
    unsigned long long tot = 0;
    for (int j = 0; j < njobs; j++) tot += ctx->h_job_counts[j];
    if (stats) stats->candidates = (int64_t)tot;
  }
  if (n_aps_out) *n_aps_out = n_aps;
  const unsigned err = ctx->h_st->err_flags;
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

static void fill_job(KJob &J, int K, int shift, int item, int64_t q0, int64_t q1,
                     int word_begin = 0) {
  memset(&J, 0, sizeof(J));
  J.K = K;
  J.shift = shift;
  J.item = item;
  J.q_begin = q0;
  J.q_end = q1;
  J.word_begin = word_begin;
}

// Runs jobs, retrying with smaller chunks on a candidate-buffer overflow.
static int run_jobs_retry(ap26_ctx *ctx, int njobs, bool count_only, ap26_stats *stats,
                          long long *n_aps, bool overlap = false) {
  const int saved = ctx->opts.chunk_tiles;
  std::vector<KJob> keep(ctx->h_jobs, ctx->h_jobs + njobs);
  int rc = run_jobs(ctx, njobs, count_only, stats, n_aps, overlap);
  int tries = 0;
  while (rc == AP26_E_OVERFLOW && (ctx->h_st->err_flags & ERR_CAND_OVERFLOW) &&
         ctx->opts.chunk_tiles > 64 && tries < 6) {
    ctx->opts.chunk_tiles /= 4;
    if (ctx->chunk_graph) { cudaGraphExecDestroy(ctx->chunk_graph); ctx->chunk_graph = nullptr; }
    memcpy(ctx->h_jobs, keep.data(), sizeof(KJob) * njobs);
    rc = run_jobs(ctx, njobs, count_only, stats, n_aps, overlap);
    if (stats) stats->error_flags |= 1;
    tries++;
  }
  if (ctx->opts.chunk_tiles != saved) {
    ctx->opts.chunk_tiles = saved;
    if (ctx->chunk_graph) { cudaGraphExecDestroy(ctx->chunk_graph); ctx->chunk_graph = nullptr; }
  }
  return rc;
}

static void aprec_to_ap(const ap26_ctx *ctx, const APRec &r, ap26_ap &a) {
  a.k = r.k;
  a.K = ctx->h_jobs[r.job].K;
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

constexpr long long kMaxIntV = 2000000000;   // MAXINTV, AP26.cpp:88

// result_hash after adding `add` through ReportSolution calls, each of which
// adds first%1000 + len and subtracts MAXINTV when above it (AP26.cpp:556-560):
// for a start in [0, MAXINTV] the value stays in [0, MAXINTV], is congruent
// to the total and is 0 only for a zero total.
static int32_t hash_fold(int32_t h0, unsigned long long add) {
  const unsigned long long total = (unsigned long long)h0 + add;
  if (total == 0) return 0;
  return (int32_t)((total - 1) % (unsigned long long)kMaxIntV + 1);
}

// A report with its ReportSolution result and AVX2 order key.
struct RepOut {
  ap26_ap ap;
  FinRec fin;
  uint64_t key;
};

// Reports of run_jobs' last call, job index alongside.
static std::vector<std::pair<int, RepOut>> collect_reports(const ap26_ctx *ctx, long long n) {
  std::vector<std::pair<int, RepOut>> v((size_t)n);
  for (long long i = 0; i < n; i++) {
    const APRec &r = ctx->h_aps[i];
    v[i].first = r.job;
    aprec_to_ap(ctx, r, v[i].second.ap);
    v[i].second.fin = ctx->h_fin[i];
    v[i].second.key = ap26h_order_key(v[i].second.ap.K, ctx->h_jobs[r.job].shift, r.n);
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
  fill_job(ctx->h_jobs[0], K, shift, 0, 0, N53_PER_K);
  long long n = 0;
  int rc = run_jobs_retry(ctx, 1, false, stats, &n);
  if (rc != AP26_OK) return rc;
  *n_out = (int)n;
  if (n > cap) return AP26_E_CAPACITY;
  for (long long i = 0; i < n; i++) aprec_to_ap(ctx, ctx->h_aps[i], out[i]);
  ap26_sort_aps(out, (int)n, shift);
  return AP26_OK;
}

extern "C" int ap26_search_k_sol(ap26_ctx *ctx, int K, int shift, int iter,
                                 int32_t *result_hash, ap26_sol *sol, int cap, int *n_sol,
                                 ap26_stats *stats) {
  if (!ctx || !result_hash || !n_sol || cap < 0 || (cap > 0 && !sol)) return AP26_E_ARG;
  if (iter < 0 || iter >= WORDS) return AP26_E_ARG;
  if (*result_hash < 0 || *result_hash > kMaxIntV) return AP26_E_ARG;
  if (!k_in_domain(K, shift)) return AP26_E_DOMAIN;
  if (!ap26_will_search(K)) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  fill_job(ctx->h_jobs[0], K, shift, 0, 0, N53_PER_K, iter);
  long long n = 0;
  int rc = run_jobs_retry(ctx, 1, false, stats, &n);
  if (rc != AP26_OK) return rc;
  auto v = collect_reports(ctx, n);
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
      o++;
    }
  *result_hash = hash_fold(*result_hash, ctx->h_job_hash[0]);
  return AP26_OK;
}

// ---- batched persistent form ------------------------------------------------------
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
  int rc;
  if ((rc = ensure_jobs(ctx, (int)jobs.size())) != AP26_OK) return rc;
  for (size_t j = 0; j < jobs.size(); j++)
    fill_job(ctx->h_jobs[j], jobs[j].second, items[jobs[j].first].shift, jobs[j].first, 0,
             N53_PER_K);
  long long n = 0;
  if (!jobs.empty()) {
    rc = run_jobs_retry(ctx, (int)jobs.size(), false, stats, &n, true);
    if (rc != AP26_OK) return rc;
  } else if (stats) {
    memset(stats, 0, sizeof(*stats));
  }
  // group reports: item, K ascending, AVX2 order inside K
  std::vector<std::vector<RepOut>> per_item(n_items);
  for (auto &r : collect_reports(ctx, n)) per_item[ctx->h_jobs[r.first].item].push_back(r.second);
  int64_t total = 0;
  std::vector<unsigned long long> hash_add(n_items, 0);
  for (size_t j = 0; j < jobs.size(); j++) hash_add[jobs[j].first] += ctx->h_job_hash[j];
  for (int i = 0; i < n_items; i++) {
    auto &v = per_item[i];
    std::sort(v.begin(), v.end(), rep_less);
    res[i].id = items[i].id;
    res[i].status = AP26_OK;
    for (const auto &r : v)
      if (r.fin.status != AP26_OK) { res[i].status = r.fin.status; break; }
    res[i].n_aps = (int32_t)v.size();
    res[i].first_ap = total;
    res[i].candidates = 0;
    res[i].ks_searched = 0;
    res[i].result_hash = hash_fold(0, hash_add[i]);
    res[i].latency_ms = 0;
    total += (int64_t)v.size();
  }
  for (size_t j = 0; j < jobs.size(); j++) {
    res[jobs[j].first].candidates += (int64_t)ctx->h_job_counts[j];
    res[jobs[j].first].ks_searched++;
  }
  *n_aps = total;
  if (total > ap_cap) return AP26_E_CAPACITY;
  for (int i = 0; i < n_items; i++)
    for (size_t e = 0; e < per_item[i].size(); e++) aps[res[i].first_ap + e] = per_item[i][e].ap;
  return AP26_OK;
}

// ---- serving: continuous batching ----------------------------------------------------
// A unit costs its K-job tables and descriptors while admitted.
static int64_t unit_bytes(size_t nk) { return (int64_t)nk * (TABLE_WORDS * 4 + sizeof(KJob) + 8); }

extern "C" int ap26_serve_submit(ap26_ctx *ctx, const ap26_item *item) {
  if (!ctx || !item || item->kmax < item->kmin) return AP26_E_ARG;
  if (!k_in_domain(item->kmin, item->shift) || !k_in_domain(item->kmax, item->shift))
    return AP26_E_DOMAIN;
  ServeUnit u;
  u.item = *item;
  for (int K = item->kmin; K <= item->kmax; K++)
    if (ap26_will_search(K)) u.ks.push_back(K);
  const int64_t need = unit_bytes(u.ks.size());
  if (ctx->bytes_in_use + need > ctx->opts.mem_budget || ctx->free_slots.empty())
    return AP26_E_NOMEM;
  CK(cudaSetDevice(ctx->device));
  u.slot = ctx->free_slots.back();
  CK(cudaMemsetAsync(ctx->d_units + u.slot, 0, sizeof(UnitState), ctx->stream));
  ctx->free_slots.pop_back();
  ctx->bytes_in_use += need;
  u.t_submit = std::chrono::steady_clock::now();
  ctx->units.push_back(std::move(u));
  return AP26_OK;
}

// One slice: up to `slice_k` K-jobs drawn round-robin from the admitted units
// run as one batched launch chain; finished units move to the poll queue.
extern "C" int ap26_serve_step(ap26_ctx *ctx, int *active_units) {
  if (!ctx) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  // One K-job per admitted unit per slice (round-robin), at most 8: a slice
  // then lasts about one K of device time however many units are waiting,
  // and a unit that arrives during a slice starts with the next one.
  const int slice_k = std::max(1, std::min<int>(8, (int)ctx->units.size()));
  std::vector<std::pair<ServeUnit *, int>> picked;
  bool progress = true;
  while ((int)picked.size() < slice_k && progress) {
    progress = false;
    for (auto &u : ctx->units) {
      if ((int)picked.size() >= slice_k) break;
      if (u.next_k < u.ks.size()) {
        picked.push_back({&u, u.ks[u.next_k++]});
        progress = true;
      }
    }
  }
  if (!picked.empty()) {
    int rc;
    if ((rc = ensure_jobs(ctx, (int)picked.size())) != AP26_OK) return rc;
    for (size_t j = 0; j < picked.size(); j++)
      fill_job(ctx->h_jobs[j], picked[j].second, picked[j].first->item.shift,
               picked[j].first->slot, 0, N53_PER_K);
    long long n = 0;
    ap26_stats st;
    rc = run_jobs_retry(ctx, (int)picked.size(), false, &st, &n, true);
    if (rc != AP26_OK) {
      for (auto &pk : picked) pk.first->status = rc;
    } else {
      // the units' running sums stay on the device
      unit_accumulate_kernel<<<1, 256, 0, ctx->stream>>>(ctx->d_jobs, (int)picked.size(),
                                                         ctx->d_job_counts, ctx->d_job_hash,
                                                         ctx->d_units);
      CK(cudaGetLastError());
      std::vector<std::vector<RepOut>> per_job(picked.size());
      for (auto &r : collect_reports(ctx, n)) per_job[r.first].push_back(r.second);
      for (size_t j = 0; j < picked.size(); j++) {
        ServeUnit *u = picked[j].first;
        std::sort(per_job[j].begin(), per_job[j].end(), rep_less);
        for (const auto &r : per_job[j]) {
          u->aps.push_back(r.ap);
          if (r.fin.status != AP26_OK && u->status == AP26_OK) u->status = r.fin.status;
        }
        u->done_k++;
      }
    }
  }
  for (auto it = ctx->units.begin(); it != ctx->units.end();) {
    if (it->done_k == (int)it->ks.size() || it->status != AP26_OK) {
      it->latency_ms = std::chrono::duration<double, std::milli>(
                           std::chrono::steady_clock::now() - it->t_submit).count();
      ctx->bytes_in_use -= unit_bytes(it->ks.size());
      ctx->finished.push_back(std::move(*it));
      it = ctx->units.erase(it);
    } else {
      ++it;
    }
  }
  if (active_units) *active_units = (int)ctx->units.size();
  return AP26_OK;
}

extern "C" int ap26_serve_poll(ap26_ctx *ctx, ap26_item_result *res, ap26_ap *aps,
                               int64_t ap_cap, int64_t *n_aps) {
  if (!ctx || !res || !n_aps) return AP26_E_ARG;
  if (ctx->finished.empty()) return 0;
  ServeUnit &u = ctx->finished.front();
  *n_aps = (int64_t)u.aps.size();
  if ((int64_t)u.aps.size() > ap_cap) return AP26_E_CAPACITY;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  UnitState us;
  CK(cudaMemcpyAsync(&us, ctx->d_units + u.slot, sizeof(us), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
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
  res->result_hash = hash_fold(0, us.hash_add);
  res->latency_ms = u.latency_ms;
  ctx->free_slots.push_back(u.slot);
  ctx->finished.pop_front();
  return 1;
}

// ---- kernel-level entry points ---------------------------------------------------------
extern "C" int ap26_sieve_range(ap26_ctx *ctx, int K, int shift, int64_t q_begin, int64_t q_end,
                                int64_t *cand, int64_t cap, int64_t *n_cand, ap26_stats *stats) {
  if (!ctx || !n_cand || q_begin < 0 || q_end > N53_PER_K || q_end < q_begin) return AP26_E_ARG;
  if (!k_in_domain(K, shift)) return AP26_E_DOMAIN;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  fill_job(ctx->h_jobs[0], K, shift, 0, q_begin, q_end);
  // sieve without the chain walk: one chunk covering everything, candidates kept
  const int saved = ctx->opts.chunk_tiles;
  const int64_t tile_n53 = (int64_t)kVariants[ctx->variant].WARPS * 32;
  const int64_t tiles = (q_end - q_begin + tile_n53 - 1) / tile_n53;
  ctx->opts.chunk_tiles = (int)std::max<int64_t>(1, tiles);
  if (ctx->chunk_graph) { cudaGraphExecDestroy(ctx->chunk_graph); ctx->chunk_graph = nullptr; }
  const int saved_graph = ctx->opts.use_graphs;
  ctx->opts.use_graphs = 0;
  // run setup + sieve only (no chain) by hand
  int rc = AP26_OK;
  {
    KJob &J = ctx->h_jobs[0];
    J.ntiles = (int32_t)tiles;
    J.tile_begin = 0;
    memset(ctx->h_st, 0, sizeof(DevState));
    ctx->h_st->chunk_size = (unsigned long long)std::max<int64_t>(1, tiles);
    ctx->h_st->total_tiles = (unsigned long long)tiles;
    cudaStream_t s = ctx->stream;
    const SieveVariant &V = kVariants[ctx->variant];
    CK(cudaEventRecord(ctx->ev0, s));
    CK(cudaMemcpyAsync(ctx->d_jobs, ctx->h_jobs, sizeof(KJob), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->d_st, ctx->h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->d_job_counts, 0, sizeof(unsigned long long), s));
    setup_jobs_kernel<<<1, 256, 0, s>>>(ctx->d_jobs, 1, ctx->d_tables);
    chunk_begin_kernel<<<1, 1, 0, s>>>(ctx->d_st, 0);
    const SieveArgs sa = sieve_args(ctx->d_jobs, 1, ctx->d_tables, ctx->d_st, ctx->d_cand[0],
                                    ctx->cand_cap, ctx->d_job_counts, 0,
                                    &ctx->d_st->cand_count[0]);
    V.kernel<<<ctx->sieve_blocks, V.WARPS * 32, V.smem(), s>>>(sa);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(ctx->ev1, s));
    rc = wait_stream(ctx, ctx->opts.wait_timeout_s);
    if (rc == AP26_OK) {
      const long long nc = (long long)ctx->h_st->cand_count[0];
      *n_cand = nc;
      if (nc > ctx->cand_cap) rc = AP26_E_OVERFLOW;
      else if (nc > cap) rc = AP26_E_CAPACITY;
      else if (nc > 0) {
        std::vector<Cand> tmp(nc);
        CK(cudaMemcpy(tmp.data(), ctx->d_cand[0], sizeof(Cand) * nc, cudaMemcpyDeviceToHost));
        for (long long i = 0; i < nc; i++) cand[i] = tmp[i].n;
      }
      if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        memset(stats, 0, sizeof(*stats));
        stats->candidates = nc;
        stats->late_items = (int64_t)ctx->h_st->late_items;
        stats->device_ms = ms;
        stats->error_flags = (int32_t)ctx->h_st->err_flags;
        stats->launches = 3;
      }
    }
  }
  ctx->opts.chunk_tiles = saved;
  ctx->opts.use_graphs = saved_graph;
  return rc;
}

extern "C" int ap26_sieve_count(ap26_ctx *ctx, const int32_t *Ks, int nK, int shift,
                                int64_t *counts, ap26_stats *stats) {
  if (!ctx || !Ks || nK <= 0 || !counts) return AP26_E_ARG;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  int rc;
  if ((rc = ensure_jobs(ctx, nK)) != AP26_OK) return rc;
  for (int i = 0; i < nK; i++) {
    if (!k_in_domain(Ks[i], shift)) return AP26_E_DOMAIN;
    fill_job(ctx->h_jobs[i], Ks[i], shift, i, 0, N53_PER_K);
  }
  rc = run_jobs(ctx, nK, true, stats, nullptr);
  if (rc != AP26_OK) return rc;
  for (int i = 0; i < nK; i++) counts[i] = (int64_t)ctx->h_job_counts[i];
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
  fill_job(ctx->h_jobs[0], K, 0, 0, 0, 0);
  DevBuf<int64_t> dn, df;
  DevBuf<int32_t> dk;
  CK(dn.alloc(count));
  CK(df.alloc(count));
  CK(dk.alloc(count));
  cudaStream_t s = ctx->stream;
  memset(ctx->h_st, 0, sizeof(DevState));
  CK(cudaMemcpyAsync(ctx->d_jobs, ctx->h_jobs, sizeof(KJob), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->d_st, ctx->h_st, sizeof(DevState), cudaMemcpyHostToDevice, s));
  setup_jobs_kernel<<<1, 256, 0, s>>>(ctx->d_jobs, 1, ctx->d_tables);
  CK(cudaMemcpyAsync(dn.p, n, sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(ctx->ev0, s));
  chain_explicit_kernel<<<ctx->num_sms * 8, 128, 0, s>>>(ctx->d_jobs, dn.p, count, dk.p, df.p,
                                                         ctx->d_st);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev1, s));
  CK(cudaMemcpyAsync(k_out, dk.p, sizeof(int32_t) * count, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(first_out, df.p, sizeof(int64_t) * count, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->device_ms = ms;
    stats->error_flags = (int32_t)ctx->h_st->err_flags;
    stats->launches = 2;
  }
  return (ctx->h_st->err_flags & ERR_DOMAIN) ? AP26_E_DOMAIN : AP26_OK;
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
// Times every compiled sieve variant (and two chunk sizes) on the same slice
// of K's lattice (count-only, so only the sieve is measured) and keeps the
// fastest.  The slice is the first 1/64 of the K's starts.
extern "C" int ap26_autotune(ap26_ctx *ctx, int K, int shift, ap26_opts *chosen) {
  if (!ctx) return AP26_E_ARG;
  if (!k_in_domain(K, shift)) return AP26_E_DOMAIN;
  CK(cudaSetDevice(ctx->device));
  drain(ctx);
  const int64_t q1 = N53_PER_K / 64;
  double best_ms = 1e30;
  int best_v = ctx->variant, best_chunk = ctx->opts.chunk_tiles;
  const int chunks[2] = {8192, 32768};
  for (int vi = 0; vi < kNumVariants; vi++) {
    int rc = set_variant(ctx, vi);
    if (rc != AP26_OK) return rc;
    for (int ci = 0; ci < 2; ci++) {
      ctx->opts.chunk_tiles = chunks[ci];
      double t = 0;
      for (int rep = 0; rep < 2; rep++) {
        fill_job(ctx->h_jobs[0], K, shift, 0, 0, q1);
        ap26_stats st;
        rc = run_jobs(ctx, 1, true, &st, nullptr);
        if (rc != AP26_OK) return rc;
        if (rep == 1) t = st.device_ms;   // first run warms up
      }
      if (t < best_ms) { best_ms = t; best_v = vi; best_chunk = chunks[ci]; }
    }
  }
  int rc = set_variant(ctx, best_v);
  ctx->opts.chunk_tiles = best_chunk;
  if (chosen) *chosen = ctx->opts;
  return rc;
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
  uint32_t tables[AP26_NOALLOC_MAX_K][TABLE_WORDS];
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
      setup_jobs_kernel<<<nK, 256, 0, s>>>(S->jobs, nK, &S->tables[0][0]);
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
