// ap26_kernels.cuh -- sm_100a kernels of the AP26 per-K search.
//
// Pipeline for a set of K-jobs (one (K, SHIFT) pair each), run chunk by chunk
// on one stream (ap26_capi.cu):
//
//   setup_jobs_kernel   per-K residue setup (the reference's split
//                       multiplications, src/opencl/AP26.h:112-120) and the
//                       per-K sieve bitstrings (replaces clearok/setok/
//                       setupokok/offset, src/opencl/kernels/*.cl)
//   chunk_begin_kernel  resets per-chunk counters
//   sieve_kernel        persistent, work-stealing over tiles of n53 starts;
//                       replaces setupn.cl + sieve.cl (the 1.1 GB n59 array
//                       of the reference is never materialised: starts are
//                       generated from a flat index)
//   chain_kernel        base-2 SPRP chain walk (replaces checkn.cl)
//   chunk_end_kernel    advances the chunk window
//   report_kernel       after the last chunk: ReportSolution of every raw
//                       report (9-base validation, split recursion, hash;
//                       src/common/AP26.cpp:484-602), per-job hash sums
//
// ---------------------------------------------------------------------------
// Sieve formulation.  The reference ANDs, for every lattice value n59 and
// every shift word w (absolute shift SHIFT+64w), the 83 table words
// OKOK_{p,w}[n59 mod p] (sieve.cl:28-113), where bit b of OKOK_{p,w}[r] is
// OK_p[(r + (SHIFT+64w+b)*MOD) mod p] (setupokok.cl, cpusse2.cpp:38-43).
// Multiplying the index by MOD^-1 mod p turns the 640 bits of all 10 words
// into ONE window of a p-periodic bitstring:
//     B_p[j] = OK_p[((j + SHIFT) * MOD) mod p],
//     bit i of the 640-bit mask = B_p[s + i],  s = n59 * MOD^-1 mod p.
// So each prime needs a (p + 672)-bit string and, per n59, one window
// offset: 2806 words (11.2 KB) per (K, SHIFT) with the pair strings below,
// staged in shared memory per CTA (the dense primes' words as overlapping
// 128-bit quads, the rest once: 20.8 KB for G = 22).  Reading a window is
// conflict-free: all lanes read the same prime's string at word offsets
// that differ by at most (p-1)/32 < 17, within one 32-bank row.
// Primes 61 and 67 share one string of period 4087 (bit j = B_61[j] &
// B_67[j], window start n59 * MOD^-1 mod 4087), and 71 and 73 one of
// period 5183; their windows are read conflict-free because the starts of
// an n43 value are visited sorted by those window starts (ap26_const.cuh),
// so a warp's 32 starts lie close together in both strings.
//
//   dense phase  the first G primes for all 10 words of every n59: G-2
//                windows (the two pairs, primes 4..G-1), each five 128-bit
//                loads and one 32-bit load + 20 funnel shifts
//   tail         live (n59, word) pairs are compacted into a per-warp shared
//                queue (ballot/popc) and advanced R primes at a time, all
//                lanes on the same prime, until stage SL
//   late         pairs alive at SL wait in a second per-warp queue until
//                enough have gathered to go through primes SL..82 together;
//                surviving bits pass the 7..23 filter (sieve.cl:123-142) and
//                become candidates n = n59 + (SHIFT + 64w + b) * MOD.
#pragma once
#include <stdint.h>
#include <utility>
#include "ap26_const.cuh"

namespace ap26 {

// ---- device data ------------------------------------------------------------
struct KJob {
  int64_t STEP, n0, S31, S37, S41, S43, S47, S53, S59;
  int64_t q_begin, q_end;     // n53 start range [q_begin, q_end)
  int64_t tile_begin;         // global index of this job's first tile
  int32_t K, shift, item, ntiles;
  int32_t word_begin;         // first shift word reported (the reference's ITER)
  int32_t table;              // index of this job's block in SieveArgs::tables
  int32_t flags;              // JOB_SORTED: n53 starts in the sorted lattice order
  int32_t pad;
};

enum : int32_t { JOB_SORTED = 1 };

struct Cand {
  int64_t n;
  int32_t job;
  int32_t pad;
};

struct APRec {
  int32_t k;
  int32_t job;
  int64_t first;
  int64_t n;
};

struct DevState {
  unsigned long long tile_next, tile_end;      // current chunk window
  unsigned long long chunk_begin, chunk_size, total_tiles;
  unsigned long long cand_count[2];            // per chunk, per candidate ring
  unsigned long long chain_next[2];            // chain walk's next candidate, per ring
  unsigned long long ap_count, prp_tests, cand_total, late_items;  // per run
  unsigned int err_flags;
  unsigned int pad;
  unsigned long long chain_walks;              // candidates the chain walk took, per run
  unsigned long long chain_check;              // sum of n over the rings' filled entries
                                               // minus sum of n over the walked ones: 0
};

enum : unsigned int {
  ERR_CAND_OVERFLOW = 1u,
  ERR_DOMAIN = 4u,
  ERR_AP_OVERFLOW = 8u,
  ERR_CHAIN_LIMIT = 16u,   // a chain walk ran kMaxChainTests tests: bad candidate data
};

struct SieveArgs {
  const KJob *jobs;
  int njobs;
  const uint32_t *tables;       // [*][JOB_TABLE_WORDS] (bitstrings, lattice order),
                                // job j's at KJob::table
  DevState *st;
  Cand *cand;
  long long cand_cap;
  unsigned long long *job_counts;  // per-job survivor counts
  int count_only;               // 1: count survivors, emit no candidates
  unsigned long long *cand_count;  // fill count of `cand` (DevState::cand_count[ring])
};

struct ChainArgs {
  const KJob *jobs;
  DevState *st;
  const Cand *cand;
  long long cand_cap;
  APRec *aps;
  long long ap_cap;
  const unsigned long long *cand_count;
  unsigned long long *chain_next;   // DevState::chain_next[ring], zero at the chunk's start
};

// A tile is one n53 start per thread of a sieve CTA: WARPS * 32 starts.
constexpr uint32_t FULL = 0xffffffffu;

// (i31, i37, i41) triples in the reference's loop order (AP26.h:127-131),
// packed 5 bits each, and the per-prime parameters; filled by the host.
// (This header is compiled into exactly one translation unit.)
__constant__ uint16_t c_triples[NUM_TRIPLES];
__constant__ PrimeParam c_params[NPRIMES];

// ---- 64-bit helpers -----------------------------------------------------------
// x mod MOD for 0 <= x < 2^62 via a double quotient estimate corrected once
// (the estimate is within one of floor(x/MOD)).
__device__ __forceinline__ int64_t mod_MOD(uint64_t x) {
  const double inv = 1.0 / (double)MOD;
  int64_t q = (int64_t)((double)x * inv);
  int64_t r = (int64_t)x - q * MOD;
  if (r < 0) r += MOD;
  else if (r >= MOD) r -= MOD;
  return r;
}

// ---- sieve pieces -----------------------------------------------------------
// The shared table holds the bitstrings in two regions.  The dense primes'
// words [0, D), D = word_offset(G), come first as overlapping 128-bit quads,
// quad[i] = (word i .. word i+3), so a 640-bit window starting at any word
// is five aligned 128-bit loads and one 32-bit load; a quarter warp's quads
// at one step lie within (p-1)/32 + 1 < 8 consecutive entries (distinct
// banks or broadcast).  The tail primes' words [D, TABLE_WORDS) follow once
// each: a 64-bit window at any bit is three 32-bit loads, and a warp's loads
// for one prime lie within floor((p + 575)/32) + 3 consecutive words, at
// most 32 (conflict-free) for every p below 385.
constexpr int table_bytes(int G) {
  return 16 * word_offset(G) + 4 * (TABLE_WORDS - word_offset(G));
}

__device__ __forceinline__ const uint4 *quad_at(const uint32_t *tab, uint32_t off, uint32_t w) {
  return reinterpret_cast<const uint4 *>(tab) + off + w;
}

template <int u>
__device__ __forceinline__ uint32_t unit_start(uint32_t a, uint32_t b, uint32_t c) {
  constexpr PrimeParam P = dense_param(u);
  uint32_t x = a * (uint32_t)P.A + b * (uint32_t)P.B + c * (uint32_t)P.C;
  return x - (uint32_t)P.p * (__umulhi(x, P.M) >> P.k);
}

// Units u and u+1 together: acc &= window_u & window_{u+1}, one 3-input
// LOP3 per word instead of two ANDs.
template <int u>
__device__ __forceinline__ void dense_two(const uint32_t *__restrict__ tab, uint32_t a,
                                          uint32_t b, uint32_t c, uint32_t (&acc)[20]) {
  constexpr PrimeParam P = dense_param(u), Q = dense_param(u + 1);
  const uint32_t s = unit_start<u>(a, b, c), t = unit_start<u + 1>(a, b, c);
  const uint4 *tp = quad_at(tab, P.off, s >> 5);
  const uint4 *tq = quad_at(tab, Q.off, t >> 5);
  const uint32_t sp = s & 31, sq = t & 31;
  uint32_t vp[21], vq[21];
#pragma unroll
  for (int i = 0; i < 5; i++) {
    const uint4 x = tp[4 * i], y = tq[4 * i];
    vp[4 * i] = x.x;
    vp[4 * i + 1] = x.y;
    vp[4 * i + 2] = x.z;
    vp[4 * i + 3] = x.w;
    vq[4 * i] = y.x;
    vq[4 * i + 1] = y.y;
    vq[4 * i + 2] = y.z;
    vq[4 * i + 3] = y.w;
  }
  vp[20] = *reinterpret_cast<const uint32_t *>(tp + 20);
  vq[20] = *reinterpret_cast<const uint32_t *>(tq + 20);
#pragma unroll
  for (int i = 0; i < 20; i++)
    acc[i] &= __funnelshift_r(vp[i], vp[i + 1], sp) & __funnelshift_r(vq[i], vq[i + 1], sq);
}

template <int... I>
__device__ __forceinline__ void dense_twos(const uint32_t *tab, uint32_t a, uint32_t b,
                                           uint32_t c, uint32_t (&acc)[20],
                                           std::integer_sequence<int, I...>) {
  (dense_two<2 * I>(tab, a, b, c, acc), ...);
}

// The first G primes (G even): the two pair bitstrings (primes 0..3) and
// primes 4..G-1, G-2 windows, two at a time.
template <int G>
__device__ __forceinline__ void dense_all(const uint32_t *tab, uint32_t a, uint32_t b,
                                          uint32_t c, uint32_t (&acc)[20]) {
  static_assert(G % 2 == 0 && G >= 6, "dense phase: both pairs and an even number of primes");
  dense_twos(tab, a, b, c, acc, std::make_integer_sequence<int, (G - 2) / 2>{});
}

// Queue item: x = n59 bits 0..31, y = n59 bits 32..47 | w << 16, z/w = mask.
__device__ __forceinline__ void split_n59(uint32_t x, uint32_t y, uint32_t &a, uint32_t &b,
                                          uint32_t &c) {
  a = x & 0xffffu;
  b = x >> 16;
  c = y & 0xffffu;
}

// Emits the candidates of one fully sieved word: each set bit b gives
// n = n59 + (shift + 64w + b) * MOD, kept when n has no factor 7..23.
__device__ __forceinline__ int emit_word(const SieveArgs &A, uint64_t n59, int w, uint64_t mask,
                                         int shift, int job) {
  int kept = 0;
  while (mask) {
    int b = __ffsll((long long)mask) - 1;
    mask &= mask - 1;
    int64_t n = (int64_t)n59 + (int64_t)(shift + 64 * w + b) * MOD;
    if (n % 7 && n % 11 && n % 13 && n % 17 && n % 19 && n % 23) {
      kept++;
      if (!A.count_only) {
        unsigned long long i = atomicAdd(A.cand_count, 1ull);
        if ((long long)i < A.cand_cap) {
          A.cand[i].n = n;
          A.cand[i].job = job;
        } else {
          atomicOr(&A.st->err_flags, ERR_CAND_OVERFLOW);
        }
      }
    }
  }
  return kept;
}

// One word of prime P (runtime parameters, identical for all lanes): the 64
// bits of the window at pos..pos+63, i.e. words j, j+1, j+2 (j = pos / 32)
// funnel-shifted by pos mod 32.  `tab` is the tail region's base moved back
// by D words, so a tail prime's global word offset indexes it directly.
__device__ __forceinline__ void word_prime_rt(const uint32_t *__restrict__ tab,
                                              const PrimeParam &P, uint32_t a, uint32_t b,
                                              uint32_t c, uint32_t w64, uint32_t &lo,
                                              uint32_t &hi) {
  const uint32_t x = a * (uint32_t)P.A + b * (uint32_t)P.B + c * (uint32_t)P.C;
  const uint32_t pos = x - (uint32_t)P.p * (__umulhi(x, P.M) >> P.k) + w64;
  const uint32_t *v = tab + (uint32_t)P.off + (pos >> 5);
  const uint32_t sh = pos & 31;
  const uint32_t v0 = v[0], v1 = v[1], v2 = v[2];
  lo &= __funnelshift_r(v0, v1, sh);
  hi &= __funnelshift_r(v1, v2, sh);
}

// Tail stages g_begin..g_end-1: every queued item advances R primes per pass
// (all lanes on the same primes, read warp-uniformly from constant memory),
// then the survivors are compacted in place (write index <= read index).
// One copy of this code serves every stage of both queues.
template <int R>
__device__ __forceinline__ void tail_stages(const uint32_t *tab, uint4 *q, int &cnt, int lane,
                                            int g_begin, int g_end) {
  for (int g0 = g_begin; g0 < g_end && cnt > 0; g0 += R) {
    PrimeParam P[R];
#pragma unroll
    for (int r = 0; r < R; r++) P[r] = c_params[min(g0 + r, NPRIMES - 1)];
    const int nr = min(R, g_end - g0);
    int out = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int i = base + lane;
      const bool valid = i < cnt;
      const uint4 it = valid ? q[i] : make_uint4(0, 0, 0, 0);
      __syncwarp();
      uint32_t a, b, c;
      split_n59(it.x, it.y, a, b, c);
      const uint32_t w64 = ((it.y >> 16) & 15u) * 64u;
      uint32_t lo = it.z, hi = it.w;
#pragma unroll
      for (int r = 0; r < R; r++)
        if (r < nr) word_prime_rt(tab, P[r], a, b, c, w64, lo, hi);
      const bool alive = valid && ((lo | hi) != 0u);
      const unsigned bal = __ballot_sync(FULL, alive);
      if (alive) q[out + __popc(bal & ((1u << lane) - 1u))] = make_uint4(it.x, it.y, lo, hi);
      out += __popc(bal);
      __syncwarp();
    }
    cnt = out;
  }
}

// Per-warp late queue: items alive at stage SL wait there until 3/4 of its
// LCAP slots are used, then go through the last primes together
// (stage-synchronous, so the rare late items do not run lane-by-lane in
// otherwise idle warps).

// Late drain: primes SL..82 for every queued item, then emission of the
// surviving bits of the fully sieved words.
template <int R, int SL>
__device__ __forceinline__ int late_drain(const SieveArgs &A, const uint32_t *tab, uint4 *buf,
                                          int &n, int lane, int shift, int job) {
  tail_stages<R>(tab, buf, n, lane, SL, NPRIMES);
  int kept = 0;
  // a K resumed at shift word ITER reports words ITER..9 only
  const int word_begin = A.jobs[job].word_begin;
  for (int i = lane; i < n; i += 32) {
    const uint4 it = buf[i];
    const uint64_t n59 = (uint64_t)it.x | ((uint64_t)(it.y & 0xffffu) << 32);
    const int w = (int)((it.y >> 16) & 15u);
    if (w >= word_begin)
      kept += emit_word(A, n59, w, ((uint64_t)it.w << 32) | it.z, shift, job);
  }
  __syncwarp();
  n = 0;
  return kept;
}

// Front drain: stage-synchronous groups G..SL-1 over the main queue, then
// the survivors move to the late queue (drained when it passes 3/4 full).
// With force, the late queue is drained too (job change / end of work).
// The late queue is drained at a single call site: moving items in, it is
// drained whenever it fills, and finally once it passes 3/4 of LCAP.
template <int G, int R, int SL, int LCAP>
__device__ __forceinline__ int front_drain(const SieveArgs &A, const uint32_t *tab, uint4 *q,
                                           int &cnt, uint4 *lq, int &lcnt, int lane, int shift,
                                           int job, unsigned long long &late, bool force) {
  tail_stages<R>(tab, q, cnt, lane, G, SL);
  late += (unsigned long long)cnt;
  int kept = 0;
  int moved = 0;
  for (;;) {
    const int take = min(LCAP - lcnt, cnt - moved);
    for (int i = lane; i < take; i += 32) lq[lcnt + i] = q[moved + i];
    lcnt += take;
    moved += take;
    __syncwarp();
    const bool more = moved < cnt;
    if (more || lcnt >= LCAP * 3 / 4 || (force && lcnt > 0))
      kept += late_drain<R, SL>(A, tab, lq, lcnt, lane, shift, job);
    if (!more) break;
  }
  cnt = 0;
  return kept;
}

// n53 start of lattice index q (0 <= q < N53_PER_K) of job J:
// n43 = (n0 + i3*S3 + i5*S5 + i31*S31 + i37*S37 + i41*S41) mod MOD
// (AP26.h:134) and n53 = n43 + j43*S43 + j47*S47 + j53*S53 mod MOD, the
// value the reference's nested increments reach (setupn.cl:31-53).
// With the sorted lattice order (perm != null) the q-th start of an n43
// value is the perm[q mod 12673]-th of its natural order.
__device__ __forceinline__ int64_t n53_at(const KJob &J, int64_t q, const uint16_t *perm) {
  int n43i = (int)(q / N53_PER_N43);
  int rem = (int)(q - (int64_t)n43i * N53_PER_N43);
  if (perm) rem = perm[rem];
  int j43 = rem / 667;
  rem -= j43 * 667;
  int j47 = rem / 29;
  int j53 = rem - j47 * 29;
  uint32_t tr = c_triples[n43i >> 3];
  int i31 = tr & 31, i37 = (tr >> 5) & 31, i41 = (tr >> 10) & 31;
  int i3 = (n43i >> 2) & 1, i5 = n43i & 3;
  uint64_t x = (uint64_t)J.n0 + (uint64_t)i3 * (uint64_t)S3 + (uint64_t)i5 * (uint64_t)S5 +
               (uint64_t)i31 * (uint64_t)J.S31 + (uint64_t)i37 * (uint64_t)J.S37 +
               (uint64_t)i41 * (uint64_t)J.S41;
  uint64_t n43 = (uint64_t)mod_MOD(x);
  uint64_t y = n43 + (uint64_t)j43 * (uint64_t)J.S43 + (uint64_t)j47 * (uint64_t)J.S47 +
               (uint64_t)j53 * (uint64_t)J.S53;
  return mod_MOD(y);
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

__device__ __forceinline__ int find_job(const KJob *jobs, int njobs, unsigned long long tile) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if ((unsigned long long)jobs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ---- the sieve kernel -----------------------------------------------------------
// Persistent: each CTA grabs tiles (one n53 start per thread) from
// DevState::tile_next until the chunk window ends; 35 n59 per start.  The
// per-warp queues carry over from tile to tile and are flushed only when the
// CTA moves to another K-job (the shared table changes) or runs out of work.
template <int G, int R, int SL, int QCAP, int LCAP, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 24 / WARPS)   // 24 resident warps per SM
sieve_kernel(SieveArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint4 *queues = reinterpret_cast<uint4 *>(smem_raw);
  uint4 *lqueues = queues + QCAP * WARPS;
  uint32_t *tab = reinterpret_cast<uint32_t *>(lqueues + LCAP * WARPS);
  constexpr int D = word_offset(G);
  static_assert(D + 3 <= TABLE_WORDS, "quad entries read past the table");
  uint32_t *ptab = tab + 3 * D;   // tail words: ptab[off + w], off >= D
  __shared__ unsigned long long s_tile;
  __shared__ int s_job;
  __shared__ unsigned long long s_kept[WARPS];
  __shared__ unsigned long long s_late[WARPS];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint4 *q = queues + warp * QCAP;
  uint4 *lq = lqueues + warp * LCAP;
  // The queue is drained when the next dense batch would not fit, so QCAP
  // only has to hold one worst-case batch and drains run on a full queue.
  static_assert(QCAP >= 32 * WORDS, "queue too small for one dense batch");

  int cur_job = -1, cur_shift = 0;
  const uint16_t *cur_perm = nullptr;
  int cnt = 0, lcnt = 0;
  unsigned long long kept_acc = 0, late_acc = 0;

  for (;;) {
    if (threadIdx.x == 0) {
      unsigned long long t = atomicAdd(&A.st->tile_next, 1ull);
      s_tile = t;
      s_job = (t < A.st->tile_end) ? find_job(A.jobs, A.njobs, t) : -1;
    }
    __syncthreads();
    const unsigned long long tile = s_tile;
    const int job = s_job;
    // job < 0: the chunk window is exhausted (also on a CTA's first grab,
    // when the chunk has fewer tiles than CTAs) -- flush and leave.
    if (job != cur_job || job < 0) {
      if (cur_job >= 0) {
        // finish the previous job's items with its table still in place
        kept_acc += front_drain<G, R, SL, LCAP>(A, ptab, q, cnt, lq, lcnt, lane, cur_shift,
                                                cur_job, late_acc, true);
        const unsigned long long v = warp_sum(kept_acc);
        if (lane == 0) s_kept[warp] = v;
        kept_acc = 0;
        __syncthreads();
        if (threadIdx.x == 0) {
          unsigned long long s = 0;
          for (int i = 0; i < WARPS; i++) s += s_kept[i];
          if (s) atomicAdd(&A.job_counts[cur_job], s);
        }
      }
      if (job < 0) break;
      const uint32_t *src = A.tables + (size_t)A.jobs[job].table * JOB_TABLE_WORDS;
      cur_perm = (A.jobs[job].flags & JOB_SORTED)
                     ? reinterpret_cast<const uint16_t *>(src + TABLE_WORDS) : nullptr;
      for (int i = threadIdx.x; i < D; i += blockDim.x)   // D + 3 <= TABLE_WORDS
        reinterpret_cast<uint4 *>(tab)[i] = make_uint4(src[i], src[i + 1], src[i + 2], src[i + 3]);
      for (int i = D + threadIdx.x; i < TABLE_WORDS; i += blockDim.x) ptab[i] = src[i];
      cur_job = job;
      cur_shift = A.jobs[job].shift;
      __syncthreads();
    }
    const KJob &J = A.jobs[job];
    const int64_t S59 = J.S59;
    const int64_t qi = J.q_begin +
                       (int64_t)(tile - (unsigned long long)J.tile_begin) * (WARPS * 32) +
                       warp * 32 + lane;
    const bool valid = qi < J.q_end;
    int64_t n59 = valid ? n53_at(J, qi, cur_perm) : 0;

    for (int j = 0; j < J59; j++) {
      uint32_t acc[20];
#pragma unroll
      for (int i = 0; i < 20; i++) acc[i] = valid ? FULL : 0u;
      const uint32_t x = (uint32_t)n59, y = (uint32_t)((uint64_t)n59 >> 32);
      uint32_t a, b, c;
      split_n59(x, y, a, b, c);
      dense_all<G>(tab, a, b, c, acc);
      unsigned bal[WORDS];
      int incoming = 0;
#pragma unroll
      for (int w = 0; w < WORDS; w++) {
        bal[w] = __ballot_sync(FULL, (acc[2 * w] | acc[2 * w + 1]) != 0u);
        incoming += __popc(bal[w]);
      }
      if (cnt + incoming > QCAP)
        kept_acc += front_drain<G, R, SL, LCAP>(A, ptab, q, cnt, lq, lcnt, lane, cur_shift, job,
                                                late_acc, false);
#pragma unroll
      for (int w = 0; w < WORDS; w++) {
        if ((bal[w] >> lane) & 1u)
          q[cnt + __popc(bal[w] & ((1u << lane) - 1u))] =
              make_uint4(x, y | ((uint32_t)w << 16), acc[2 * w], acc[2 * w + 1]);
        cnt += __popc(bal[w]);
      }
      __syncwarp();
      n59 += S59;
      if (n59 >= MOD) n59 -= MOD;
    }
    __syncthreads();   // the next grab overwrites s_tile / s_job
  }
  if (lane == 0) s_late[warp] = late_acc;   // warp-uniform
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long l = 0;
    for (int i = 0; i < WARPS; i++) l += s_late[i];
    if (l) atomicAdd(&A.st->late_items, l);
  }
}

// ---- Montgomery arithmetic mod odd N < 2^63 ---------------------------------------
// REDC with R = 2^64: for a, b < N, t = a*b, m = t_lo * (-N^-1) mod 2^64,
// (t + m*N) / 2^64 = t_hi + mulhi(m, N) + (t_lo != 0) < 2N.
__device__ __forceinline__ uint64_t mont_mul(uint64_t a, uint64_t b, uint64_t N, uint64_t ninv) {
  uint64_t lo = a * b, hi = __umul64hi(a, b);
  uint64_t m = lo * ninv;
  uint64_t r = hi + __umul64hi(m, N) + (lo != 0 ? 1ull : 0ull);
  return r >= N ? r - N : r;
}

__device__ __forceinline__ uint64_t neg_inv64(uint64_t N) {
  uint64_t x = N;               // correct to 3 bits for odd N
#pragma unroll
  for (int i = 0; i < 5; i++) x *= 2 - N * x;
  return 0 - x;
}

// 2^64 mod N by binary long division from N << clz(N) (>= 2^63).
__device__ __forceinline__ uint64_t r_mod(uint64_t N) {
  int s = __clzll((long long)N);
  uint64_t r = 0 - (N << s);
  for (int i = s - 1; i >= 0; i--)
    if (r >= (N << i)) r -= (N << i);
  return r;
}

// Base-2 strong probable prime test, same verdict as the reference's
// strong_prp(2, N) (PrimeQ_x86.h:143-182, checkn.cl:59-122) for odd N in
// [3, 2^63): left-to-right exponentiation by d = (N-1)/2^t in Montgomery
// form, the multiplications by the base 2 done as modular doublings.
// *sq counts the modular squarings.
__device__ __forceinline__ bool sprp2(uint64_t N, unsigned &sq) {
  if (N < 3) return false;
  const uint64_t nm1 = N - 1;
  const int t = __ffsll((long long)nm1) - 1;
  const uint64_t d = nm1 >> t;
  const uint64_t ninv = neg_inv64(N);
  const uint64_t one = r_mod(N);
  const uint64_t mone = N - one;
  uint64_t x = one + one;
  if (x >= N) x -= N;                   // 2 in Montgomery form
  const int top = 63 - __clzll((long long)d);
  for (int i = top - 1; i >= 0; i--) {
    x = mont_mul(x, x, N, ninv);
    sq++;
    if ((d >> i) & 1) {
      x += x;
      if (x >= N) x -= N;
    }
  }
  if (x == one || x == mone) return true;
  for (int s = 1; s < t; s++) {
    x = mont_mul(x, x, N, ninv);
    sq++;
    if (x == mone) return true;
    if (x == one) return false;
  }
  return false;
}

__device__ __forceinline__ bool prp_term(DevState *st, int64_t m, unsigned &tests, unsigned &sq) {
  if ((uint64_t)m >= (1ull << 62)) {       // PrimeQ's domain (PrimeQ_x86.h:191)
    atomicOr(&st->err_flags, ERR_DOMAIN);
    return false;
  }
  tests++;
  return sprp2((uint64_t)m, sq);
}

// ---- chain walk: checkn.cl:128-206 / cpuavx2.cpp:532-552 ------------------------
// For each candidate n (a sieve survivor), with S = K * 23#:
//   k = 0; m = n + 5S; while (PRP(m)) { k++; m += S; }
//   if (k >= 10) { m = n + 4S; while (m > 0 && PRP(m)) { k++; m -= S; } }
//   if (k >= 10) report (k, first = m + S)
// Walked as a stream of single SPRP tests: each lane holds one chain, runs
// one test per step, and when its chain ends takes the next candidate of
// the warp's claimed batch (32 at a time from DevState::chain_next).  A warp
// that gave each thread a whole chain would run as many tests as its
// longest chain (about 3.7 for 32 chains) for a mean of about 1.4.
__device__ __forceinline__ void emit_chain(const ChainArgs &A, int k, int job, int64_t first,
                                           int64_t n) {
  unsigned long long j = atomicAdd(&A.st->ap_count, 1ull);
  if ((long long)j < A.ap_cap) {
    A.aps[j].k = k;
    A.aps[j].job = job;
    A.aps[j].first = first;
    A.aps[j].n = n;
  } else {
    atomicOr(&A.st->err_flags, ERR_AP_OVERFLOW);
  }
}

// No AP of valid candidates comes near this length (the longest known has 27
// terms); a walk that reaches it ends with ERR_CHAIN_LIMIT, so the kernel
// ends whatever its input holds.
constexpr int kMaxChainTests = 4096;

__global__ void chain_kernel(ChainArgs A) {
  const unsigned long long n_c = min(*A.cand_count, (unsigned long long)A.cand_cap);
  const int lane = threadIdx.x & 31;
  unsigned tests = 0, sq = 0, walks = 0;
  // coverage check: each of the ring's n_c filled entries is walked once, so
  // the sum of their n minus the sum of the walked n is 0 (mod 2^64)
  unsigned long long chk = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n_c;
       i += (unsigned long long)gridDim.x * blockDim.x)
    chk += (unsigned long long)A.cand[i].n;
  bool active = false, bwd = false;
  int64_t n = 0, m = 0, S = 0;
  int k = 0, job = 0, walk = 0;
  unsigned long long base = 0;
  int got = 0;                  // candidates in the warp's current batch (<= 32)
  int left = 0;                 // of them, not yet taken by a lane
  bool exhausted = false;
  for (;;) {
    // refill: idle lanes take the next candidates of the warp's batch
    for (;;) {
      const unsigned idle = __ballot_sync(FULL, !active);
      if (!idle || exhausted) break;
      if (left == 0) {
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(A.chain_next, 32ull);
        b = __shfl_sync(FULL, b, 0);
        base = b;
        left = b < n_c ? (int)min(32ull, n_c - b) : 0;
        got = left;
        if (left == 0) {
          exhausted = true;
          break;
        }
      }
      const int rank = __popc(idle & ((1u << lane) - 1u));
      const int take = min(__popc(idle), left);
      if (!active && rank < take) {
        const Cand cd = A.cand[base + (got - left) + rank];
        n = cd.n;
        job = cd.job;
        chk -= (unsigned long long)n;
        S = A.jobs[job].STEP;
        m = n + S * 5;
        k = 0;
        walk = 0;
        walks++;
        bwd = false;
        active = true;
      }
      left -= take;
    }
    if (!__any_sync(FULL, active)) break;
    if (active && ++walk > kMaxChainTests) {
      atomicOr(&A.st->err_flags, ERR_CHAIN_LIMIT);
      active = false;
    }
    if (active) {
      if (bwd && m <= 0) {          // the backward walk stops below zero, untested
        emit_chain(A, k, job, m + S, n);
        active = false;
      } else if (prp_term(A.st, m, tests, sq)) {
        k++;
        m = bwd ? m - S : m + S;
      } else if (!bwd && k >= 10) {
        bwd = true;
        m = n + S * 4;
      } else {
        if (k >= 10) emit_chain(A, k, job, m + S, n);
        active = false;
      }
    }
  }
  // warp-aggregated test and walk counters
  unsigned v = tests, w = walks;
  for (int o = 16; o; o >>= 1) {
    v += __shfl_xor_sync(FULL, v, o);
    w += __shfl_xor_sync(FULL, w, o);
    chk += __shfl_xor_sync(FULL, chk, o);
  }
  if (lane == 0 && v) atomicAdd(&A.st->prp_tests, (unsigned long long)v);
  if (lane == 0 && w) atomicAdd(&A.st->chain_walks, (unsigned long long)w);
  if (lane == 0 && chk) atomicAdd(&A.st->chain_check, chk);
}

// ---- ReportSolution on the device: AP26.cpp:484-602 ------------------------------
// Strong probable-prime test to base a (2 <= a < N), same verdict as the
// reference's strong_prp(a, N) (PrimeQ_x86.h:143-182) for odd N in (a, 2^63):
// x = a^d in Montgomery form, left to right, then up to t-1 squarings.
__device__ __forceinline__ bool sprp_base(uint32_t a, uint64_t N) {
  const uint64_t nm1 = N - 1;
  const int t = __ffsll((long long)nm1) - 1;
  const uint64_t d = nm1 >> t;
  const uint64_t ninv = neg_inv64(N);
  const uint64_t one = r_mod(N);
  const uint64_t mone = N - one;
  uint64_t am = 0;                      // a·2^64 mod N by double-and-add over a's bits
  for (int b = 4; b >= 0; b--) {
    am += am;
    if (am >= N) am -= N;
    if ((a >> b) & 1u) {
      am += one;
      if (am >= N) am -= N;
    }
  }
  uint64_t x = am;
  const int top = 63 - __clzll((long long)d);
  for (int i = top - 1; i >= 0; i--) {
    x = mont_mul(x, x, N, ninv);
    if ((d >> i) & 1) x = mont_mul(x, am, N, ninv);
  }
  if (x == one || x == mone) return true;
  for (int s = 1; s < t; s++) {
    x = mont_mul(x, x, N, ninv);
    if (x == mone) return true;
    if (x == one) return false;
  }
  return false;
}

// Status codes of one report (the library's public codes).
enum : int32_t { REP_OK = 0, REP_ARG = -1, REP_DOMAIN = -4, REP_OVERFLOW = -6, REP_INVALID = -8 };
constexpr int FIN_MAX_SOL = 3;       // runs of >= 20 valid terms in one report of <= 128
constexpr int FIN_MAX_TERMS = 128;
constexpr int MIN_REPORT = 20;       // MINIMUM_AP_LENGTH_TO_REPORT, AP26.cpp:104

// One raw report after ReportSolution (layout of the public ap26_final).
struct FinRec {
  int64_t hash_add;                  // sum of first%1000 + len over every call
  int32_t status;
  int32_t n_sol;
  int32_t sol_len[FIN_MAX_SOL];
  int32_t pad;
  int64_t sol_first[FIN_MAX_SOL];
};

struct ReportArgs {
  const APRec *aps;                  // k, job (or K when jobs is null), first
  const unsigned long long *count;   // device-side report count, or null
  long long n;                       // reports (cap when count is set)
  const KJob *jobs;
  FinRec *fin;
  unsigned long long *job_hash;      // per job and shift word: sum of hash_add
                                     // (status OK), [job * WORDS + w], or null
};

// Shift word (0..9) of a raw report: its candidate n = n59 + (shift + 64w +
// b) * MOD with 0 <= n59 < MOD.
__device__ __forceinline__ int report_word(int64_t n, int shift) {
  const int t = (int)((uint64_t)n / (uint64_t)MOD) - shift;
  return min(max(t >> 6, 0), WORDS - 1);
}

constexpr int REPORT_WARPS = 4;
enum : uint8_t { TERM_DOM = 1, TERM_P2 = 2, TERM_P9 = 4 };

// One warp per report: lane j tests terms j, j+32, ... (domain 0 <= N <
// 2^62 of the reference's mulmod, AP26.cpp:494/529; base 2; the 8 further
// bases of validate_ap26, AP26.cpp:519), then lane 0 replays the recursion
// of ReportSolution over the per-term verdicts: every call adds
// first%1000 + len; a piece whose first 9-base failure is at i is checked
// to base 2 as a whole (Computation error otherwise), its leading i terms
// are one call (valid, reported at length >= 20) and its trailing
// len-(i+1) terms the next piece.
__global__ void __launch_bounds__(REPORT_WARPS * 32) report_kernel(ReportArgs A) {
  __shared__ uint8_t flags[REPORT_WARPS][FIN_MAX_TERMS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long n = A.count ? min((long long)*A.count, A.n) : A.n;
  uint8_t *fl = flags[warp];
  for (long long r = (long long)blockIdx.x * REPORT_WARPS + warp; r < n;
       r += (long long)gridDim.x * REPORT_WARPS) {
    const APRec rec = A.aps[r];
    const int K = A.jobs ? A.jobs[rec.job].K : rec.job;
    const int k = rec.k;
    const int64_t first = rec.first;
    FinRec out;
    out.hash_add = 0;
    out.status = REP_OK;
    out.n_sol = 0;
    out.pad = 0;
    for (int i = 0; i < FIN_MAX_SOL; i++) { out.sol_len[i] = 0; out.sol_first[i] = 0; }
    const bool args_ok = k >= 0 && first > 23 && K >= 1 && K <= 400000000;
    if (args_ok && k > FIN_MAX_TERMS) out.status = REP_OVERFLOW;
    else if (!args_ok) out.status = REP_ARG;
    if (out.status == REP_OK) {
      const uint64_t D = (uint64_t)K * (uint64_t)PRIM23;     // < 2^57
      for (int j = lane; j < k; j += 32) {
        uint8_t f = 0;
        const uint64_t jd = (uint64_t)j * D;                   // < 2^64
        const uint64_t N = (uint64_t)first + jd;
        if (jd < (1ull << 62) && N < (1ull << 62)) {
          f = TERM_DOM;
          unsigned sq = 0;
          if ((N & 1) && sprp2(N, sq)) {
            f |= TERM_P2;
            bool all = true;
            const uint32_t bases[8] = {3, 5, 7, 11, 13, 17, 19, 23};
            for (int b = 0; b < 8 && all; b++) all = sprp_base(bases[b], N);
            if (all) f |= TERM_P9;
          }
        }
        fl[j] = f;
      }
    }
    __syncwarp();
    if (lane == 0) {
      if (out.status == REP_OK) {
        const int64_t D = (int64_t)K * PRIM23;
        int s = 0;
        const int e = k;
        int64_t f = first;
        for (;;) {
          out.hash_add += f % 1000 + (e - s);
          // validate_ap26 over [s, e): first term failing any of the 9 bases
          int i = e;
          if (f % 2 == 0) {
            i = s;
          } else {
            for (int j = s; j < e; j++) {
              if (!(fl[j] & TERM_DOM)) { out.status = REP_DOMAIN; break; }
              if (!(fl[j] & TERM_P9)) { i = j; break; }
            }
          }
          if (out.status != REP_OK) break;
          if (i == e) {
            if (e - s >= MIN_REPORT) {
              if (out.n_sol < FIN_MAX_SOL) {
                out.sol_len[out.n_sol] = e - s;
                out.sol_first[out.n_sol] = f;
                out.n_sol++;
              } else {
                out.status = REP_OVERFLOW;
              }
            }
            break;
          }
          // Non-Solution: the whole piece must still be a base-2 AP
          if (f % 2 == 0) {
            out.status = REP_INVALID;
            break;
          }
          for (int j = s; j < e; j++) {
            if (!(fl[j] & TERM_DOM)) { out.status = REP_DOMAIN; break; }
            if (!(fl[j] & TERM_P2)) { out.status = REP_INVALID; break; }
          }
          if (out.status != REP_OK) break;
          // leading i-s terms: one call, valid by construction
          out.hash_add += f % 1000 + (i - s);
          if (i - s >= MIN_REPORT) {
            if (out.n_sol < FIN_MAX_SOL) {
              out.sol_len[out.n_sol] = i - s;
              out.sol_first[out.n_sol] = f;
              out.n_sol++;
            } else {
              out.status = REP_OVERFLOW;
              break;
            }
          }
          // trailing piece
          f += (int64_t)(i + 1 - s) * D;
          s = i + 1;
        }
      }
      A.fin[r] = out;
      if (A.job_hash && out.status == REP_OK)
        atomicAdd(&A.job_hash[rec.job * WORDS + report_word(rec.n, A.jobs[rec.job].shift)],
                  (unsigned long long)out.hash_add);
    }
    __syncwarp();
  }
}

}  // namespace ap26
