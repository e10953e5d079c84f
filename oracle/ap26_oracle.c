/* ap26_oracle.c -- THE ORACLE.  Test infrastructure only.
 *
 * A plain-C restatement of the reference's per-K AP26 search (ibethune/ap26),
 * used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
 * the CHECKER of the CUDA path.  Nothing in ap26_b200/ links, loads or calls
 * this file.  It favours obviousness over speed (scalar, 128-bit mulmod).
 *
 * Pinned against: the reference's golden SOL/hash files (tests/TEST-366384.txt,
 * TEST-44121555.txt, TEST-47715109.txt), the reference's sieve survivor known
 * answer (38,838,420 for K=366384 SHIFT=0, src/opencl/AP26.h:343) and raw AP
 * records produced by the reference's own Search_avx2 (oracle/ref_harness.cpp,
 * tests/golden/ref_raw/).
 *
 * Every function cites the reference lines it restates.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <pthread.h>

#define PRIM23 INT64_C(223092870)            /* src/common/CONST.H:7  */
#define MOD    INT64_C(258559632607830)      /* src/common/CONST.H:16 */
#define N0     INT64_C(106990415896110)      /* CONST.H:17 */
#define N30    INT64_C(94805198622871)       /* CONST.H:18 */
#define S3     INT64_C(172373088405220)      /* CONST.H:19 */
#define S5     INT64_C(51711926521566)       /* CONST.H:20 */
#define PRES2  INT64_C(16681266619860)       /* CONST.H:21-27 */
#define PRES3  INT64_C(181690552643340)
#define PRES4  INT64_C(132432982555230)
#define PRES5  INT64_C(126273308948010)
#define PRES6  INT64_C(115526644356690)
#define PRES7  INT64_C(48784836341100)
#define PRES8  INT64_C(100794433050510)

#define NPRIMES 83
#define NUM_N43 10840
#define PER_N43 443555            /* 19 * 23 * 29 * 35 */
#define MAXINTV 2000000000        /* src/common/AP26.cpp:88 */
#define MIN_REPORT 20             /* AP26.cpp:104 */

/* the 83 sieve primes 61..541 (src/cpu/cpusse2.cpp:62-144) */
static const int PR[NPRIMES] = {
  61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127, 131, 137, 139,
  149, 151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223, 227,
  229, 233, 239, 241, 251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311,
  313, 317, 331, 337, 347, 349, 353, 359, 367, 373, 379, 383, 389, 397, 401,
  409, 419, 421, 431, 433, 439, 443, 449, 457, 461, 463, 467, 479, 487, 491,
  499, 503, 509, 521, 523, 541};

int ao_num_primes(void) { return NPRIMES; }
int ao_prime(int i) { return (i >= 0 && i < NPRIMES) ? PR[i] : 0; }

/* ---- per-K setup: src/opencl/AP26.h:112-120, src/cpu/cpuavx2.cpp:223-232 -- */
typedef struct {
  int64_t STEP, n0, S31, S37, S41, S43, S47, S53, S59;
} ksetup;

static int64_t kmul(int64_t c, int K) {
  return (c * (K % 17835) + ((c * 17835) % MOD) * (K / 17835)) % MOD;
}

static void setup_k(int K, ksetup *s) {
  s->STEP = (int64_t)K * PRIM23;
  s->n0 = (N0 * (K % 17835) + ((N0 * 17835) % MOD) * (K / 17835) + N30) % MOD;
  s->S31 = kmul(PRES2, K);
  s->S37 = kmul(PRES3, K);
  s->S41 = kmul(PRES4, K);
  s->S43 = kmul(PRES5, K);
  s->S47 = kmul(PRES6, K);
  s->S53 = kmul(PRES7, K);
  s->S59 = kmul(PRES8, K);
}

/* out[9] = STEP, n0, S31, S37, S41, S43, S47, S53, S59 */
int ao_setup(int K, int64_t *out) {
  ksetup s;
  setup_k(K, &s);
  memcpy(out, &s, sizeof s);
  return 0;
}

/* ---- n43 lattice in the reference's loop order: AP26.h:127-136 ---------- */
static int n43_table(const ksetup *s, int64_t *out) {
  int count = 0;
  for (int i31 = 0; i31 < 7; ++i31)
    for (int i37 = 0; i37 < 13; ++i37)
      if (i37 - i31 <= 10 && i31 - i37 <= 4)
        for (int i41 = 0; i41 < 17; ++i41)
          if (i41 - i31 <= 14 && i41 - i37 <= 14 && i31 - i41 <= 4 && i37 - i41 <= 10)
            for (int i3 = 0; i3 < 2; ++i3)
              for (int i5 = 0; i5 < 4; ++i5)
                out[count++] = (s->n0 + i3 * S3 + i5 * S5 + i31 * s->S31 +
                                i37 * s->S37 + i41 * s->S41) % MOD;
  return count;
}

int ao_n43(int K, int64_t *out) {
  ksetup s;
  setup_k(K, &s);
  return n43_table(&s, out);
}

/* n59 at flat position f, f = n43idx*443555 + j43*23345 + j47*1015 + j53*35 + j59.
 * Equals the value the reference's nested loops reach (cpuavx2.cpp:397-410,
 * 822-851): each level adds its step and reduces once, so the partial sums
 * are the true residues mod MOD. */
static int64_t n59_at(const ksetup *s, const int64_t *n43, int64_t f) {
  int64_t i = f / PER_N43, r = f % PER_N43;
  int j43 = (int)(r / 23345); r %= 23345;
  int j47 = (int)(r / 1015);  r %= 1015;
  int j53 = (int)(r / 35);
  int j59 = (int)(r % 35);
  int64_t v = n43[i];
  v = (v + (int64_t)j43 * s->S43 % MOD) % MOD;   /* j*S < 2^53: no overflow */
  v = (v + (int64_t)j47 * s->S47 % MOD) % MOD;
  v = (v + (int64_t)j53 * s->S53 % MOD) % MOD;
  v = (v + (int64_t)j59 * s->S59 % MOD) % MOD;
  return v;
}

int64_t ao_n59(int K, int64_t f) {
  ksetup s;
  int64_t n43[NUM_N43];
  setup_k(K, &s);
  n43_table(&s, n43);
  return n59_at(&s, n43, f);
}

/* ---- OK_p: MAKE_OK, src/cpu/cpusse2.cpp:32-36 --------------------------- */
static void make_ok(int64_t STEP, int p, uint8_t *ok) {
  for (int j = 0; j < p; j++) ok[j] = 1;
  for (int j = p - 23; j <= p; j++) ok[(j * (STEP % p)) % p] = 0;
}

int ao_ok_table(int K, int p, uint8_t *out) {
  make_ok((int64_t)K * PRIM23, p, out);
  return 0;
}

/* ---- OKOK_p for one shift word: MAKE_OKOK, cpusse2.cpp:38-43 ------------- */
static void make_okok(const uint8_t *ok, int p, int shift, uint64_t *okok) {
  for (int j = 0; j < p; j++) {
    uint64_t w = 0;
    for (int jj = 0; jj < 64; jj++)
      w |= ((uint64_t)ok[(j + (jj + shift) * MOD) % p]) << jj;
    okok[j] = w;
  }
}

int ao_okok(int K, int shift, int p, uint64_t *out) {
  uint8_t ok[541];
  make_ok((int64_t)K * PRIM23, p, ok);
  make_okok(ok, p, shift, out);
  return 0;
}

/* ---- strong PRP: src/common/PrimeQ_x86.h:143-182 -------------------------
 * Same control flow (t = ctz(N-1), left-to-right square-and-multiply over the
 * bits of d below its top bit, then up to t-1 squarings); the x87 quotient
 * estimate of mulmod (PrimeQ_x86.h:114-136) is replaced by an exact 128-bit
 * remainder, which is the value that estimate computes for N < 2^62.  Valid
 * here for odd N < 2^63, a < N. */
static uint64_t mulmod128(uint64_t a, uint64_t b, uint64_t n) {
  return (uint64_t)(((unsigned __int128)a * b) % n);
}

int ao_sprp(int64_t N, int64_t a_in) {
  uint64_t n = (uint64_t)N, a = (uint64_t)a_in, r, d;
  unsigned t = (unsigned)__builtin_ctzll(n - 1), s;
  d = n >> t;
  for (r = a, d >>= 1; d > 0; d >>= 1) {
    a = mulmod128(a, a, n);
    if (d & 1) r = mulmod128(r, a, n);
  }
  if (r == 1 || r == n - 1) return 1;
  for (s = 1; s < t; s++)
    if ((r = mulmod128(r, r, n)) == n - 1) return 1;
  return 0;
}

/* Number of Montgomery-style mulmods the SPRP performs on N: squarings over
 * the bits of d below its top bit, one multiply per set bit below the top,
 * then the clause-2 squarings actually executed.  Used for the PRP roofline's
 * algorithmic work count. */
int ao_sprp_mulmods(int64_t N) {
  uint64_t n = (uint64_t)N, a = 2, r, d;
  unsigned t = (unsigned)__builtin_ctzll(n - 1), s;
  int cnt = 0;
  d = n >> t;
  for (r = a, d >>= 1; d > 0; d >>= 1) {
    a = mulmod128(a, a, n); cnt++;
    if (d & 1) { r = mulmod128(r, a, n); cnt++; }
  }
  if (r == 1 || r == n - 1) return cnt;
  for (s = 1; s < t; s++) {
    cnt++;
    if ((r = mulmod128(r, r, n)) == n - 1) return cnt;
  }
  return cnt;
}

/* PrimeQ (PrimeQ_x86.h:189-198): the reference exits for N >= 2^62; here the
 * caller gets -1 so tests can see the domain violation. */
static int primeq(int64_t N) {
  if ((uint64_t)N >= (UINT64_C(1) << 62)) return -1;
  return ao_sprp(N, 2);
}

/* ---- PRP chain: src/cpu/cpuavx2.cpp:532-552 (= cpusse2.cpp:570-590) ------ */
int ao_chain(int64_t n, int64_t STEP, int *k_out, int64_t *first_out) {
  int64_t m;
  int k = 0, q;
  m = n + STEP * 5;
  while ((q = primeq(m)) == 1) { k++; m += STEP; }
  if (q < 0) return -1;
  if (k >= 10) {
    m = n + STEP * 4;
    while (m > 0 && (q = primeq(m)) == 1) { k++; m -= STEP; }
    if (q < 0 && m > 0) return -1;
  }
  *k_out = k;
  *first_out = m + STEP;
  return 0;
}

/* ---- sieve over a flat range of n59 positions, all 10 shift words --------
 * Restates the per-n59 body of cpusse2.cpp:465-594: for each word (absolute
 * shift SHIFT+64w), sito = AND_p OKOK_p[n59 % p]; every set bit b gives
 * n = n59 + (b + SHIFT + 64w) * MOD, kept if n is not divisible by 7..23.
 * Candidate positions are encoded pos = (f << 10) | (w << 6) | b.
 * `consults` counts table lookups under the canonical order (ascending
 * primes, early exit per word when sito reaches zero). */
static inline int fmod_p(int64_t x, int p, double inv);
static double INVP[NPRIMES];
typedef struct {
  int K, shift;
  int64_t f0, f1;
  const ksetup *s;
  const int64_t *n43;
  uint64_t (*okok)[541];      /* [83*10][541] */
  int64_t *cand_n;
  uint64_t *cand_pos;
  int64_t cap, count;
  uint64_t consults;
} sieve_job;

static void *sieve_worker(void *arg) {
  sieve_job *J = (sieve_job *)arg;
  for (int64_t f = J->f0; f < J->f1; f++) {
    int64_t n59 = n59_at(J->s, J->n43, f);
    int rem[NPRIMES];
    int have = 0;
    for (int w = 0; w < 10; w++) {
      uint64_t sito = ~UINT64_C(0);
      for (int i = 0; i < NPRIMES && sito; i++) {
        if (i >= have) { rem[have] = fmod_p(n59, PR[i], INVP[i]); have++; }
        sito &= J->okok[i * 10 + w][rem[i]];
        J->consults++;
      }
      while (sito) {
        int b = __builtin_ctzll(sito);
        sito &= sito - 1;
        int64_t n = n59 + (int64_t)(b + J->shift + 64 * w) * MOD;
        if (n % 7 && n % 11 && n % 13 && n % 17 && n % 19 && n % 23) {
          if (J->count < J->cap) {
            J->cand_n[J->count] = n;
            J->cand_pos[J->count] = ((uint64_t)f << 10) | ((uint64_t)w << 6) | (uint64_t)b;
          }
          J->count++;
        }
      }
    }
  }
  return NULL;
}

/* x mod p for 0 <= x < 2^53 through a double-precision quotient estimate,
 * corrected by one step (the estimate is off by at most one). */
static inline int fmod_p(int64_t x, int p, double inv) {
  int64_t q = (int64_t)((double)x * inv);
  int64_t r = x - q * p;
  if (r < 0) r += p;
  else if (r >= p) r -= p;
  return (int)r;
}

static void init_invp(void) {
  for (int i = 0; i < NPRIMES; i++) INVP[i] = 1.0 / PR[i];
}

static uint64_t (*build_okok(int K, int shift))[541] {
  init_invp();
  uint64_t (*okok)[541] = malloc(sizeof(uint64_t[541]) * NPRIMES * 10);
  uint8_t ok[541];
  for (int i = 0; i < NPRIMES; i++) {
    make_ok((int64_t)K * PRIM23, PR[i], ok);
    for (int w = 0; w < 10; w++) make_okok(ok, PR[i], shift + 64 * w, okok[i * 10 + w]);
  }
  return okok;
}

/* Returns the candidate count (may exceed cap; only cap are stored, in
 * (f, w, b) order).  nthreads > 1 splits [f0, f1) into contiguous pieces. */
int64_t ao_sieve(int K, int shift, int64_t f0, int64_t f1, int64_t *cand_n,
                 uint64_t *cand_pos, int64_t cap, uint64_t *consults, int nthreads) {
  ksetup s;
  int64_t n43[NUM_N43];
  setup_k(K, &s);
  n43_table(&s, n43);
  uint64_t (*okok)[541] = build_okok(K, shift);
  if (nthreads < 1) nthreads = 1;
  sieve_job *jobs = calloc(nthreads, sizeof(sieve_job));
  pthread_t *th = calloc(nthreads, sizeof(pthread_t));
  int64_t span = f1 - f0;
  for (int t = 0; t < nthreads; t++) {
    sieve_job *J = &jobs[t];
    J->K = K; J->shift = shift; J->s = &s; J->n43 = n43; J->okok = okok;
    J->f0 = f0 + span * t / nthreads;
    J->f1 = f0 + span * (t + 1) / nthreads;
    J->cap = cap;  /* each worker stores into its own scratch, merged below */
    J->cand_n = cap ? malloc(sizeof(int64_t) * cap) : NULL;
    J->cand_pos = cap ? malloc(sizeof(uint64_t) * cap) : NULL;
    pthread_create(&th[t], NULL, sieve_worker, J);
  }
  int64_t total = 0;
  uint64_t cons = 0;
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    sieve_job *J = &jobs[t];
    int64_t stored = J->count < J->cap ? J->count : J->cap;
    for (int64_t i = 0; i < stored && total + i < cap; i++) {
      cand_n[total + i] = J->cand_n[i];
      cand_pos[total + i] = J->cand_pos[i];
    }
    total += J->count;
    cons += J->consults;
    free(J->cand_n);
    free(J->cand_pos);
  }
  if (consults) *consults = cons;
  free(jobs); free(th); free(okok);
  return total;
}

/* ---- whole search over a flat range: sieve + chain ------------------------
 * Emits the raw reports (k >= 10) the reference would pass to ReportSolution
 * (cpuavx2.cpp:548-552), with the candidate position of each.  The caller
 * orders them (see ao_avx2_order_key).  Returns #reports (may exceed cap),
 * -1 on a PrimeQ domain violation. */
typedef struct {
  int K, shift;
  int64_t f0, f1;
  const ksetup *s;
  const int64_t *n43;
  uint64_t (*okok)[541];
  int *ks; int64_t *firsts; uint64_t *pos;
  int64_t cap, count, ncand;
  int err;
} search_job;

static void *search_worker(void *arg) {
  search_job *J = (search_job *)arg;
  int rem[NPRIMES];
  for (int64_t f = J->f0; f < J->f1; f++) {
    int64_t n59 = n59_at(J->s, J->n43, f);
    int have = 0;
    for (int w = 0; w < 10; w++) {
      uint64_t sito = ~UINT64_C(0);
      for (int i = 0; i < NPRIMES && sito; i++) {
        if (i >= have) { rem[have] = fmod_p(n59, PR[i], INVP[i]); have++; }
        sito &= J->okok[i * 10 + w][rem[i]];
      }
      while (sito) {
        int b = __builtin_ctzll(sito);
        sito &= sito - 1;
        int64_t n = n59 + (int64_t)(b + J->shift + 64 * w) * MOD;
        if (!(n % 7 && n % 11 && n % 13 && n % 17 && n % 19 && n % 23)) continue;
        J->ncand++;
        int k; int64_t first;
        if (ao_chain(n, J->s->STEP, &k, &first) < 0) { J->err = 1; continue; }
        if (k >= 10) {
          if (J->count < J->cap) {
            J->ks[J->count] = k;
            J->firsts[J->count] = first;
            J->pos[J->count] = ((uint64_t)f << 10) | ((uint64_t)w << 6) | (uint64_t)b;
          }
          J->count++;
        }
      }
    }
  }
  return NULL;
}

int64_t ao_search(int K, int shift, int64_t f0, int64_t f1, int *ks, int64_t *firsts,
                  uint64_t *pos, int64_t cap, int64_t *ncand, int nthreads) {
  ksetup s;
  int64_t n43[NUM_N43];
  setup_k(K, &s);
  n43_table(&s, n43);
  uint64_t (*okok)[541] = build_okok(K, shift);
  if (nthreads < 1) nthreads = 1;
  search_job *jobs = calloc(nthreads, sizeof(search_job));
  pthread_t *th = calloc(nthreads, sizeof(pthread_t));
  int64_t span = f1 - f0;
  for (int t = 0; t < nthreads; t++) {
    search_job *J = &jobs[t];
    J->K = K; J->shift = shift; J->s = &s; J->n43 = n43; J->okok = okok;
    J->f0 = f0 + span * t / nthreads;
    J->f1 = f0 + span * (t + 1) / nthreads;
    J->cap = cap;
    J->ks = malloc(sizeof(int) * (cap ? cap : 1));
    J->firsts = malloc(sizeof(int64_t) * (cap ? cap : 1));
    J->pos = malloc(sizeof(uint64_t) * (cap ? cap : 1));
    pthread_create(&th[t], NULL, search_worker, J);
  }
  int64_t total = 0, nc = 0;
  int err = 0;
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    search_job *J = &jobs[t];
    int64_t stored = J->count < J->cap ? J->count : J->cap;
    for (int64_t i = 0; i < stored && total + i < cap; i++) {
      ks[total + i] = J->ks[i];
      firsts[total + i] = J->firsts[i];
      pos[total + i] = J->pos[i];
    }
    total += J->count;
    nc += J->ncand;
    err |= J->err;
    free(J->ks); free(J->firsts); free(J->pos);
  }
  if (ncand) *ncand = nc;
  free(jobs); free(th); free(okok);
  return err ? -1 : total;
}

/* Order in which the reference's AVX2 search reaches a candidate position:
 * 4-word passes (cpuavx2.cpp:334), then the n59 loop order (= f), then the
 * word inside the pass (sito0..sito3, cpuavx2.cpp:465-817), then the bit. */
uint64_t ao_avx2_order_key(uint64_t pos) {
  uint64_t f = pos >> 10, w = (pos >> 6) & 15, b = pos & 63;
  return ((w / 4) << 60) | (f << 8) | ((w % 4) << 6) | b;
}

/* ---- ReportSolution / validation / hash: src/common/AP26.cpp:484-602 ----- */
static int validate_ap26(int k, int d, int64_t f) {            /* 513-543 */
  static const int base[] = {2, 3, 5, 7, 11, 13, 17, 19, 23};
  int64_t N;
  int j;
  if (f % 2 == 0) return 0;
  for (j = 0, N = f; j < k; j++) {
    if (N < 0 || N >= (INT64_C(1) << 62)) return -1;
    for (int i = 0; i < 9; i++)
      if (!ao_sprp(N, base[i])) return j;
    N += (int64_t)d * 2 * 3 * 5 * 7 * 11 * 13 * 17 * 19 * 23;
  }
  return j;
}

static int val_base2_ap26(int k, int d, int64_t f) {           /* 484-506 */
  int64_t N;
  int j;
  if (f % 2 == 0) return 0;
  for (j = 0, N = f; j < k; j++) {
    if (N < 0 || N >= (INT64_C(1) << 62)) return -1;
    if (!ao_sprp(N, 2)) return j;
    N += (int64_t)d * 2 * 3 * 5 * 7 * 11 * 13 * 17 * 19 * 23;
  }
  return j;
}

/* One ReportSolution call (AP26.cpp:549-602) against hash state *hash.
 * Appends "len K first\n" lines for reported APs (len >= 20) to sol (cap
 * bytes, NUL-terminated).  Returns 0, or -1 where the reference would exit
 * ("Computation error": not even a base-2 AP, or modulus out of range). */
int ao_report(int *hash, int len, int K, int64_t first, char *sol, int sol_cap) {
  *hash += (int)(first % 1000);
  *hash += len;
  if (*hash > MAXINTV) *hash -= MAXINTV;
  int i = validate_ap26(len, K, first);
  if (i < 0) return -1;
  if (i < len) {
    int b2 = val_base2_ap26(len, K, first);
    if (b2 < 0 || b2 < len) return -1;
    if (ao_report(hash, i, K, first, sol, sol_cap) < 0) return -1;
    return ao_report(hash, len - (i + 1), K,
                     first + (int64_t)(i + 1) * K * 2 * 3 * 5 * 7 * 11 * 13 * 17 * 19 * 23,
                     sol, sol_cap);
  }
  if (len >= MIN_REPORT && sol) {
    size_t used = strlen(sol);
    snprintf(sol + used, sol_cap > (int)used ? (size_t)sol_cap - used : 0, "%d %d %lld\n",
             len, K, (long long)first);
  }
  return 0;
}

/* write_hash (AP26.cpp:295-357): 16 uppercase hex digits. */
int ao_hash_hex(int kmin, int kmax, int hash, char *out17) {
  uint64_t minmax = (uint64_t)(kmin + kmax);
  while (minmax > MAXINTV) minmax -= MAXINTV;
  unsigned int solhash = (unsigned int)hash;
  int64_t h = (int64_t)((minmax << 32) | solhash);
  char hex[16];
  memset(hex, '0', 16);
  int i = 0;
  while (h != 0) {
    int t = (int)(h % 16);
    hex[i++] = (char)(t < 10 ? t + 48 : t + 55);
    h /= 16;
  }
  for (int j = 0; j < 16; j++) out17[j] = hex[15 - j];
  out17[16] = 0;
  return 0;
}

/* will_search (AP26.cpp:649-653) */
int ao_will_search(int K) {
  return K % 29 && K % 31 && K % 37 && K % 41 && K % 43 && K % 47 && K % 53 && K % 59;
}
