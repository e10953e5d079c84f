/* ap26_avx512.c -- test infrastructure and CPU baseline companion, not
 * product code: nothing in ap26_b200/ links, loads or calls it.
 *
 * A second CPU restatement of the per-K search (ibethune/ap26), written for
 * AVX-512 (F/VL/BW/DQ + VBMI2) where the reference stops at AVX2
 * (src/cpu/cpuavx2.cpp).  Same results as the plain oracle (ap26_oracle.c):
 * the candidate set of a lattice range, and the raw reports with the
 * candidate each comes from.  Two changes of method, both exact:
 *
 *   sieve  Instead of one OKOK_{p,w} table per prime and shift word
 *          (cpusse2.cpp:38-43, sieve.cl:28-113), bit i of the 640-bit
 *          mask of all 10 words is B_p[s + i] with s = n59 * MOD^-1 mod p and
 *          B_p[j] = OK_p[((j + SHIFT) * MOD) mod p], a p-periodic bitstring.
 *          61 and 67 share one string of period 61*67 (bit j = B_61[j] &
 *          B_67[j]), as do 71 and 73: 81 strings for the 83 primes, about
 *          12 KB per K and SHIFT.  The ten 64-bit window words of a string
 *          are two unaligned vector loads each and one VPSHRDVQ
 *          (concatenate-and-shift) per 8 words, ANDed into the mask; the
 *          strings run in ascending order and stop when all ten words are
 *          zero.  The window starts of a lattice value are computed for 8
 *          strings at a time in double precision (exact below 2^53) and
 *          advanced with the n59 step as 16-lane integer adds.
 *   chain  The base-2 strong-PRP walk of cpuavx2.cpp:532-552 with a 64-bit
 *          Montgomery product (REDC, R = 2^64, N < 2^62) instead of the x87
 *          quotient estimate of PrimeQ_x86.h:114-136; same verdicts.
 *
 * Entry points return -2 when the CPU lacks AVX-512 VBMI2 (a5_supported()).
 */
#include <immintrin.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int ao_setup(int K, int64_t *out);
int ao_n43(int K, int64_t *out);
int ao_ok_table(int K, int p, uint8_t *out);
int ao_prime(int i);
uint64_t ao_avx2_order_key(uint64_t pos);

#define MOD INT64_C(258559632607830)       /* src/common/CONST.H:16 */
#define NPR 83
#define NUM_N43 10840
#define PER_N43 443555
#define TGT __attribute__((target("avx512f,avx512vl,avx512bw,avx512dq,avx512vbmi2")))

int a5_supported(void) {
  __builtin_cpu_init();
  return __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512vl") &&
         __builtin_cpu_supports("avx512bw") && __builtin_cpu_supports("avx512dq") &&
         __builtin_cpu_supports("avx512vbmi2");
}

/* ---- per-(K, SHIFT) tables ------------------------------------------------ */
/* Sieve units: the pair strings of 61*67 and 71*73 (bit t = B_p[t] & B_q[t],
 * period p*q; a lattice value's window starts at n59 * MOD^-1 mod p*q,
 * whose residues mod p and q are the two primes' own starts), then primes
 * 79..541 one string each: 81 units for the 83 primes. */
#define NU 81
#define NUV 96                       /* padded to 6 vectors of 16 lanes */
typedef struct {
  uint32_t P[NUV];                   /* unit period                                */
  uint32_t minv[NUV];                /* MOD^-1 mod P                               */
  uint32_t dv[NUV], dw[NUV];         /* S59 * MOD^-1 mod P, and that minus 1 (wrap) */
  uint32_t off[NUV];                 /* the unit's first word in tabs               */
  double invP[NUV];
  uint64_t *tabs;                    /* all units' strings, bit t = unit bit t mod P */
  int64_t s[9];                      /* STEP, n0, S31, S37, S41, S43, S47, S53, S59 */
  int64_t n43[NUM_N43];
  int shift;
} a5_k;

static int inv_mod(int a, int p) {   /* a^-1 mod p by the extended Euclid */
  int t = 0, nt = 1, r = p, nr = ((a % p) + p) % p;
  while (nr) {
    int q = r / nr, x = t - q * nt;
    t = nt; nt = x;
    x = r - q * nr; r = nr; nr = x;
  }
  return t < 0 ? t + p : t;
}

static a5_k *a5_build(int K, int shift) {
  a5_k *k = calloc(1, sizeof(a5_k));
  ao_setup(K, k->s);
  ao_n43(K, k->n43);
  k->shift = shift;
  static const int pair[2][2] = {{61, 67}, {71, 73}};
  uint8_t ok[NPR][541];
  int pr[NPR];
  for (int i = 0; i < NPR; i++) {
    pr[i] = ao_prime(i);
    ao_ok_table(K, pr[i], ok[i]);
  }
  uint32_t total = 0;
  for (int u = 0; u < NU; u++) {
    const int P = u < 2 ? pair[u][0] * pair[u][1] : pr[u + 2];
    k->P[u] = (uint32_t)P;
    k->off[u] = total;
    total += (uint32_t)((P - 1) / 64 + 12);   /* window words up to (s >> 6) + 10 */
  }
  k->tabs = calloc(total, sizeof(uint64_t));
  for (int u = 0; u < NU; u++) {
    const int P = (int)k->P[u];
    const int np = u < 2 ? 2 : 1;
    const int ps[2] = {u < 2 ? pair[u][0] : P, u < 2 ? pair[u][1] : P};
    const int nw = (P - 1) / 64 + 12;
    uint64_t *tab = k->tabs + k->off[u];
    for (int t = 0; t < nw * 64; t++) {
      int on = 1;
      for (int q = 0; q < np && on; q++) {
        const int p = ps[q], gi = u < 2 ? 2 * u + q : u + 2;
        const int mp = (int)(MOD % p), j = t % p;
        on = ok[gi][(int)(((int64_t)(j + shift % p) * mp) % p)];
      }
      if (on) tab[t >> 6] |= 1ull << (t & 63);
    }
    const int mP = (int)(MOD % P);
    k->minv[u] = (uint32_t)inv_mod(mP, P);
    k->invP[u] = 1.0 / P;
    k->dv[u] = (uint32_t)((int64_t)(k->s[8] % P) * k->minv[u] % P);
    k->dw[u] = (k->dv[u] + (uint32_t)P - 1) % (uint32_t)P;
  }
  for (int u = NU; u < NUV; u++) {
    k->P[u] = 1; k->minv[u] = 0; k->dv[u] = 0; k->dw[u] = 0; k->off[u] = 0; k->invP[u] = 1.0;
  }
  return k;
}

static void a5_free(a5_k *k) {
  free(k->tabs);
  free(k);
}

/* n59 at flat position f (cpuavx2.cpp:397-410, 822-851), as ap26_oracle.c */
static int64_t n59_of(const a5_k *k, int64_t f) {
  int64_t i = f / PER_N43, r = f % PER_N43;
  int j43 = (int)(r / 23345); r %= 23345;
  int j47 = (int)(r / 1015);  r %= 1015;
  int j53 = (int)(r / 35);
  int j59 = (int)(r % 35);
  int64_t v = k->n43[i];
  v = (v + (int64_t)j43 * k->s[5] % MOD) % MOD;
  v = (v + (int64_t)j47 * k->s[6] % MOD) % MOD;
  v = (v + (int64_t)j53 * k->s[7] % MOD) % MOD;
  v = (v + (int64_t)j59 * k->s[8] % MOD) % MOD;
  return v;
}

/* x mod P for 8 lanes of doubles holding integers below 2^53: the quotient
 * estimate floor(x / P) is off by at most one, so one correction each way. */
TGT static inline __m512d mod_pd(__m512d x, __m512d P, __m512d iP) {
  const __m512d q = _mm512_roundscale_pd(_mm512_mul_pd(x, iP),
                                         _MM_FROUND_TO_NEG_INF | _MM_FROUND_NO_EXC);
  __m512d r = _mm512_fnmadd_pd(q, P, x);
  r = _mm512_mask_add_pd(r, _mm512_cmp_pd_mask(r, _mm512_setzero_pd(), _CMP_LT_OQ), r, P);
  r = _mm512_mask_sub_pd(r, _mm512_cmp_pd_mask(r, P, _CMP_GE_OQ), r, P);
  return r;
}

/* Window starts s_u = n59 * MOD^-1 mod P_u of all units (n59 < 2^48). */
TGT static void starts_of(const a5_k *k, int64_t n59, uint32_t *st) {
  const __m512d x = _mm512_set1_pd((double)n59);
  for (int v = 0; v < NUV; v += 8) {
    const __m512d P = _mm512_cvtepu32_pd(_mm256_loadu_si256((const __m256i *)(k->P + v)));
    const __m512d iP = _mm512_loadu_pd(k->invP + v);
    const __m512d mi = _mm512_cvtepu32_pd(_mm256_loadu_si256((const __m256i *)(k->minv + v)));
    const __m512d r = mod_pd(x, P, iP);                       /* n59 mod P */
    const __m512d s = mod_pd(_mm512_mul_pd(r, mi), P, iP);    /* < 2^25 before the mod */
    _mm256_storeu_si256((__m256i *)(st + v), _mm512_cvttpd_epu32(s));
  }
}

/* n59 -> n59 + S59 (mod MOD): every start advances by S59 * MOD^-1 mod P,
 * and by one less when the sum wrapped (MOD is not 0 mod P). */
TGT static void advance_starts(const a5_k *k, uint32_t *st, int wrapped) {
  const uint32_t *d = wrapped ? k->dw : k->dv;
  for (int v = 0; v < NUV; v += 16) {
    __m512i x = _mm512_add_epi32(_mm512_loadu_si512(st + v), _mm512_loadu_si512(d + v));
    x = _mm512_min_epu32(x, _mm512_sub_epi32(x, _mm512_loadu_si512(k->P + v)));
    _mm512_storeu_si512(st + v, x);
  }
}

/* First table word of each unit's window: off_u + s_u / 64. */
TGT static void window_words(const a5_k *k, const uint32_t *st, uint32_t *idx) {
  for (int v = 0; v < NUV; v += 16)
    _mm512_storeu_si512(idx + v, _mm512_add_epi32(_mm512_loadu_si512(k->off + v),
                                                  _mm512_srli_epi32(_mm512_loadu_si512(st + v), 6)));
}

/* The sieved 640-bit mask of n59 (window starts st, first words idx):
 * m[0..9] = words 0..9.  All ten words in every step (8 + 2 lanes).  The
 * first 20 units run unconditionally (the mask of under 1% of lattice
 * values dies before unit 20) and the mask is then tested for zero every
 * second unit, in one test of the OR of both parts.  (A scalar per-word
 * tail after 12-24 vector primes, as the GPU kernel does, measured
 * 1.3-2.7x slower here: the branch on each word's death mispredicts.)  The
 * shift of a window is broadcast as a 32-bit value: VPSHRDVQ reads the low
 * 6 bits of each 64-bit count, s mod 64. */
TGT static void sieve_n59(const a5_k *k, const uint32_t *st, const uint32_t *idx, uint64_t m[10]) {
  __m512i acc8 = _mm512_set1_epi64(-1);
  __m128i acc2 = _mm_set1_epi64x(-1);
  const uint64_t *tabs = k->tabs;
  for (int u = 0; u < NU; u++) {
    const uint64_t *t = tabs + idx[u];
    const __m512i sh = _mm512_set1_epi32((int)st[u]);
    acc8 = _mm512_and_si512(acc8, _mm512_shrdv_epi64(_mm512_loadu_si512(t),
                                                     _mm512_loadu_si512(t + 1), sh));
    acc2 = _mm_and_si128(acc2, _mm_shrdv_epi64(_mm_loadu_si128((const __m128i *)(t + 8)),
                                               _mm_loadu_si128((const __m128i *)(t + 9)),
                                               _mm512_castsi512_si128(sh)));
    if (u >= 19 && (u & 1) == 1 &&
        !_mm512_test_epi64_mask(_mm512_or_si512(acc8, _mm512_zextsi128_si512(acc2)),
                                _mm512_or_si512(acc8, _mm512_zextsi128_si512(acc2))))
      break;
  }
  _mm512_storeu_si512(m, acc8);
  _mm_storeu_si128((__m128i *)(m + 8), acc2);
}

/* ---- base-2 strong PRP, 64-bit Montgomery (N odd, 3 <= N < 2^62) ---------- */
typedef unsigned __int128 u128;
static inline uint64_t redc(u128 t, uint64_t N, uint64_t ninv) {
  uint64_t m = (uint64_t)t * ninv;
  uint64_t r = (uint64_t)((t + (u128)m * N) >> 64);
  return r >= N ? r - N : r;
}
static int sprp2(uint64_t N) {                /* verdict of strong_prp(2, N) */
  uint64_t ninv = N;
  for (int i = 0; i < 5; i++) ninv *= 2 - N * ninv;
  ninv = 0 - ninv;
  const uint64_t one = (uint64_t)(((u128)1 << 64) % N), mone = N - one;
  const uint64_t nm1 = N - 1;
  const int t = __builtin_ctzll(nm1);
  const uint64_t d = nm1 >> t;
  uint64_t x = one + one;
  if (x >= N) x -= N;
  for (int i = 62 - __builtin_clzll(d); i >= 0; i--) {
    x = redc((u128)x * x, N, ninv);
    if ((d >> i) & 1) { x += x; if (x >= N) x -= N; }
  }
  if (x == one || x == mone) return 1;
  for (int s = 1; s < t; s++) {
    x = redc((u128)x * x, N, ninv);
    if (x == mone) return 1;
    if (x == one) return 0;
  }
  return 0;
}
/* PrimeQ (PrimeQ_x86.h:189-198): -1 outside its domain */
static int primeq(int64_t N) {
  if ((uint64_t)N >= (UINT64_C(1) << 62)) return -1;
  if (N < 3 || !(N & 1)) return 0;
  return sprp2((uint64_t)N);
}
/* chain walk, cpuavx2.cpp:532-552 */
static int chain(int64_t n, int64_t STEP, int *k_out, int64_t *first_out) {
  int k = 0, q;
  int64_t m = n + STEP * 5;
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

/* ---- workers ---------------------------------------------------------------- */
typedef struct {
  const a5_k *k;
  int64_t f0, f1, cap, count, ncand;
  int walk, err;
  int64_t *cand;               /* sieve: candidate n */
  int *ks; int64_t *firsts, *ns; uint64_t *pos;
} a5_job;

static void *worker(void *arg) {
  a5_job *J = (a5_job *)arg;
  const a5_k *k = J->k;
  uint64_t m[10];
  uint32_t st[NUV] __attribute__((aligned(64)));
  uint32_t idx[NUV] __attribute__((aligned(64)));
  int64_t n59 = 0;
  for (int64_t f = J->f0; f < J->f1; f++) {
    if (f == J->f0 || f % 35 == 0) {        /* new n53: starts from scratch */
      n59 = n59_of(k, f);
      starts_of(k, n59, st);
    } else {                                /* next j59: n59 += S59 (mod MOD) */
      n59 += k->s[8];
      const int wrapped = n59 >= MOD;
      if (wrapped) n59 -= MOD;
      advance_starts(k, st, wrapped);
    }
    window_words(k, st, idx);
    sieve_n59(k, st, idx, m);
    for (int w = 0; w < 10; w++) {
      uint64_t bits = m[w];
      while (bits) {
        const int b = __builtin_ctzll(bits);
        bits &= bits - 1;
        const int64_t n = n59 + (int64_t)(b + k->shift + 64 * w) * MOD;
        if (!(n % 7 && n % 11 && n % 13 && n % 17 && n % 19 && n % 23)) continue;
        if (!J->walk) {
          if (J->count < J->cap) J->cand[J->count] = n;
          J->count++;
          continue;
        }
        J->ncand++;
        int kk;
        int64_t first;
        if (chain(n, k->s[0], &kk, &first) < 0) { J->err = 1; continue; }
        if (kk >= 10) {
          if (J->count < J->cap) {
            J->ks[J->count] = kk;
            J->firsts[J->count] = first;
            J->ns[J->count] = n;
            J->pos[J->count] = ((uint64_t)f << 10) | ((uint64_t)w << 6) | (uint64_t)b;
          }
          J->count++;
        }
      }
    }
  }
  return NULL;
}

static int64_t run(int K, int shift, int64_t f0, int64_t f1, int walk, int64_t *cand, int *ks,
                   int64_t *firsts, int64_t *ns, uint64_t *pos, int64_t cap, int64_t *ncand,
                   int nthreads) {
  if (!a5_supported()) return -2;
  if (nthreads < 1) nthreads = 1;
  a5_k *k = a5_build(K, shift);
  a5_job *jobs = calloc(nthreads, sizeof(a5_job));
  pthread_t *th = calloc(nthreads, sizeof(pthread_t));
  const int64_t span = f1 - f0;
  for (int t = 0; t < nthreads; t++) {
    a5_job *J = &jobs[t];
    J->k = k;
    J->walk = walk;
    J->f0 = f0 + span * t / nthreads;
    J->f1 = f0 + span * (t + 1) / nthreads;
    J->cap = cap;
    const int64_t c = cap ? cap : 1;
    if (walk) {
      J->ks = malloc(sizeof(int) * c);
      J->firsts = malloc(sizeof(int64_t) * c);
      J->ns = malloc(sizeof(int64_t) * c);
      J->pos = malloc(sizeof(uint64_t) * c);
    } else {
      J->cand = malloc(sizeof(int64_t) * c);
    }
    pthread_create(&th[t], NULL, worker, J);
  }
  int64_t total = 0, nc = 0;
  int err = 0;
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    a5_job *J = &jobs[t];
    const int64_t stored = J->count < J->cap ? J->count : J->cap;
    for (int64_t i = 0; i < stored && total + i < cap; i++) {
      if (walk) {
        ks[total + i] = J->ks[i];
        firsts[total + i] = J->firsts[i];
        ns[total + i] = J->ns[i];
        pos[total + i] = J->pos[i];
      } else {
        cand[total + i] = J->cand[i];
      }
    }
    total += J->count;
    nc += J->ncand;
    err |= J->err;
    free(J->cand); free(J->ks); free(J->firsts); free(J->ns); free(J->pos);
  }
  if (ncand) *ncand = nc;
  free(jobs);
  free(th);
  a5_free(k);
  return err ? -1 : total;
}

/* Candidates (after the 7..23 filter) of lattice positions [f0, f1) of
 * (K, SHIFT), unordered; returns the count (may exceed cap). */
int64_t a5_sieve(int K, int shift, int64_t f0, int64_t f1, int64_t *cand, int64_t cap,
                 int nthreads) {
  return run(K, shift, f0, f1, 0, cand, NULL, NULL, NULL, NULL, cap, NULL, nthreads);
}

/* Raw reports (k >= 10) of lattice positions [f0, f1): k, first, candidate n
 * and position (f << 10 | w << 6 | b, ordered by ao_avx2_order_key as the
 * reference's AVX2 build meets them); returns the count, -1 on a PrimeQ
 * domain violation. */
int64_t a5_search(int K, int shift, int64_t f0, int64_t f1, int *ks, int64_t *firsts,
                  int64_t *ns, uint64_t *pos, int64_t cap, int64_t *ncand, int nthreads) {
  return run(K, shift, f0, f1, 1, NULL, ks, firsts, ns, pos, cap, ncand, nthreads);
}
