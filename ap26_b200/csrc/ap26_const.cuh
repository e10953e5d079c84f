// ap26_const.cuh -- compile-time constants of the AP26 search.
//
// The numeric constants are the reference's (ibethune/ap26,
// src/common/CONST.H:7-27); the per-prime parameters below are derived from
// them at compile time for the bitstring-window sieve formulation described
// at the top of ap26_kernels.cuh.
#pragma once
#include <stdint.h>

namespace ap26 {

constexpr int64_t PRIM23 = 223092870LL;            // 23#          CONST.H:7
constexpr int64_t MOD = 258559632607830LL;         // 30*29*...*59 CONST.H:16
constexpr int64_t N0 = 106990415896110LL;          // CONST.H:17
constexpr int64_t N30 = 94805198622871LL;          // CONST.H:18
constexpr int64_t S3 = 172373088405220LL;          // CONST.H:19
constexpr int64_t S5 = 51711926521566LL;           // CONST.H:20
constexpr int64_t PRES2 = 16681266619860LL;        // CONST.H:21-27
constexpr int64_t PRES3 = 181690552643340LL;
constexpr int64_t PRES4 = 132432982555230LL;
constexpr int64_t PRES5 = 126273308948010LL;
constexpr int64_t PRES6 = 115526644356690LL;
constexpr int64_t PRES7 = 48784836341100LL;
constexpr int64_t PRES8 = 100794433050510LL;

// Lattice sizes (src/opencl/AP26.h:122-123, setupn.cl:31-35).
constexpr int NUM_TRIPLES = 1355;        // admissible (i31, i37, i41)
constexpr int NUM_N43 = 10840;           // NUM_TRIPLES * 2 (i3) * 4 (i5)
constexpr int N53_PER_N43 = 12673;       // 19 * 23 * 29
constexpr int64_t N53_PER_K = 137375320; // NUM_N43 * N53_PER_N43
constexpr int J59 = 35;                  // i59 steps per n53
constexpr int WORDS = 10;                // 64-bit shift words per K

constexpr int NPRIMES = 83;
constexpr int PRIMES[NPRIMES] = {
    61,  67,  71,  73,  79,  83,  89,  97,  101, 103, 107, 109, 113, 127, 131,
    137, 139, 149, 151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211,
    223, 227, 229, 233, 239, 241, 251, 257, 263, 269, 271, 277, 281, 283, 293,
    307, 311, 313, 317, 331, 337, 347, 349, 353, 359, 367, 373, 379, 383, 389,
    397, 401, 409, 419, 421, 431, 433, 439, 443, 449, 457, 461, 463, 467, 479,
    487, 491, 499, 503, 509, 521, 523, 541};

// Each bitstring covers its period + WIN_EXTRA bits: enough for a 640-bit
// window (plus a 32-bit funnel word) starting anywhere in one period,
// rounded up to an even word count.  The first four primes are held in two
// pair bitstrings, of periods 61 * 67 (PAIR1_P) and 71 * 73 (PAIR2_P): bit j
// of a pair's string is B_p[j] & B_q[j], and a lattice value's window in it
// starts at n59 * MOD^-1 mod (p*q), whose residues mod p and mod q are the
// two primes' own starts.  Primes 4..82 follow, one bitstring each.
constexpr int WIN_EXTRA = 672;
constexpr int PAIR1_P = 61 * 67;                     // 4087
constexpr int PAIR2_P = 71 * 73;                     // 5183
constexpr int nwords(int p) { return ((p + WIN_EXTRA + 31) / 32 + 1) & ~1; }
constexpr int PAIR1_WORDS = nwords(PAIR1_P);         // 150
constexpr int PAIR2_WORDS = nwords(PAIR2_P);         // 184
constexpr int PAIR_PRIMES = 4;                       // primes held in the pairs
constexpr int word_offset(int g) {                   // g >= PAIR_PRIMES
  int o = PAIR1_WORDS + PAIR2_WORDS;
  for (int i = PAIR_PRIMES; i < g; i++) o += nwords(PRIMES[i]);
  return o;
}
constexpr int TABLE_WORDS = word_offset(NPRIMES);   // 2806 words, 11224 bytes

// Lattice order.  The 12673 n53 starts of one n43 value (index j43*667 +
// j47*29 + j53) are visited sorted by their window starts in the pair
// bitstrings: the start in the 61*67 string is k1 = (j43*d43 + j47*d47 +
// j53*d53) mod 4087 (d = S * MOD^-1 mod 4087) up to the reductions mod MOD
// (at most 3), and k2 likewise mod 5183.  Starts are ordered by k1 in
// buckets of ORDER_BUCKET values, and by k2 inside a bucket (about 320
// starts each).  The 32 starts of a warp then lie within about 230 bits of
// each other in the first string and 870 bits in the second, and the 8
// starts of a quarter warp (one phase of a 128-bit load) nearly always
// within 8 consecutive quad entries: a CPU model of the order counts no
// extra wavefronts for the first string and 1-3% for the second.  The
// order is one 16-bit index per start, built with the tables.
constexpr int ORDER_BUCKET = 103;
constexpr int PERM_WORDS = (N53_PER_N43 + 1) / 2;   // 6337 words
constexpr int JOB_TABLE_WORDS = TABLE_WORDS + PERM_WORDS;   // per K-job, 36,572 bytes

constexpr int64_t mod_pos(int64_t a, int64_t m) { return ((a % m) + m) % m; }
constexpr int inv_mod(int a, int p) {                // a^-1 mod p, a coprime to p
  int t = 0, nt = 1, r = p, nr = ((a % p) + p) % p;
  while (nr != 0) {
    int q = r / nr, tmp = t - q * nt;
    t = nt; nt = tmp;
    tmp = r - q * nr; r = nr; nr = tmp;
  }
  return t < 0 ? t + p : t;
}
constexpr int ilog2(int x) { int k = 0; while ((2 << k) <= x) k++; return k; }

// Window start of prime p for a lattice value n59 = a + b*2^16 + c*2^32:
//   s = n59 * MOD^-1  (mod p) = (a*A + b*B + c*C) mod p.
// x = a*A + b*B + c*C < 3 * 2^16 * 541 < 2^28, and
//   x mod p = x - p * (umulhi(x, M) >> k),  k = floor(log2 p),
//   M = ceil(2^(32+k) / p) < 2^32,
// is exact for every x < 2^31 (round-up reciprocal, error x*(M*p-2^(32+k))
// / (p*2^(32+k)) < 1/p).
// For the pair bitstrings (p = 4087, 5183) x < 3 * 2^16 * 5183 < 2^30, and
// the reduction was checked exhaustively for every x < 2^30 with both.
struct PrimeParam {
  int p, A, B, C, k, off;
  uint32_t M;
};
constexpr PrimeParam make_param_p(int p, int off) {
  int minv = inv_mod((int)(MOD % p), p);
  int A = minv;
  int B = (int)(((int64_t)65536 % p) * minv % p);
  int C = (int)((((int64_t)1 << 32) % p) * minv % p);
  int k = ilog2(p);
  uint64_t M = ((uint64_t)1 << (32 + k)) / (uint64_t)p + 1;
  return PrimeParam{p, A, B, C, k, off, (uint32_t)M};
}
// Prime g's own bitstring (g >= 4; primes 0..3 only exist in the pairs).
constexpr PrimeParam make_param(int g) {
  return make_param_p(PRIMES[g], g >= PAIR_PRIMES ? word_offset(g) : 0);
}
constexpr PrimeParam PAIR1_PARAM = make_param_p(PAIR1_P, 0);
constexpr PrimeParam PAIR2_PARAM = make_param_p(PAIR2_P, PAIR1_WORDS);
// Dense-phase windows: units 0 and 1 are the pair bitstrings (primes 0..3),
// unit u >= 2 is prime u + 2.
constexpr PrimeParam dense_param(int u) {
  return u == 0 ? PAIR1_PARAM : u == 1 ? PAIR2_PARAM : make_param(u + 2);
}

// Residue 0 test helpers for the 7..23 filter (sieve.cl:123-142,
// cpusse2.cpp:563-568).
constexpr int SMALL_PRIMES[6] = {7, 11, 13, 17, 19, 23};

}  // namespace ap26
