/* ref_harness.cpp -- test infrastructure, not product code.
 *
 * Drives the reference CPU search (ibethune/ap26, src/cpu/cpuavx2.cpp:72
 * Search_avx2 and src/cpu/cpusse2.cpp:46 Search_sse2), compiled unmodified
 * from the reference sources by oracle/build_ref.sh, through the callback ABI
 * the reference declares in src/cpu/cpuavx2.h:5-9.  This file supplies those
 * callbacks itself:
 *
 *   ReportSolution  records every RAW report (k, K, first) exactly as the
 *                   search emits it (src/cpu/cpuavx2.cpp:551), before any
 *                   hash update or validation, so the record is the
 *                   reference's own candidate->AP output;
 *   PrimeQ          is the reference's own, from src/common/PrimeQ_x86.h
 *                   (included from the reference tree at build time), behind
 *                   a thin wrapper that counts sieve survivors: every
 *                   candidate n that passes the reference's sieve and its
 *                   7..23 / OK_p filters starts exactly one chain walk, whose
 *                   first call is PrimeQ(n + 5*STEP) (cpuavx2.cpp:532-546);
 *                   the wrapper tells first calls from the walk's
 *                   continuations (below) and counts them;
 *   checkpoint      no-op (the CLI's state handling is not under test here);
 *   Progress        counts ticks; in "sample" mode it ends the search early
 *                   with longjmp after a bounded number of ticks, which turns
 *                   the reference's whole-K search into a bounded CPU sample.
 *
 * Modes:
 *   ref_harness raw    K SHIFT [avx2|sse2]   -> "R k K first" lines, then
 *                      "COUNT survivors" and the summary
 *   ref_harness sample K SHIFT TICKS [avx2|sse2] [ITER]
 *                      -> "SAMPLE K n43_done total_n43_units seconds isa ITER
 *                          setup_seconds tick_seconds"
 *                      the pass starting at shift word ITER (0, 4 or 8 for
 *                      AVX2: Search_avx2's own resume point), aborted after
 *                      TICKS pairs; setup_seconds = start to the first tick
 *                      (tables of the pass), tick_seconds = first tick to the
 *                      abort (exactly n43_done lattice values of the pass)
 *
 * Progress accounting (sample mode): the AVX2 search calls Progress once per
 * admissible (i31, i37) pair of each 4-word pass (cpuavx2.cpp:380-388), the
 * SSE2 search once per pair of each 1-word pass (cpusse2.cpp:434-441).  Each
 * pair covers 8 * (#admissible i41) n43 values.  Aborting at tick T+1 of the
 * first pass therefore means exactly the n43 values of the first T pairs were
 * searched for that pass's words; a whole K is 10840 n43 values times the
 * number of passes (3 for AVX2, 10 for SSE2).
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>
#include <setjmp.h>
#include <time.h>

/* the reference's PrimeQ under another name; PrimeQ itself is the counting
 * wrapper defined below */
#define PrimeQ ref_PrimeQ
#include "PrimeQ_x86.h"   /* reference: src/common/PrimeQ_x86.h */
#undef PrimeQ

void Search_avx2(int K, int startSHIFT, int ITER, int K_COUNT, int K_DONE);
void Search_sse2(int K, int startSHIFT, int ITER, int K_COUNT, int K_DONE);

static int g_mode_sample = 0;
static long g_ticks = 0, g_tick_limit = 0;
static double g_t_first = 0, g_t_end = 0;
static double now_s(void);
static jmp_buf g_abort;
static long g_reports = 0;

void Progress(double prog) {
  (void)prog;
  g_ticks++;
  if (g_ticks == 1) g_t_first = now_s();
  if (g_mode_sample && g_ticks > g_tick_limit) {
    g_t_end = now_s();
    longjmp(g_abort, 1);
  }
}

/* Survivor count from the chain walk's call pattern (cpuavx2.cpp:532-546):
 *   k=0; m=n+5S; while (PrimeQ(m)) { k++; m+=S; }
 *   if (k>=10) { m=n+4S; while (m>0 && PrimeQ(m)) { k++; m-=S; } }
 * After a call that returned true the next call continues the same walk at
 * m+S (forward) or m-S (backward).  After a forward walk that ended false
 * with k >= 10 the next call is the backward start n+4S.  Every other call
 * is the first call of a new candidate.  A backward walk that stops at
 * m <= 0 makes no call, so a continuation is also checked by its argument. */
static int64_t g_step = 0;
static long long g_survivors = 0;
static int64_t g_last = 0, g_first = 0;
static int g_last_true = 0, g_fwd = 1, g_fwd_k = 0, g_started = 0;

int PrimeQ(int64_t N) {
  const int r = ref_PrimeQ(N);
  int cont = 0;
  if (g_started && g_last_true) {
    if (g_fwd && N == g_last + g_step) cont = 1;
    else if (!g_fwd && N == g_last - g_step) cont = 1;
  } else if (g_started && g_fwd && g_fwd_k >= 10 && N == g_first - g_step) {
    g_fwd = 0;                       /* backward start n + 4S */
    cont = 1;
  }
  if (!cont) {
    g_survivors++;
    g_started = 1;
    g_first = N;
    g_fwd = 1;
    g_fwd_k = 0;
  }
  if (g_fwd && r) g_fwd_k++;
  g_last = N;
  g_last_true = r;
  return r;
}

void ReportSolution(int AP_Length, int difference, int64_t First_Term) {
  g_reports++;
  if (!g_mode_sample)
    printf("R %d %d %lld\n", AP_Length, difference, (long long)First_Term);
}

void checkpoint(int SHIFT, int K, int force, int ITER) {
  (void)SHIFT; (void)K; (void)force; (void)ITER;
}

/* n43 count of the t-th admissible (i31, i37) pair, in the reference's loop
 * order (src/opencl/AP26.h:127-136, src/cpu/cpuavx2.cpp:380-395). */
static long n43_in_first_pairs(long T) {
  long pair = 0, n43 = 0;
  for (int i31 = 0; i31 < 7; ++i31)
    for (int i37 = 0; i37 < 13; ++i37) {
      if (!(i37 - i31 <= 10 && i31 - i37 <= 4)) continue;
      if (pair >= T) return n43;
      pair++;
      for (int i41 = 0; i41 < 17; ++i41)
        if (i41 - i31 <= 14 && i41 - i37 <= 14 && i31 - i41 <= 4 && i37 - i41 <= 10)
          n43 += 8;
    }
  return n43;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s raw K SHIFT [avx2|sse2] | sample K SHIFT TICKS [avx2|sse2]\n", argv[0]);
    return 2;
  }
  int K = atoi(argv[2]);
  int SHIFT = atoi(argv[3]);
  const char *isa = "avx2";
  int iter = 0;
  if (!strcmp(argv[1], "sample")) {
    if (argc < 5) return 2;
    g_mode_sample = 1;
    g_tick_limit = atol(argv[4]);
    if (argc > 5) isa = argv[5];
    if (argc > 6) iter = atoi(argv[6]);
  } else if (argc > 4) {
    isa = argv[4];
  }
  int use_sse2 = !strcmp(isa, "sse2");
  int passes = use_sse2 ? 10 : 3;

  g_step = (int64_t)K * 223092870LL;   /* K * 23#, CONST.H:7 */
  double t0 = now_s();
  if (setjmp(g_abort) == 0) {
    if (use_sse2) Search_sse2(K, SHIFT, iter, 1, 0);
    else Search_avx2(K, SHIFT, iter, 1, 0);
  }
  double dt = now_s() - t0;
  fflush(stdout);
  if (g_mode_sample) {
    long T = g_ticks - 1;           /* pairs fully searched in the pass */
    if (T < 0) T = 0;
    long done = n43_in_first_pairs(T);
    if (g_t_end == 0) g_t_end = now_s();   /* the pass ended before the limit */
    printf("SAMPLE %d %ld %ld %.6f %s %d %.6f %.6f\n", K, done, 10840L * passes, dt, isa, iter,
           g_t_first - t0, g_t_end - g_t_first);
  } else {
    printf("COUNT %lld\n", g_survivors);
    printf("DONE %d %ld %.3f %s\n", K, g_reports, dt, isa);
  }
  return 0;
}
