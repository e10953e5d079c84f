/* ap26_cli.c -- the `ap26` command: AP26 KMIN KMAX SHIFT [-compute]
 *                [-device N] [-batch N] [-stop-after N] [-stop-at-word W]
 *
 * Keeps the reference's command-line contract (ibethune/ap26
 * src/common/AP26.cpp:660-1041): resume from AP26-state.{a,b}.txt, search
 * every K in [KMIN, KMAX] with will_search(K), checkpoint before each K,
 * append "len K first" lines for APs of length >= 20 and, at the end, the
 * 16-hex-digit result hash to SOL-AP26.txt.  The per-K search runs on the
 * GPU through libap26.so: ap26_search_k_sol in place of SearchAP26 at
 * AP26.cpp:976 and of the ReportSolution calls on its results (hash,
 * 9-base validation and splits computed on the device).  -batch N searches
 * N K at a time through the batched persistent form and reports through
 * ap26_report_batch; output is identical.  -stop-after N ends the process
 * after N searched K with the checkpoint of the next K written and no hash
 * line, the way a BOINC client stops a task between K; running the command
 * again resumes there.
 *
 * Inside a K the command writes the states the reference's CPU build writes
 * between its 4-word passes (src/cpu/cpuavx2.cpp:858-861): the SOL lines of
 * shift words 0-3, then the state (K, ITER 4, hash of those words), the
 * lines of words 4-7, then (K, ITER 8, hash), from the per-word hash sums
 * the device keeps (ap26_search_k_sol_words).  -stop-at-word W (4 or 8)
 * ends the process right after the state with ITER W, as a client stopped
 * there would; running the command again continues K at shift word W.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "../../include/ap26.h"

#define RESULTS_FILENAME "SOL-AP26.txt"

static int KMIN, KMAX, K_DONE, K_COUNT;
static int32_t result_hash;
static double last_trickle;
static int write_state_a_next;
static FILE *results_file;

static void checkpoint(int SHIFT, int K, int ITER) {       /* AP26.cpp:607-645 */
  if (results_file) {
    fflush(results_file);
    fsync(fileno(results_file));
  }
  ap26_write_state("", KMIN, KMAX, SHIFT, K, ITER, result_hash, last_trickle, &write_state_a_next);
  printf("Checkpoint: KMIN:%d KMAX:%d SHIFT:%d K:%d ITER:%d\n", KMIN, KMAX, SHIFT, K, ITER);
}

static void die(const char *msg) {
  fprintf(stderr, "%s\n", msg);
  exit(EXIT_FAILURE);
}

static void computation_error(void) {                      /* AP26.cpp:569-574 */
  printf("Error: Computation error, found invalid AP, exiting...\n");
  die("Error: Computation error, found invalid AP");
}

/* Appends solutions to SOL-AP26.txt (AP26.cpp:585-598). */
static void write_sols(const ap26_sol *sol, int n) {
  for (int i = 0; i < n; i++) {
    if (!results_file) results_file = fopen(RESULTS_FILENAME, "a");
    if (!results_file) die("Cannot open " RESULTS_FILENAME " !!!");
    printf("Solution: %d %d %lld\n", sol[i].len, sol[i].K, (long long)sol[i].first);
    if (fprintf(results_file, "%d %d %lld\n", sol[i].len, sol[i].K, (long long)sol[i].first) < 0)
      die("Cannot write to " RESULTS_FILENAME " !!!");
  }
}

/* ReportSolution of raw reports, on the device (ap26_report_batch): the
 * hash advances and the solutions are written in report order. */
static void report_all(ap26_ctx *ctx, const ap26_ap *aps, int64_t n) {
  if (n <= 0) return;
  ap26_final *fin = (ap26_final *)malloc(sizeof(ap26_final) * (size_t)n);
  if (!fin) die("out of memory");
  int rc = ap26_report_batch(ctx, aps, n, fin, &result_hash, NULL);
  if (rc == AP26_E_INVALID) computation_error();
  if (rc != AP26_OK) die(ap26_strerror(rc));
  for (int64_t i = 0; i < n; i++)
    for (int j = 0; j < fin[i].n_sol; j++) {
      ap26_sol s = {fin[i].sol_len[j], aps[i].K, fin[i].sol_first[j]};
      write_sols(&s, 1);
    }
  free(fin);
}

static void write_hash_line(void) {                         /* AP26.cpp:295-357 */
  char hex[17];
  ap26_hash_hex(KMIN, KMAX, result_hash, hex);
  if (!results_file) results_file = fopen(RESULTS_FILENAME, "a");
  if (!results_file) die("Cannot open " RESULTS_FILENAME " !!!");
  if (fprintf(results_file, "%s\n", hex) < 0) die("Cannot write to " RESULTS_FILENAME " !!!");
  fclose(results_file);
  results_file = NULL;
}

int main(int argc, char **argv) {
  int K, SHIFT, ITER = 0, device = 0, batch = 0, stop_after = 0, searched = 0, stop_word = 0;
  printf("AP26 B200 10-shift search version 1.0 (sm_100a, libap26 %d)\n", ap26_version());
  fprintf(stderr, "Command line: ");
  for (int i = 0; i < argc; i++) fprintf(stderr, "%s ", argv[i]);
  fprintf(stderr, "\n");
  if (argc < 4) {
    printf("Usage: %s KMIN KMAX SHIFT [-compute] [-device N] [-batch N] [-stop-after N] "
           "[-stop-at-word W]\n", argv[0]);
    exit(EXIT_FAILURE);
  }
  sscanf(argv[1], "%d", &KMIN);
  sscanf(argv[2], "%d", &KMAX);
  sscanf(argv[3], "%d", &SHIFT);
  for (int i = 4; i < argc; i++) {
    if (!strcmp(argv[i], "-compute")) fprintf(stderr, "Compute mode enabled.\n");
    else if (!strcmp(argv[i], "-device") && i + 1 < argc) device = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-batch") && i + 1 < argc) batch = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-stop-after") && i + 1 < argc) stop_after = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-stop-at-word") && i + 1 < argc) stop_word = atoi(argv[++i]);
  }
  if (ap26_read_state("", KMIN, KMAX, SHIFT, &K, &ITER, &result_hash, &last_trickle,
                      &write_state_a_next)) {
    printf("Resuming search from checkpoint.\n");
    fprintf(stderr, "Resuming from checkpoint. K: %d ITER: %d\n", K, ITER);
    if (ITER < 0 || ITER > 9) {   /* not a shift word: restart (AP26.cpp:792-801) */
      printf("Checkpoint was from a different version. Restarting workunit.\n");
      fprintf(stderr, "Checkpoint was from a different version. Restarting workunit.\n");
      K = KMIN;
      ITER = 0;
      result_hash = 0;
      last_trickle = (double)time(NULL);
    } else if (ITER != 0) {
      /* A mid-K checkpoint of the reference's CPU build (ITER 4 or 8 before
         its 4-word passes): the reference's GPU build restarts the workunit
         here; this one continues K at shift word ITER with the hash of the
         words before it, which gives the uninterrupted run's output. */
      fprintf(stderr, "Continuing K %d from shift word %d.\n", K, ITER);
    }
  } else {
    printf("Beginning a new search with parameters from the command line\n");
    K = KMIN;
    ITER = 0;
    result_hash = 0;
    last_trickle = (double)time(NULL);
    write_state_a_next = 1;
  }

  ap26_ctx *ctx = NULL;
  int rc = ap26_create(device, NULL, &ctx);
  if (rc != AP26_OK) {
    fprintf(stderr, "ap26_create: %s\n", ap26_strerror(rc));
    exit(EXIT_FAILURE);
  }
  for (int i = KMIN; i <= KMAX; i++)
    if (ap26_will_search(i)) {
      K_COUNT++;
      if (K > i) K_DONE++;
    }
  printf("%d K in this range remaining to be searched (%d skipped, %d done).\n", K_COUNT - K_DONE,
         KMAX + 1 - KMIN - K_COUNT, K_DONE);

  const int cap = 1 << 16;
  ap26_ap *aps = (ap26_ap *)malloc(sizeof(ap26_ap) * cap);
  ap26_sol *sols = (ap26_sol *)malloc(sizeof(ap26_sol) * cap);
  int32_t *sol_word = (int32_t *)malloc(sizeof(int32_t) * cap);
  if (!aps || !sols || !sol_word) die("out of memory");
  while (K <= KMAX) {
    if (batch > 1 && ITER == 0) {   /* a K resumed mid-way goes through the per-K path */
      /* next group of up to `batch` searchable K */
      int kend = K, nk = 0;
      while (kend <= KMAX && nk < batch) { if (ap26_will_search(kend)) nk++; kend++; }
      if (nk == 0) { K = kend; continue; }
      checkpoint(SHIFT, K, ITER);
      ap26_item it = {0, K, kend - 1, SHIFT, 0};
      ap26_item_result res;
      int64_t n = 0;
      ap26_stats st;
      time_t t0 = time(NULL);
      rc = ap26_search_batch(ctx, &it, 1, aps, cap, &n, &res, &st);
      if (rc != AP26_OK) die(ap26_strerror(rc));
      report_all(ctx, aps, n);
      fprintf(stderr, "K %d..%d done in %d sec (%.1f ms device).\n", K, kend - 1,
              (int)(time(NULL) - t0), st.device_ms);
      K_DONE += nk;
      K = kend;
      ITER = 0;
      searched += nk;
      if (stop_after > 0 && searched >= stop_after && K <= KMAX) break;
      continue;
    }
    if (ap26_will_search(K)) {
      checkpoint(SHIFT, K, ITER);
      int n = 0;
      ap26_stats st;
      int32_t h = result_hash, hash_at[10];
      time_t t0 = time(NULL);
      /* SearchAP26 + ReportSolution of its results, both on the device */
      rc = ap26_search_k_sol_words(ctx, K, SHIFT, ITER, &h, hash_at, sols, sol_word, cap, &n,
                                   &st);
      if (rc == AP26_E_INVALID) computation_error();
      if (rc != AP26_OK) die(ap26_strerror(rc));
      /* the reference CPU build's pass boundaries: lines of the pass, then
         the checkpoint with the hash of the words before ITER */
      int written = 0;
      for (int it = 4; it < 10; it += 4) {
        if (it <= ITER) continue;
        int e = written;
        while (e < n && sol_word[e] < it) e++;
        write_sols(sols + written, e - written);
        written = e;
        result_hash = hash_at[it - 1];
        checkpoint(SHIFT, K, it);
        if (stop_word == it) {
          if (results_file) fclose(results_file);
          fprintf(stderr, "Stopped at shift word %d of K %d; resume with the same command.\n",
                  it, K);
          free(aps);
          free(sols);
          free(sol_word);
          ap26_destroy(ctx);
          return EXIT_SUCCESS;
        }
      }
      write_sols(sols + written, n - written);
      result_hash = h;
      fprintf(stderr, "K %d done in %d sec (%.1f ms device, %lld candidates).\n", K,
              (int)(time(NULL) - t0), st.device_ms, (long long)st.candidates);
      ITER = 0;
      K_DONE++;
      searched++;
    }
    K++;
    if (stop_after > 0 && searched >= stop_after && K <= KMAX) break;
  }
  if (K <= KMAX) {                /* stopped early: checkpoint, no hash line */
    checkpoint(SHIFT, K, 0);
    if (results_file) fclose(results_file);
    fprintf(stderr, "Stopped after %d K; resume with the same command.\n", searched);
    free(aps);
    free(sols);
    free(sol_word);
    ap26_destroy(ctx);
    return EXIT_SUCCESS;
  }
  checkpoint(SHIFT, K, ITER);     /* final, K = KMAX + 1 (AP26.cpp:989) */
  write_hash_line();
  fprintf(stderr, "Workunit complete.\n");
  free(aps);
  free(sols);
  free(sol_word);
  ap26_destroy(ctx);
  return EXIT_SUCCESS;
}
