/* ap26_cli.c -- the `ap26` command: AP26 KMIN KMAX SHIFT [-compute]
 *                [-device N] [-batch N]
 *
 * Keeps the reference's command-line contract (ibethune/ap26
 * src/common/AP26.cpp:660-1041): resume from AP26-state.{a,b}.txt, search
 * every K in [KMIN, KMAX] with will_search(K), checkpoint before each K,
 * append "len K first" lines for APs of length >= 20 and, at the end, the
 * 16-hex-digit result hash to SOL-AP26.txt.  The per-K search runs on the
 * GPU through libap26.so (ap26_search_k in place of SearchAP26 at
 * AP26.cpp:976).  -batch N searches N K at a time through the batched
 * persistent form; output is identical.
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

/* ReportSolution (AP26.cpp:549-602) through the library's hash/validation,
 * writing the SOL lines it produces. */
static void report_all(const ap26_ap *aps, int n) {
  for (int i = 0; i < n; i++) {
    char sol[4096];
    int sol_len = 0;
    sol[0] = 0;
    int rc = ap26_report(&result_hash, aps[i].k, aps[i].K, aps[i].first, sol, sizeof sol, &sol_len);
    if (rc == AP26_E_INVALID) {
      printf("Error: Computation error, found invalid AP, exiting...\n");
      die("Error: Computation error, found invalid AP");
    }
    if (rc != AP26_OK) die(ap26_strerror(rc));
    if (sol_len) {
      if (!results_file) results_file = fopen(RESULTS_FILENAME, "a");
      if (!results_file) die("Cannot open " RESULTS_FILENAME " !!!");
      char *line = sol;
      while (*line) {
        char *nl = strchr(line, '\n');
        printf("Solution: %.*s\n", (int)(nl - line), line);
        line = nl + 1;
      }
      if (fputs(sol, results_file) < 0) die("Cannot write to " RESULTS_FILENAME " !!!");
    }
  }
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
  int K, SHIFT, ITER = 0, device = 0, batch = 0;
  printf("AP26 B200 10-shift search version 1.0 (sm_100a, libap26 %d)\n", ap26_version());
  fprintf(stderr, "Command line: ");
  for (int i = 0; i < argc; i++) fprintf(stderr, "%s ", argv[i]);
  fprintf(stderr, "\n");
  if (argc < 4) {
    printf("Usage: %s KMIN KMAX SHIFT [-compute] [-device N] [-batch N]\n", argv[0]);
    exit(EXIT_FAILURE);
  }
  sscanf(argv[1], "%d", &KMIN);
  sscanf(argv[2], "%d", &KMAX);
  sscanf(argv[3], "%d", &SHIFT);
  for (int i = 4; i < argc; i++) {
    if (!strcmp(argv[i], "-compute")) fprintf(stderr, "Compute mode enabled.\n");
    else if (!strcmp(argv[i], "-device") && i + 1 < argc) device = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-batch") && i + 1 < argc) batch = atoi(argv[++i]);
  }
  if (ap26_read_state("", KMIN, KMAX, SHIFT, &K, &ITER, &result_hash, &last_trickle,
                      &write_state_a_next)) {
    printf("Resuming search from checkpoint.\n");
    fprintf(stderr, "Resuming from checkpoint. K: %d ITER: %d\n", K, ITER);
    if (ITER != 0) {   /* GPU builds restart a K from its first word (AP26.cpp:792-801) */
      printf("Checkpoint was from a different version. Restarting workunit.\n");
      fprintf(stderr, "Checkpoint was from a different version. Restarting workunit.\n");
      K = KMIN;
      ITER = 0;
      result_hash = 0;
      last_trickle = (double)time(NULL);
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
  while (K <= KMAX) {
    if (batch > 1) {
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
      report_all(aps, (int)n);
      fprintf(stderr, "K %d..%d done in %d sec (%.1f ms device).\n", K, kend - 1,
              (int)(time(NULL) - t0), st.device_ms);
      K_DONE += nk;
      K = kend;
      ITER = 0;
      continue;
    }
    if (ap26_will_search(K)) {
      checkpoint(SHIFT, K, ITER);
      int n = 0;
      ap26_stats st;
      time_t t0 = time(NULL);
      rc = ap26_search_k(ctx, K, SHIFT, aps, cap, &n, &st);
      if (rc != AP26_OK) die(ap26_strerror(rc));
      report_all(aps, n);
      fprintf(stderr, "K %d done in %d sec (%.1f ms device, %lld candidates).\n", K,
              (int)(time(NULL) - t0), st.device_ms, (long long)st.candidates);
      ITER = 0;
      K_DONE++;
    }
    K++;
  }
  checkpoint(SHIFT, K, ITER);     /* final, K = KMAX + 1 (AP26.cpp:989) */
  write_hash_line();
  fprintf(stderr, "Workunit complete.\n");
  free(aps);
  ap26_destroy(ctx);
  return EXIT_SUCCESS;
}
