/* ap26_host.c -- host services of libap26.so: the reference's result hash,
 * ReportSolution with 9-base re-validation, SOL line format, A/B checkpoint
 * files, and the ordering of raw reports.
 *
 * Restates ibethune/ap26 src/common/AP26.cpp:295-653 so that SOL-AP26.txt,
 * the hash line and the AP26-state.{a,b}.txt files written through this
 * library are byte-identical to the reference's.  Host-side only: no GPU
 * work happens here.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/ap26.h"
#include "ap26_hostcore.h"

#define PRIM23 INT64_C(223092870)
#define MOD INT64_C(258559632607830)
#define N0 INT64_C(106990415896110)
#define N30 INT64_C(94805198622871)
#define PRES2 INT64_C(16681266619860)
#define PRES3 INT64_C(181690552643340)
#define PRES4 INT64_C(132432982555230)
#define PRES5 INT64_C(126273308948010)
#define PRES6 INT64_C(115526644356690)
#define PRES7 INT64_C(48784836341100)
#define PRES8 INT64_C(100794433050510)
#define MAXINTV 2000000000               /* AP26.cpp:88  */
#define MIN_REPORT 20                    /* AP26.cpp:104 */
#define STATE_A "AP26-state.a.txt"       /* AP26.cpp:93  */
#define STATE_B "AP26-state.b.txt"       /* AP26.cpp:94  */

/* ---- lattice -------------------------------------------------------------- */
int ap26h_triples(uint16_t *out) {
  int n = 0;
  for (int i31 = 0; i31 < 7; ++i31)
    for (int i37 = 0; i37 < 13; ++i37)
      if (i37 - i31 <= 10 && i31 - i37 <= 4)
        for (int i41 = 0; i41 < 17; ++i41)
          if (i41 - i31 <= 14 && i41 - i37 <= 14 && i31 - i41 <= 4 && i37 - i41 <= 10) {
            if (out) out[n] = (uint16_t)(i31 | (i37 << 5) | (i41 << 10));
            n++;
          }
  return n;
}

static int64_t kmul(int64_t c, int K) {
  return (c * (K % 17835) + ((c * 17835) % MOD) * (K / 17835)) % MOD;
}

void ap26h_setup_k(int K, int64_t out[9]) {
  out[0] = (int64_t)K * PRIM23;
  out[1] = (N0 * (K % 17835) + ((N0 * 17835) % MOD) * (K / 17835) + N30) % MOD;
  out[2] = kmul(PRES2, K);
  out[3] = kmul(PRES3, K);
  out[4] = kmul(PRES4, K);
  out[5] = kmul(PRES5, K);
  out[6] = kmul(PRES6, K);
  out[7] = kmul(PRES7, K);
  out[8] = kmul(PRES8, K);
}

int ap26_will_search(int K) {                        /* AP26.cpp:649-653 */
  return (K % 29 && K % 31 && K % 37 && K % 41 && K % 43 && K % 47 && K % 53 && K % 59) ? 1 : 0;
}

static int mod_int(int64_t a, int m) { int r = (int)(a % m); return r < 0 ? r + m : r; }
static int inv_int(int a, int p) {
  int t = 0, nt = 1, r = p, nr = mod_int(a, p);
  while (nr) {
    int q = r / nr, tmp = t - q * nt;
    t = nt; nt = tmp;
    tmp = r - q * nr; r = nr; nr = tmp;
  }
  return t < 0 ? t + p : t;
}

/* Each wheel step S_q is 0 modulo every wheel prime but q (S3 = 1 mod 3,
 * S5 = 1 mod 5, S31 = 6K mod 31, ..., CONST.H:19-27), so n59 - n0 determines
 * every lattice index by one modular division. */
uint64_t ap26h_order_key(int K, int shift, int64_t n) {
  static int tri_index[7][13][17];
  static int tri_ready = 0;
  if (!tri_ready) {
    uint16_t t[1355];
    memset(tri_index, 0xff, sizeof tri_index);
    int cnt = ap26h_triples(t);
    for (int i = 0; i < cnt; i++) tri_index[t[i] & 31][(t[i] >> 5) & 31][(t[i] >> 10) & 31] = i;
    tri_ready = 1;
  }
  if (n < 0) return UINT64_MAX;
  int64_t s[9];
  ap26h_setup_k(K, s);
  const int64_t n59 = n % MOD;
  const int64_t bp = n / MOD - shift;
  if (bp < 0 || bp >= 640) return UINT64_MAX;
  const int w = (int)(bp / 64), b = (int)(bp % 64);
  const int64_t d = n59 - s[1];
  const int i3 = mod_int(d, 3), i5 = mod_int(d, 5);
  const int i31 = mod_int(d, 31) * inv_int(mod_int(s[2], 31), 31) % 31;
  const int i37 = mod_int(d, 37) * inv_int(mod_int(s[3], 37), 37) % 37;
  const int i41 = mod_int(d, 41) * inv_int(mod_int(s[4], 41), 41) % 41;
  const int j43 = mod_int(d, 43) * inv_int(mod_int(s[5], 43), 43) % 43;
  const int j47 = mod_int(d, 47) * inv_int(mod_int(s[6], 47), 47) % 47;
  const int j53 = mod_int(d, 53) * inv_int(mod_int(s[7], 53), 53) % 53;
  const int j59 = mod_int(d, 59) * inv_int(mod_int(s[8], 59), 59) % 59;
  if (i3 > 1 || i5 > 3 || i31 > 6 || i37 > 12 || i41 > 16 || j43 > 18 || j47 > 22 || j53 > 28 ||
      j59 > 34)
    return UINT64_MAX;
  const int t = tri_index[i31][i37][i41];
  if (t < 0) return UINT64_MAX;
  const uint64_t f = ((uint64_t)(t * 8 + i3 * 4 + i5)) * 443555u + (uint64_t)j43 * 23345u +
                     (uint64_t)j47 * 1015u + (uint64_t)j53 * 35u + (uint64_t)j59;
  return ((uint64_t)(w / 4) << 60) | (f << 8) | ((uint64_t)(w % 4) << 6) | (uint64_t)b;
}

typedef struct { uint64_t key; ap26_ap ap; } keyed_ap;
static int cmp_keyed(const void *x, const void *y) {
  const keyed_ap *a = (const keyed_ap *)x, *b = (const keyed_ap *)y;
  if (a->key != b->key) return a->key < b->key ? -1 : 1;
  if (a->ap.first != b->ap.first) return a->ap.first < b->ap.first ? -1 : 1;
  return a->ap.k - b->ap.k;
}

int ap26_sort_aps(ap26_ap *aps, int n, int shift) {
  if (n < 0 || (n > 0 && !aps)) return AP26_E_ARG;
  if (n < 2) return AP26_OK;
  keyed_ap *tmp = (keyed_ap *)malloc(sizeof(keyed_ap) * (size_t)n);
  if (!tmp) return AP26_E_NOMEM;
  for (int i = 0; i < n; i++) {
    tmp[i].key = ap26h_order_key(aps[i].K, shift, aps[i].n);
    tmp[i].ap = aps[i];
  }
  qsort(tmp, (size_t)n, sizeof(keyed_ap), cmp_keyed);
  for (int i = 0; i < n; i++) aps[i] = tmp[i].ap;
  free(tmp);
  return AP26_OK;
}

/* ---- strong PRP (exact 128-bit remainder; PrimeQ_x86.h:143-182) ---------- */
static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t n) {
  return (uint64_t)(((unsigned __int128)a * b) % n);
}

int ap26h_strong_prp(int64_t a_in, int64_t N) {
  uint64_t n = (uint64_t)N, a = (uint64_t)a_in, r, d;
  unsigned t = (unsigned)__builtin_ctzll(n - 1), s;
  d = n >> t;
  for (r = a, d >>= 1; d > 0; d >>= 1) {
    a = mulmod(a, a, n);
    if (d & 1) r = mulmod(r, a, n);
  }
  if (r == 1 || r == n - 1) return 1;
  for (s = 1; s < t; s++)
    if ((r = mulmod(r, r, n)) == n - 1) return 1;
  return 0;
}

/* validate_ap26 / val_base2_ap26 (AP26.cpp:484-543); -1 = modulus out of
 * range (the reference exits). */
static int validate(int k, int d, int64_t f, int nbases) {
  static const int base[9] = {2, 3, 5, 7, 11, 13, 17, 19, 23};
  int64_t N;
  int j;
  if (f % 2 == 0) return 0;
  for (j = 0, N = f; j < k; j++) {
    if (N < 0 || N >= (INT64_C(1) << 62)) return -1;
    for (int i = 0; i < nbases; i++)
      if (!ap26h_strong_prp(base[i], N)) return j;
    N += (int64_t)d * 2 * 3 * 5 * 7 * 11 * 13 * 17 * 19 * 23;
  }
  return j;
}

int ap26_report(int32_t *result_hash, int len, int K, int64_t first, char *sol, int sol_cap,
                int *sol_len) {
  if (!result_hash) return AP26_E_ARG;
  /* hash before validation (AP26.cpp:557-561) */
  *result_hash += (int32_t)(first % 1000);
  *result_hash += len;
  if (*result_hash > MAXINTV) *result_hash -= MAXINTV;
  int i = validate(len, K, first, 9);
  if (i < 0) return AP26_E_DOMAIN;
  if (i < len) {
    /* "Non-Solution" (AP26.cpp:565-582) */
    int b2 = validate(len, K, first, 1);
    if (b2 < 0) return AP26_E_DOMAIN;
    if (b2 < len) return AP26_E_INVALID;
    int rc = ap26_report(result_hash, i, K, first, sol, sol_cap, sol_len);
    if (rc != AP26_OK) return rc;
    return ap26_report(result_hash, len - (i + 1), K,
                       first + (int64_t)(i + 1) * K * 2 * 3 * 5 * 7 * 11 * 13 * 17 * 19 * 23,
                       sol, sol_cap, sol_len);
  }
  if (len >= MIN_REPORT && sol) {
    int used = sol_len ? *sol_len : (int)strlen(sol);
    int w = snprintf(sol + used, sol_cap > used ? (size_t)(sol_cap - used) : 0, "%d %d %lld\n",
                     len, K, (long long)first);
    if (w < 0 || used + w >= sol_cap) return AP26_E_CAPACITY;
    if (sol_len) *sol_len = used + w;
  }
  return AP26_OK;
}

int ap26_hash_hex(int kmin, int kmax, int32_t result_hash, char *out17) {   /* 295-357 */
  if (!out17) return AP26_E_ARG;
  uint64_t minmax = (uint64_t)(int64_t)(kmin + kmax);
  while (minmax > MAXINTV) minmax -= MAXINTV;
  unsigned int solhash = (unsigned int)result_hash;
  int64_t hash = (int64_t)((minmax << 32) | solhash);
  char hex[16];
  memset(hex, '0', sizeof hex);
  int i = 0;
  while (hash != 0 && i < 16) {
    int tmp = (int)(hash % 16);
    hex[i++] = (char)(tmp < 10 ? tmp + 48 : tmp + 55);
    hash /= 16;
  }
  for (int j = 0; j < 16; j++) out17[j] = hex[15 - j];
  out17[16] = '\0';
  return AP26_OK;
}

/* ---- A/B state files (AP26.cpp:360-476) ----------------------------------- */
static void state_path(char *buf, size_t n, const char *dir, const char *name) {
  if (dir && dir[0]) snprintf(buf, n, "%s/%s", dir, name);
  else snprintf(buf, n, "%s", name);
}

int ap26_write_state(const char *dir, int kmin, int kmax, int shift, int K, int ITER,
                     int32_t result_hash, double last_trickle, int *write_a_next) {
  if (!write_a_next) return AP26_E_ARG;
  char path[4096];
  state_path(path, sizeof path, dir, *write_a_next ? STATE_A : STATE_B);
  FILE *out = fopen(path, "w");
  if (!out) {
    fprintf(stderr, "Cannot open %s !!!\n", *write_a_next ? STATE_A : STATE_B);
    return AP26_E_ARG;
  }
  if (fprintf(out, "%d %d %d %d %d %d %lf\n", kmin, kmax, shift, K, ITER, result_hash,
              last_trickle) < 0) {
    fprintf(stderr, "Cannot write to %s !!! Continuing...\n", *write_a_next ? STATE_A : STATE_B);
    fclose(out);
    return AP26_E_ARG;
  }
  if (fclose(out) == 0) *write_a_next = !*write_a_next;
  return AP26_OK;
}

static int read_one(const char *path, int kmin, int kmax, int shift, int *K, int *ITER, int *h,
                    double *tr) {
  FILE *in = fopen(path, "r");
  if (!in) return 0;
  int a, b, c;
  if (fscanf(in, "%d %d %d %d %d %d %lf\n", &a, &b, &c, K, ITER, h, tr) != 7) {
    fprintf(stderr, "Cannot parse %s !!!\n", path);
    fclose(in);
    return 0;
  }
  fclose(in);
  return (a == kmin && b == kmax && c == shift) ? 1 : 0;
}

int ap26_read_state(const char *dir, int kmin, int kmax, int shift, int *K, int *ITER,
                    int32_t *result_hash, double *last_trickle, int *write_a_next) {
  if (!K || !ITER || !result_hash || !last_trickle || !write_a_next) return AP26_E_ARG;
  char pa[4096], pb[4096];
  state_path(pa, sizeof pa, dir, STATE_A);
  state_path(pb, sizeof pb, dir, STATE_B);
  int Ka = 0, Ia = 0, ha = 0, Kb = 0, Ib = 0, hb = 0;
  double ta = 0, tb = 0;
  int ga = read_one(pa, kmin, kmax, shift, &Ka, &Ia, &ha, &ta);
  int gb = read_one(pb, kmin, kmax, shift, &Kb, &Ib, &hb, &tb);
  if (ga && gb) {
    if (Ka > Kb || (Ka == Kb && Ia > Ib)) gb = 0;
    else ga = 0;
  }
  if (ga) {
    *K = Ka; *ITER = Ia; *result_hash = ha; *last_trickle = ta; *write_a_next = 0;
    return 1;
  }
  if (gb) {
    *K = Kb; *ITER = Ib; *result_hash = hb; *last_trickle = tb; *write_a_next = 1;
    return 1;
  }
  return 0;
}
