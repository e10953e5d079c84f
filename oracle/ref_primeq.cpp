/* ref_primeq.cpp -- test infrastructure: prints the reference's own
 * strong_prp(a, N) verdicts (ibethune/ap26 src/common/PrimeQ_x86.h:143-182,
 * included from the reference tree at build time) for "N a" pairs read from
 * stdin, one "N a verdict" line each.  N must be odd, a < N < 2^62 (the
 * reference's domain, PrimeQ_x86.h:191). */
#include <stdio.h>
#include <stdint.h>
#include "PrimeQ_x86.h"

int main(void) {
  long long N, a;
  check_fpu_mode();
  while (scanf("%lld %lld", &N, &a) == 2)
    printf("%lld %lld %d\n", N, a, strong_prp((int64_t)a, (int64_t)N));
  return 0;
}
