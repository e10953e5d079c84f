/* ref_report.cpp -- test infrastructure, not product code.
 *
 * Runs the reference's own ReportSolution (ibethune/ap26
 * src/common/AP26.cpp:549-602, with validate_ap26 / val_base2_ap26 at
 * 484-543), compiled unmodified from the reference sources by
 * oracle/build_ref.sh (AP26.cpp with its main renamed), on one raw report:
 *
 *   ref_report k K first [result_hash]
 *
 * sets result_hash (AP26.cpp:110) to the start value, calls
 * ReportSolution(k, K, first) once and prints "HASH <result_hash>".  The
 * reference itself prints "Solution: ..." / "Non-Solution: ..." lines and
 * appends solutions to SOL-AP26.txt in the working directory; on a
 * computation error or a modulus out of range it exits with EXIT_FAILURE,
 * as it does in the real program. */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>

extern int result_hash;
void ReportSolution(int AP_Length, int difference, int64_t First_Term);

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s k K first [result_hash]\n", argv[0]);
    return 2;
  }
  result_hash = argc > 4 ? atoi(argv[4]) : 0;
  ReportSolution(atoi(argv[1]), atoi(argv[2]), (int64_t)strtoll(argv[3], NULL, 10));
  printf("HASH %d\n", result_hash);
  return 0;
}
