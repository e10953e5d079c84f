#!/usr/bin/env bash
# build_ref.sh -- test infrastructure: compile the reference CPU build of
# ibethune/ap26 from its own sources, where they lie, into oracle/_ref/.
#
# Outputs (git-ignored, but shipped with the working tree):
#   oracle/_ref/AP26         the reference CLI (AP26 KMIN KMAX SHIFT), -DAP26_CPU,
#                            runtime SSE2/SSE4.1/AVX/AVX2 dispatch, no BOINC
#   oracle/_ref/ref_harness  oracle/ref_harness.cpp linked with the reference's
#                            Search_avx2 / Search_sse2 objects (raw AP records and
#                            bounded timing samples)
#   oracle/_ref/ref_primeq   the reference's strong_prp on "N a" pairs
#   oracle/_ref/ref_report   the reference's ReportSolution on one raw report
#                            (AP26.cpp compiled again with main renamed)
#
# Flags follow the reference's own makefile (src/cpu/Makefile_linux:10-38) minus
# BOINC: -O3 -m64, per-file -mavx2 / -mavx / -msse4.1 / -msse2.
# Usage: oracle/build_ref.sh [--if-present] [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $AP26_REFERENCE, else the read-only tree this
#   recipe was written against (/root/reference).  With --if-present a missing
#   tree is not an error: the recipe builds nothing and exits 0.
set -euo pipefail
IF_PRESENT=0
if [ "${1:-}" = "--if-present" ]; then IF_PRESENT=1; shift; fi
REF="${1:-${AP26_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/common/AP26.cpp" ]; then
  if [ "$IF_PRESENT" = 1 ]; then exit 0; fi
  echo "reference sources not found under $REF" >&2
  exit 1
fi
mkdir -p "$OUT"
CXX="${CXX:-g++}"
CF="-w -O3 -m64 -DAP26_CPU -I$REF/src/cpu -I$REF/src/common"
$CXX $CF -c -o "$OUT/AP26.o"     "$REF/src/common/AP26.cpp"
$CXX $CF -mavx2   -c -o "$OUT/cpuavx2.o"  "$REF/src/cpu/cpuavx2.cpp"
$CXX $CF -mavx    -c -o "$OUT/cpuavx.o"   "$REF/src/cpu/cpuavx.cpp"
$CXX $CF -msse4.1 -c -o "$OUT/cpusse41.o" "$REF/src/cpu/cpusse41.cpp"
$CXX $CF -msse2   -c -o "$OUT/cpusse2.o"  "$REF/src/cpu/cpusse2.cpp"
$CXX -o "$OUT/AP26" "$OUT/AP26.o" "$OUT/cpuavx2.o" "$OUT/cpuavx.o" \
     "$OUT/cpusse41.o" "$OUT/cpusse2.o" -lm
$CXX $CF -c -o "$OUT/ref_harness.o" "$HERE/ref_harness.cpp"
$CXX -o "$OUT/ref_harness" "$OUT/ref_harness.o" "$OUT/cpuavx2.o" "$OUT/cpusse2.o" -lm
echo "built $OUT/AP26 $OUT/ref_harness"
$CXX $CF -o "$OUT/ref_primeq" "$HERE/ref_primeq.cpp"
echo "built $OUT/ref_primeq"
$CXX $CF -Dmain=ap26_reference_main -c -o "$OUT/AP26_nomain.o" "$REF/src/common/AP26.cpp"
$CXX $CF -c -o "$OUT/ref_report.o" "$HERE/ref_report.cpp"
$CXX -o "$OUT/ref_report" "$OUT/ref_report.o" "$OUT/AP26_nomain.o" "$OUT/cpuavx2.o" \
     "$OUT/cpuavx.o" "$OUT/cpusse41.o" "$OUT/cpusse2.o" -lm
echo "built $OUT/ref_report"
