/* ap26_hostcore.h -- internal helpers shared by the CUDA host layer and the
 * C host services of libap26.so (not part of the public ABI). */
#ifndef AP26_HOSTCORE_H
#define AP26_HOSTCORE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The 1355 admissible (i31, i37, i41) triples in the reference's loop order
 * (src/opencl/AP26.h:127-131), packed i31 | i37 << 5 | i41 << 10.
 * Returns the count. */
int ap26h_triples(uint16_t *out);

/* Per-K constants exactly as the reference computes them
 * (src/opencl/AP26.h:112-120): out = STEP, n0, S31, S37, S41, S43, S47,
 * S53, S59. */
void ap26h_setup_k(int K, int64_t out[9]);

/* Position at which the reference's AVX2 search meets candidate n of K
 * (4-word pass, lattice order, word in pass, bit); UINT64_MAX if n is not a
 * lattice candidate of (K, shift). */
uint64_t ap26h_order_key(int K, int shift, int64_t n);

/* Exact base-a strong-PRP test for odd N < 2^63, a < N (same verdict as
 * src/common/PrimeQ_x86.h:143-182 for N < 2^62). */
int ap26h_strong_prp(int64_t a, int64_t N);

#ifdef __cplusplus
}
#endif
#endif
