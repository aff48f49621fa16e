/*
 * gcz_gen.h -- seeded synthetic inputs for the match-find workloads.
 *
 * The reference measures on one ISO image that is not available here; these
 * generators stand in for it with seeded spans of three kinds:
 *   - Markov: order-1 over a 64-symbol alphabet (a seeded subset of byte
 *     values); each row is a Zipf(s=1) distribution over a seeded permutation
 *     of the 64 symbols, quantised to 1/1024;
 *   - copy: a repeat of earlier output, length 4 + geometric (mean 48 in all),
 *     offset log-uniform over [1, max_offset], clamped to the current position;
 *   - random: uniform bytes.
 * Markov and random span lengths are geometric with mean 48.  The span kind is
 * drawn with probabilities (f_markov, f_copy, f_random), which are then also the
 * expected byte fractions.  Output depends only on the arguments (xoshiro256**
 * seeded through splitmix64).
 */
#ifndef GCZ_GEN_H
#define GCZ_GEN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Fill out[0..n) from `seed`.  Fractions are normalised; all zero means 0.4/0.4/0.2. */
void gcz_gen_synthetic(uint64_t seed, uint8_t *out, uint64_t n, uint64_t max_offset,
                       double f_markov, double f_copy, double f_random);

/* `count` file sizes log-uniform over [min_size, max_size] and, per file, a
 * Dirichlet(1,1,1) mix written to mix[3*i .. 3*i+2] (may be NULL). */
void gcz_gen_file_sizes(uint64_t seed, uint64_t count, uint64_t min_size, uint64_t max_size,
                        uint64_t *sizes, double *mix);

#ifdef __cplusplus
}
#endif

#endif /* GCZ_GEN_H */
