/* Oracle for the FFT plan-execution path: TEST INFRASTRUCTURE ONLY.
 *
 * Nothing in the product library links, loads or calls this code. Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark use it, and
 * only as the checker.
 *
 * Conventions (as in the reference library): complex data is interleaved
 * [re, im]; forward is sign = -1 (X[k] = sum x[n] e^{-2 pi i nk/N}); both
 * directions are unnormalised; strides count complex elements.
 */
#ifndef AOCLFFTZ_DFT_ORACLE_H
#define AOCLFFTZ_DFT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Naive FP64 DFT (long-double accumulation), exact integer reduction of
 * (j*k) mod n before the angle is formed. howmany transforms, distances idist,
 * odist; element strides is, os (complex elements). */
void orc_dft_1d(int64_t n, int sign, const double *in, int64_t is, int64_t idist,
                double *out, int64_t os, int64_t odist, int64_t howmany);

/* Naive DFT evaluated at selected output bins only (unit-stride input). */
void orc_dft_bins(int64_t n, int sign, const double *in, int64_t nbins,
                  const int64_t *bins, double *out);

/* Multi-dimensional exact DFT of a dense row-major array; dims[0] is the
 * innermost (fastest) dimension, as in the reference's descriptors. In place. */
void orc_dft_nd(int rank, const int64_t *dims, int sign, double *data);

/* Restated fast FFT in double precision: mixed-radix Cooley-Tukey over the
 * radix menu {2..13}, Bluestein for larger prime factors. Unit stride, one
 * transform, out of place (in != out). Returns 0 on success. */
int orc_fft(int64_t n, int sign, const double *in, double *out);

/* Batched version of orc_fft over contiguous transforms (OpenMP over batch). */
int orc_fft_batch(int64_t n, int sign, const double *in, double *out, int64_t howmany);

/* Multi-dimensional fast FFT (row-column with orc_fft), dense row-major,
 * dims[0] innermost; in place. */
int orc_fft_nd(int rank, const int64_t *dims, int sign, double *data);

/* Packed real transforms (even n): r2c writes n/2+1 complex bins, c2r reads
 * n/2+1 bins and writes n reals (unnormalised). */
int orc_rfft_packed(int64_t n, const double *in, double *out_half);
int orc_irfft_packed(int64_t n, const double *in_half, double *out);

/* Plan-shape helpers restated from the reference. */
int orc_pow2_radix_balanced(int64_t n, int64_t *radixes);
int orc_pow2_balanced_split(int64_t n, int64_t *n1, int64_t *n2);
int64_t orc_bluestein_extended_length(int64_t n);
void orc_bluestein_chirp(int64_t n, int64_t m, double *b);

#ifdef __cplusplus
}
#endif
#endif
