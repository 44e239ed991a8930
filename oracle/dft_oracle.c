/* Oracle for the FFT plan-execution path: TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the GPU library, never part of it. It restates,
 * in plain C99 double / long-double arithmetic, the algorithms of the
 * reference library (AOCL-FFTZ) that the GPU path re-implements:
 *
 *   orc_dft_1d / orc_dft_nd    test/bench/dft_reference.c:458-636 (naive DFT,
 *                              sign -1 forward, N-D angle = sum k_i n_i / N_i);
 *                              here the index product is reduced exactly in
 *                              integers and accumulated in long double.
 *   orc_fft                    mixed-radix Cooley-Tukey over the reference's
 *                              prime radix menu {2,3,5,7,11,13}
 *                              (core/common/bluestein_utils.c:26-28,
 *                              selector/complex/selector_ct_dft.c:104-326) and
 *                              Bluestein for larger primes
 *                              (core/solvers/complex/bluestein_solver_dft.c:137-234).
 *   orc_bluestein_*            core/common/bluestein_utils.c:39-67 (extended
 *                              length) and :88-159 (chirp, exact (i*i) % 2n).
 *   orc_pow2_*                 core/common/pow2_radix_decompose.c:15-35, :122-150.
 *   orc_rfft_packed / irfft    core/solvers/real/packed_solver_rdft.c:154-226 with
 *                              the recombine / separate butterflies of
 *                              core/kernels/non_dft/real_packed/packed_rdft_common.h:42-63,
 *                              :179-196 and the DC/Nyquist case :307-340.
 */
#include "dft_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI_L 3.141592653589793238462643383279502884L

/* W_n^r = exp(sign * 2 pi i r / n) for 0 <= r < n, computed in long double
 * and rounded once. The angle uses the reduced integer r, so no large-argument
 * trig is ever evaluated. */
static long double *twiddle_table_l(int64_t n, int sign)
{
    long double *t = (long double *)malloc(sizeof(long double) * 2 * (size_t)n);
    if (!t) return NULL;
    for (int64_t r = 0; r < n; r++)
    {
        long double a = 2.0L * ORC_PI_L * (long double)r / (long double)n;
        t[2 * r] = cosl(a);
        t[2 * r + 1] = (long double)sign * sinl(a);
    }
    return t;
}

void orc_dft_1d(int64_t n, int sign, const double *in, int64_t is, int64_t idist,
                double *out, int64_t os, int64_t odist, int64_t howmany)
{
    long double *w = twiddle_table_l(n, sign);
    if (!w) return;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t b = 0; b < howmany; b++)
    {
        for (int64_t k = 0; k < n; k++)
        {
            const double *x = in + 2 * b * idist;
            long double sr = 0.0L, si = 0.0L;
            int64_t r = 0; /* (j * k) mod n, advanced by k each step */
            for (int64_t j = 0; j < n; j++)
            {
                long double xr = x[2 * j * is], xi = x[2 * j * is + 1];
                long double wr = w[2 * r], wi = w[2 * r + 1];
                sr += xr * wr - xi * wi;
                si += xr * wi + xi * wr;
                r += k;
                if (r >= n) r -= n;
            }
            out[2 * (b * odist + k * os)] = (double)sr;
            out[2 * (b * odist + k * os) + 1] = (double)si;
        }
    }
    free(w);
}

void orc_dft_bins(int64_t n, int sign, const double *in, int64_t nbins,
                  const int64_t *bins, double *out)
{
    long double *w = twiddle_table_l(n, sign);
    if (!w) return;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < nbins; q++)
    {
        int64_t k = ((bins[q] % n) + n) % n;
        long double sr = 0.0L, si = 0.0L;
        int64_t r = 0;
        for (int64_t j = 0; j < n; j++)
        {
            long double xr = in[2 * j], xi = in[2 * j + 1];
            sr += xr * w[2 * r] - xi * w[2 * r + 1];
            si += xr * w[2 * r + 1] + xi * w[2 * r];
            r += k;
            if (r >= n) r -= n;
        }
        out[2 * q] = (double)sr;
        out[2 * q + 1] = (double)si;
    }
    free(w);
}

/* Applies a 1-D transform along dimension d of a dense row-major array
 * (dims[0] innermost) with the supplied line transform. */
typedef int (*line_fn)(int64_t n, int sign, const double *in, double *out);

static int naive_line(int64_t n, int sign, const double *in, double *out)
{
    orc_dft_1d(n, sign, in, 1, n, out, 1, n, 1);
    return 0;
}

static int along_dims(int rank, const int64_t *dims, int sign, double *data, line_fn fn)
{
    int64_t total = 1;
    for (int d = 0; d < rank; d++) total *= dims[d];
    int64_t stride = 1;
    for (int d = 0; d < rank; d++)
    {
        int64_t n = dims[d];
        int64_t outer = total / (n * stride);
        int err = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(| : err)
        for (int64_t o = 0; o < outer; o++)
        {
            for (int64_t s = 0; s < stride; s++)
            {
                double *line = (double *)malloc(sizeof(double) * 4 * (size_t)n);
                if (!line) { err |= 1; continue; }
                double *res = line + 2 * n;
                double *base = data + 2 * (o * n * stride + s);
                for (int64_t j = 0; j < n; j++)
                {
                    line[2 * j] = base[2 * j * stride];
                    line[2 * j + 1] = base[2 * j * stride + 1];
                }
                err |= fn(n, sign, line, res) != 0;
                for (int64_t j = 0; j < n; j++)
                {
                    base[2 * j * stride] = res[2 * j];
                    base[2 * j * stride + 1] = res[2 * j + 1];
                }
                free(line);
            }
        }
        if (err) return -1;
        stride *= n;
    }
    return 0;
}

void orc_dft_nd(int rank, const int64_t *dims, int sign, double *data)
{
    /* Parallelism lives in the line loop; the naive line itself is then serial
     * because nested OpenMP regions run with one thread by default. */
    along_dims(rank, dims, sign, data, naive_line);
}

/* ------------------------------------------------------------------ fast FFT */

static int64_t smallest_factor(int64_t n)
{
    static const int64_t menu[] = {2, 3, 5, 7, 11, 13};
    for (int i = 0; i < 6; i++)
        if (n % menu[i] == 0) return menu[i];
    return n;
}

static int only_menu_factors(int64_t n)
{
    static const int64_t menu[] = {2, 3, 5, 7, 11, 13};
    for (int i = 0; i < 6; i++)
        while (n % menu[i] == 0) n /= menu[i];
    return n == 1;
}

/* Recursive decimation-in-time. tw holds W_N^r (double, length N); the
 * sub-transform of size n uses W_n^x = tw[(x mod n) * tws], tws = N / n. */
static void ct_rec(int64_t n, const double *in, int64_t is, double *out,
                   const double *tw, int64_t tws, double *tmp)
{
    if (n == 1)
    {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    int64_t p = smallest_factor(n);
    int64_t m = n / p;
    for (int64_t r = 0; r < p; r++)
        ct_rec(m, in + 2 * r * is, is * p, out + 2 * r * m, tw, tws * p, tmp);
    /* Butterflies: X[k + m q] = sum_r (W_n^{r k} Y_r[k]) W_p^{r q}. */
    for (int64_t k = 0; k < m; k++)
    {
        double t[2 * 13];
        for (int64_t r = 0; r < p; r++)
        {
            int64_t e = (r * k) % n;
            double wr = tw[2 * e * tws], wi = tw[2 * e * tws + 1];
            double yr = out[2 * (r * m + k)], yi = out[2 * (r * m + k) + 1];
            t[2 * r] = yr * wr - yi * wi;
            t[2 * r + 1] = yr * wi + yi * wr;
        }
        for (int64_t q = 0; q < p; q++)
        {
            double sr = 0.0, si = 0.0;
            for (int64_t r = 0; r < p; r++)
            {
                int64_t e = ((r * q) % p) * m; /* W_p^{rq} = W_n^{m rq} */
                double wr = tw[2 * e * tws], wi = tw[2 * e * tws + 1];
                sr += t[2 * r] * wr - t[2 * r + 1] * wi;
                si += t[2 * r] * wi + t[2 * r + 1] * wr;
            }
            tmp[2 * (k + m * q)] = sr;
            tmp[2 * (k + m * q) + 1] = si;
        }
    }
    memcpy(out, tmp, sizeof(double) * 2 * (size_t)n);
}

static double *twiddle_table_d(int64_t n, int sign)
{
    double *t = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    if (!t) return NULL;
    for (int64_t r = 0; r < n; r++)
    {
        long double a = 2.0L * ORC_PI_L * (long double)r / (long double)n;
        t[2 * r] = (double)cosl(a);
        t[2 * r + 1] = (double)((long double)sign * sinl(a));
    }
    return t;
}

static int ct_fft(int64_t n, int sign, const double *in, double *out)
{
    double *tw = twiddle_table_d(n, sign);
    double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    if (!tw || !tmp)
    {
        free(tw);
        free(tmp);
        return -1;
    }
    ct_rec(n, in, 1, out, tw, 1, tmp);
    free(tw);
    free(tmp);
    return 0;
}

int64_t orc_bluestein_extended_length(int64_t n)
{
    for (int64_t m = 2 * n - 1;; m++)
        if (only_menu_factors(m)) return m;
}

void orc_bluestein_chirp(int64_t n, int64_t m, double *b)
{
    /* b[i] = exp(+i pi (i*i mod 2n) / n) for i < n, mirrored at m - i, zero
     * elsewhere; the square is reduced exactly in 64-bit integers. */
    memset(b, 0, sizeof(double) * 2 * (size_t)m);
    int64_t n2 = 2 * n;
    for (int64_t i = 0; i < n; i++)
    {
        int64_t sq = (int64_t)(((unsigned __int128)i * (unsigned __int128)i) % (unsigned __int128)n2);
        long double a = ORC_PI_L * (long double)sq / (long double)n;
        double re = (double)cosl(a), im = (double)sinl(a);
        b[2 * i] = re;
        b[2 * i + 1] = im;
        if (i > 0)
        {
            b[2 * (m - i)] = re;
            b[2 * (m - i) + 1] = im;
        }
    }
}

static int bluestein_fft(int64_t n, int sign, const double *in, double *out)
{
    int64_t m = orc_bluestein_extended_length(n);
    double *a = (double *)calloc(2 * (size_t)m, sizeof(double));
    double *b = (double *)malloc(sizeof(double) * 2 * (size_t)m);
    double *A = (double *)malloc(sizeof(double) * 2 * (size_t)m);
    double *B = (double *)malloc(sizeof(double) * 2 * (size_t)m);
    double *c = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    int rc = -1;
    if (!a || !b || !A || !B || !c) goto done;
    orc_bluestein_chirp(n, m, b); /* b = conj of the forward chirp */
    for (int64_t i = 0; i < n; i++)
    {
        /* chirp c_i = exp(sign * i pi (i^2 mod 2n) / n) */
        c[2 * i] = b[2 * i];
        c[2 * i + 1] = (sign < 0) ? -b[2 * i + 1] : b[2 * i + 1];
    }
    if (sign > 0)
        for (int64_t i = 0; i < m; i++) b[2 * i + 1] = -b[2 * i + 1];
    for (int64_t i = 0; i < n; i++)
    {
        double xr = in[2 * i], xi = in[2 * i + 1];
        a[2 * i] = xr * c[2 * i] - xi * c[2 * i + 1];
        a[2 * i + 1] = xr * c[2 * i + 1] + xi * c[2 * i];
    }
    if (ct_fft(m, -1, a, A) || ct_fft(m, -1, b, B)) goto done;
    for (int64_t i = 0; i < m; i++)
    {
        double ar = A[2 * i], ai = A[2 * i + 1], br = B[2 * i], bi = B[2 * i + 1];
        a[2 * i] = ar * br - ai * bi;
        a[2 * i + 1] = ar * bi + ai * br;
    }
    if (ct_fft(m, +1, a, A)) goto done;
    for (int64_t i = 0; i < n; i++)
    {
        double yr = A[2 * i] / (double)m, yi = A[2 * i + 1] / (double)m;
        out[2 * i] = yr * c[2 * i] - yi * c[2 * i + 1];
        out[2 * i + 1] = yr * c[2 * i + 1] + yi * c[2 * i];
    }
    rc = 0;
done:
    free(a);
    free(b);
    free(A);
    free(B);
    free(c);
    return rc;
}

int orc_fft(int64_t n, int sign, const double *in, double *out)
{
    if (n < 1) return -1;
    if (only_menu_factors(n)) return ct_fft(n, sign, in, out);
    return bluestein_fft(n, sign, in, out);
}

int orc_fft_batch(int64_t n, int sign, const double *in, double *out, int64_t howmany)
{
    int err = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : err)
    for (int64_t b = 0; b < howmany; b++)
        err |= orc_fft(n, sign, in + 2 * b * n, out + 2 * b * n) != 0;
    return err ? -1 : 0;
}

int orc_fft_nd(int rank, const int64_t *dims, int sign, double *data)
{
    return along_dims(rank, dims, sign, data, orc_fft);
}

/* ------------------------------------------------------------- packed real */

int orc_rfft_packed(int64_t n, const double *in, double *out_half)
{
    if (n < 2 || (n & 1)) return -1;
    int64_t M = n / 2;
    double *Z = (double *)malloc(sizeof(double) * 2 * (size_t)M);
    if (!Z) return -1;
    /* n reals are read as M interleaved complex values z_j = x_2j + i x_2j+1 */
    if (orc_fft(M, -1, in, Z))
    {
        free(Z);
        return -1;
    }
    out_half[0] = Z[0] + Z[1];
    out_half[1] = 0.0;
    out_half[2 * M] = Z[0] - Z[1];
    out_half[2 * M + 1] = 0.0;
    for (int64_t k = 1; k < M; k++)
    {
        /* X_k = (Z_k + conj Z_{M-k})/2 + W_n^k (Z_k - conj Z_{M-k})/(2i) */
        long double a = 2.0L * ORC_PI_L * (long double)k / (long double)n;
        double c = (double)cosl(a), s = (double)sinl(a);
        double zr = Z[2 * k], zi = Z[2 * k + 1];
        double mr = Z[2 * (M - k)], mi = Z[2 * (M - k) + 1];
        double er = 0.5 * (zr + mr), ei = 0.5 * (zi - mi);
        double orr = 0.5 * (zi + mi), oi = 0.5 * (mr - zr);
        out_half[2 * k] = er + (c * orr + s * oi);
        out_half[2 * k + 1] = ei + (c * oi - s * orr);
    }
    free(Z);
    return 0;
}

int orc_irfft_packed(int64_t n, const double *in_half, double *out)
{
    if (n < 2 || (n & 1)) return -1;
    int64_t M = n / 2;
    double *Z = (double *)malloc(sizeof(double) * 2 * (size_t)M);
    if (!Z) return -1;
    for (int64_t k = 0; k < M; k++)
    {
        /* 2 Z_k = (X_k + conj X_{M-k}) + i e^{+2 pi i k/n} (X_k - conj X_{M-k}) */
        long double a = 2.0L * ORC_PI_L * (long double)k / (long double)n;
        double c = (double)cosl(a), s = (double)sinl(a);
        double xr = in_half[2 * k], xi = in_half[2 * k + 1];
        double mr = in_half[2 * (M - k)], mi = in_half[2 * (M - k) + 1];
        double sr = xr + mr, si = xi - mi;
        double dr = xr - mr, di = xi + mi;
        double rr = c * dr - s * di, ri = c * di + s * dr; /* e^{+i a} * d */
        Z[2 * k] = sr - ri;
        Z[2 * k + 1] = si + rr;
    }
    int rc = orc_fft(M, +1, Z, out);
    free(Z);
    return rc;
}

/* ------------------------------------------------------------ plan helpers */

int orc_pow2_balanced_split(int64_t n, int64_t *n1, int64_t *n2)
{
    if (n < 2 || (n & (n - 1))) return 0;
    int k = 0;
    while (((int64_t)1 << k) < n) k++;
    int64_t b = (int64_t)1 << (k / 2);
    int64_t a = n / b;
    if (a < 2 || b < 2) return 0;
    *n1 = a;
    *n2 = b;
    return 1;
}

int orc_pow2_radix_balanced(int64_t n, int64_t *radixes)
{
    if (n < 2 || (n & (n - 1))) return 0;
    int log2n = 0;
    while (((int64_t)1 << log2n) < n) log2n++;
    int stages = (log2n + 3) / 4;
    if (stages < 1) stages = 1;
    int base = log2n / stages, extra = log2n % stages;
    for (int s = 0; s < stages; s++) radixes[s] = (int64_t)1 << (base + (s < extra ? 1 : 0));
    return stages;
}
