/* Plan-time tables in FP64 (C99 host layer).
 *
 * Every twiddle, four-step factor, Bluestein chirp and packed-real twiddle is
 * formed in double (long double where the argument needs it) from an exactly
 * reduced integer index, then rounded once to the working precision. The
 * reference forms its float tables in float (core/common/twiddle.c:24-98) and
 * only the four-step step twiddles in double
 * (core/solvers/complex/pow2_fourstep_solver_dft.c:124-171); here every table
 * is FP64-formed, which is where the stability of a long transform comes from.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fz_internal.h"

#define FZ_PI_L 3.141592653589793238462643383279502884L

/* exp(-2 pi i r / N) for an exactly reduced 0 <= r < N. The angle is folded
 * into the first octant so that the long-double cosl/sinl see |x| <= pi/4. */
static void w_n(int64_t r, int64_t N, double *re, double *im)
{
    r %= N;
    if (r < 0) r += N;
    /* angle = 2 pi r / N; use 8r/N octants */
    long double t = (long double)r / (long double)N; /* in [0, 1) turns */
    long double c, s;
    long double x = t * 8.0L;
    int oct = (int)floorl(x);
    long double f = (x - oct) / 8.0L; /* remaining turns in [0, 1/8) */
    long double a = 2.0L * FZ_PI_L * f;
    long double ca = cosl(a), sa = sinl(a);
    /* exact quarter-turn rotations of (cos a, sin a) */
    switch (oct & 7)
    {
    case 0: c = ca; s = sa; break;
    case 1: { long double b = 2.0L * FZ_PI_L * (0.125L - f); c = sinl(b); s = cosl(b); break; }
    case 2: c = -sa; s = ca; break;
    case 3: { long double b = 2.0L * FZ_PI_L * (0.125L - f); c = -cosl(b); s = sinl(b); break; }
    case 4: c = -ca; s = -sa; break;
    case 5: { long double b = 2.0L * FZ_PI_L * (0.125L - f); c = -sinl(b); s = -cosl(b); break; }
    case 6: c = sa; s = -ca; break;
    default: { long double b = 2.0L * FZ_PI_L * (0.125L - f); c = cosl(b); s = -sinl(b); break; }
    }
    *re = (double)c;
    *im = (double)(-s);
}

int64_t fz_blob_reserve(fz_blob *b, size_t bytes)
{
    size_t off = (b->len + 255) & ~(size_t)255; /* 256-byte aligned tables */
    size_t need = off + bytes;
    if (need > b->cap)
    {
        size_t nc = b->cap ? b->cap : 4096;
        while (nc < need) nc *= 2;
        unsigned char *np = (unsigned char *)realloc(b->p, nc);
        if (!np) return -1;
        b->p = np;
        b->cap = nc;
    }
    memset(b->p + b->len, 0, need - b->len);
    b->len = need;
    return (int64_t)off;
}

int64_t fz_blob_add(fz_blob *b, const void *data, size_t bytes)
{
    int64_t off = fz_blob_reserve(b, bytes);
    if (off >= 0 && bytes) memcpy(b->p + off, data, bytes);
    return off;
}

static void put_c(fz_blob *b, int64_t off, int dtype, int64_t idx, double re, double im)
{
    if (dtype == 0)
    {
        float *f = (float *)(b->p + off);
        f[2 * idx] = (float)re;
        f[2 * idx + 1] = (float)im;
    }
    else
    {
        double *d = (double *)(b->p + off);
        d[2 * idx] = re;
        d[2 * idx + 1] = im;
    }
}

int64_t fz_stage_twiddles(fz_blob *b, int dtype, int n, int nstages, const int32_t *radix, int32_t *tw_off)
{
    /* stage s >= 1 uses W_{Ns*R}^{k*r}, k < Ns, r = 1..R-1, at [(r-1)*Ns + k] */
    int64_t total = 1, ns = 1;
    for (int s = 0; s < nstages; s++)
    {
        tw_off[s] = (int32_t)total;
        if (s > 0) total += (int64_t)(radix[s] - 1) * ns;
        ns *= radix[s];
    }
    (void)n;
    size_t esz = dtype == 0 ? 8 : 16;
    int64_t off = fz_blob_reserve(b, (size_t)total * esz);
    if (off < 0) return -1;
    ns = 1;
    put_c(b, off, dtype, 0, 1.0, 0.0);
    for (int s = 0; s < nstages; s++)
    {
        int64_t R = radix[s];
        if (s > 0)
            for (int64_t r = 1; r < R; r++)
                for (int64_t k = 0; k < ns; k++)
                {
                    double re, im;
                    w_n(k * r, ns * R, &re, &im);
                    put_c(b, off, dtype, tw_off[s] + (r - 1) * ns + k, re, im);
                }
        ns *= R;
    }
    return off;
}

int fz_tw4_tables(fz_blob *b, int dtype, int64_t N, int64_t *L, int64_t *off_hi, int64_t *off_lo)
{
    /* W_N^r = hi[r / L] * lo[r % L]: both factors formed in FP64 and stored in
     * the working precision (the product is taken in the working precision) */
    int64_t l = 1;
    while (l * l < N) l *= 2;
    /* lo holds at most 1024 factors while hi stays <= 2^20 entries: the
     * four-step epilogue's random lookups (r = column * k) then stay within
     * two 1024-entry tables that remain in L1 beside the stage twiddles */
    if (l > 1024 && (N + 1023) / 1024 <= ((int64_t)1 << 20)) l = 1024;
    int64_t nhi = (N + l - 1) / l;
    size_t esz = dtype == 0 ? 8 : 16;
    *L = l;
    *off_hi = fz_blob_reserve(b, (size_t)nhi * esz);
    if (*off_hi < 0) return -1;
    for (int64_t j = 0; j < nhi; j++)
    {
        double re, im;
        w_n(j * l, N, &re, &im);
        put_c(b, *off_hi, dtype, j, re, im);
    }
    *off_lo = fz_blob_reserve(b, (size_t)l * esz);
    if (*off_lo < 0) return -1;
    for (int64_t j = 0; j < l; j++)
    {
        double re, im;
        w_n(j, N, &re, &im);
        put_c(b, *off_lo, dtype, j, re, im);
    }
    return 0;
}

/* in-place iterative radix-2 FFT in double (forward), m a power of two */
static void host_fft_pow2(double *x, int64_t m)
{
    for (int64_t i = 1, j = 0; i < m; i++)
    {
        int64_t bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j)
        {
            double t0 = x[2 * i], t1 = x[2 * i + 1];
            x[2 * i] = x[2 * j];
            x[2 * i + 1] = x[2 * j + 1];
            x[2 * j] = t0;
            x[2 * j + 1] = t1;
        }
    }
    double *w = (double *)malloc(sizeof(double) * (size_t)m);
    if (!w) return;
    for (int64_t k = 0; k < m / 2; k++) w_n(k, m, &w[2 * k], &w[2 * k + 1]);
    for (int64_t len = 2; len <= m; len <<= 1)
    {
        int64_t step = m / len;
        for (int64_t i = 0; i < m; i += len)
            for (int64_t k = 0; k < len / 2; k++)
            {
                double wr = w[2 * k * step], wi = w[2 * k * step + 1];
                double *a = x + 2 * (i + k), *c = x + 2 * (i + k + len / 2);
                double tr = c[0] * wr - c[1] * wi, ti = c[0] * wi + c[1] * wr;
                c[0] = a[0] - tr;
                c[1] = a[1] - ti;
                a[0] += tr;
                a[1] += ti;
            }
    }
    free(w);
}

int fz_bluestein_tables(fz_blob *b, int dtype, int64_t n, int64_t m, int direction, int64_t *off_pre,
                        int64_t *off_post, int64_t *off_mid)
{
    /* forward chirp c_j = exp(-i pi (j^2 mod 2n) / n) = W_{2n}^{j^2 mod 2n}
     * (core/common/bluestein_utils.c:88-159 keeps the square exact in integers) */
    size_t esz = dtype == 0 ? 8 : 16;
    double *c = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *bb = (double *)calloc(2 * (size_t)m, sizeof(double));
    if (!c || !bb)
    {
        free(c);
        free(bb);
        return -1;
    }
    const int64_t n2 = 2 * n;
    for (int64_t j = 0; j < n; j++)
    {
        int64_t sq = (int64_t)(((unsigned __int128)j * (unsigned __int128)j) % (unsigned __int128)n2);
        w_n(sq, n2, &c[2 * j], &c[2 * j + 1]);
    }
    /* b_j = conj(c_j) at j and m - j, zero between */
    for (int64_t j = 0; j < n; j++)
    {
        bb[2 * j] = c[2 * j];
        bb[2 * j + 1] = -c[2 * j + 1];
        if (j > 0)
        {
            bb[2 * (m - j)] = c[2 * j];
            bb[2 * (m - j) + 1] = -c[2 * j + 1];
        }
    }
    host_fft_pow2(bb, m);
    *off_pre = fz_blob_reserve(b, (size_t)n * esz);
    *off_post = fz_blob_reserve(b, (size_t)n * esz);
    *off_mid = fz_blob_reserve(b, (size_t)m * esz);
    if (*off_pre < 0 || *off_post < 0 || *off_mid < 0)
    {
        free(c);
        free(bb);
        return -1;
    }
    const double inv_m = 1.0 / (double)m;
    for (int64_t j = 0; j < n; j++)
    {
        put_c(b, *off_pre, dtype, j, c[2 * j], c[2 * j + 1]);
        if (direction == 0)
            put_c(b, *off_post, dtype, j, c[2 * j] * inv_m, c[2 * j + 1] * inv_m);
        else
            put_c(b, *off_post, dtype, j, c[2 * j] * inv_m, -c[2 * j + 1] * inv_m);
    }
    for (int64_t j = 0; j < m; j++) put_c(b, *off_mid, dtype, j, bb[2 * j], -bb[2 * j + 1]);
    free(c);
    free(bb);
    return 0;
}

int64_t fz_real_twiddles(fz_blob *b, int dtype, int64_t M)
{
    size_t esz = dtype == 0 ? 8 : 16;
    int64_t off = fz_blob_reserve(b, (size_t)(M + 1) * esz);
    if (off < 0) return -1;
    for (int64_t k = 0; k < M; k++)
    {
        double re, im;
        w_n(k, 2 * M, &re, &im);
        put_c(b, off, dtype, k, re, im);
    }
    put_c(b, off, dtype, M, -1.0, 0.0);
    return off;
}

int64_t fz_blob_permute(fz_blob *b, int dtype, int64_t off, int64_t n1, int64_t n2)
{
    /* T'[k1 * n2 + k2] = T[k1 + n1 * k2]: the rows of an n1 x n2 table become
     * contiguous (a table read along k2 for a fixed k1) */
    const size_t esz = dtype == 0 ? 8 : 16;
    int64_t o = fz_blob_reserve(b, (size_t)(n1 * n2) * esz);
    if (o < 0) return -1;
    for (int64_t k1 = 0; k1 < n1; k1++)
        for (int64_t k2 = 0; k2 < n2; k2++)
            memcpy(b->p + o + (size_t)(k1 * n2 + k2) * esz, b->p + off + (size_t)(k1 + n1 * k2) * esz, esz);
    return o;
}

/* IEEE binary32 -> bfloat16 bits, round to nearest even */
static uint16_t bf16_bits(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

static double bf16_value(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

int64_t fz_tc64_tables(fz_blob *b)
{
    /* [A_hi | A_mid | A_lo | W_4096]: the real 128 x 128 matrix of the
     * 64-point DFT (rows 2k / 2k+1 = re / im of output k, columns 2j / 2j+1 =
     * re / im of input j: [[C, S], [-S, C]], C = cos(2 pi jk/64), S =
     * sin(2 pi jk/64)) formed in FP64, split as hi + mid + lo in BF16 (each
     * term the rounding of what the earlier ones left) and placed in the
     * tensor cores' canonical K-major layout (8 x 16-byte core matrices,
     * K-chunks 128 B apart, 8-row groups 2048 B apart); then
     * (cos, sin)(2 pi r / 4096) for r < 4096 as floats. */
    const size_t abytes = 128 * 256;
    int64_t off = fz_blob_reserve(b, 3 * abytes + 4096 * 8);
    if (off < 0) return -1;
    unsigned char *hi = b->p + off, *mid = hi + abytes, *lo = mid + abytes;
    for (int row = 0; row < 128; row++)
        for (int kk = 0; kk < 128; kk++)
        {
            const int k = row >> 1, j = kk >> 1;
            double c, ms;
            w_n((int64_t)j * k, 64, &c, &ms); /* (cos, -sin) */
            const double sn = -ms;
            double f;
            if ((row & 1) == 0)
                f = (kk & 1) == 0 ? c : sn;
            else
                f = (kk & 1) == 0 ? -sn : c;
            const uint16_t h = bf16_bits((float)f);
            const double r1 = f - bf16_value(h);
            const uint16_t m = bf16_bits((float)r1);
            const uint16_t l = bf16_bits((float)(r1 - bf16_value(m)));
            const size_t o = (size_t)((row >> 3) * 2048 + (kk >> 3) * 128 + (row & 7) * 16 + (kk & 7) * 2);
            memcpy(hi + o, &h, 2);
            memcpy(mid + o, &m, 2);
            memcpy(lo + o, &l, 2);
        }
    float *w = (float *)(b->p + off + 3 * abytes);
    for (int r = 0; r < 4096; r++)
    {
        double c, ms;
        w_n(r, 4096, &c, &ms);
        w[2 * r] = (float)c;
        w[2 * r + 1] = (float)(-ms);
    }
    return off;
}
