/* FFTW3-compatible surface (C99 host layer): translates fftw_plan_* calls into
 * aoclfftz descriptors and plans, as the reference's wrapper does
 * (wrappers/fftw/src/translator/fftz_translator.c:13-291 and
 * wrappers/fftw/src/c/fftw_{plan,execute,destroy,misc}_wrapper.c):
 *   - FFTW's n[] is row-major (n[rank-1] contiguous); dims[] runs innermost
 *     first, so n is reversed;
 *   - placement is in-place exactly when in == out;
 *   - FFTW_FORWARD (-1) selects the forward direction;
 *   - plan_many: strides of dim i (innermost first) are
 *     stride * prod(embed[rank-1], ..., embed[rank-i]); a NULL embed means n,
 *     zero strides / distances mean 1;
 *   - r2c / c2r without embeds pad the real rows of an in-place transform to
 *     2 (n0/2 + 1) reals;
 *   - planner flags are ignored and execute discards the status.
 */
#include <cuda_runtime_api.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "aoclfftz_gpu.h"
#include "fftw3.h"
#include "fz_internal.h"

typedef struct
{
    int64_t n, is, os;
} fw_dim;

static void *fw_make(int dtype, int type, int dir, int rank, const fw_dim *dims, int hrank, const fw_dim *hdims,
                     void *in, void *out)
{
    aoclfftz_dim_t_64_ d[16], v[16];
    if (rank < 0 || rank > 16 || hrank < 0 || hrank > 16) return NULL;
    int dr = 0, vr = 0;
    if (rank == 0)
    {
        d[0].n = 1;
        d[0].in_stride = d[0].out_stride = 1;
        dr = 1;
    }
    for (int i = 0; i < rank; i++)
    {
        d[i].n = dims[rank - 1 - i].n;
        d[i].in_stride = dims[rank - 1 - i].is;
        d[i].out_stride = dims[rank - 1 - i].os;
        dr = rank;
    }
    if (hrank == 0)
    {
        v[0].n = 1;
        v[0].in_stride = v[0].out_stride = 1;
        vr = 1;
    }
    for (int i = 0; i < hrank; i++)
    {
        v[i].n = hdims[hrank - 1 - i].n;
        v[i].in_stride = hdims[hrank - 1 - i].is ? hdims[hrank - 1 - i].is : 1;
        v[i].out_stride = hdims[hrank - 1 - i].os ? hdims[hrank - 1 - i].os : 1;
        vr = hrank;
    }
    if (dtype == 0)
    {
        aoclfftz_prob_desc_f_64_ p;
        memset(&p, 0, sizeof(p));
        p.in = (float *)in;
        p.out = (float *)out;
        p.dim_rank = dr;
        p.vec_rank = vr;
        p.dims = d;
        p.vecs = v;
        p.flags.fft_type = (FFTZ_UINT8)type;
        p.flags.fft_direction = (FFTZ_UINT8)dir;
        p.flags.fft_placement = in == out ? 0 : 1;
        p.pthr_fft.num_threads = 1;
        p.pthr_fft.dynamic_load_model = 1;
        p.cntrl_params.opt_level = 3;
        return aoclfftz_setup_f_64_(&p);
    }
    aoclfftz_prob_desc_d_64_ p;
    memset(&p, 0, sizeof(p));
    p.in = (double *)in;
    p.out = (double *)out;
    p.dim_rank = dr;
    p.vec_rank = vr;
    p.dims = d;
    p.vecs = v;
    p.flags.fft_type = (FFTZ_UINT8)type;
    p.flags.fft_direction = (FFTZ_UINT8)dir;
    p.flags.fft_placement = in == out ? 0 : 1;
    p.pthr_fft.num_threads = 1;
    p.pthr_fft.dynamic_load_model = 1;
    p.cntrl_params.opt_level = 3;
    return aoclfftz_setup_d_64_(&p);
}

/* contiguous row-major c2c dims (FFTW order) */
static int fw_dense(int rank, const int *n, fw_dim *dims)
{
    if (rank < 0 || rank > 16 || (rank > 0 && !n)) return -1;
    int64_t s = 1;
    for (int i = rank - 1; i >= 0; i--)
    {
        dims[i].n = n[i];
        dims[i].is = dims[i].os = s;
        s *= n[i];
    }
    return 0;
}

/* plan_many strides: innermost dim gets stride, dim i the product of the
 * embeds of the dims inside it */
static void fw_many_side(int rank, const int *n, const int *embed, int stride, fw_dim *dims, int side_in)
{
    const int *e = embed ? embed : n;
    int64_t s = stride ? stride : 1;
    for (int i = rank - 1; i >= 0; i--)
    {
        if (side_in)
            dims[i].is = s;
        else
            dims[i].os = s;
        s *= e[i];
    }
}

/* real-side / half-side strides without embeds: row of the real side padded
 * to 2 (n0/2 + 1) reals when in place */
static void fw_real_side(int rank, const int *n, int stride, int half, int inplace, fw_dim *dims, int side_in)
{
    int64_t s = stride ? stride : 1;
    for (int i = rank - 1; i >= 0; i--)
    {
        if (side_in)
            dims[i].is = s;
        else
            dims[i].os = s;
        int64_t len = n[i];
        if (i == rank - 1) len = half ? n[i] / 2 + 1 : (inplace ? 2 * (n[i] / 2 + 1) : n[i]);
        s *= len;
    }
}

static int g_nthreads = 1;

/* FFTW defines only FFTW_FORWARD (-1) and FFTW_BACKWARD (+1): 0 / 1 for the
 * planner's direction, -1 (no plan) for any other sign */
static int fw_sign(int sign)
{
    if (sign == FFTW_FORWARD) return 0;
    if (sign == FFTW_BACKWARD) return 1;
    fz_set_error("FFTW sign %d is neither FFTW_FORWARD (-1) nor FFTW_BACKWARD (+1)", sign);
    return -1;
}

#define FW_DEFINE(P, DT, R, Cx)                                                                                       \
    P##_plan P##_plan_dft(int rank, const int *n, Cx *in, Cx *out, int sign, unsigned flags)                          \
    {                                                                                                                  \
        fw_dim d[16];                                                                                                  \
        (void)flags;                                                                                                   \
        if (fw_sign(sign) < 0 || fw_dense(rank, n, d)) return NULL;                                                    \
        return fw_make(DT, 0, fw_sign(sign), rank, d, 0, NULL, in, out);                              \
    }                                                                                                                  \
    P##_plan P##_plan_dft_1d(int n, Cx *in, Cx *out, int sign, unsigned flags)                                        \
    {                                                                                                                  \
        return P##_plan_dft(1, &n, in, out, sign, flags);                                                             \
    }                                                                                                                  \
    P##_plan P##_plan_dft_2d(int n0, int n1, Cx *in, Cx *out, int sign, unsigned flags)                               \
    {                                                                                                                  \
        int n[2] = {n0, n1};                                                                                           \
        return P##_plan_dft(2, n, in, out, sign, flags);                                                              \
    }                                                                                                                  \
    P##_plan P##_plan_dft_3d(int n0, int n1, int n2, Cx *in, Cx *out, int sign, unsigned flags)                       \
    {                                                                                                                  \
        int n[3] = {n0, n1, n2};                                                                                       \
        return P##_plan_dft(3, n, in, out, sign, flags);                                                              \
    }                                                                                                                  \
    P##_plan P##_plan_many_dft(int rank, const int *n, int howmany, Cx *in, const int *inembed, int istride,          \
                               int idist, Cx *out, const int *onembed, int ostride, int odist, int sign,               \
                               unsigned flags)                                                                         \
    {                                                                                                                  \
        fw_dim d[16], h;                                                                                               \
        (void)flags;                                                                                                   \
        if (rank < 0 || rank > 16 || (rank > 0 && !n) || fw_sign(sign) < 0) return NULL;                              \
        for (int i = 0; i < rank; i++) d[i].n = n[i];                                                                  \
        fw_many_side(rank, n, inembed, istride, d, 1);                                                                 \
        fw_many_side(rank, n, onembed, ostride, d, 0);                                                                 \
        h.n = howmany;                                                                                                 \
        h.is = idist;                                                                                                  \
        h.os = odist;                                                                                                  \
        return fw_make(DT, 0, fw_sign(sign), rank, d, 1, &h, in, out);                                \
    }                                                                                                                  \
    P##_plan P##_plan_guru64_dft(int rank, const P##_iodim64 *dims, int hr, const P##_iodim64 *hd, Cx *in, Cx *out,   \
                                 int sign, unsigned flags)                                                             \
    {                                                                                                                  \
        fw_dim d[16], h[16];                                                                                           \
        (void)flags;                                                                                                   \
        if (rank < 0 || rank > 16 || hr < 0 || hr > 16 || (rank && !dims) || (hr && !hd) || fw_sign(sign) < 0)       \
            return NULL;                                                                                               \
        for (int i = 0; i < rank; i++)                                                                                 \
        {                                                                                                              \
            d[i].n = dims[i].n;                                                                                        \
            d[i].is = dims[i].is;                                                                                      \
            d[i].os = dims[i].os;                                                                                      \
        }                                                                                                              \
        for (int i = 0; i < hr; i++)                                                                                   \
        {                                                                                                              \
            h[i].n = hd[i].n;                                                                                          \
            h[i].is = hd[i].is;                                                                                        \
            h[i].os = hd[i].os;                                                                                        \
        }                                                                                                              \
        return fw_make(DT, 0, fw_sign(sign), rank, d, hr, h, in, out);                                \
    }                                                                                                                  \
    P##_plan P##_plan_guru_dft(int rank, const P##_iodim *dims, int hr, const P##_iodim *hd, Cx *in, Cx *out,         \
                               int sign, unsigned flags)                                                               \
    {                                                                                                                  \
        P##_iodim64 d[16], h[16];                                                                                      \
        if (rank < 0 || rank > 16 || hr < 0 || hr > 16 || (rank && !dims) || (hr && !hd) || fw_sign(sign) < 0)       \
            return NULL;                                                                                               \
        for (int i = 0; i < rank; i++)                                                                                 \
        {                                                                                                              \
            d[i].n = dims[i].n;                                                                                        \
            d[i].is = dims[i].is;                                                                                      \
            d[i].os = dims[i].os;                                                                                      \
        }                                                                                                              \
        for (int i = 0; i < hr; i++)                                                                                   \
        {                                                                                                              \
            h[i].n = hd[i].n;                                                                                          \
            h[i].is = hd[i].is;                                                                                        \
            h[i].os = hd[i].os;                                                                                        \
        }                                                                                                              \
        return P##_plan_guru64_dft(rank, d, hr, h, in, out, sign, flags);                                             \
    }

/* r2c (sign 0 -> forward) and c2r (backward) planning shared by both precisions */
#define FW_DEFINE_REAL(P, DT, R, Cx)                                                                                  \
    static P##_plan P##_real_many(int dir, int rank, const int *n, int howmany, void *in, const int *inembed,          \
                                  int istride, int idist, void *out, const int *onembed, int ostride, int odist)       \
    {                                                                                                                  \
        fw_dim d[16], h;                                                                                               \
        if (rank <= 0 || rank > 16 || !n) return NULL;                                                                 \
        const int inplace = in == out;                                                                                 \
        for (int i = 0; i < rank; i++) d[i].n = n[i];                                                                  \
        /* the input side is real for r2c, half-complex for c2r; the output side the other way */                     \
        if (inembed)                                                                                                   \
            fw_many_side(rank, n, inembed, istride, d, 1);                                                             \
        else                                                                                                           \
            fw_real_side(rank, n, istride, dir == 1, inplace, d, 1);                                                   \
        if (onembed)                                                                                                   \
            fw_many_side(rank, n, onembed, ostride, d, 0);                                                             \
        else                                                                                                           \
            fw_real_side(rank, n, ostride, dir == 0, inplace, d, 0);                                                   \
        h.n = howmany;                                                                                                 \
        h.is = idist;                                                                                                  \
        h.os = odist;                                                                                                  \
        return fw_make(DT, 1, dir, rank, d, 1, &h, in, out);                                                          \
    }                                                                                                                  \
    P##_plan P##_plan_many_dft_r2c(int rank, const int *n, int howmany, R *in, const int *inembed, int istride,       \
                                   int idist, Cx *out, const int *onembed, int ostride, int odist, unsigned flags)     \
    {                                                                                                                  \
        (void)flags;                                                                                                   \
        return P##_real_many(0, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist);         \
    }                                                                                                                  \
    P##_plan P##_plan_many_dft_c2r(int rank, const int *n, int howmany, Cx *in, const int *inembed, int istride,      \
                                   int idist, R *out, const int *onembed, int ostride, int odist, unsigned flags)      \
    {                                                                                                                  \
        (void)flags;                                                                                                   \
        return P##_real_many(1, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist);         \
    }                                                                                                                  \
    P##_plan P##_plan_dft_r2c(int rank, const int *n, R *in, Cx *out, unsigned flags)                                 \
    {                                                                                                                  \
        return P##_plan_many_dft_r2c(rank, n, 1, in, NULL, 1, 1, out, NULL, 1, 1, flags);                             \
    }                                                                                                                  \
    P##_plan P##_plan_dft_c2r(int rank, const int *n, Cx *in, R *out, unsigned flags)                                 \
    {                                                                                                                  \
        return P##_plan_many_dft_c2r(rank, n, 1, in, NULL, 1, 1, out, NULL, 1, 1, flags);                             \
    }                                                                                                                  \
    P##_plan P##_plan_dft_r2c_1d(int n, R *in, Cx *out, unsigned flags) { return P##_plan_dft_r2c(1, &n, in, out, flags); } \
    P##_plan P##_plan_dft_c2r_1d(int n, Cx *in, R *out, unsigned flags) { return P##_plan_dft_c2r(1, &n, in, out, flags); } \
    P##_plan P##_plan_dft_r2c_2d(int n0, int n1, R *in, Cx *out, unsigned flags)                                      \
    {                                                                                                                  \
        int n[2] = {n0, n1};                                                                                           \
        return P##_plan_dft_r2c(2, n, in, out, flags);                                                                \
    }                                                                                                                  \
    P##_plan P##_plan_dft_c2r_2d(int n0, int n1, Cx *in, R *out, unsigned flags)                                      \
    {                                                                                                                  \
        int n[2] = {n0, n1};                                                                                           \
        return P##_plan_dft_c2r(2, n, in, out, flags);                                                                \
    }                                                                                                                  \
    P##_plan P##_plan_dft_r2c_3d(int n0, int n1, int n2, R *in, Cx *out, unsigned flags)                              \
    {                                                                                                                  \
        int n[3] = {n0, n1, n2};                                                                                       \
        return P##_plan_dft_r2c(3, n, in, out, flags);                                                                \
    }                                                                                                                  \
    P##_plan P##_plan_dft_c2r_3d(int n0, int n1, int n2, Cx *in, R *out, unsigned flags)                              \
    {                                                                                                                  \
        int n[3] = {n0, n1, n2};                                                                                       \
        return P##_plan_dft_c2r(3, n, in, out, flags);                                                                \
    }                                                                                                                  \
    static P##_plan P##_real_guru(int dir, int rank, const P##_iodim64 *dims, int hr, const P##_iodim64 *hd, void *in, \
                                  void *out)                                                                           \
    {                                                                                                                  \
        fw_dim d[16], h[16];                                                                                           \
        if (rank <= 0 || rank > 16 || hr < 0 || hr > 16 || !dims || (hr && !hd)) return NULL;                         \
        for (int i = 0; i < rank; i++)                                                                                 \
        {                                                                                                              \
            d[i].n = dims[i].n;                                                                                        \
            d[i].is = dims[i].is;                                                                                      \
            d[i].os = dims[i].os;                                                                                      \
        }                                                                                                              \
        for (int i = 0; i < hr; i++)                                                                                   \
        {                                                                                                              \
            h[i].n = hd[i].n;                                                                                          \
            h[i].is = hd[i].is;                                                                                        \
            h[i].os = hd[i].os;                                                                                        \
        }                                                                                                              \
        return fw_make(DT, 1, dir, rank, d, hr, h, in, out);                                                          \
    }                                                                                                                  \
    P##_plan P##_plan_guru64_dft_r2c(int rank, const P##_iodim64 *dims, int hr, const P##_iodim64 *hd, R *in,         \
                                     Cx *out, unsigned flags)                                                          \
    {                                                                                                                  \
        (void)flags;                                                                                                   \
        return P##_real_guru(0, rank, dims, hr, hd, in, out);                                                         \
    }                                                                                                                  \
    P##_plan P##_plan_guru64_dft_c2r(int rank, const P##_iodim64 *dims, int hr, const P##_iodim64 *hd, Cx *in,        \
                                     R *out, unsigned flags)                                                           \
    {                                                                                                                  \
        (void)flags;                                                                                                   \
        return P##_real_guru(1, rank, dims, hr, hd, in, out);                                                         \
    }                                                                                                                  \
    static int P##_widen(int rank, const P##_iodim *dims, int hr, const P##_iodim *hd, P##_iodim64 *d,                 \
                         P##_iodim64 *h)                                                                               \
    {                                                                                                                  \
        if (rank < 0 || rank > 16 || hr < 0 || hr > 16 || (rank && !dims) || (hr && !hd)) return -1;                  \
        for (int i = 0; i < rank; i++)                                                                                 \
        {                                                                                                              \
            d[i].n = dims[i].n;                                                                                        \
            d[i].is = dims[i].is;                                                                                      \
            d[i].os = dims[i].os;                                                                                      \
        }                                                                                                              \
        for (int i = 0; i < hr; i++)                                                                                   \
        {                                                                                                              \
            h[i].n = hd[i].n;                                                                                          \
            h[i].is = hd[i].is;                                                                                        \
            h[i].os = hd[i].os;                                                                                        \
        }                                                                                                              \
        return 0;                                                                                                      \
    }                                                                                                                  \
    P##_plan P##_plan_guru_dft_r2c(int rank, const P##_iodim *dims, int hr, const P##_iodim *hd, R *in, Cx *out,       \
                                   unsigned flags)                                                                     \
    {                                                                                                                  \
        P##_iodim64 d[16], h[16];                                                                                      \
        if (P##_widen(rank, dims, hr, hd, d, h)) return NULL;                                                          \
        return P##_plan_guru64_dft_r2c(rank, d, hr, h, in, out, flags);                                               \
    }                                                                                                                  \
    P##_plan P##_plan_guru_dft_c2r(int rank, const P##_iodim *dims, int hr, const P##_iodim *hd, Cx *in, R *out,       \
                                   unsigned flags)                                                                     \
    {                                                                                                                  \
        P##_iodim64 d[16], h[16];                                                                                      \
        if (P##_widen(rank, dims, hr, hd, d, h)) return NULL;                                                          \
        return P##_plan_guru64_dft_c2r(rank, d, hr, h, in, out, flags);                                               \
    }                                                                                                                  \
    P##_plan P##_plan_r2r(int rank, const int *n, R *in, R *out, const P##_r2r_kind *kind, unsigned flags)            \
    {                                                                                                                  \
        (void)rank, (void)n, (void)in, (void)out, (void)kind, (void)flags;                                            \
        fprintf(stderr, "[aoclfftz-gpu] WARNING: %s: r2r transforms are not supported\n", #P "_plan_r2r");             \
        return NULL;                                                                                                   \
    }                                                                                                                  \
    P##_plan P##_plan_r2r_1d(int n, R *in, R *out, P##_r2r_kind kind, unsigned flags)                                 \
    {                                                                                                                  \
        return P##_plan_r2r(1, &n, in, out, &kind, flags);                                                            \
    }                                                                                                                  \
    void P##_execute(const P##_plan p) { (void)aoclfftz_execute(p); }                                                 \
    void P##_execute_dft(const P##_plan p, Cx *in, Cx *out) { (void)aoclfftz_execute_io(p, in, out); }                \
    void P##_execute_dft_r2c(const P##_plan p, R *in, Cx *out) { (void)aoclfftz_execute_io(p, in, out); }             \
    void P##_execute_dft_c2r(const P##_plan p, Cx *in, R *out) { (void)aoclfftz_execute_io(p, in, out); }             \
    void P##_execute_r2r(const P##_plan p, R *in, R *out)                                                             \
    {                                                                                                                  \
        (void)p, (void)in, (void)out;                                                                                  \
        fprintf(stderr, "[aoclfftz-gpu] WARNING: %s: r2r transforms are not supported\n", #P "_execute_r2r");          \
    }                                                                                                                  \
    void P##_destroy_plan(P##_plan p) { aoclfftz_destroy(p); }                                                        \
    void *P##_malloc(size_t n) { return fw_malloc(n); }                                                               \
    R *P##_alloc_real(size_t n) { return n > (size_t)-1 / sizeof(R) ? NULL : (R *)fw_malloc(n * sizeof(R)); }         \
    Cx *P##_alloc_complex(size_t n) { return n > (size_t)-1 / sizeof(Cx) ? NULL : (Cx *)fw_malloc(n * sizeof(Cx)); }  \
    void P##_free(void *p) { fw_free(p); }                                                                            \
    void P##_cleanup(void) {}                                                                                         \
    int P##_init_threads(void) { return 1; }                                                                          \
    void P##_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }                           \
    int P##_planner_nthreads(void) { return g_nthreads; }                                                             \
    void P##_cleanup_threads(void) {}                                                                                 \
    void P##_set_timelimit(double t) { (void)t; }                                                                     \
    void P##_fprint_plan(const P##_plan p, FILE *f)                                                                   \
    {                                                                                                                  \
        char buf[1024];                                                                                                \
        if (aoclfftz_gpu_describe(p, buf, sizeof(buf)) >= 0 && f) fprintf(f, "%s", buf);                              \
    }                                                                                                                  \
    void P##_print_plan(const P##_plan p) { P##_fprint_plan(p, stdout); }                                           \
    /* FFTW's contract: a string the caller releases with free() */                                                 \
    char *P##_sprint_plan(const P##_plan p)                                                                            \
    {                                                                                                                  \
        char buf[1024];                                                                                                \
        buf[0] = 0;                                                                                                    \
        if (p) aoclfftz_gpu_describe(p, buf, sizeof(buf));                                                            \
        char *s = (char *)malloc(strlen(buf) + 1);                                                                     \
        if (s) strcpy(s, buf);                                                                                         \
        return s;                                                                                                      \
    }                                                                                                                  \
    /* nominal counts of the plan's transforms: 5 N log2 N real operations per                                       \
     * complex transform (half for real ones), split 3 : 2 between adds and                                          \
     * multiplies; the GPU kernels fuse many of them into FMAs */                                                    \
    void P##_flops(const P##_plan p, double *add, double *mul, double *fmas)                                          \
    {                                                                                                                  \
        const double f = fw_nominal_flops(p);                                                                          \
        if (add) *add = 0.6 * f;                                                                                       \
        if (mul) *mul = 0.4 * f;                                                                                       \
        if (fmas) *fmas = 0;                                                                                           \
    }                                                                                                                  \
    double P##_estimate_cost(const P##_plan p) { return fw_nominal_flops(p); }                                         \
    double P##_cost(const P##_plan p) { return fw_nominal_flops(p); }                                                  \
    int P##_alignment_of(R *p) { return (int)(((uintptr_t)p) % 16); }                                                 \
    void P##_make_planner_thread_safe(void) {}                                                                        \
    void P##_threads_set_callback(void (*parallel_loop)(void *(*work)(char *), char *jobdata, size_t elsize,          \
                                                        int njobs, void *data),                                        \
                                  void *data)                                                                          \
    {                                                                                                                  \
        (void)parallel_loop, (void)data; /* the GPU runs the transform, not a host thread team */                     \
    }                                                                                                                  \
    P##_plan P##_plan_r2r_2d(int n0, int n1, R *in, R *out, P##_r2r_kind k0, P##_r2r_kind k1, unsigned flags)         \
    {                                                                                                                  \
        const int n[2] = {n0, n1};                                                                                     \
        const P##_r2r_kind k[2] = {k0, k1};                                                                            \
        return P##_plan_r2r(2, n, in, out, k, flags);                                                                  \
    }                                                                                                                  \
    P##_plan P##_plan_r2r_3d(int n0, int n1, int n2, R *in, R *out, P##_r2r_kind k0, P##_r2r_kind k1,                 \
                             P##_r2r_kind k2, unsigned flags)                                                          \
    {                                                                                                                  \
        const int n[3] = {n0, n1, n2};                                                                                 \
        const P##_r2r_kind k[3] = {k0, k1, k2};                                                                        \
        return P##_plan_r2r(3, n, in, out, k, flags);                                                                  \
    }                                                                                                                  \
    P##_plan P##_plan_many_r2r(int rank, const int *n, int howmany, R *in, const int *inembed, int istride,           \
                               int idist, R *out, const int *onembed, int ostride, int odist,                          \
                               const P##_r2r_kind *kind, unsigned flags)                                               \
    {                                                                                                                  \
        (void)howmany, (void)inembed, (void)istride, (void)idist, (void)onembed, (void)ostride, (void)odist;          \
        return P##_plan_r2r(rank, n, in, out, kind, flags);                                                            \
    }                                                                                                                  \
    P##_plan P##_plan_guru_r2r(int rank, const P##_iodim *dims, int hr, const P##_iodim *hd, R *in, R *out,           \
                               const P##_r2r_kind *kind, unsigned flags)                                               \
    {                                                                                                                  \
        (void)dims, (void)hr, (void)hd;                                                                                \
        return P##_plan_r2r(rank, NULL, in, out, kind, flags);                                                         \
    }                                                                                                                  \
    P##_plan P##_plan_guru64_r2r(int rank, const P##_iodim64 *dims, int hr, const P##_iodim64 *hd, R *in, R *out,     \
                                 const P##_r2r_kind *kind, unsigned flags)                                             \
    {                                                                                                                  \
        (void)dims, (void)hr, (void)hd;                                                                                \
        return P##_plan_r2r(rank, NULL, in, out, kind, flags);                                                         \
    }                                                                                                                  \
    /* Wisdom: plans are rebuilt from the descriptor each time, so there is                                          \
     * nothing to store -- exports succeed and write nothing, imports report                                         \
     * that nothing was loaded (FFTW's "failure" value 0), and the exported                                          \
     * string is an empty string the caller frees with free(). */                                                    \
    void P##_forget_wisdom(void) {}                                                                                   \
    int P##_export_wisdom_to_filename(const char *filename)                                                           \
    {                                                                                                                  \
        (void)filename;                                                                                                \
        return 1;                                                                                                      \
    }                                                                                                                  \
    void P##_export_wisdom_to_file(FILE *f) { (void)f; }                                                              \
    char *P##_export_wisdom_to_string(void)                                                                           \
    {                                                                                                                  \
        char *s = (char *)malloc(1);                                                                                   \
        if (s) s[0] = 0;                                                                                               \
        return s;                                                                                                      \
    }                                                                                                                  \
    void P##_export_wisdom(P##_write_char_func write_char, void *data) { (void)write_char, (void)data; }              \
    int P##_import_system_wisdom(void) { return 0; }                                                                  \
    int P##_import_wisdom_from_filename(const char *filename)                                                         \
    {                                                                                                                  \
        (void)filename;                                                                                                \
        return 0;                                                                                                      \
    }                                                                                                                  \
    int P##_import_wisdom_from_file(FILE *f)                                                                          \
    {                                                                                                                  \
        (void)f;                                                                                                       \
        return 0;                                                                                                      \
    }                                                                                                                  \
    int P##_import_wisdom_from_string(const char *s)                                                                  \
    {                                                                                                                  \
        (void)s;                                                                                                       \
        return 0;                                                                                                      \
    }                                                                                                                  \
    int P##_import_wisdom(P##_read_char_func read_char, void *data)                                                   \
    {                                                                                                                  \
        (void)read_char, (void)data;                                                                                   \
        return 0;                                                                                                      \
    }                                                                                                                  \
    const char P##_version[] = AOCLFFTZ_LIBRARY_VERSION " B200 (FFTW compatible)";

/* 5 N log2 N real operations per complex transform of the plan (N the
 * product of its dims; half for real transforms), summed over its batch */
static double fw_nominal_flops(const void *h)
{
    const fz_plan *pl = (const fz_plan *)h;
    if (!pl || pl->magic != FZ_MAGIC || pl->nop) return 0.0;
    double n = 1.0, howmany = 1.0;
    for (int i = 0; i < pl->sv_rank; i++) n *= (double)pl->sv_dims[i].n;
    for (int i = 0; i < pl->sv_vrank; i++) howmany *= (double)pl->sv_vecs[i].n;
    const double f = n > 1 ? 5.0 * n * log2(n) * howmany : 0.0;
    return pl->fft_type == 0 ? f : 0.5 * f;
}

/* fftw_malloc: page-locked host memory (host-visible, and the library's
 * staging copies from it run at full bus speed); ordinary heap memory when
 * pinning is unavailable */
static void *fw_malloc(size_t n)
{
    void *p = NULL;
    if (n == 0) n = 1;
    if (cudaMallocHost(&p, n) == cudaSuccess) return p;
    cudaGetLastError();
    return malloc(n);
}

static void fw_free(void *p)
{
    if (!p) return;
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost)
        cudaFreeHost(p);
    else
    {
        cudaGetLastError();
        free(p);
    }
}

FW_DEFINE(fftw, 1, double, fftw_complex)
FW_DEFINE(fftwf, 0, float, fftwf_complex)
FW_DEFINE_REAL(fftw, 1, double, fftw_complex)
FW_DEFINE_REAL(fftwf, 0, float, fftwf_complex)
