/* Fortran-callable FFTW interface (C99 host layer): arguments by reference,
 * dimension lists in Fortran order, reversed here before the C planners of
 * fftw_api.c are called. The entry points and their argument order are the
 * reference wrapper's (wrappers/fftw/src/fortran/fftw_plan_wrapper.c,
 * fftw_execute_wrapper.c, fftw_destroy_wrapper.c, fftw_misc_wrapper.c). */
#include <stddef.h>

#include "fftw3_fortran.h"

#define FZ_FORTRAN_MAX_RANK 16

static int fz_reverse(int rank, const int *src, int *dst)
{
    if (rank < 0 || rank > FZ_FORTRAN_MAX_RANK) return -1;
    for (int i = 0; i < rank; i++) dst[i] = src[rank - 1 - i];
    return 0;
}

#define FZ_FORTRAN_DEFINE(F, P, R, C)                                                                           \
    static int F##_guru_dims(int rank, const int *n, const int *is, const int *os, int hr, const int *hn,       \
                             const int *his, const int *hos, P##_iodim *d, P##_iodim *h)                       \
    {                                                                                                           \
        if (rank < 0 || rank > FZ_FORTRAN_MAX_RANK || hr < 0 || hr > FZ_FORTRAN_MAX_RANK) return -1;           \
        for (int i = 0; i < rank; i++)                                                                          \
        {                                                                                                       \
            d[i].n = n[rank - 1 - i];                                                                           \
            d[i].is = is[rank - 1 - i];                                                                         \
            d[i].os = os[rank - 1 - i];                                                                         \
        }                                                                                                       \
        for (int i = 0; i < hr; i++)                                                                            \
        {                                                                                                       \
            h[i].n = hn[hr - 1 - i];                                                                            \
            h[i].is = his[hr - 1 - i];                                                                          \
            h[i].os = hos[hr - 1 - i];                                                                          \
        }                                                                                                       \
        return 0;                                                                                               \
    }                                                                                                           \
    void F##_plan_dft_(P##_plan *p, int *rank, const int *n, C *in, C *out, int *sign, int *flags)             \
    {                                                                                                           \
        int rn[FZ_FORTRAN_MAX_RANK];                                                                            \
        *p = fz_reverse(*rank, n, rn) ? NULL : P##_plan_dft(*rank, rn, in, out, *sign, (unsigned)*flags);       \
    }                                                                                                           \
    void F##_plan_dft_1d_(P##_plan *p, int *n, C *in, C *out, int *sign, int *flags)                           \
    {                                                                                                           \
        *p = P##_plan_dft_1d(*n, in, out, *sign, (unsigned)*flags);                                             \
    }                                                                                                           \
    void F##_plan_dft_2d_(P##_plan *p, int *nx, int *ny, C *in, C *out, int *sign, int *flags)                 \
    {                                                                                                           \
        *p = P##_plan_dft_2d(*ny, *nx, in, out, *sign, (unsigned)*flags);                                       \
    }                                                                                                           \
    void F##_plan_dft_3d_(P##_plan *p, int *nx, int *ny, int *nz, C *in, C *out, int *sign, int *flags)        \
    {                                                                                                           \
        *p = P##_plan_dft_3d(*nz, *ny, *nx, in, out, *sign, (unsigned)*flags);                                  \
    }                                                                                                           \
    void F##_plan_many_dft_(P##_plan *p, int *rank, const int *n, int *howmany, C *in, const int *inembed,     \
                            int *istride, int *idist, C *out, const int *onembed, int *ostride, int *odist,    \
                            int *sign, int *flags)                                                              \
    {                                                                                                           \
        int rn[FZ_FORTRAN_MAX_RANK], ri[FZ_FORTRAN_MAX_RANK], ro[FZ_FORTRAN_MAX_RANK];                          \
        *p = NULL;                                                                                              \
        if (fz_reverse(*rank, n, rn) || (inembed && fz_reverse(*rank, inembed, ri)) ||                          \
            (onembed && fz_reverse(*rank, onembed, ro)))                                                        \
            return;                                                                                             \
        *p = P##_plan_many_dft(*rank, rn, *howmany, in, inembed ? ri : NULL, *istride, *idist, out,            \
                               onembed ? ro : NULL, *ostride, *odist, *sign, (unsigned)*flags);                 \
    }                                                                                                           \
    void F##_plan_guru_dft_(P##_plan *p, int *rank, const int *n, const int *is, const int *os,                \
                            int *howmany_rank, const int *h_n, const int *h_is, const int *h_os, C *in,        \
                            C *out, int *sign, int *flags)                                                      \
    {                                                                                                           \
        P##_iodim d[FZ_FORTRAN_MAX_RANK], h[FZ_FORTRAN_MAX_RANK];                                               \
        *p = F##_guru_dims(*rank, n, is, os, *howmany_rank, h_n, h_is, h_os, d, h)                              \
                 ? NULL                                                                                         \
                 : P##_plan_guru_dft(*rank, d, *howmany_rank, h, in, out, *sign, (unsigned)*flags);             \
    }                                                                                                           \
    void F##_plan_dft_r2c_(P##_plan *p, int *rank, const int *n, R *in, C *out, int *flags)                    \
    {                                                                                                           \
        int rn[FZ_FORTRAN_MAX_RANK];                                                                            \
        *p = fz_reverse(*rank, n, rn) ? NULL : P##_plan_dft_r2c(*rank, rn, in, out, (unsigned)*flags);          \
    }                                                                                                           \
    void F##_plan_dft_r2c_1d_(P##_plan *p, int *n, R *in, C *out, int *flags)                                  \
    {                                                                                                           \
        *p = P##_plan_dft_r2c_1d(*n, in, out, (unsigned)*flags);                                                \
    }                                                                                                           \
    void F##_plan_dft_r2c_2d_(P##_plan *p, int *nx, int *ny, R *in, C *out, int *flags)                        \
    {                                                                                                           \
        *p = P##_plan_dft_r2c_2d(*ny, *nx, in, out, (unsigned)*flags);                                          \
    }                                                                                                           \
    void F##_plan_dft_r2c_3d_(P##_plan *p, int *nx, int *ny, int *nz, R *in, C *out, int *flags)               \
    {                                                                                                           \
        *p = P##_plan_dft_r2c_3d(*nz, *ny, *nx, in, out, (unsigned)*flags);                                     \
    }                                                                                                           \
    void F##_plan_many_dft_r2c_(P##_plan *p, int *rank, const int *n, int *howmany, R *in, const int *inembed, \
                                int *istride, int *idist, C *out, const int *onembed, int *ostride,            \
                                int *odist, int *flags)                                                         \
    {                                                                                                           \
        int rn[FZ_FORTRAN_MAX_RANK], ri[FZ_FORTRAN_MAX_RANK], ro[FZ_FORTRAN_MAX_RANK];                          \
        *p = NULL;                                                                                              \
        if (fz_reverse(*rank, n, rn) || (inembed && fz_reverse(*rank, inembed, ri)) ||                          \
            (onembed && fz_reverse(*rank, onembed, ro)))                                                        \
            return;                                                                                             \
        *p = P##_plan_many_dft_r2c(*rank, rn, *howmany, in, inembed ? ri : NULL, *istride, *idist, out,        \
                                   onembed ? ro : NULL, *ostride, *odist, (unsigned)*flags);                    \
    }                                                                                                           \
    void F##_plan_guru_dft_r2c_(P##_plan *p, int *rank, const int *n, const int *is, const int *os,            \
                                int *howmany_rank, const int *h_n, const int *h_is, const int *h_os, R *in,    \
                                C *out, int *flags)                                                             \
    {                                                                                                           \
        P##_iodim d[FZ_FORTRAN_MAX_RANK], h[FZ_FORTRAN_MAX_RANK];                                               \
        *p = F##_guru_dims(*rank, n, is, os, *howmany_rank, h_n, h_is, h_os, d, h)                              \
                 ? NULL                                                                                         \
                 : P##_plan_guru_dft_r2c(*rank, d, *howmany_rank, h, in, out, (unsigned)*flags);                \
    }                                                                                                           \
    void F##_plan_dft_c2r_(P##_plan *p, int *rank, const int *n, C *in, R *out, int *flags)                    \
    {                                                                                                           \
        int rn[FZ_FORTRAN_MAX_RANK];                                                                            \
        *p = fz_reverse(*rank, n, rn) ? NULL : P##_plan_dft_c2r(*rank, rn, in, out, (unsigned)*flags);          \
    }                                                                                                           \
    void F##_plan_dft_c2r_1d_(P##_plan *p, int *n, C *in, R *out, int *flags)                                  \
    {                                                                                                           \
        *p = P##_plan_dft_c2r_1d(*n, in, out, (unsigned)*flags);                                                \
    }                                                                                                           \
    void F##_plan_dft_c2r_2d_(P##_plan *p, int *nx, int *ny, C *in, R *out, int *flags)                        \
    {                                                                                                           \
        *p = P##_plan_dft_c2r_2d(*ny, *nx, in, out, (unsigned)*flags);                                          \
    }                                                                                                           \
    void F##_plan_dft_c2r_3d_(P##_plan *p, int *nx, int *ny, int *nz, C *in, R *out, int *flags)               \
    {                                                                                                           \
        *p = P##_plan_dft_c2r_3d(*nz, *ny, *nx, in, out, (unsigned)*flags);                                     \
    }                                                                                                           \
    void F##_plan_many_dft_c2r_(P##_plan *p, int *rank, const int *n, int *howmany, C *in, const int *inembed, \
                                int *istride, int *idist, R *out, const int *onembed, int *ostride,            \
                                int *odist, int *flags)                                                         \
    {                                                                                                           \
        int rn[FZ_FORTRAN_MAX_RANK], ri[FZ_FORTRAN_MAX_RANK], ro[FZ_FORTRAN_MAX_RANK];                          \
        *p = NULL;                                                                                              \
        if (fz_reverse(*rank, n, rn) || (inembed && fz_reverse(*rank, inembed, ri)) ||                          \
            (onembed && fz_reverse(*rank, onembed, ro)))                                                        \
            return;                                                                                             \
        *p = P##_plan_many_dft_c2r(*rank, rn, *howmany, in, inembed ? ri : NULL, *istride, *idist, out,        \
                                   onembed ? ro : NULL, *ostride, *odist, (unsigned)*flags);                    \
    }                                                                                                           \
    void F##_plan_guru_dft_c2r_(P##_plan *p, int *rank, const int *n, const int *is, const int *os,            \
                                int *howmany_rank, const int *h_n, const int *h_is, const int *h_os, C *in,    \
                                R *out, int *flags)                                                             \
    {                                                                                                           \
        P##_iodim d[FZ_FORTRAN_MAX_RANK], h[FZ_FORTRAN_MAX_RANK];                                               \
        *p = F##_guru_dims(*rank, n, is, os, *howmany_rank, h_n, h_is, h_os, d, h)                              \
                 ? NULL                                                                                         \
                 : P##_plan_guru_dft_c2r(*rank, d, *howmany_rank, h, in, out, (unsigned)*flags);                \
    }                                                                                                           \
    void F##_execute_(P##_plan *const p) { P##_execute(*p); }                                                   \
    void F##_execute_dft_(P##_plan *p, C *in, C *out) { P##_execute_dft(*p, in, out); }                        \
    void F##_execute_dft_r2c_(P##_plan *p, R *in, C *out) { P##_execute_dft_r2c(*p, in, out); }                \
    void F##_execute_dft_c2r_(P##_plan *p, C *in, R *out) { P##_execute_dft_c2r(*p, in, out); }                \
    void F##_destroy_plan_(P##_plan *p) { P##_destroy_plan(*p); }                                               \
    void F##_cleanup_(void) { P##_cleanup(); }                                                                  \
    void F##_plan_with_nthreads_(int *nthreads) { P##_plan_with_nthreads(*nthreads); }                          \
    void F##_init_threads_(int *ret) { *ret = P##_init_threads(); }                                             \
    void F##_cleanup_threads_(void) { P##_cleanup_threads(); }                                                  \
    void F##_flops_(P##_plan *p, double *add, double *mul, double *fma) { P##_flops(*p, add, mul, fma); }      \
    void F##_estimate_cost_(double *cost, P##_plan *const p) { *cost = P##_estimate_cost(*p); }                \
    void F##_cost_(double *cost, P##_plan *const p) { *cost = P##_cost(*p); }

FZ_FORTRAN_DEFINE(dfftw, fftw, double, fftw_complex)
FZ_FORTRAN_DEFINE(dfftwf, fftwf, float, fftwf_complex)
