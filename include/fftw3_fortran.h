/* fftw3_fortran.h -- the Fortran-callable FFTW planner interface.
 *
 * Same entry points as the reference wrapper's Fortran layer
 * (wrappers/fftw/src/fortran/fftw_plan_wrapper.c, fftw_execute_wrapper.c,
 * fftw_destroy_wrapper.c, fftw_misc_wrapper.c): every argument by reference,
 * the plan returned through the first argument, dimension lists in Fortran
 * (column-major) order -- reversed here before the C planner of fftw3.h is
 * called. dfftw_* is double precision, dfftwf_* single precision (the
 * reference's names). Fortran code calls them with the usual trailing
 * underscore mangling, e.g. `call dfftw_plan_dft_1d(plan, n, in, out,
 * FFTW_FORWARD, FFTW_ESTIMATE)`.
 */
#ifndef AOCLFFTZ_FFTW3_FORTRAN_H
#define AOCLFFTZ_FFTW3_FORTRAN_H

#include "fftw3.h"

#ifdef __cplusplus
extern "C" {
#endif

#define AOCLFFTZ_FFTW_FORTRAN_DECLARE(F, P, R, C)                                                               \
    void F##_plan_dft_(P##_plan *p, int *rank, const int *n, C *in, C *out, int *sign, int *flags);            \
    void F##_plan_dft_1d_(P##_plan *p, int *n, C *in, C *out, int *sign, int *flags);                          \
    void F##_plan_dft_2d_(P##_plan *p, int *nx, int *ny, C *in, C *out, int *sign, int *flags);                \
    void F##_plan_dft_3d_(P##_plan *p, int *nx, int *ny, int *nz, C *in, C *out, int *sign, int *flags);       \
    void F##_plan_many_dft_(P##_plan *p, int *rank, const int *n, int *howmany, C *in, const int *inembed,    \
                            int *istride, int *idist, C *out, const int *onembed, int *ostride, int *odist,   \
                            int *sign, int *flags);                                                            \
    void F##_plan_guru_dft_(P##_plan *p, int *rank, const int *n, const int *is, const int *os,               \
                            int *howmany_rank, const int *h_n, const int *h_is, const int *h_os, C *in,       \
                            C *out, int *sign, int *flags);                                                    \
    void F##_plan_dft_r2c_(P##_plan *p, int *rank, const int *n, R *in, C *out, int *flags);                  \
    void F##_plan_dft_r2c_1d_(P##_plan *p, int *n, R *in, C *out, int *flags);                                \
    void F##_plan_dft_r2c_2d_(P##_plan *p, int *nx, int *ny, R *in, C *out, int *flags);                      \
    void F##_plan_dft_r2c_3d_(P##_plan *p, int *nx, int *ny, int *nz, R *in, C *out, int *flags);             \
    void F##_plan_many_dft_r2c_(P##_plan *p, int *rank, const int *n, int *howmany, R *in, const int *inembed, \
                                int *istride, int *idist, C *out, const int *onembed, int *ostride,          \
                                int *odist, int *flags);                                                       \
    void F##_plan_guru_dft_r2c_(P##_plan *p, int *rank, const int *n, const int *is, const int *os,           \
                                int *howmany_rank, const int *h_n, const int *h_is, const int *h_os, R *in,   \
                                C *out, int *flags);                                                           \
    void F##_plan_dft_c2r_(P##_plan *p, int *rank, const int *n, C *in, R *out, int *flags);                  \
    void F##_plan_dft_c2r_1d_(P##_plan *p, int *n, C *in, R *out, int *flags);                                \
    void F##_plan_dft_c2r_2d_(P##_plan *p, int *nx, int *ny, C *in, R *out, int *flags);                      \
    void F##_plan_dft_c2r_3d_(P##_plan *p, int *nx, int *ny, int *nz, C *in, R *out, int *flags);             \
    void F##_plan_many_dft_c2r_(P##_plan *p, int *rank, const int *n, int *howmany, C *in, const int *inembed, \
                                int *istride, int *idist, R *out, const int *onembed, int *ostride,          \
                                int *odist, int *flags);                                                       \
    void F##_plan_guru_dft_c2r_(P##_plan *p, int *rank, const int *n, const int *is, const int *os,           \
                                int *howmany_rank, const int *h_n, const int *h_is, const int *h_os, C *in,   \
                                R *out, int *flags);                                                           \
    void F##_execute_(P##_plan *const p);                                                                      \
    void F##_execute_dft_(P##_plan *p, C *in, C *out);                                                         \
    void F##_execute_dft_r2c_(P##_plan *p, R *in, C *out);                                                     \
    void F##_execute_dft_c2r_(P##_plan *p, C *in, R *out);                                                     \
    void F##_destroy_plan_(P##_plan *p);                                                                       \
    void F##_cleanup_(void);                                                                                   \
    void F##_plan_with_nthreads_(int *nthreads);                                                               \
    void F##_init_threads_(int *ret);                                                                          \
    void F##_cleanup_threads_(void);                                                                           \
    void F##_flops_(P##_plan *p, double *add, double *mul, double *fma);                                       \
    void F##_estimate_cost_(double *cost, P##_plan *const p);                                                  \
    void F##_cost_(double *cost, P##_plan *const p);

AOCLFFTZ_FFTW_FORTRAN_DECLARE(dfftw, fftw, double, fftw_complex)
AOCLFFTZ_FFTW_FORTRAN_DECLARE(dfftwf, fftwf, float, fftwf_complex)

#ifdef __cplusplus
}
#endif
#endif
