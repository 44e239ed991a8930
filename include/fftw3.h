/* fftw3.h -- FFTW3-compatible planning / execution surface of the B200 FFT library.
 *
 * The same entry points as the reference library's FFTW wrapper
 * (wrappers/fftw/api/fftw_wrapper.h:51-300, installed there as fftw3.h), for
 * double (fftw_*) and float (fftwf_*). Plans are aoclfftz handles: the
 * translation follows wrappers/fftw/src/translator/fftz_translator.c (FFTW's
 * row-major n[] becomes dims[] innermost-first; placement is in == out; the
 * sign picks the direction; planner flags are accepted and ignored).
 * Buffers may live in host memory (the library stages them through the GPU)
 * or on the device. fftw_malloc returns page-locked host memory so that the
 * staging copies run at full bus speed.
 * r2r kinds are not supported, as in the reference: planning returns NULL
 * and prints a warning.
 */
#ifndef AOCLFFTZ_FFTW3_H
#define AOCLFFTZ_FFTW3_H

#include <stddef.h>
#include <stdio.h>

#include "aoclfftz.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

#if !defined(FFTW_NO_Complex) && defined(_Complex_I) && defined(complex) && defined(I)
typedef double _Complex fftw_complex;
typedef float _Complex fftwf_complex;
#else
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
#endif

typedef void *fftw_plan;
typedef void *fftwf_plan;

typedef struct
{
    int n, is, os;
} fftw_iodim;
typedef fftw_iodim fftwf_iodim;
typedef struct
{
    ptrdiff_t n, is, os;
} fftw_iodim64;
typedef fftw_iodim64 fftwf_iodim64;
typedef int fftw_r2r_kind;
typedef int fftwf_r2r_kind;
typedef void (*fftw_write_char_func)(char c, void *data);
typedef int (*fftw_read_char_func)(void *data);
typedef fftw_write_char_func fftwf_write_char_func;
typedef fftw_read_char_func fftwf_read_char_func;

/* Declares one precision's API: P = prefix tag (fftw / fftwf), R = real type,
 * C = complex type. */
#define AOCLFFTZ_FFTW_DECLARE(P, R, C)                                                                       \
    P##_plan P##_plan_dft(int rank, const int *n, C *in, C *out, int sign, unsigned flags);                \
    P##_plan P##_plan_dft_1d(int n, C *in, C *out, int sign, unsigned flags);                              \
    P##_plan P##_plan_dft_2d(int n0, int n1, C *in, C *out, int sign, unsigned flags);                     \
    P##_plan P##_plan_dft_3d(int n0, int n1, int n2, C *in, C *out, int sign, unsigned flags);             \
    P##_plan P##_plan_many_dft(int rank, const int *n, int howmany, C *in, const int *inembed, int istride, \
                               int idist, C *out, const int *onembed, int ostride, int odist, int sign,    \
                               unsigned flags);                                                           \
    P##_plan P##_plan_guru_dft(int rank, const P##_iodim *dims, int howmany_rank,                          \
                               const P##_iodim *howmany_dims, C *in, C *out, int sign, unsigned flags);    \
    P##_plan P##_plan_guru64_dft(int rank, const P##_iodim64 *dims, int howmany_rank,                      \
                                 const P##_iodim64 *howmany_dims, C *in, C *out, int sign, unsigned flags); \
    P##_plan P##_plan_dft_r2c(int rank, const int *n, R *in, C *out, unsigned flags);                      \
    P##_plan P##_plan_dft_r2c_1d(int n, R *in, C *out, unsigned flags);                                    \
    P##_plan P##_plan_dft_r2c_2d(int n0, int n1, R *in, C *out, unsigned flags);                           \
    P##_plan P##_plan_dft_r2c_3d(int n0, int n1, int n2, R *in, C *out, unsigned flags);                   \
    P##_plan P##_plan_many_dft_r2c(int rank, const int *n, int howmany, R *in, const int *inembed,          \
                                   int istride, int idist, C *out, const int *onembed, int ostride,        \
                                   int odist, unsigned flags);                                            \
    P##_plan P##_plan_guru_dft_r2c(int rank, const P##_iodim *dims, int howmany_rank,                      \
                                   const P##_iodim *howmany_dims, R *in, C *out, unsigned flags);          \
    P##_plan P##_plan_guru64_dft_r2c(int rank, const P##_iodim64 *dims, int howmany_rank,                  \
                                     const P##_iodim64 *howmany_dims, R *in, C *out, unsigned flags);      \
    P##_plan P##_plan_dft_c2r(int rank, const int *n, C *in, R *out, unsigned flags);                      \
    P##_plan P##_plan_dft_c2r_1d(int n, C *in, R *out, unsigned flags);                                    \
    P##_plan P##_plan_dft_c2r_2d(int n0, int n1, C *in, R *out, unsigned flags);                           \
    P##_plan P##_plan_dft_c2r_3d(int n0, int n1, int n2, C *in, R *out, unsigned flags);                   \
    P##_plan P##_plan_many_dft_c2r(int rank, const int *n, int howmany, C *in, const int *inembed,          \
                                   int istride, int idist, R *out, const int *onembed, int ostride,        \
                                   int odist, unsigned flags);                                            \
    P##_plan P##_plan_guru_dft_c2r(int rank, const P##_iodim *dims, int howmany_rank,                      \
                                   const P##_iodim *howmany_dims, C *in, R *out, unsigned flags);          \
    P##_plan P##_plan_guru64_dft_c2r(int rank, const P##_iodim64 *dims, int howmany_rank,                  \
                                     const P##_iodim64 *howmany_dims, C *in, R *out, unsigned flags);      \
    P##_plan P##_plan_r2r(int rank, const int *n, R *in, R *out, const P##_r2r_kind *kind, unsigned flags); \
    P##_plan P##_plan_r2r_1d(int n, R *in, R *out, P##_r2r_kind kind, unsigned flags);                     \
    void P##_execute(const P##_plan p);                                                                    \
    void P##_execute_dft(const P##_plan p, C *in, C *out);                                                 \
    void P##_execute_dft_r2c(const P##_plan p, R *in, C *out);                                             \
    void P##_execute_dft_c2r(const P##_plan p, C *in, R *out);                                             \
    void P##_execute_r2r(const P##_plan p, R *in, R *out);                                                 \
    void P##_destroy_plan(P##_plan p);                                                                     \
    void *P##_malloc(size_t n);                                                                            \
    R *P##_alloc_real(size_t n);                                                                           \
    C *P##_alloc_complex(size_t n);                                                                        \
    void P##_free(void *p);                                                                                \
    void P##_cleanup(void);                                                                                \
    int P##_init_threads(void);                                                                            \
    void P##_plan_with_nthreads(int nthreads);                                                             \
    int P##_planner_nthreads(void);                                                                        \
    void P##_cleanup_threads(void);                                                                        \
    void P##_set_timelimit(double t);                                                                      \
    void P##_print_plan(const P##_plan p);                                                                 \
    void P##_fprint_plan(const P##_plan p, FILE *f);                                                       \
    char *P##_sprint_plan(const P##_plan p);                                                               \
    void P##_flops(const P##_plan p, double *add, double *mul, double *fmas);                              \
    double P##_estimate_cost(const P##_plan p);                                                            \
    double P##_cost(const P##_plan p);                                                                     \
    int P##_alignment_of(R *p);                                                                            \
    void P##_make_planner_thread_safe(void);                                                               \
    void P##_threads_set_callback(void (*parallel_loop)(void *(*work)(char *), char *jobdata, size_t elsize, \
                                                        int njobs, void *data),                            \
                                  void *data);                                                             \
    P##_plan P##_plan_r2r_2d(int n0, int n1, R *in, R *out, P##_r2r_kind k0, P##_r2r_kind k1, unsigned flags); \
    P##_plan P##_plan_r2r_3d(int n0, int n1, int n2, R *in, R *out, P##_r2r_kind k0, P##_r2r_kind k1,      \
                             P##_r2r_kind k2, unsigned flags);                                             \
    P##_plan P##_plan_many_r2r(int rank, const int *n, int howmany, R *in, const int *inembed, int istride,  \
                               int idist, R *out, const int *onembed, int ostride, int odist,              \
                               const P##_r2r_kind *kind, unsigned flags);                                  \
    P##_plan P##_plan_guru_r2r(int rank, const P##_iodim *dims, int howmany_rank,                          \
                               const P##_iodim *howmany_dims, R *in, R *out, const P##_r2r_kind *kind,     \
                               unsigned flags);                                                            \
    P##_plan P##_plan_guru64_r2r(int rank, const P##_iodim64 *dims, int howmany_rank,                      \
                                 const P##_iodim64 *howmany_dims, R *in, R *out, const P##_r2r_kind *kind, \
                                 unsigned flags);                                                          \
    void P##_forget_wisdom(void);                                                                          \
    int P##_export_wisdom_to_filename(const char *filename);                                               \
    void P##_export_wisdom_to_file(FILE *f);                                                               \
    char *P##_export_wisdom_to_string(void);                                                               \
    void P##_export_wisdom(P##_write_char_func write_char, void *data);                                    \
    int P##_import_system_wisdom(void);                                                                    \
    int P##_import_wisdom_from_filename(const char *filename);                                             \
    int P##_import_wisdom_from_file(FILE *f);                                                              \
    int P##_import_wisdom_from_string(const char *s);                                                      \
    int P##_import_wisdom(P##_read_char_func read_char, void *data);                                       \
    extern const char P##_version[];

AOCLFFTZ_FFTW_DECLARE(fftw, double, fftw_complex)
AOCLFFTZ_FFTW_DECLARE(fftwf, float, fftwf_complex)

#ifdef __cplusplus
}
#endif
#endif
