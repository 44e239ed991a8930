/* aoclfftz.h -- plan / execute / destroy C ABI of the B200 FFT library.
 *
 * This header declares the same entry points, structures and error codes as the
 * reference library's public header (AOCL-FFTZ 6.0.0, api/aoclfftz.h), so that
 * a program written against that header relinks against libaoclfftz_gpu.so
 * unchanged. Each declaration names the reference declaration it replaces.
 *
 * Conventions (identical to the reference):
 *   - complex data is interleaved [re, im];
 *   - dims[0] is the innermost (contiguous) dimension;
 *   - strides count complex elements for c2c, real elements on the real side of
 *     r2c/c2r and complex elements on the half-complex side;
 *   - forward uses exp(-2 pi i jk/N); neither direction is normalised;
 *   - r2c output / c2r input holds n0/2+1 complex bins along dims[0].
 *
 * Buffers may be device pointers (the computation runs in place on the GPU)
 * or host pointers (the library stages them through device memory: copy in,
 * compute, copy out), so existing CPU callers work unchanged.
 */
#ifndef AOCLFFTZ_H
#define AOCLFFTZ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scalar types of the reference ABI (api/types.h:22-56). */
typedef int64_t FFTZ_INT64;
typedef int32_t FFTZ_INT32;
typedef ptrdiff_t FFTZ_INTP;
typedef uint64_t FFTZ_UINT64;
typedef uint32_t FFTZ_UINT32;
typedef size_t FFTZ_UINTP;
typedef char FFTZ_CHAR;
typedef unsigned char FFTZ_UCHAR;
typedef short FFTZ_SHORT;
typedef unsigned short FFTZ_USHORT;
typedef void FFTZ_VOID;
typedef float FFTZ_FLOAT32;
typedef float FFTZ_FLOAT;
typedef double FFTZ_FLOAT64;
typedef double FFTZ_DOUBLE;
typedef uint8_t FFTZ_UINT8;

#define AOCLFFTZ_LIBRARY_VERSION "AOCL-FFTZ 6.0.0"

/* Status codes; values equal the reference's (api/aoclfftz.h:60-68). */
typedef enum
{
    AOCLFFTZ_TIME_OUT = -5,     /* an operation did not finish in time          */
    AOCLFFTZ_MEMORY_FAILURE,    /* allocation or memory access failed (-4)      */
    AOCLFFTZ_INVALID_INPUT,     /* invalid descriptor or buffers (-3)           */
    AOCLFFTZ_SETUP_FAILURE,     /* plan construction failed (-2)                */
    AOCLFFTZ_EXECUTION_FAILURE, /* execution failed (-1)                        */
    AOCLFFTZ_SUCCESS            /* 0                                            */
} aoclfftz_error_type;

/* Logging verbosity (api/aoclfftz.h:74-80). */
typedef enum
{
    AOCLFFTZ_LOG_NONE = 0,
    AOCLFFTZ_LOG_INFO = 1,
    AOCLFFTZ_LOG_TRACE = 2,
    AOCLFFTZ_LOG_DEBUG = 3,
} aoclfftz_logger_mode;

/* Problem flags (api/aoclfftz.h:86-102). */
typedef struct aoclfftz_flags
{
    FFTZ_UINT8 fft_type;            /* 0 complex, 1 real                               */
    FFTZ_UINT8 fft_direction;       /* 0 forward, 1 backward                           */
    FFTZ_UINT8 storage_order;       /* must be 0 (in-order); 1 is rejected              */
    FFTZ_UINT8 fft_placement;       /* 0 in-place (in == out), 1 out-of-place          */
    FFTZ_UINT8 transpose_mode;      /* must be 0; standalone transpose is rejected     */
    FFTZ_UINT8 bit_reproducibility; /* 0 or 1; results are bitwise reproducible always */
} aoclfftz_flags_t;

/* One tensor dimension, LP64 (api/aoclfftz.h:108-113). */
typedef struct aoclfftz_dim
{
    FFTZ_INT32 n;
    FFTZ_INT32 in_stride;
    FFTZ_INT32 out_stride;
} aoclfftz_dim_t;

/* One tensor dimension, ILP64 (api/aoclfftz.h:119-124). */
typedef struct aoclfftz_dim_64_
{
    FFTZ_INTP n;
    FFTZ_INTP in_stride;
    FFTZ_INTP out_stride;
} aoclfftz_dim_t_64_;

/* Threading parameters (api/aoclfftz.h:130-140); accepted and ignored on the
 * GPU, where the grid replaces the thread team. */
typedef struct aoclfftz_smp_pfft
{
    FFTZ_INT32 num_threads;
    FFTZ_UINT32 dynamic_load_model;
} aoclfftz_smp_pfft_t;

/* Control parameters (api/aoclfftz.h:146-165). opt_level selects an x86 ISA in
 * the reference; it is validated the same way and otherwise ignored here. */
typedef struct aoclfftz_cntrl_params
{
    FFTZ_INT32 opt_level;
    FFTZ_INT32 opt_off;
    aoclfftz_logger_mode logger_mode;
    FFTZ_INT32 measure_stats;
} aoclfftz_cntrl_params_t;

/* Problem descriptors (api/aoclfftz.h:174-311): the same four layouts. */
typedef struct
{
    FFTZ_FLOAT *in;
    FFTZ_FLOAT *out;
    FFTZ_INT32 vec_rank;
    FFTZ_INT32 dim_rank;
    aoclfftz_dim_t *dims;
    aoclfftz_dim_t *vecs;
    aoclfftz_flags_t flags;
    aoclfftz_smp_pfft_t pthr_fft;
    aoclfftz_cntrl_params_t cntrl_params;
} aoclfftz_prob_desc_f;

typedef struct
{
    FFTZ_DOUBLE *in;
    FFTZ_DOUBLE *out;
    FFTZ_INT32 vec_rank;
    FFTZ_INT32 dim_rank;
    aoclfftz_dim_t *dims;
    aoclfftz_dim_t *vecs;
    aoclfftz_flags_t flags;
    aoclfftz_smp_pfft_t pthr_fft;
    aoclfftz_cntrl_params_t cntrl_params;
} aoclfftz_prob_desc_d;

typedef struct
{
    FFTZ_FLOAT *in;
    FFTZ_FLOAT *out;
    FFTZ_INT32 vec_rank;
    FFTZ_INT32 dim_rank;
    aoclfftz_dim_t_64_ *dims;
    aoclfftz_dim_t_64_ *vecs;
    aoclfftz_flags_t flags;
    aoclfftz_smp_pfft_t pthr_fft;
    aoclfftz_cntrl_params_t cntrl_params;
} aoclfftz_prob_desc_f_64_;

typedef struct
{
    FFTZ_DOUBLE *in;
    FFTZ_DOUBLE *out;
    FFTZ_INT32 vec_rank;
    FFTZ_INT32 dim_rank;
    aoclfftz_dim_t_64_ *dims;
    aoclfftz_dim_t_64_ *vecs;
    aoclfftz_flags_t flags;
    aoclfftz_smp_pfft_t pthr_fft;
    aoclfftz_cntrl_params_t cntrl_params;
} aoclfftz_prob_desc_d_64_;

/* Builds a plan for the descriptor; NULL on any failure. The descriptor and its
 * dims/vecs arrays may be freed after the call. in/out may be NULL, in which
 * case the plan runs only through aoclfftz_execute_io.
 * Replaces api/aoclfftz.h:343 (float LP64), :371 (double LP64),
 * :399 (float ILP64), :428 (double ILP64). */
FFTZ_VOID *aoclfftz_setup_f(aoclfftz_prob_desc_f *problem);
FFTZ_VOID *aoclfftz_setup_d(aoclfftz_prob_desc_d *problem);
FFTZ_VOID *aoclfftz_setup_f_64_(aoclfftz_prob_desc_f_64_ *problem);
FFTZ_VOID *aoclfftz_setup_d_64_(aoclfftz_prob_desc_d_64_ *problem);

/* Runs the plan on the setup-time buffers. Returns AOCLFFTZ_EXECUTION_FAILURE
 * for a NULL handle or when a setup-time buffer was NULL. Device buffers: the
 * call returns once the work is enqueued on the plan's stream (see
 * aoclfftz_gpu.h); host buffers: the call returns when the result is in out.
 * Not safe to call concurrently on one handle. Replaces api/aoclfftz.h:452. */
aoclfftz_error_type aoclfftz_execute(FFTZ_VOID *handle);

/* Runs the plan on new buffers of the same placement (in == out for in-place
 * plans, in != out otherwise). Safe to call concurrently on one handle: the
 * first caller uses the plan's scratch, concurrent callers get their own.
 * Replaces api/aoclfftz.h:484. */
aoclfftz_error_type aoclfftz_execute_io(FFTZ_VOID *handle, FFTZ_VOID *in, FFTZ_VOID *out);

/* Releases the plan and all device memory it owns. Replaces api/aoclfftz.h:499. */
FFTZ_VOID aoclfftz_destroy(FFTZ_VOID *handle);

/* Version string. Replaces api/aoclfftz.h:507. */
const FFTZ_CHAR *aoclfftz_version(FFTZ_VOID);

#ifdef __cplusplus
}
#endif

#endif /* AOCLFFTZ_H */
