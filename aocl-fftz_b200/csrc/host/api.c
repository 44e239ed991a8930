/* Public C ABI: aoclfftz_setup_* / execute / execute_io / destroy / version
 * and the GPU extensions of aoclfftz_gpu.h (C99 host layer).
 *
 * Mirrors api/aoclfftz_api.c of the reference: setup validates the descriptor
 * with the rules of api/validate_problem.h:346 and returns NULL on any failure;
 * execute refuses NULL setup-time buffers (api/aoclfftz_api.c:66-82);
 * execute_io lets the first concurrent caller use the plan's scratch and gives
 * the others their own (api/aoclfftz_api.c:88-135) -- here a stream-ordered
 * device allocation instead of a host slab.
 */
#include <cuda_runtime_api.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "aoclfftz_gpu.h"
#include "fz_internal.h"

static __thread char g_err[512];

void fz_set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

static int g_log_mode = 0;
static __thread aoclfftz_gpu_hints_t g_hints;

aoclfftz_error_type aoclfftz_gpu_set_hints(const aoclfftz_gpu_hints_t *hints)
{
    if (hints)
        g_hints = *hints;
    else
        memset(&g_hints, 0, sizeof(g_hints));
    return AOCLFFTZ_SUCCESS;
}

void fz_log(const fz_plan *pl, const char *fmt, ...)
{
    int mode = pl ? pl->log_mode : g_log_mode;
    if (mode < AOCLFFTZ_LOG_INFO) return;
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "[aoclfftz-gpu] ");
    vfprintf(stderr, fmt, ap);
    fprintf(stderr, "\n");
    va_end(ap);
}

const FFTZ_CHAR *aoclfftz_gpu_last_error(FFTZ_VOID) { return g_err; }

int64_t fz_inj_tma_short = 0, fz_inj_ragged_wait = 0, fz_inj_ragged_dep = 0, fz_inj_alloc_fail = 0;

int fz_dev_malloc(void **p, size_t bytes)
{
    if (__atomic_load_n(&fz_inj_alloc_fail, __ATOMIC_ACQUIRE) > 0 &&
        __atomic_sub_fetch(&fz_inj_alloc_fail, 1, __ATOMIC_ACQ_REL) >= 0)
    {
        *p = NULL;
        return -1;
    }
    if (cudaMalloc(p, bytes) != cudaSuccess)
    {
        cudaGetLastError();
        *p = NULL;
        return -1;
    }
    return 0;
}

static int device_usable(const void *p);

aoclfftz_error_type aoclfftz_gpu_transpose(FFTZ_INT32 dtype, FFTZ_INT32 is_real, const FFTZ_VOID *in, FFTZ_VOID *out,
                                           FFTZ_INT64 rows, FFTZ_INT64 cols, FFTZ_INT64 row_is, FFTZ_INT64 col_is,
                                           FFTZ_INT64 row_os, FFTZ_INT64 col_os, FFTZ_VOID *stream)
{
    if (dtype != 0 && dtype != 1)
    {
        fz_set_error("transpose: dtype must be 0 (float) or 1 (double)");
        return AOCLFFTZ_INVALID_INPUT;
    }
    if (is_real != 0 && is_real != 1)
    {
        fz_set_error("transpose: is_real must be 0 (complex) or 1 (real)");
        return AOCLFFTZ_INVALID_INPUT;
    }
    if (rows < 1 || cols < 1 || row_is < 1 || col_is < 1 || row_os < 1 || col_os < 1)
    {
        fz_set_error("transpose: sizes and strides must be positive");
        return AOCLFFTZ_INVALID_INPUT;
    }
    if (!in || !out)
    {
        fz_set_error("transpose: in and out cannot be NULL");
        return AOCLFFTZ_INVALID_INPUT;
    }
    /* the largest element index on each side, and the element count, must
     * fit 63 bits (checked without overflowing) */
    if ((cols - 1) > INT64_MAX / col_is || (cols - 1) > INT64_MAX / col_os ||
        (rows - 1) > (INT64_MAX - (cols - 1) * col_is) / row_is ||
        (rows - 1) > (INT64_MAX - (cols - 1) * col_os) / row_os || rows > INT64_MAX / 16 / cols)
    {
        fz_set_error("transpose: the strides address beyond 2^63 elements");
        return AOCLFFTZ_INVALID_INPUT;
    }
    if (!device_usable(in) || !device_usable(out))
    {
        fz_set_error("transpose: in and out must be device memory");
        return AOCLFFTZ_INVALID_INPUT;
    }
    const int eb = (dtype == 0 ? 4 : 8) * (is_real ? 1 : 2);
    cudaStream_t st = (cudaStream_t)stream;
    int e;
    if (in != out)
        e = fftz_launch_transpose(in, out, rows, cols, row_is, col_is, row_os, col_os, eb, st);
    else if (rows == cols && row_os == col_is && col_os == row_is)
        e = fftz_launch_transpose_square_inplace(out, rows, row_is, col_is, eb, st);
    else
    {
        /* any other in-place layout: copy the input to a dense temporary, then
         * transpose from there */
        void *tmp = NULL;
        if (cudaMallocAsync(&tmp, (size_t)(rows * cols * eb), st) != cudaSuccess)
        {
            cudaGetLastError();
            fz_set_error("transpose: temporary of %lld bytes could not be allocated", (long long)(rows * cols * eb));
            return AOCLFFTZ_MEMORY_FAILURE;
        }
        e = fftz_launch_transpose(in, tmp, rows, cols, row_is, col_is, cols, 1, eb, st);
        if (!e) e = fftz_launch_transpose(tmp, out, rows, cols, cols, 1, row_os, col_os, eb, st);
        cudaFreeAsync(tmp, st);
    }
    if (e)
    {
        fz_set_error("transpose launch failed: %s", cudaGetErrorString((cudaError_t)e));
        cudaGetLastError();
        return AOCLFFTZ_EXECUTION_FAILURE;
    }
    return AOCLFFTZ_SUCCESS;
}

FFTZ_INT32 aoclfftz_gpu_inject_fault(FFTZ_INT32 kind, FFTZ_INT64 value)
{
    if (value < 0) return -1;
    switch (kind)
    {
    case AOCLFFTZ_GPU_FAULT_NONE:
        fz_inj_tma_short = fz_inj_ragged_wait = fz_inj_ragged_dep = fz_inj_alloc_fail = 0;
        return 0;
    case AOCLFFTZ_GPU_FAULT_TMA_SHORT:
        if (value > (1 << 20)) return -1;
        fz_inj_tma_short = value;
        return 0;
    case AOCLFFTZ_GPU_FAULT_RAGGED_WAIT: fz_inj_ragged_wait = value; return 0;
    case AOCLFFTZ_GPU_FAULT_RAGGED_DEP: fz_inj_ragged_dep = value; return 0;
    case AOCLFFTZ_GPU_FAULT_ALLOC: __atomic_store_n(&fz_inj_alloc_fail, value, __ATOMIC_RELEASE); return 0;
    }
    return -1;
}

/* ------------------------------------------------------------- validation */

typedef struct
{
    void *in, *out;
    int vec_rank, dim_rank;
    fz_dim dims[16], vecs[16];
    aoclfftz_flags_t *flags;
    aoclfftz_cntrl_params_t *cp;
    aoclfftz_smp_pfft_t *pt;
} fz_desc;

#define FZ_FAIL(...)                                                                                                   \
    do                                                                                                                 \
    {                                                                                                                  \
        fz_set_error(__VA_ARGS__);                                                                                     \
        if (d->cp && d->cp->logger_mode >= AOCLFFTZ_LOG_INFO) fprintf(stderr, "[aoclfftz-gpu] %s\n", g_err);         \
        return AOCLFFTZ_INVALID_INPUT;                                                                                 \
    } while (0)

/* the reference's VALIDATE_PROBLEM_DESCRIPTOR (api/validate_problem.h:346-414)
 * and its helpers (:24-344), same checks in the same order */
static int validate(fz_desc *d)
{
    aoclfftz_flags_t *f = d->flags;
    aoclfftz_cntrl_params_t *cp = d->cp;
    if (cp->logger_mode < 0 || cp->logger_mode > 3) cp->logger_mode = AOCLFFTZ_LOG_NONE;
    if (cp->measure_stats != 0) cp->measure_stats = 0;
    if (!cp->opt_off && (cp->opt_level < 0 || cp->opt_level > 3)) cp->opt_level = 3;
    if (f->fft_type > 1) FZ_FAIL("fft_type can be Complex(0) or Real(1)");
    if (f->fft_direction > 1) FZ_FAIL("fft_direction can be Forward(0) or Backward(1)");
    if (f->storage_order) FZ_FAIL("out-of-order outputs are not supported");
    if (f->fft_placement > 1) FZ_FAIL("fft_placement can be In-place(0) or Out-of-place(1)");
    if (f->transpose_mode) FZ_FAIL("standalone transpose is not supported");
    if (f->bit_reproducibility > 1) FZ_FAIL("bit_reproducibility can be Disable(0) or Enable(1)");
    if (!f->fft_placement)
    {
        if (d->in != d->out) FZ_FAIL("input and output buffer must be the same for in-place problems");
        if (!f->fft_type)
        {
            for (int i = 0; i < d->dim_rank; i++)
                if (d->dims[i].is != d->dims[i].os) FZ_FAIL("dimension[%d]: in_stride != out_stride", i);
            for (int i = 0; i < d->vec_rank; i++)
                if (d->vecs[i].is != d->vecs[i].os) FZ_FAIL("vecs[%d]: in_stride != out_stride", i);
        }
        else
        {
            int64_t in_scale = f->fft_direction == 0 ? 2 : 1;
            int64_t out_scale = f->fft_direction == 1 ? 2 : 1;
            for (int i = 0; i < d->dim_rank; i++)
                if (d->dims[i].is * out_scale != d->dims[i].os * in_scale)
                {
                    if (i == 0 && d->dims[i].is == d->dims[i].os) continue;
                    FZ_FAIL("dimension[%d]: real in-place strides must differ by a factor of 2", i);
                }
            for (int i = 0; i < d->vec_rank; i++)
                if (d->vecs[i].is * out_scale != d->vecs[i].os * in_scale && !(i == 0 && d->vecs[i].n == 1))
                    FZ_FAIL("vecs[%d]: real in-place strides must differ by a factor of 2", i);
        }
    }
    else if (d->in == d->out)
        FZ_FAIL("input and output buffer cannot be the same for out-of-place problems");
    if (d->pt->dynamic_load_model != 0 && d->pt->dynamic_load_model != 1) d->pt->dynamic_load_model = 1;
    return AOCLFFTZ_SUCCESS;
}

/* ---------------------------------------------------------------- setup */

static int64_t span_elems(const fz_dim *dims, int rank, const fz_dim *vecs, int vrank, int use_out, int64_t n0)
{
    int64_t s = 1;
    for (int i = 0; i < rank; i++)
    {
        int64_t n = (i == 0 && n0 > 0) ? n0 : dims[i].n;
        s += (n - 1) * (use_out ? dims[i].os : dims[i].is);
    }
    for (int i = 0; i < vrank; i++)
        if (vecs[i].n > 0) s += (vecs[i].n - 1) * (use_out ? vecs[i].os : vecs[i].is);
    return s;
}

void fz_plan_free(fz_plan *pl)
{
    if (!pl) return;
    if (pl->rg) fz_ragged_free(pl->rg);
    if (pl->dtab) cudaFree(pl->dtab);
    if (pl->scratch) cudaFree(pl->scratch);
    if (pl->stage) cudaFree(pl->stage);
    if (pl->prof_ev)
    {
        for (int i = 0; i < 2 * pl->prof_cap * pl->npass; i++)
            if (pl->prof_ev[i]) cudaEventDestroy((cudaEvent_t)pl->prof_ev[i]);
        free(pl->prof_ev);
    }
    if (pl->chunk) fz_plan_free(pl->chunk);
    for (int i = 0; i < 3; i++)
        if (pl->pipe_stream[i]) cudaStreamDestroy((cudaStream_t)pl->pipe_stream[i]);
    if (pl->pipe_buf) cudaFree(pl->pipe_buf);
    free(pl->pass);
    free(pl->blob.p);
    pl->magic = 0;
    free(pl);
}

static void *setup_impl(fz_desc *d, int dtype)
{
    fz_plan *pl = NULL;
    g_err[0] = 0;
    if (validate(d) != AOCLFFTZ_SUCCESS) return NULL;
    g_log_mode = d->cp->logger_mode;
    pl = (fz_plan *)calloc(1, sizeof(fz_plan));
    if (!pl)
    {
        fz_set_error("out of host memory");
        return NULL;
    }
    pl->magic = FZ_MAGIC;
    pl->dtype = dtype;
    pl->fft_type = d->flags->fft_type;
    pl->direction = d->flags->fft_direction;
    pl->placement = d->flags->fft_placement;
    pl->log_mode = d->cp->logger_mode;
    pl->setup_in = d->in;
    pl->setup_out = d->out;
    pl->stream = NULL;
    pl->hints = g_hints;
    if (cudaGetDevice(&pl->device) != cudaSuccess)
    {
        fz_set_error("no CUDA device available");
        fz_plan_free(pl);
        return NULL;
    }
    const int64_t esz = dtype == 0 ? 4 : 8;
    const int64_t n0 = d->dims[0].n;
    if (pl->fft_type == 0)
    {
        pl->in_bytes = span_elems(d->dims, d->dim_rank, d->vecs, d->vec_rank, 0, 0) * 2 * esz;
        pl->out_bytes = span_elems(d->dims, d->dim_rank, d->vecs, d->vec_rank, 1, 0) * 2 * esz;
    }
    else if (pl->direction == 0)
    {
        pl->in_bytes = span_elems(d->dims, d->dim_rank, d->vecs, d->vec_rank, 0, 0) * esz;
        pl->out_bytes = span_elems(d->dims, d->dim_rank, d->vecs, d->vec_rank, 1, n0 / 2 + 1) * 2 * esz;
    }
    else
    {
        pl->in_bytes = span_elems(d->dims, d->dim_rank, d->vecs, d->vec_rank, 0, n0 / 2 + 1) * 2 * esz;
        pl->out_bytes = span_elems(d->dims, d->dim_rank, d->vecs, d->vec_rank, 1, 0) * esz;
    }
    pl->sv_rank = d->dim_rank;
    pl->sv_vrank = d->vec_rank;
    memcpy(pl->sv_dims, d->dims, sizeof(fz_dim) * (size_t)d->dim_rank);
    memcpy(pl->sv_vecs, d->vecs, sizeof(fz_dim) * (size_t)d->vec_rank);
    if (fz_plan_build(pl, d->dim_rank, d->dims, d->vec_rank, d->vecs))
    {
        fz_log(pl, "setup failed: %s", g_err);
        fz_plan_free(pl);
        return NULL;
    }
    /* device tables: one allocation, then every pass's pointers */
    if (pl->blob.len)
    {
        if (fz_dev_malloc(&pl->dtab, pl->blob.len) ||
            cudaMemcpy(pl->dtab, pl->blob.p, pl->blob.len, cudaMemcpyHostToDevice) != cudaSuccess)
        {
            cudaGetLastError();
            fz_set_error("device allocation of %zu table bytes failed", pl->blob.len);
            fz_plan_free(pl);
            return NULL;
        }
    }
    for (int i = 0; i < pl->npass; i++)
    {
        fz_pass *p = &pl->pass[i];
        unsigned char *base = (unsigned char *)pl->dtab;
        p->k.tw = p->off_tw >= 0 ? base + p->off_tw : NULL;
        p->k.tw4_hi = p->off_tw4hi >= 0 ? base + p->off_tw4hi : NULL;
        p->k.tw4_lo = p->off_tw4lo >= 0 ? base + p->off_tw4lo : NULL;
        p->k.pre_tab = p->off_pre >= 0 ? base + p->off_pre : NULL;
        p->k.post_tab = p->off_post >= 0 ? base + p->off_post : NULL;
        p->k.mid_tab = p->off_mid >= 0 ? base + p->off_mid : NULL;
        p->k.rtw = p->off_rtw >= 0 ? base + p->off_rtw : NULL;
        if (p->is_elem) p->e.tab = p->off_rtw >= 0 ? base + p->off_rtw : NULL;
    }
    pl->nlaunch = pl->npass;
    const int64_t csz = 2 * esz;
    pl->scratch_bytes = 0;
    for (int i = 0; i < pl->nscratch; i++)
        pl->scratch_bytes += (pl->scratch_elems[i] * csz + 255) & ~(int64_t)255;
    if (pl->scratch_bytes > 0 && fz_dev_malloc(&pl->scratch, (size_t)pl->scratch_bytes))
    {
        cudaGetLastError();
        fz_set_error("device allocation of %lld scratch bytes failed", (long long)pl->scratch_bytes);
        fz_plan_free(pl);
        return NULL;
    }
    if (pl->log_mode >= AOCLFFTZ_LOG_INFO)
    {
        char buf[1024];
        aoclfftz_gpu_describe(pl, buf, sizeof(buf));
        fz_log(pl, "plan: %s", buf);
    }
    return pl;
}

#define FILL_DESC(problem)                                                                                             \
    fz_desc d;                                                                                                         \
    memset(&d, 0, sizeof(d));                                                                                          \
    if (!(problem))                                                                                                    \
    {                                                                                                                  \
        fz_set_error("problem descriptor is NULL");                                                                    \
        return NULL;                                                                                                   \
    }                                                                                                                  \
    d.in = (problem)->in;                                                                                              \
    d.out = (problem)->out;                                                                                            \
    d.vec_rank = (problem)->vec_rank;                                                                                  \
    d.dim_rank = (problem)->dim_rank;                                                                                  \
    d.flags = &(problem)->flags;                                                                                       \
    d.cp = &(problem)->cntrl_params;                                                                                   \
    d.pt = &(problem)->pthr_fft;                                                                                       \
    if (d.dim_rank <= 0)                                                                                               \
    {                                                                                                                  \
        fz_set_error("dim rank must be at least 1");                                                                   \
        return NULL;                                                                                                   \
    }                                                                                                                  \
    if (d.vec_rank <= 0)                                                                                               \
    {                                                                                                                  \
        fz_set_error("vec rank must be at least 1");                                                                   \
        return NULL;                                                                                                   \
    }                                                                                                                  \
    if (d.dim_rank > 16 || d.vec_rank > 16)                                                                            \
    {                                                                                                                  \
        fz_set_error("ranks above 16 are not supported");                                                             \
        return NULL;                                                                                                   \
    }                                                                                                                  \
    if (!(problem)->dims)                                                                                              \
    {                                                                                                                  \
        fz_set_error("dims cannot be NULL");                                                                           \
        return NULL;                                                                                                   \
    }                                                                                                                  \
    for (int i_ = 0; i_ < d.dim_rank; i_++)                                                                            \
    {                                                                                                                  \
        d.dims[i_].n = (problem)->dims[i_].n;                                                                          \
        d.dims[i_].is = (problem)->dims[i_].in_stride;                                                                 \
        d.dims[i_].os = (problem)->dims[i_].out_stride;                                                                \
        if (d.dims[i_].n <= 0 || d.dims[i_].is <= 0 || d.dims[i_].os <= 0)                                             \
        {                                                                                                              \
            fz_set_error("dimension[%d]: size and strides must be positive", i_);                                     \
            return NULL;                                                                                               \
        }                                                                                                              \
    }                                                                                                                  \
    if (!(problem)->vecs)                                                                                              \
    {                                                                                                                  \
        fz_set_error("vecs cannot be NULL");                                                                           \
        return NULL;                                                                                                   \
    }                                                                                                                  \
    for (int i_ = 0; i_ < d.vec_rank; i_++)                                                                            \
    {                                                                                                                  \
        d.vecs[i_].n = (problem)->vecs[i_].n;                                                                          \
        d.vecs[i_].is = (problem)->vecs[i_].in_stride;                                                                 \
        d.vecs[i_].os = (problem)->vecs[i_].out_stride;                                                                \
        if (d.vecs[i_].n < 0 || d.vecs[i_].is <= 0 || d.vecs[i_].os <= 0)                                              \
        {                                                                                                              \
            fz_set_error("vector[%d]: size must be >= 0 and strides positive", i_);                                   \
            return NULL;                                                                                               \
        }                                                                                                              \
    }

FFTZ_VOID *aoclfftz_setup_f(aoclfftz_prob_desc_f *problem)
{
    FILL_DESC(problem)
    return setup_impl(&d, 0);
}

FFTZ_VOID *aoclfftz_setup_d(aoclfftz_prob_desc_d *problem)
{
    FILL_DESC(problem)
    return setup_impl(&d, 1);
}

FFTZ_VOID *aoclfftz_setup_f_64_(aoclfftz_prob_desc_f_64_ *problem)
{
    FILL_DESC(problem)
    return setup_impl(&d, 0);
}

FFTZ_VOID *aoclfftz_setup_d_64_(aoclfftz_prob_desc_d_64_ *problem)
{
    FILL_DESC(problem)
    return setup_impl(&d, 1);
}

/* -------------------------------------------------------------- execute */

static fz_plan *as_plan(void *h)
{
    fz_plan *pl = (fz_plan *)h;
    if (!pl || pl->magic != FZ_MAGIC) return NULL;
    return pl;
}

/* 1 if the GPU can use the pointer directly (device or managed memory) */
static int device_usable(const void *p)
{
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static void *setup_impl(fz_desc *d, int dtype);

static int is_pinned(const void *p)
{
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeHost;
}

/* Builds the chunk plan: the same descriptor with the outermost batch
 * dimension cut to chunk_c entries (a divisor of its length), so that
 * consecutive chunks are contiguous byte ranges on both sides. */
static int prepare_chunks(fz_plan *pl)
{
    pl->chunk_state = -1;
    if (pl->sv_vrank < 1 || pl->nop) return -1;
    int o = 0;
    for (int i = 1; i < pl->sv_vrank; i++)
        if (pl->sv_vecs[i].is > pl->sv_vecs[o].is) o = i;
    const fz_dim outer = pl->sv_vecs[o];
    if (outer.n < 2) return -1;
    /* everything below the outer dimension must fit inside one outer stride on
     * both sides, so that chunks are disjoint byte ranges */
    int64_t span_in = 1, span_out = 1;
    for (int i = 0; i < pl->sv_rank; i++)
    {
        span_in += (pl->sv_dims[i].n - 1) * pl->sv_dims[i].is;
        span_out += (pl->sv_dims[i].n - 1) * pl->sv_dims[i].os;
    }
    for (int i = 0; i < pl->sv_vrank; i++)
        if (i != o && pl->sv_vecs[i].n > 0)
        {
            span_in += (pl->sv_vecs[i].n - 1) * pl->sv_vecs[i].is;
            span_out += (pl->sv_vecs[i].n - 1) * pl->sv_vecs[i].os;
        }
    if (span_in > outer.is || span_out > outer.os) return -1;
    /* about 8 chunks of at least 4 MiB each */
    const int64_t per_entry = pl->in_bytes / outer.n + 1;
    int64_t target = outer.n / 8;
    if (target < 1) target = 1;
    while (target > 1 && target * per_entry < (4 << 20) && target * 2 <= outer.n / 2) target *= 2;
    int64_t c = target;
    while (c > 1 && outer.n % c) c--;
    if (outer.n / c < 2) return -1;
    fz_desc d;
    memset(&d, 0, sizeof(d));
    aoclfftz_flags_t f;
    memset(&f, 0, sizeof(f));
    f.fft_type = (FFTZ_UINT8)pl->fft_type;
    f.fft_direction = (FFTZ_UINT8)pl->direction;
    f.fft_placement = (FFTZ_UINT8)pl->placement;
    aoclfftz_cntrl_params_t cp;
    memset(&cp, 0, sizeof(cp));
    cp.opt_level = 3;
    aoclfftz_smp_pfft_t pt = {1, 1};
    d.flags = &f;
    d.cp = &cp;
    d.pt = &pt;
    d.dim_rank = pl->sv_rank;
    d.vec_rank = pl->sv_vrank;
    memcpy(d.dims, pl->sv_dims, sizeof(fz_dim) * (size_t)pl->sv_rank);
    memcpy(d.vecs, pl->sv_vecs, sizeof(fz_dim) * (size_t)pl->sv_vrank);
    d.vecs[o].n = c;
    /* placeholder device-side addresses with the right placement */
    d.in = (void *)(uintptr_t)0x1000;
    d.out = pl->placement == 0 ? d.in : (void *)(uintptr_t)0x2000;
    aoclfftz_gpu_hints_t saved = g_hints;
    g_hints = pl->hints;
    fz_plan *ch = (fz_plan *)setup_impl(&d, pl->dtype);
    g_hints = saved;
    if (!ch) return -1;
    ch->stream = NULL;
    /* the chunk plan's passes run on the slot buffers below, not on its own scratch */
    if (ch->scratch) cudaFree(ch->scratch);
    ch->scratch = NULL;
    const int64_t esz_in = (pl->fft_type == 0 || pl->direction == 1) ? (pl->dtype == 0 ? 8 : 16) : (pl->dtype == 0 ? 4 : 8);
    const int64_t esz_out = (pl->fft_type == 0 || pl->direction == 0) ? (pl->dtype == 0 ? 8 : 16) : (pl->dtype == 0 ? 4 : 8);
    pl->chunk = ch;
    pl->chunk_c = c;
    pl->chunk_count = outer.n / c;
    pl->chunk_in_step = c * outer.is * esz_in;
    pl->chunk_out_step = c * outer.os * esz_out;
    pl->pipe_in_bytes = (ch->in_bytes + 255) & ~(int64_t)255;
    pl->pipe_out_bytes = pl->placement == 0 ? 0 : (ch->out_bytes + 255) & ~(int64_t)255;
    if (pl->placement == 0 && ch->out_bytes > ch->in_bytes) pl->pipe_in_bytes = (ch->out_bytes + 255) & ~(int64_t)255;
    pl->pipe_slot_bytes = pl->pipe_in_bytes + pl->pipe_out_bytes + ((ch->scratch_bytes + 255) & ~(int64_t)255);
    if (fz_dev_malloc(&pl->pipe_buf, (size_t)(3 * pl->pipe_slot_bytes)))
    {
        cudaGetLastError();
        return -1;
    }
    for (int i = 0; i < 3; i++)
        if (cudaStreamCreateWithFlags((cudaStream_t *)&pl->pipe_stream[i], cudaStreamNonBlocking) != cudaSuccess)
            return -1;
    pl->chunk_state = 1;
    return 0;
}

/* Launches the passes of plan `ch` with the given buffer bases on stream st. */
/* The blocked four-step intermediate needs its column pass on the split
 * kernel, which needs a 16-byte aligned input: for an execute whose column
 * pass input is not aligned, both passes keep the plain layout. */
static int blk4_usable(const fz_plan *pl, void *const *buf)
{
    for (int i = 0; i < pl->npass; i++)
        if (!pl->pass[i].is_elem && (pl->pass[i].k.flags & FFTZ_F_BLK4_OUT) &&
            (((uintptr_t)buf[pl->pass[i].src] + (uintptr_t)pl->pass[i].in_off) & 15) != 0)
            return 0;
    return 1;
}

static int launch_passes(fz_plan *ch, void *in, void *out, void *scratch, cudaStream_t st)
{
    void *buf[FZ_NBUF];
    buf[FZ_BUF_IN] = in;
    buf[FZ_BUF_OUT] = out;
    int64_t off = 0;
    for (int i = 0; i < ch->nscratch; i++)
    {
        buf[FZ_BUF_SCR0 + i] = (unsigned char *)scratch + off;
        off += (ch->scratch_elems[i] * 2 * (ch->dtype == 0 ? 4 : 8) + 255) & ~(int64_t)255;
    }
    const int blk = blk4_usable(ch, buf);
    for (int i = 0; i < ch->npass; i++)
    {
        int e;
        if (ch->pass[i].is_elem)
        {
            fftz_elem_t el = ch->pass[i].e;
            el.in = (const unsigned char *)buf[ch->pass[i].src] + ch->pass[i].in_off;
            el.out = (unsigned char *)buf[ch->pass[i].dst] + ch->pass[i].out_off;
            e = fftz_launch_elem(&el, st);
        }
        else
        {
            fftz_pass_t k = ch->pass[i].k;
            k.in = (const unsigned char *)buf[ch->pass[i].src] + ch->pass[i].in_off;
            k.out = (unsigned char *)buf[ch->pass[i].dst] + ch->pass[i].out_off;
            if (!blk) k.flags &= ~(FFTZ_F_BLK4_IN | FFTZ_F_BLK4_OUT);
            e = fftz_launch_pass(&k, st);
        }
        if (e) return e;
    }
    return 0;
}

/* Host buffers in page-locked memory: chunk i is copied in on slot i % 3's
 * stream, transformed, and copied out, so copy-in of one chunk, the passes
 * of the next and copy-out of the previous overlap. */
static aoclfftz_error_type run_pipelined(fz_plan *pl, void *in, void *out)
{
    cudaStream_t ps = (cudaStream_t)pl->stream;
    cudaEvent_t ready;
    if (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess) return AOCLFFTZ_EXECUTION_FAILURE;
    cudaEventRecord(ready, ps); /* work already queued on the plan's stream comes first */
    int err = 0;
    for (int i = 0; i < 3; i++) cudaStreamWaitEvent((cudaStream_t)pl->pipe_stream[i], ready, 0);
    for (int64_t c = 0; c < pl->chunk_count && !err; c++)
    {
        const int slot = (int)(c % 3);
        cudaStream_t st = (cudaStream_t)pl->pipe_stream[slot];
        unsigned char *sb = (unsigned char *)pl->pipe_buf + slot * pl->pipe_slot_bytes;
        unsigned char *din = sb, *dout = pl->placement == 0 ? sb : sb + pl->pipe_in_bytes;
        unsigned char *scr = sb + pl->pipe_in_bytes + pl->pipe_out_bytes;
        err |= cudaMemcpyAsync(din, (unsigned char *)in + c * pl->chunk_in_step, (size_t)pl->chunk->in_bytes,
                               cudaMemcpyHostToDevice, st) != cudaSuccess;
        err |= launch_passes(pl->chunk, din, dout, scr, st) != 0;
        err |= cudaMemcpyAsync((unsigned char *)out + c * pl->chunk_out_step, dout, (size_t)pl->chunk->out_bytes,
                               cudaMemcpyDeviceToHost, st) != cudaSuccess;
    }
    for (int i = 0; i < 3; i++)
        if (cudaStreamSynchronize((cudaStream_t)pl->pipe_stream[i]) != cudaSuccess) err = 1;
    cudaEventDestroy(ready);
    if (err)
    {
        fz_set_error("pipelined host execution failed: %s", cudaGetErrorString(cudaGetLastError()));
        return AOCLFFTZ_EXECUTION_FAILURE;
    }
    return AOCLFFTZ_SUCCESS;
}

static aoclfftz_error_type run_on_device(fz_plan *pl, void *in, void *out);

/* Executes on the plan's device and restores the caller's current device. */
static aoclfftz_error_type run(fz_plan *pl, void *in, void *out)
{
    if (pl->nop) return AOCLFFTZ_SUCCESS;
    int cur = -1;
    cudaGetDevice(&cur);
    const int sw = cur != pl->device;
    if (sw) cudaSetDevice(pl->device);
    aoclfftz_error_type r = run_on_device(pl, in, out);
    if (sw && cur >= 0) cudaSetDevice(cur);
    return r;
}

static aoclfftz_error_type run_on_device(fz_plan *pl, void *in, void *out)
{
    cudaStream_t st = (cudaStream_t)pl->stream;
    const int in_dev = device_usable(in);
    const int out_dev = device_usable(out);
    const int inplace = (in == out);
    if (!in_dev && !out_dev && !pl->prof_ev && is_pinned(in) && is_pinned(out))
    {
        /* one pipelined execute at a time per plan (the staging slots are shared) */
        int expect = 0;
        if (__atomic_compare_exchange_n(&pl->scratch_busy, &expect, 1, 0, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE))
        {
            if (pl->chunk_state == 0) prepare_chunks(pl);
            aoclfftz_error_type r = AOCLFFTZ_SUCCESS;
            int used = pl->chunk_state == 1;
            if (used) r = run_pipelined(pl, in, out);
            __atomic_store_n(&pl->scratch_busy, 0, __ATOMIC_RELEASE);
            if (used) return r;
        }
    }
    /* ownership of the plan's scratch and staging memory */
    int expected = 0;
    const int owner = __atomic_compare_exchange_n(&pl->scratch_busy, &expected, 1, 0, __ATOMIC_ACQ_REL,
                                                  __ATOMIC_ACQUIRE);
    void *scratch = NULL, *stage = NULL;
    int64_t stage_need = 0;
    if (!in_dev || !out_dev)
    {
        int64_t a = (pl->in_bytes + 255) & ~(int64_t)255;
        stage_need = inplace ? (pl->in_bytes > pl->out_bytes ? pl->in_bytes : pl->out_bytes) : a + pl->out_bytes;
    }
    aoclfftz_error_type ret = AOCLFFTZ_SUCCESS;
    if (owner)
    {
        scratch = pl->scratch;
        if (stage_need > pl->stage_bytes)
        {
            if (pl->stage) cudaFree(pl->stage);
            pl->stage = NULL;
            pl->stage_bytes = 0;
            if (fz_dev_malloc(&pl->stage, (size_t)stage_need))
            {
                cudaGetLastError();
                fz_set_error("staging allocation of %lld bytes failed", (long long)stage_need);
                __atomic_store_n(&pl->scratch_busy, 0, __ATOMIC_RELEASE);
                return AOCLFFTZ_MEMORY_FAILURE;
            }
            pl->stage_bytes = stage_need;
        }
        stage = pl->stage;
    }
    else
    {
        if (pl->scratch_bytes > 0 && cudaMallocAsync(&scratch, (size_t)pl->scratch_bytes, st) != cudaSuccess)
        {
            cudaGetLastError();
            fz_set_error("per-call scratch allocation failed");
            return AOCLFFTZ_MEMORY_FAILURE;
        }
        if (stage_need > 0 && cudaMallocAsync(&stage, (size_t)stage_need, st) != cudaSuccess)
        {
            cudaGetLastError();
            if (scratch) cudaFreeAsync(scratch, st);
            fz_set_error("per-call staging allocation failed");
            return AOCLFFTZ_MEMORY_FAILURE;
        }
    }
    void *buf[FZ_NBUF];
    buf[FZ_BUF_IN] = in;
    buf[FZ_BUF_OUT] = out;
    if (!in_dev || !out_dev)
    {
        unsigned char *sb = (unsigned char *)stage;
        void *din = in_dev ? in : (void *)sb;
        void *dout = out_dev ? out : (inplace ? (void *)sb : (void *)(sb + ((pl->in_bytes + 255) & ~(int64_t)255)));
        if (!in_dev && cudaMemcpyAsync(din, in, (size_t)pl->in_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
            ret = AOCLFFTZ_EXECUTION_FAILURE;
        buf[FZ_BUF_IN] = din;
        buf[FZ_BUF_OUT] = dout;
    }
    {
        int64_t off = 0;
        for (int i = 0; i < pl->nscratch; i++)
        {
            buf[FZ_BUF_SCR0 + i] = scratch ? (void *)((unsigned char *)scratch + off) : NULL;
            off += (pl->scratch_elems[i] * 2 * (pl->dtype == 0 ? 4 : 8) + 255) & ~(int64_t)255;
        }
    }
    const int blk = blk4_usable(pl, buf);
    for (int i = 0; i < pl->npass && ret == AOCLFFTZ_SUCCESS; i++)
    {
        cudaEvent_t *ev = NULL;
        if (pl->prof_ev && pl->prof_n < pl->prof_cap)
        {
            ev = (cudaEvent_t *)&pl->prof_ev[2 * (pl->prof_n * pl->npass + i)];
            cudaEventRecord(ev[0], st);
        }
        int e;
        if (pl->pass[i].is_elem)
        {
            fftz_elem_t el = pl->pass[i].e;
            el.in = (const unsigned char *)buf[pl->pass[i].src] + pl->pass[i].in_off;
            el.out = (unsigned char *)buf[pl->pass[i].dst] + pl->pass[i].out_off;
            e = fftz_launch_elem(&el, st);
        }
        else
        {
            fftz_pass_t k = pl->pass[i].k;
            k.in = (const unsigned char *)buf[pl->pass[i].src] + pl->pass[i].in_off;
            k.out = (unsigned char *)buf[pl->pass[i].dst] + pl->pass[i].out_off;
            k.test_tx_short = (int32_t)fz_inj_tma_short;
            if (!blk) k.flags &= ~(FFTZ_F_BLK4_IN | FFTZ_F_BLK4_OUT);
            e = fftz_launch_pass(&k, st);
        }
        if (ev) cudaEventRecord(ev[1], st);
        if (e != 0)
        {
            fz_set_error("launch of pass %d (%s) failed: %s", i, pl->pass[i].what, cudaGetErrorString((cudaError_t)e));
            ret = AOCLFFTZ_EXECUTION_FAILURE;
        }
    }
    if (pl->prof_ev && pl->prof_n < pl->prof_cap) pl->prof_n++;
    if (ret == AOCLFFTZ_SUCCESS && !out_dev)
    {
        if (cudaMemcpyAsync(out, buf[FZ_BUF_OUT], (size_t)pl->out_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            ret = AOCLFFTZ_EXECUTION_FAILURE;
    }
    if (!owner)
    {
        if (scratch) cudaFreeAsync(scratch, st);
        if (stage) cudaFreeAsync(stage, st);
    }
    if (!in_dev || !out_dev || !owner)
    {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
        {
            fz_set_error("execution failed: %s", cudaGetErrorString(e));
            ret = AOCLFFTZ_EXECUTION_FAILURE;
        }
    }
    if (owner) __atomic_store_n(&pl->scratch_busy, 0, __ATOMIC_RELEASE);
    return ret;
}

aoclfftz_error_type aoclfftz_execute(FFTZ_VOID *handle)
{
    fz_plan *pl = as_plan(handle);
    if (!pl) return AOCLFFTZ_EXECUTION_FAILURE;
    if (!pl->setup_in || !pl->setup_out)
    {
        fz_set_error("one or both setup-time buffers are NULL; use aoclfftz_execute_io");
        return AOCLFFTZ_EXECUTION_FAILURE;
    }
    return run(pl, pl->setup_in, pl->setup_out);
}

aoclfftz_error_type aoclfftz_execute_io(FFTZ_VOID *handle, FFTZ_VOID *in, FFTZ_VOID *out)
{
    fz_plan *pl = as_plan(handle);
    if (!pl || !in || !out) return AOCLFFTZ_EXECUTION_FAILURE;
    if ((pl->placement == 0) != (in == out))
    {
        fz_set_error("buffers do not match the plan's placement");
        return AOCLFFTZ_EXECUTION_FAILURE;
    }
    return run(pl, in, out);
}

FFTZ_VOID aoclfftz_destroy(FFTZ_VOID *handle)
{
    fz_plan *pl = as_plan(handle);
    if (!pl) return;
    if (pl->stream) cudaStreamSynchronize((cudaStream_t)pl->stream);
    else cudaDeviceSynchronize();
    fz_plan_free(pl);
}

const FFTZ_CHAR *aoclfftz_version(FFTZ_VOID) { return AOCLFFTZ_LIBRARY_VERSION " B200 (sm_100a)"; }

/* ------------------------------------------------------- GPU extensions */

aoclfftz_error_type aoclfftz_gpu_set_stream(FFTZ_VOID *handle, FFTZ_VOID *stream)
{
    fz_plan *pl = as_plan(handle);
    if (!pl) return AOCLFFTZ_INVALID_INPUT;
    pl->stream = stream;
    return AOCLFFTZ_SUCCESS;
}

FFTZ_VOID *aoclfftz_gpu_get_stream(FFTZ_VOID *handle)
{
    fz_plan *pl = as_plan(handle);
    return pl ? pl->stream : NULL;
}

aoclfftz_error_type aoclfftz_gpu_synchronize(FFTZ_VOID *handle)
{
    fz_plan *pl = as_plan(handle);
    if (!pl) return AOCLFFTZ_INVALID_INPUT;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)pl->stream);
    if (e != cudaSuccess)
    {
        fz_set_error("%s", cudaGetErrorString(e));
        return AOCLFFTZ_EXECUTION_FAILURE;
    }
    for (int i = 0; i < pl->npass; i++)
        if (!pl->pass[i].is_elem && pl->pass[i].k.variant == FFTZ_VAR_TC)
        {
            if (fftz_tc_wait_failed())
            {
                fz_set_error("a tensor-core pass gave up waiting for its MMAs (results invalid)");
                return AOCLFFTZ_EXECUTION_FAILURE;
            }
            break;
        }
    for (int i = 0; i < pl->npass; i++)
        if (!pl->pass[i].is_elem && pl->pass[i].k.use_tma)
        {
            if (fftz_tma_wait_failed())
            {
                fz_set_error("a TMA-fed pass gave up waiting for its tile copies (its results, and those of "
                             "later work on the same stream, are invalid)");
                return AOCLFFTZ_EXECUTION_FAILURE;
            }
            break;
        }
    if (pl->rg && pl->rg->d_err)
    {
        int flag = 0;
        if (cudaMemcpy(&flag, pl->rg->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess || flag)
        {
            /* reported once: later runs on the handle start with a clear flag */
            if (flag) cudaMemset(pl->rg->d_err, 0, sizeof(int));
            fz_set_error("ragged executor: a dependency wait gave up (results invalid)");
            return AOCLFFTZ_EXECUTION_FAILURE;
        }
    }
    return AOCLFFTZ_SUCCESS;
}

FFTZ_INT32 aoclfftz_gpu_num_launches(FFTZ_VOID *handle)
{
    fz_plan *pl = as_plan(handle);
    if (!pl) return -1;
    if (pl->rg) return 1;
    return pl->nop ? 0 : pl->nlaunch;
}

FFTZ_INT32 aoclfftz_gpu_describe(FFTZ_VOID *handle, FFTZ_CHAR *buf, FFTZ_INT32 len)
{
    fz_plan *pl = as_plan(handle);
    if (!pl || !buf || len <= 0) return -1;
    int w = snprintf(buf, (size_t)len, "%s %s %s %s:", pl->dtype ? "f64" : "f32", pl->fft_type ? "real" : "c2c",
                     pl->direction ? "bwd" : "fwd", pl->placement ? "oop" : "inplace");
    if (pl->nop && w < len) w += snprintf(buf + w, (size_t)(len - w), " empty batch");
    if (pl->rg && w < len) w += snprintf(buf + w, (size_t)(len - w), " %s", pl->rg->summary);
    for (int i = 0; i < pl->npass && w < len; i++)
        w += pl->pass[i].is_elem ? snprintf(buf + w, (size_t)(len - w), " [%s]", pl->pass[i].what)
                                  : snprintf(buf + w, (size_t)(len - w), " [%s tpc=%d tpt=%d%s]", pl->pass[i].what,
                                             pl->pass[i].k.tpc, pl->pass[i].k.tpt,
                                             (pl->pass[i].k.flags & (FFTZ_F_BLK4_IN | FFTZ_F_BLK4_OUT)) ? " blk4 tma-split"
                                             : pl->pass[i].k.use_tma == 7 ? " tma-stream"
                                             : pl->pass[i].k.use_tma == 6 ? " tma-split3"
                                             : pl->pass[i].k.use_tma == 5 ? " tma-split2"
                                             : pl->pass[i].k.use_tma == 4 ? " tma-split"
                                             : pl->pass[i].k.use_tma == 3 ? " tma-prefetch"
                                             : pl->pass[i].k.use_tma == 2 ? " tma-half-prefetch"
                                             : pl->pass[i].k.use_tma      ? " tma"
                                                                          : "");
    return w < len ? w : len - 1;
}

FFTZ_INT64 aoclfftz_gpu_device_bytes(FFTZ_VOID *handle)
{
    fz_plan *pl = as_plan(handle);
    if (!pl) return -1;
    return (FFTZ_INT64)pl->blob.len + pl->scratch_bytes + pl->stage_bytes;
}

aoclfftz_error_type aoclfftz_gpu_profile_begin(FFTZ_VOID *handle, FFTZ_INT32 max_executes)
{
    fz_plan *pl = as_plan(handle);
    if (!pl || max_executes <= 0) return AOCLFFTZ_INVALID_INPUT;
    if (pl->prof_ev)
    {
        for (int i = 0; i < 2 * pl->prof_cap * pl->npass; i++)
            if (pl->prof_ev[i]) cudaEventDestroy((cudaEvent_t)pl->prof_ev[i]);
        free(pl->prof_ev);
        pl->prof_ev = NULL;
    }
    int n = 2 * max_executes * pl->npass;
    pl->prof_ev = (void **)calloc((size_t)(n > 0 ? n : 1), sizeof(void *));
    if (!pl->prof_ev) return AOCLFFTZ_MEMORY_FAILURE;
    for (int i = 0; i < n; i++)
        if (cudaEventCreate((cudaEvent_t *)&pl->prof_ev[i]) != cudaSuccess)
        {
            cudaGetLastError();
            return AOCLFFTZ_MEMORY_FAILURE;
        }
    pl->prof_cap = max_executes;
    pl->prof_n = 0;
    return AOCLFFTZ_SUCCESS;
}

FFTZ_INT32 aoclfftz_gpu_profile_end(FFTZ_VOID *handle, float *ms_per_pass, FFTZ_INT32 max_passes)
{
    fz_plan *pl = as_plan(handle);
    if (!pl || !pl->prof_ev) return -1;
    cudaStreamSynchronize((cudaStream_t)pl->stream);
    for (int i = 0; i < pl->npass && i < max_passes; i++)
    {
        float tot = 0.f;
        for (int r = 0; r < pl->prof_n; r++)
        {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, (cudaEvent_t)pl->prof_ev[2 * (r * pl->npass + i)],
                                 (cudaEvent_t)pl->prof_ev[2 * (r * pl->npass + i) + 1]);
            tot += ms;
        }
        ms_per_pass[i] = tot;
    }
    int n = pl->prof_n;
    for (int i = 0; i < 2 * pl->prof_cap * pl->npass; i++) cudaEventDestroy((cudaEvent_t)pl->prof_ev[i]);
    free(pl->prof_ev);
    pl->prof_ev = NULL;
    pl->prof_cap = pl->prof_n = 0;
    return n;
}

FFTZ_INT32 aoclfftz_gpu_pass_info(FFTZ_VOID *handle, FFTZ_INT32 i, FFTZ_CHAR *buf, FFTZ_INT32 len,
                                  FFTZ_INT64 *elems_in, FFTZ_INT64 *elems_out)
{
    fz_plan *pl = as_plan(handle);
    if (!pl || i < 0 || i >= pl->npass) return -1;
    const fftz_pass_t *k = &pl->pass[i].k;
    if (buf && len > 0) snprintf(buf, (size_t)len, "%s", pl->pass[i].what);
    if (pl->pass[i].is_elem)
    {
        if (elems_in) *elems_in = pl->pass[i].e.nlines * pl->pass[i].e.nout;
        if (elems_out) *elems_out = pl->pass[i].e.nlines * pl->pass[i].e.nout;
        return pl->npass;
    }
    if (elems_in) *elems_in = k->ntf * (int64_t)(k->pre_n > 0 ? k->pre_n : k->nload);
    if (elems_out) *elems_out = k->ntf * (int64_t)(k->post_n > 0 ? k->post_n : k->nstore);
    return pl->npass;
}
