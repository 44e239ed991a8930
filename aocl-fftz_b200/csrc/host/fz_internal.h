/* Internal plan structures of the B200 FFT library (C99 host layer).
 *
 * A plan is a flat list of kernel passes (fftz_pass_t, see
 * ../kernels/fftz_kernels.h) over four logical buffers: the caller's input,
 * the caller's output and two plan-owned scratch arrays. The reference keeps a
 * linked tree of solver nodes walked at execute time
 * (api/aoclfftz_internal.h:797-805, core/executor.c:17-44); on the GPU the
 * tree is flattened at setup into this pass list, so execute is a loop of
 * kernel launches with no host-side recursion.
 */
#ifndef FZ_INTERNAL_H
#define FZ_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "../kernels/fftz_kernels.h"
#include "aoclfftz.h"
#include "aoclfftz_gpu.h"

#define FZ_MAGIC 0x475a4646u /* "FFZG" */

/* fault injection for the failure-path tests (aoclfftz_gpu_inject_fault):
 * process-wide, read by setup and execute */
extern int64_t fz_inj_tma_short;   /* extra bytes each TMA tile waits for */
extern int64_t fz_inj_ragged_wait; /* ragged dependency-wait limit (spins), 0 = default */
extern int64_t fz_inj_ragged_dep;  /* raise the first dependent item's count at ragged setup */
extern int64_t fz_inj_alloc_fail;  /* fail this many of the next device allocations */

/* cudaMalloc, or a failure while an injected allocation failure is pending */
int fz_dev_malloc(void **p, size_t bytes);

/* shared memory a ragged executor tile may use (its CTAs run several per SM) */
int64_t fz_ragged_smem_cap(int dtype);

/* logical buffers: the caller's in / out, then plan-owned scratch arrays,
 * one per use (four-step intermediates, Bluestein work arrays, the
 * half-complex work array of an out-of-place multi-dimensional c2r, dense
 * lines of a multi-pass real line) */
enum { FZ_BUF_IN = 0, FZ_BUF_OUT = 1, FZ_BUF_SCR0 = 2 };
#define FZ_MAX_SCRATCH 16
#define FZ_NBUF (FZ_BUF_SCR0 + FZ_MAX_SCRATCH)

/* one tensor dimension, strides in elements of the side's type */
typedef struct
{
    int64_t n, is, os;
} fz_dim;

typedef struct
{
    int is_elem; /* 0: FFT pass (k), 1: elementwise pass (e) */
    fftz_elem_t e;
    fftz_pass_t k;
    int src, dst;
    int64_t in_off, out_off; /* byte offsets added to the src / dst base pointers */
    /* byte offsets of the pass's tables in the plan's table blob (-1: none) */
    int64_t off_tw, off_tw4hi, off_tw4lo, off_pre, off_post, off_mid, off_rtw;
    char what[64];
} fz_pass;

/* growable host byte buffer holding every table of a plan before upload */
typedef struct
{
    unsigned char *p;
    size_t len, cap;
} fz_blob;

/* ragged batch state (ragged.c): one persistent launch over all tiles */
typedef struct fz_ragged
{
    int64_t count, npasses, nitems;
    int64_t in_elems, out_elems; /* complex elements the buffers span */
    void *d_passes, *d_items, *d_done, *d_queue, *d_err;
    void *d_ind;                  /* per-transform element offsets of grouped passes */
    int64_t ngroups;
    int grid, smem;
    void *cap_stream;             /* stream used to capture the graph */
    void *graph, *graph_exec;     /* cudaGraph_t / cudaGraphExec_t */
    int64_t g_spin;               /* dependency-wait limit the graph was captured with */
    const void *g_in;             /* buffers the graph was captured with */
    void *g_out;
    char summary[224];
} fz_ragged;

typedef struct fz_plan
{
    uint32_t magic;
    int dtype;     /* 0 float, 1 double */
    int fft_type;  /* 0 complex, 1 real */
    int direction; /* 0 forward, 1 backward */
    int placement; /* 0 in-place, 1 out-of-place */
    int log_mode;
    int nop;       /* empty batch: execute succeeds without work */
    void *setup_in, *setup_out;
    int64_t in_bytes, out_bytes; /* bytes spanned by the input / output buffers */
    int npass, cap;
    fz_pass *pass;
    fz_blob blob;
    int64_t scratch_elems[FZ_MAX_SCRATCH]; /* complex elements of each scratch array */
    int nscratch;
    int depth; /* planner recursion depth (hints apply at depth 0) */
    /* device state */
    int device;
    void *dtab;
    void *scratch; /* all scratch arrays in one allocation */
    int64_t scratch_bytes;
    void *stage; /* staging buffer for host-memory callers (in, then out) */
    int64_t stage_bytes;
    void *stream; /* cudaStream_t; NULL = legacy default stream */
    int scratch_busy; /* 1 while an execute holds the plan's scratch */
    int nlaunch;
    aoclfftz_gpu_hints_t hints;
    fz_ragged *rg; /* non-NULL for ragged-batch handles */
    /* the descriptor (for the chunk plan of pipelined host staging) */
    fz_dim sv_dims[16], sv_vecs[16];
    int sv_rank, sv_vrank;
    /* pipelined host staging: chunks of the outermost batch dimension run
     * copy-in / passes / copy-out on FZ_PIPE_SLOTS streams */
    struct fz_plan *chunk;   /* plan of one chunk (built at the first pinned-host execute) */
    int64_t chunk_c, chunk_count, chunk_in_step, chunk_out_step; /* entries, chunks, bytes */
    int chunk_state;         /* 0 not tried, 1 ready, -1 not chunkable */
    void *pipe_stream[3];
    void *pipe_buf;          /* per slot: staging in, staging out, scratch */
    int64_t pipe_slot_bytes, pipe_in_bytes, pipe_out_bytes;
    /* per-pass event timing: prof_cap executes x npass x {start, end} */
    void **prof_ev;
    int prof_cap, prof_n;
} fz_plan;

/* ---- logging / errors (api.c) ---- */
void fz_set_error(const char *fmt, ...);
void fz_log(const fz_plan *pl, const char *fmt, ...);

/* ---- tables (tables.c) ---- */
int64_t fz_blob_add(fz_blob *b, const void *data, size_t bytes);
int64_t fz_blob_reserve(fz_blob *b, size_t bytes);
/* stage twiddles for a radix list; returns blob offset, fills tw_off[] */
int64_t fz_stage_twiddles(fz_blob *b, int dtype, int n, int nstages, const int32_t *radix, int32_t *tw_off);
/* four-step factor tables W_N^(hi*L), W_N^lo in the working dtype */
int fz_tw4_tables(fz_blob *b, int dtype, int64_t N, int64_t *L, int64_t *off_hi, int64_t *off_lo);
/* Bluestein tables for length n, pow2 convolution length m, direction */
int fz_bluestein_tables(fz_blob *b, int dtype, int64_t n, int64_t m, int direction, int64_t *off_pre,
                        int64_t *off_post, int64_t *off_mid);
/* appends the row-major copy T'[k1 * n2 + k2] = T[k1 + n1 * k2] of the table
 * at off; returns its offset (-1 on allocation failure) */
int64_t fz_blob_permute(fz_blob *b, int dtype, int64_t off, int64_t n1, int64_t n2);
/* tables of the tensor-core 4096-point kernel (DFT-64 operand halves in BF16,
 * canonical layout, then W_4096 as float (cos, sin)); returns their offset */
int64_t fz_tc64_tables(fz_blob *b);
/* packed-real twiddles W_{2M}^k, k = 0..M (W^M = -1) */
int64_t fz_real_twiddles(fz_blob *b, int dtype, int64_t M);

/* ---- shared by api.c and ragged.c ---- */
void fz_plan_free(fz_plan *pl);
void fz_ragged_free(fz_ragged *rg);

/* ---- planner (plan.c) ---- */
int fz_plan_build(fz_plan *pl, int rank, const fz_dim *dims, int vrank, const fz_dim *vecs);

#endif
