/* Thin C-ABI between the C99 host layer and the sm_100a CUDA kernels.
 *
 * The host planner describes every kernel launch as one plain-old-data
 * fftz_pass_t (no C++ or CUDA types), and calls fftz_launch_pass() with a raw
 * stream handle. All device pointers are plain void pointers.
 *
 * One pass = one launch of the shared-memory FFT kernel: a batch of ntf
 * transforms of length n, each held whole in shared memory by one CTA
 * (tf_per_cta transforms per CTA), computed as a sequence of Stockham
 * radix stages in registers with shared-memory exchanges, with optional fused
 * prologue (conjugation, chirp / real-pair / Hermitian loads) and epilogue
 * (four-step twiddle, conjugation, table product, scale, Hermitian
 * recombination, real stores).
 */
#ifndef FFTZ_KERNELS_H
#define FFTZ_KERNELS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFTZ_MAX_STAGES 12
#define FFTZ_MAX_BDIMS 8

/* element kinds of the load phase */
enum fftz_in_kind {
    FFTZ_IN_COMPLEX = 0,   /* complex element e at in + base + e*ies           */
    FFTZ_IN_REAL_PAIRS,    /* (x[2e], x[2e+1]) of a real row, real stride ies   */
    FFTZ_IN_REAL,          /* (x[e], 0), real stride ies                        */
    FFTZ_IN_HERM_FULL,     /* e <= n/2 ? X[e] : conj(X[n-e]), complex stride ies */
    FFTZ_IN_HERM_SEPARATE  /* packed c2r: 2Z[k] from X[k], X[M-k]; k < M        */
};

/* element kinds of the store phase */
enum fftz_out_kind {
    FFTZ_OUT_COMPLEX = 0,  /* complex element k at out + base + k*oes           */
    FFTZ_OUT_REAL_PAIRS,   /* (out[2k], out[2k+1]) = (re, im), real stride oes   */
    FFTZ_OUT_REAL,         /* out[k] = re, real stride oes                      */
    FFTZ_OUT_HALF,         /* first n/2+1 bins of a complex result              */
    FFTZ_OUT_HALF_RECOMBINE /* packed r2c: X[k], k <= M, from Z[k], Z[M-k]      */
};

/* kernel families */
#define FFTZ_VAR_GENERIC 0 /* runtime radix list, any element kind, <= 256 threads   */
#define FFTZ_VAR_FAST    1 /* compile-time power-of-two shape, complex in/out fused  */
#define FFTZ_VAR_FAST_TW4 2 /* as FAST with the four-step twiddle epilogue          */
#define FFTZ_VAR_FAST_TABS 3 /* as FAST with load/store tables, bounds and scale     */
#define FFTZ_VAR_FAST_TW4_TABS 4 /* both of the above                               */
#define FFTZ_VAR_FAST_BLUE 5 /* tables plus two sweeps around a mid-table product   */
#define FFTZ_VAR_PIPE 6      /* persistent, cp.async double-buffered, complex in/out */
#define FFTZ_VAR_PIPE_TW4 7  /* as PIPE with the four-step twiddle epilogue         */
#define FFTZ_VAR_TC 8        /* 4096-point rows as two radix-64 tensor-core GEMM stages */
#define FFTZ_VAR_FAST_REAL 9 /* packed real line: generic load/store phases, compile-time stages */
#define FFTZ_VAR_GENERIC_PP 10 /* runtime radix list over two shared-memory buffers, 256 threads */

/* pass flags */
#define FFTZ_F_CONJ_IN    0x01 /* conjugate each loaded value (after kind decode) */
#define FFTZ_F_CONJ_OUT   0x02 /* conjugate each stored value (after TW4)         */
#define FFTZ_F_TW4        0x04 /* multiply output k of column c by W_{tw4_n}^{c*k}  */
#define FFTZ_F_PRE_TAB    0x08 /* multiply loaded value e by pre_tab[e*pre_es + col*pre_cs] */
#define FFTZ_F_POST_TAB   0x10 /* multiply stored value k by post_tab[k*post_es + col*post_cs] */
#define FFTZ_F_SCALE      0x20 /* multiply stored value by scale                  */
#define FFTZ_F_MID_TAB    0x40 /* two sweeps: between them v = conj(v) * mid_tab[e] */
/* 4 x 4 blocked intermediate of a 4096 x 4096 four-step (split kernels only):
 * element k of column c at (k / 4) * 4 * ncols + 4 * c + k % 4 past the line */
#define FFTZ_F_BLK4_OUT   0x80  /* the pass writes its output blocked */
#define FFTZ_F_BLK4_IN    0x100 /* the pass reads its input blocked (rows = k) */

typedef struct fftz_pass
{
    /* transform held in shared memory */
    int32_t n;                          /* length of the in-SMEM complex transform */
    int32_t nstages;
    int32_t radix[FFTZ_MAX_STAGES];
    int32_t tw_off[FFTZ_MAX_STAGES];    /* stage twiddle block offsets (complex) */
    int32_t tpt;                        /* threads per transform */
    int32_t tpc;                        /* transforms per CTA */
    int32_t sstride;                    /* SMEM complex slots between transforms */
    int32_t nload;                      /* load-phase element count per transform */
    int32_t nstore;                     /* store-phase element count per transform */
    int32_t in_kind, out_kind;
    int32_t in_mode, out_mode;          /* 0: lanes along elements, 1: along transforms */
    int32_t flags;
    int32_t fuse_load, fuse_store;      /* stage 0 reads global / last stage writes global */
    int32_t variant;                    /* FFTZ_VAR_*: which kernel family runs the pass */
    int32_t dtype;                      /* 0 float, 1 double */
    int32_t nbdims;
    /* addressing: strides in complex elements (real elements for real kinds) */
    int64_t ies, oes;
    int64_t ntf;                        /* number of transforms */
    int64_t bdim[FFTZ_MAX_BDIMS];       /* batch dims, bdim[0] fastest; col = index in bdim[0] */
    int64_t ibs[FFTZ_MAX_BDIMS];
    int64_t obs[FFTZ_MAX_BDIMS];
    /* prologue / epilogue parameters */
    int64_t tw4_n, tw4_l;               /* W_{tw4_n}^r = hi[r / tw4_l] * lo[r % tw4_l] */
    int64_t pre_n, pre_es, pre_cs;      /* load bound (0: none) and table index map */
    int64_t post_n, post_es, post_cs;   /* store bound (0: none) and table index map */
    int64_t mid_cs;                     /* mid_tab index of element e of column col: e + col * mid_cs */
    double scale;
    const void *in;
    void *out;
    const void *tw;                     /* stage twiddles, working dtype */
    const void *tw4_hi, *tw4_lo;        /* four-step twiddle factors, working dtype */
    const void *pre_tab, *post_tab, *mid_tab; /* working dtype complex */
    const void *rtw;                    /* packed-real twiddles W_{2M}^k, working dtype */
    /* persistent executor only: in / out hold byte offsets into these bases */
    int32_t src_buf, dst_buf;           /* FFTZ_RBUF_* */
    /* indirect batch dimension: when ind_in (ind_out) is set, index i of batch
     * dim ind_dim contributes ind_in[i] (ind_out[i]) elements to the input
     * (output) offset instead of i * ibs (i * obs) -- transforms of one length
     * scattered through a packed ragged buffer form one batched pass */
    int32_t ind_dim;
    int32_t use_tma;                    /* fetch the tile with TMA copies when the pass qualifies: 1 one
                                           tile per CTA, 2 half-prefetch, 3 register-resident, 4-6 split
                                           tiles, 7 streaming rows */
    int32_t smem_tw;                    /* compile-time kernels: copy the stage twiddles to shared memory */
    int32_t test_tx_short;              /* fault injection (tests): TMA tiles expect this many bytes more
                                           than their copies deliver, so the bounded tile wait runs out */
    const int64_t *ind_in, *ind_out;
} fftz_pass_t;

/* Persistent DAG executor (fft_ragged.cu): one launch runs the CTA tiles of
 * many passes; a tile of a pass with a predecessor waits until every tile of
 * the predecessor has completed. */
#define FFTZ_RBUF_IN 0
#define FFTZ_RBUF_OUT 1
#define FFTZ_RBUF_SCRATCH 2

typedef struct fftz_ritem
{
    int32_t pass;      /* index into the pass table */
    int32_t dep;       /* pass that must complete first, -1 if none */
    int64_t blk;       /* CTA tile of the pass */
    int64_t dep_count; /* tiles of dep */
    int32_t signal;    /* 1 if a later pass waits for this one: count the tile done */
    int32_t pad_;
} fftz_ritem_t;

typedef struct fftz_ragged
{
    const fftz_pass_t *passes;
    const fftz_ritem_t *items;
    int64_t nitems;
    unsigned long long *queue; /* next item to take */
    int *done;                 /* completed tiles per pass */
    int *err;                  /* set when a wait gave up */
    const void *in;
    void *out;
    void *scratch;
    int64_t spin_limit;        /* polls before a wait gives up */
    int32_t dtype;
    int32_t smem_bytes;
} fftz_ragged_t;

int fftz_launch_ragged(const fftz_ragged_t *r, int grid, void *stream);
/* 1 if the executor has a compile-time tile for a pass of length n and
 * FFTZ_VAR_FAST* variant (its tpc * tpt must then be 256). */
int fftz_ragged_fast_ok(int n, int variant);
/* CTAs of the persistent executor that fit on the device at once. */
int fftz_ragged_grid(int dtype, int smem_bytes);

/* Elementwise real-transform helpers (fft_elem.cu) */
enum fftz_elem_mode {
    FFTZ_ELEM_WIDEN_REAL = 0,
    FFTZ_ELEM_WIDEN_PAIRS,
    FFTZ_ELEM_RECOMBINE,
    FFTZ_ELEM_SEPARATE,
    FFTZ_ELEM_HERM_EXPAND,
    FFTZ_ELEM_NARROW_HALF,
    FFTZ_ELEM_REAL_OUT,
    FFTZ_ELEM_PAIRS_OUT
};

typedef struct fftz_elem
{
    int32_t mode, dtype, nbdims, pad_;
    int64_t n;      /* line length parameter of the mode (n, or M for packed) */
    int64_t nout;   /* outputs per line */
    int64_t nlines;
    int64_t is, os; /* element strides on the input / output side */
    int64_t bdim[FFTZ_MAX_BDIMS], ibs[FFTZ_MAX_BDIMS], obs[FFTZ_MAX_BDIMS];
    const void *in;
    void *out;
    const void *tab; /* packed-real twiddles W_{2M}^k, k <= M */
} fftz_elem_t;

int fftz_launch_elem(const fftz_elem_t *e, void *stream);

/* Standalone transpose (fft_transpose.cu): element (r, c) of a rows x cols
 * array of elem_bytes-byte words from in[r * row_is + c * col_is] to
 * out[r * row_os + c * col_os] (in != out); the square in-place form swaps
 * (r, c) and (c, r) of data[r * row_s + c * col_s]. cudaError_t. */
int fftz_launch_transpose(const void *in, void *out, int64_t rows, int64_t cols, int64_t row_is, int64_t col_is,
                          int64_t row_os, int64_t col_os, int elem_bytes, void *stream);
int fftz_launch_transpose_square_inplace(void *data, int64_t n, int64_t row_s, int64_t col_s, int elem_bytes,
                                         void *stream);

/* Largest in-SMEM transform length (complex elements) per dtype. */
int fftz_max_smem_n(int dtype);

/* Threads per transform of the compile-time power-of-two kernels, and the
 * largest power-of-two length they cover (0 if none). */
int fftz_fast_tpt(int n);
int fftz_fast_max_n(int dtype);
/* Radix list used by the compile-time kernel for length n (returns stages). */
int fftz_fast_radices(int n, int32_t *radix);
/* compile-time packed real-line kernel for complex length 2^log2n (NULL if
 * not instantiated) */
const void *fftz_fast_real_kernel(int dtype, int log2n);
/* Threads per CTA the generic kernel may use; the persistent kernels' bound. */
int fftz_generic_max_threads(void);
int fftz_pipe_max_threads(int n);

/* Threads-per-transform needed so that no thread holds more than the
 * register budget in any stage (returns 0 if the plan is not executable). */
int fftz_threads_per_transform(int dtype, int n, int nstages, const int32_t *radix);

/* Complex entries of the stage-twiddle table of a compile-time pass of
 * length n (0 if none). */
int32_t fftz_fast_tw_entries(int n);
/* Shared memory bytes used by a pass with the given tpc/sstride. */
int64_t fftz_pass_smem_bytes(const fftz_pass_t *p);

/* Per-transform SMEM stride (complex slots) for nslots elements; with tpc
 * transforms per CTA mapped lane-wise (column maps) the stride also spreads
 * the transforms over distinct banks. */
int32_t fftz_smem_stride(int dtype, int32_t nslots);
int32_t fftz_smem_stride_cols(int dtype, int32_t nslots, int32_t tpc);

/* Maximum dynamic SMEM bytes per CTA the kernels may use. */
int64_t fftz_smem_limit(void);

/* Launches one pass on the given stream; returns a cudaError_t value. */
int fftz_launch_pass(const fftz_pass_t *p, void *stream);
/* The TMA-fed variant of a compile-time pass (fft_tma.cu): -1 when the pass
 * or its buffers do not qualify (nothing launched), else a cudaError_t. */
int fftz_launch_pass_tma(const fftz_pass_t *p, void *stream);
/* 1 if a TMA tile gave up waiting for its copies since the last call. */
int fftz_tma_wait_failed(void);
/* Tensor-core form (fft_tc.cu): shared memory per CTA, launcher, wait flag. */
int fftz_tc_smem_bytes(void);
int fftz_launch_pass_tc(const fftz_pass_t *p, void *stream);
int fftz_tc_wait_failed(void);

#ifdef __cplusplus
}
#endif
#endif
