/* aoclfftz_gpu.h -- GPU-only extensions of the aoclfftz.h ABI.
 *
 * Nothing here exists in the reference library (which is CPU-only); these calls
 * expose what a GPU caller needs on top of the drop-in ABI: the CUDA stream a
 * plan runs on, synchronisation, plan introspection and the error state of
 * the last call. Plans created through aoclfftz.h work with every function
 * here; passing anything else returns AOCLFFTZ_INVALID_INPUT.
 */
#ifndef AOCLFFTZ_GPU_H
#define AOCLFFTZ_GPU_H

#include "aoclfftz.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Runs the plan's launches on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) instead of the plan's own stream. */
aoclfftz_error_type aoclfftz_gpu_set_stream(FFTZ_VOID *handle, FFTZ_VOID *stream);
FFTZ_VOID *aoclfftz_gpu_get_stream(FFTZ_VOID *handle);

/* Waits until all work enqueued on the plan's stream has finished; reports
 * any asynchronous CUDA error as AOCLFFTZ_EXECUTION_FAILURE. */
aoclfftz_error_type aoclfftz_gpu_synchronize(FFTZ_VOID *handle);

/* Number of kernel launches one execute enqueues (device buffers). */
FFTZ_INT32 aoclfftz_gpu_num_launches(FFTZ_VOID *handle);

/* Writes a one-line human-readable description of the plan (algorithm per
 * pass, lengths, batch, kernel family) into buf; returns the length. */
FFTZ_INT32 aoclfftz_gpu_describe(FFTZ_VOID *handle, FFTZ_CHAR *buf, FFTZ_INT32 len);

/* Device bytes the plan owns (tables, scratch, staging). */
FFTZ_INT64 aoclfftz_gpu_device_bytes(FFTZ_VOID *handle);

/* Per-pass timing with CUDA events recorded around every launch on the plan's
 * stream (no synchronisation between executes). profile_begin arms it for up
 * to max_executes executes; profile_end synchronises the stream, writes the
 * summed milliseconds of each pass into ms_per_pass and returns the number of
 * executes recorded. */
aoclfftz_error_type aoclfftz_gpu_profile_begin(FFTZ_VOID *handle, FFTZ_INT32 max_executes);
FFTZ_INT32 aoclfftz_gpu_profile_end(FFTZ_VOID *handle, float *ms_per_pass, FFTZ_INT32 max_passes);

/* Pass i of the plan: description, complex (or real-pair) elements read and
 * written per launch. Returns the number of passes, -1 on a bad index. */
FFTZ_INT32 aoclfftz_gpu_pass_info(FFTZ_VOID *handle, FFTZ_INT32 i, FFTZ_CHAR *buf, FFTZ_INT32 len,
                                  FFTZ_INT64 *elems_in, FFTZ_INT64 *elems_out);

/* Planner hints for the next aoclfftz_setup_* calls made by this thread
 * (the autotuner's knobs). Zero in a field means "planner's choice".
 *   fourstep_n1   column length n1 of a four-step split n = n1 * n2
 *   tpc_col       transforms per CTA for passes with column-mapped lanes
 *   tpc_row       transforms per CTA for row passes
 *   batch_chunk   multi-pass plans run their passes on chunks of this many
 *                 lines at a time (keeps the intermediate resident in L2)
 *   algorithm     1 one pass, 2 four-step, 3 Bluestein (0 = choose)
 *   kernel_family 1 one tile per CTA, loads by the threads; 2 persistent
 *                 double-buffered; 3 generic kernel only; 5 one tile per CTA
 *                 fetched by TMA copies wherever the pass qualifies
 *                 (0 = choose: TMA copies for column passes); 6 persistent CTAs,
 *                 half of the next tile prefetched by TMA; 7 4096-point float
 *                 row passes as tensor-core GEMM stages (three-term BF16
 *                 operands, FP32 accuracy); 8 every
 *                 4096-point float pass as persistent CTAs that keep the tile
 *                 in registers and prefetch the whole next tile by TMA; 9
 *                 every 4096-point float pass as 16 x 256 split tiles
 *                 (persistent, one exchange across the CTA per tile; 0 =
 *                 choose takes them for such passes with a column lane map);
 *                 10 / 11 the split tiles with a full-complex exchange and a
 *                 shared-memory / tensor-memory stash; 12 the in-place
 *                 runtime-radix kernel instead of the ping-pong tiles; 13
 *                 row passes of contiguous lines as persistent streaming
 *                 tiles (whole lines by bulk copies, next tile in flight)
 *   twiddles      where the stage twiddles are read from (see the field)
 * aoclfftz_gpu_set_hints(NULL) restores the defaults. */
typedef struct aoclfftz_gpu_hints
{
    FFTZ_INT64 fourstep_n1;
    FFTZ_INT32 tpc_col;
    FFTZ_INT32 tpc_row;
    FFTZ_INT64 batch_chunk;
    FFTZ_INT32 algorithm;
    FFTZ_INT32 kernel_family;
    FFTZ_INT32 twiddles;        /* 1 stage twiddles read from global memory, 2 from a
                                   shared-memory copy (compile-time passes >= 512 points) */
    FFTZ_INT32 reserved[5];
} aoclfftz_gpu_hints_t;

aoclfftz_error_type aoclfftz_gpu_set_hints(const aoclfftz_gpu_hints_t *hints);

/* Ragged batches: `count` independent 1-D c2c transforms of different lengths
 * (any length: powers of two, smooth composites, primes via Bluestein) in one
 * persistent kernel launch, captured once in a CUDA graph. dtype 0 = float,
 * 1 = double; direction 0 = forward, 1 = backward. Transform i reads sizes[i]
 * contiguous complex elements at in + in_offsets[i] and writes out +
 * out_offsets[i] (offsets in complex elements; NULL = packed back to back).
 * Execute takes device buffers (out of place); the handle is released with
 * aoclfftz_destroy and works with aoclfftz_gpu_set_stream / _synchronize
 * (which also reports a failed dependency wait). */
FFTZ_VOID *aoclfftz_gpu_ragged_setup(FFTZ_INT32 dtype, FFTZ_INT32 direction, FFTZ_INT64 count,
                                     const FFTZ_INT64 *sizes, const FFTZ_INT64 *in_offsets,
                                     const FFTZ_INT64 *out_offsets);
aoclfftz_error_type aoclfftz_gpu_ragged_execute(FFTZ_VOID *handle, FFTZ_VOID *in, FFTZ_VOID *out);

/* Learned plan selector: an MLP F -> 64 -> 64 -> 1 (ReLU) predicting the log
 * time of a candidate plan from its features, trained and evaluated by the
 * library's own CUDA kernels on device buffers. params holds W1[F][64], b1,
 * W2[64][64], b2, w3[64], b3 (float32). forward needs 2*B*64 floats of work,
 * grad 4*B*64 + 2*B; grad writes d(mean squared error)/d(params) and the loss
 * (a device float). adam performs one Adam step (step counts from 1). */
FFTZ_INT32 aoclfftz_gpu_mlp_nparams(FFTZ_INT32 features);
FFTZ_INT32 aoclfftz_gpu_mlp_forward(const float *params, FFTZ_INT32 features, const float *x, FFTZ_INT32 batch,
                                    float *y, float *work, FFTZ_VOID *stream);
FFTZ_INT32 aoclfftz_gpu_mlp_grad(const float *params, FFTZ_INT32 features, const float *x, const float *target,
                                 FFTZ_INT32 batch, float *grads, float *loss, float *work, FFTZ_VOID *stream);
FFTZ_INT32 aoclfftz_gpu_mlp_adam(float *params, const float *grads, float *m, float *v, FFTZ_INT32 n, float lr,
                                 FFTZ_INT32 step, FFTZ_VOID *stream);

/* Text of the last error recorded by this thread (empty if none). */
const FFTZ_CHAR *aoclfftz_gpu_last_error(FFTZ_VOID);

/* Fault injection for failure-path tests (no reference counterpart: the
 * reference's own tests have none). Process-wide; value 0 switches a kind
 * off, kind AOCLFFTZ_GPU_FAULT_NONE switches every kind off. Nothing here
 * makes the GPU fault or hang: every injected failure ends in a bounded wait
 * or a refused allocation that the host reports.
 *   TMA_SHORT   the TMA-fed kernels' tiles wait for `value` bytes more than
 *               their copies deliver (<= 2^20): each tile's bounded wait runs
 *               out, execute / synchronize report AOCLFFTZ_EXECUTION_FAILURE.
 *               A real wait that runs out may leave copies in flight that land
 *               later: that pass's results and those of later work on the
 *               same stream are invalid.
 *   RAGGED_WAIT dependency waits of ragged executors captured from now on
 *               give up after `value` polls (about 100 ns each).
 *   RAGGED_DEP  ragged plans set up from now on wait for `value` more tiles
 *               than the first dependency has (that wait cannot complete).
 *   ALLOC       the next `value` device allocations of setup / execute fail
 *               (setup returns NULL, execute AOCLFFTZ_MEMORY_FAILURE).
 * Returns 0, or -1 for an unknown kind or value. */
enum
{
    AOCLFFTZ_GPU_FAULT_NONE = 0,
    AOCLFFTZ_GPU_FAULT_TMA_SHORT = 1,
    AOCLFFTZ_GPU_FAULT_RAGGED_WAIT = 2,
    AOCLFFTZ_GPU_FAULT_RAGGED_DEP = 3,
    AOCLFFTZ_GPU_FAULT_ALLOC = 4
};
FFTZ_INT32 aoclfftz_gpu_inject_fault(FFTZ_INT32 kind, FFTZ_INT64 value);

/* No-allocation execute. No counterpart in the reference, which never needs
 * device memory. For callers that may not allocate device memory when they
 * transform: another allocator owns the device's memory, or a latency-critical
 * loop cannot afford cudaFree's device-wide synchronisation. Runs howmany
 * contiguous single-precision complex transforms of length n (distance n)
 * from device buffer `in` to device buffer `out` (in == out allowed), forward
 * (direction 0) or unnormalised backward (1), on `stream`, with the plan
 * path's four-step kernels and their intermediate in a 32 MiB static device
 * array. n must be a power of two in [2^15, 2^22] and n * howmany at most
 * 2^22; anything else returns AOCLFFTZ_INVALID_INPUT with a message in
 * aoclfftz_gpu_last_error. Calls no cudaMalloc, cudaFree or other allocating
 * routine. The first call on each device sets up that device's tables and
 * waits for them on `stream`; make it before any stream capture begins
 * (during capture it returns AOCLFFTZ_SETUP_FAILURE). All calls on a device
 * share the one scratch array: calls whose kernels overlap on the GPU race,
 * so order them on one stream. */
aoclfftz_error_type aoclfftz_gpu_execute_noalloc_c2c_f(const FFTZ_VOID *in, FFTZ_VOID *out, FFTZ_INT64 n,
                                                       FFTZ_INT64 howmany, FFTZ_INT32 direction,
                                                       FFTZ_VOID *stream);

/* Standalone transpose: the problem of the reference's transpose solver
 * (core/solvers/transpose_solver.c:97-141), which the reference's public API
 * does not reach (api/aoclfftz.h:97-99: transpose_mode must be 0, and
 * aoclfftz_setup_* here rejects it the same way). Element (r, c) of a
 * rows x cols array, r < rows, c < cols, is read at in[r * row_is + c * col_is]
 * and written at out[r * row_os + c * col_os] (strides in elements, positive);
 * a plain transpose of a dense row-major array is row_is = cols, col_is = 1,
 * row_os = 1, col_os = rows. Elements are complex (is_real 0) or real
 * (is_real 1), float (dtype 0) or double (dtype 1), moved bit-exactly. in and
 * out are device memory that does not overlap unless in == out; in == out
 * is allowed (a square in-place transpose
 * swaps tiles in place, any other in-place layout goes through a temporary
 * device buffer, stream-ordered). Enqueued on `stream` (NULL: the legacy
 * default stream). Returns AOCLFFTZ_SUCCESS, AOCLFFTZ_INVALID_INPUT (with the
 * reason in aoclfftz_gpu_last_error), AOCLFFTZ_MEMORY_FAILURE or
 * AOCLFFTZ_EXECUTION_FAILURE. */
aoclfftz_error_type aoclfftz_gpu_transpose(FFTZ_INT32 dtype, FFTZ_INT32 is_real, const FFTZ_VOID *in, FFTZ_VOID *out,
                                           FFTZ_INT64 rows, FFTZ_INT64 cols, FFTZ_INT64 row_is, FFTZ_INT64 col_is,
                                           FFTZ_INT64 row_os, FFTZ_INT64 col_os, FFTZ_VOID *stream);

#ifdef __cplusplus
}
#endif

#endif /* AOCLFFTZ_GPU_H */
