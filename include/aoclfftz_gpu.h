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

/* Text of the last error recorded by this thread (empty if none). */
const FFTZ_CHAR *aoclfftz_gpu_last_error(FFTZ_VOID);

#ifdef __cplusplus
}
#endif

#endif /* AOCLFFTZ_GPU_H */
