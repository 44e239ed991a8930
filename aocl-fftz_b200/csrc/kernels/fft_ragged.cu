// Persistent DAG executor for ragged batches: transforms of different lengths
// and algorithms run in ONE launch (captured in a CUDA graph by the host).
//
// The host flattens every transform's pass list into a table of CTA tiles
// ("items"), ordered so that all tiles of pass depth d precede those of
// depth d+1. Each CTA repeatedly takes the next item with an atomic counter,
// copies the item's pass descriptor into shared memory (resolving buffer
// offsets against the launch's in / out / scratch bases), waits -- with a
// bounded spin -- until every tile of the item's predecessor pass is done,
// runs the tile with the generic shared-memory FFT code, and counts itself
// done with release semantics. Only running CTAs hold items and every
// predecessor item was taken before its successors, so the waits always end;
// the spin limit turns a broken invariant into an error flag instead of a hang.
#include "fft_generic.cuh"

namespace fftz {

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename T>
__global__ void __launch_bounds__(256) fft_ragged_kernel(const __grid_constant__ fftz_ragged_t R) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ fftz_pass_t sP;
  __shared__ long long s_item;
  __shared__ int s_ok;
  for (;;) {
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(R.queue, 1ULL);
    __syncthreads();
    const long long it = s_item;
    if (it >= R.nitems) break;
    const fftz_ritem_t item = R.items[it];
    const int *src = (const int *)(R.passes + item.pass);
    int *dst = (int *)&sP;
    for (int i = threadIdx.x; i < (int)(sizeof(fftz_pass_t) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned char *ib = (const unsigned char *)(sP.src_buf == FFTZ_RBUF_IN ? R.in
                                                        : sP.src_buf == FFTZ_RBUF_OUT ? (const void *)R.out
                                                                                      : (const void *)R.scratch);
      unsigned char *ob = (unsigned char *)(sP.dst_buf == FFTZ_RBUF_IN ? (void *)R.in
                                            : sP.dst_buf == FFTZ_RBUF_OUT ? R.out
                                                                          : R.scratch);
      sP.in = ib + (size_t)sP.in;
      sP.out = ob + (size_t)sP.out;
      s_ok = 1;
      if (item.dep >= 0) {
        long long spins = 0;
        while (ld_acquire(R.done + item.dep) < item.dep_count) {
          if (++spins > R.spin_limit) {
            atomicExch(R.err, 1);
            s_ok = 0;
            break;
          }
          __nanosleep(100);
        }
        __threadfence();
      }
    }
    __syncthreads();
    if (s_ok) generic_tile<T>(sP, item.blk, smem_raw);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(R.done + item.pass, 1);
    }
  }
}

}  // namespace fftz

extern "C" int fftz_ragged_grid(int dtype, int smem_bytes) {
  const void *fn =
      dtype == 0 ? (const void *)&fftz::fft_ragged_kernel<float> : (const void *)&fftz::fft_ragged_kernel<double>;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes > 48 * 1024 ? smem_bytes : 48 * 1024);
  int occ = 0, dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, (size_t)smem_bytes) != cudaSuccess || occ < 1) {
    cudaGetLastError();
    occ = 1;
  }
  return occ * (nsm > 0 ? nsm : 148);
}

extern "C" int fftz_launch_ragged(const fftz_ragged_t *r, int grid, void *stream) {
  const void *fn =
      r->dtype == 0 ? (const void *)&fftz::fft_ragged_kernel<float> : (const void *)&fftz::fft_ragged_kernel<double>;
  void *args[1] = {(void *)r};
  return (int)cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(256), args, (size_t)r->smem_bytes, (cudaStream_t)stream);
}
