// Persistent DAG executor for ragged batches: transforms of different lengths
// and algorithms run in ONE launch (captured in a CUDA graph by the host).
//
// The host groups the transforms by length, plans each group as one batched
// plan whose transform dimension is indirect (every transform keeps its own
// offset in the packed buffers), and flattens the passes into a table of CTA
// tiles ("items"), ordered so that all tiles of pass depth d precede those of
// depth d+1. Each CTA repeatedly takes the next item with an atomic counter,
// copies the item's pass descriptor into shared memory (resolving buffer
// offsets against the launch's in / out / scratch bases), waits -- with a
// bounded spin -- until every tile of the item's predecessor pass is done,
// runs the tile and counts itself done with release semantics. Power-of-two
// tiles run the compile-time kernels' tile code (one instantiation per length
// and feature set listed below); every other tile runs the generic code. Only
// running CTAs hold items and every predecessor item was taken before its
// successors, so the waits always end; the spin limit turns a broken
// invariant into an error flag instead of a hang.
#include "fft_fast.cuh"
#include "fft_generic.cuh"

namespace fftz {

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Tiles of the compile-time kernels inside the executor (blockDim 256 =
// tpc * tpt). Kept out of line so that each has its own register allocation
// within the kernel's bound.
template <typename T, int N, int FEAT>
__device__ __noinline__ void ragged_fast_tile(const fftz_pass_t &P, int64_t blk, unsigned char *smem) {
  fast_tile<T, N, FEAT>(P, blk * P.tpc, smem);
}

#define FZ_RG_CASE(N, FEAT)                        \
  case N:                                          \
    ragged_fast_tile<T, N, FEAT>(P, blk, smem);    \
    return true;

// Lengths and feature sets that have a compile-time tile here; the host asks
// fftz_ragged_fast_ok before it leaves a pass on a FAST variant.
template <typename T>
__device__ __forceinline__ bool ragged_fast(const fftz_pass_t &P, int64_t blk, unsigned char *smem) {
  if (P.variant == FFTZ_VAR_FAST) {
    switch (P.n) {
      FZ_RG_CASE(2, 0) FZ_RG_CASE(4, 0) FZ_RG_CASE(8, 0) FZ_RG_CASE(16, 0) FZ_RG_CASE(32, 0) FZ_RG_CASE(64, 0)
      FZ_RG_CASE(128, 0) FZ_RG_CASE(256, 0) FZ_RG_CASE(512, 0) FZ_RG_CASE(1024, 0) FZ_RG_CASE(2048, 0)
      FZ_RG_CASE(4096, 0)
    }
  } else if (P.variant == FFTZ_VAR_FAST_TW4) {
    switch (P.n) { FZ_RG_CASE(64, 1) FZ_RG_CASE(128, 1) FZ_RG_CASE(256, 1) FZ_RG_CASE(512, 1) }
  } else if (P.variant == FFTZ_VAR_FAST_TABS) {
    switch (P.n) { FZ_RG_CASE(64, 2) FZ_RG_CASE(128, 2) FZ_RG_CASE(256, 2) FZ_RG_CASE(512, 2) }
  } else if (P.variant == FFTZ_VAR_FAST_TW4_TABS) {
    switch (P.n) { FZ_RG_CASE(128, 3) FZ_RG_CASE(256, 3) FZ_RG_CASE(512, 3) }
  } else if (P.variant == FFTZ_VAR_FAST_BLUE) {
    switch (P.n) {
      FZ_RG_CASE(4, 6) FZ_RG_CASE(8, 6) FZ_RG_CASE(16, 6) FZ_RG_CASE(32, 6) FZ_RG_CASE(64, 6) FZ_RG_CASE(128, 6)
      FZ_RG_CASE(256, 6) FZ_RG_CASE(512, 6) FZ_RG_CASE(1024, 6) FZ_RG_CASE(2048, 6) FZ_RG_CASE(4096, 6)
    }
  }
  return false;
}
#undef FZ_RG_CASE

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 5 : 2) fft_ragged_kernel(const __grid_constant__ fftz_ragged_t R) {
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
    // tiles without a compile-time form are ping-pong tiles (the host plans
    // every other pass that way)
    if (s_ok && !ragged_fast<T>(sP, item.blk, smem_raw)) generic_tile_pp<T>(sP, item.blk, smem_raw);
    __syncthreads();
    // only passes that another pass waits for publish their tiles (the fence
    // waits for the tile's stores, which nothing else needs to do)
    if (item.signal && threadIdx.x == 0) {
      __threadfence();
      atomicAdd(R.done + item.pass, 1);
    }
  }
}

}  // namespace fftz

extern "C" int fftz_ragged_fast_ok(int n, int variant) {
  const bool p2 = n >= 2 && n <= 4096 && (n & (n - 1)) == 0;
  if (variant == FFTZ_VAR_FAST) return p2;
  if (variant == FFTZ_VAR_FAST_TW4) return p2 && n >= 64 && n <= 512;
  if (variant == FFTZ_VAR_FAST_TABS) return p2 && n >= 64 && n <= 512;
  if (variant == FFTZ_VAR_FAST_TW4_TABS) return p2 && n >= 128 && n <= 512;
  if (variant == FFTZ_VAR_FAST_BLUE) return p2 && n >= 4;
  return 0;
}

extern "C" int fftz_ragged_grid(int dtype, int smem_bytes) {
  const void *fn =
      dtype == 0 ? (const void *)&fftz::fft_ragged_kernel<float> : (const void *)&fftz::fft_ragged_kernel<double>;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes > 48 * 1024 ? smem_bytes : 48 * 1024);
  // all of the unified L1 / shared array as shared memory: several CTAs per SM
  cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
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
