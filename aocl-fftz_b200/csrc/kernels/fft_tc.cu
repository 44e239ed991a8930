// Tensor-core form of the 4096-point line FFT: the two radix-64 stages of
// 4096 = 64 x 64 run as GEMMs on the fifth-generation tensor cores
// (tcgen05.mma, kind::f16 with BF16 operands, FP32 accumulators in tensor
// memory), each operand split into three BF16 terms x = hi + mid + lo (24
// significant bits, as many as FP32) and the product formed from the six
// terms of order >= 2^-16 relative: A_hi B_hi + A_hi B_mid + A_mid B_hi +
// A_hi B_lo + A_lo B_hi + A_mid B_mid (the dropped terms are of order 2^-24,
// the FP32 rounding level).
//
// One CTA (256 threads, persistent) takes tiles of 2 contiguous 4096-point
// lines. With j = 64 j1 + j2 and k = k1 + 64 k2:
//   stage 1  D1[k1 re/im][(t, j2)] = sum_j1 F64[k1][j1] x_t[64 j1 + j2]
//            (M = 128 real rows, K = 128, N = 2 x 64 = 128 columns)
//   twiddle  D1 * W_4096^{j2 k1} in FP32 (factors formed in FP64 on the host)
//   stage 2  D2[k2 re/im][(t, k1)] = sum_j2 F64[k2][j2] y_t[k1][j2]
//   store    X_t[k1 + 64 k2], through shared memory so the HBM stores are
//            coalesced.
// The complex 64-point DFT is the real 128 x 128 matrix
//   [Yr; Yi] = [[C, S]; [-S, C]] [Xr; Xi], C = cos(2 pi j k / 64), S = sin(...)
// interleaved by rows (re, im of each k) and columns (re, im of each j).
//
// Accuracy: with three-term operands the stages keep FP32 accuracy (the
// tests hold this form to the FP32 path's 4 log2(N) eps bound against the
// FP64 oracle). The planner only uses it when asked (kernel_family 7): the
// transform is memory-bound (at most 7.5 flop per byte), so the tensor cores
// cannot beat the SIMT path's HBM-bound stages.
//
// Operand layout in shared memory: UMMA canonical K-major without swizzle --
// 8-row x 16-byte core matrices, consecutive along K (LBO = 128 B), 8-row
// groups SBO = 2048 B apart (K = 128 BF16 = 256 B per row).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_common.cuh"

namespace fftz {

__device__ int g_tc_wait_failed;

namespace tc {

constexpr int NT = 256;          // threads per CTA
constexpr int TPC = 2;           // lines per tile
constexpr int NCOL = TPC * 64;   // GEMM N
constexpr int A_BYTES = 128 * 256;   // 128 rows x 128 BF16
constexpr int B_BYTES = NCOL * 256;  // 128 rows x 128 BF16
constexpr int SMEM = 3 * A_BYTES + 3 * B_BYTES + 1024;

__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// byte offset of element (row, k) in a canonical K-major operand (K = 128)
__device__ __forceinline__ unsigned canon(int row, int k) {
  return (unsigned)((row >> 3) * 2048 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t sdesc(unsigned addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(2048 >> 4) << 32) |
         ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both
// K-major, M = 128, N = NCOL
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NCOL >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(IDESC), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}

__device__ __forceinline__ bool try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// v = hi + mid + lo in BF16 (each term the rounding of what the earlier ones left)
__device__ __forceinline__ void split_store(unsigned char *b, unsigned off, float v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  const float r1 = v - __bfloat162float(h);
  const __nv_bfloat16 m = __float2bfloat16_rn(r1);
  const __nv_bfloat16 l = __float2bfloat16_rn(r1 - __bfloat162float(m));
  *(unsigned short *)(b + off) = __bfloat16_as_ushort(h);
  *(unsigned short *)(b + B_BYTES + off) = __bfloat16_as_ushort(m);
  *(unsigned short *)(b + 2 * B_BYTES + off) = __bfloat16_as_ushort(l);
}

// Issues the six split products of one stage (operand terms 0 hi, 1 mid,
// 2 lo; A terms A_BYTES apart, B terms B_BYTES apart) and commits them.
__device__ __forceinline__ void stage_mma(uint32_t dtmem, unsigned a0, unsigned b0, uint64_t *bar) {
  constexpr int PA[6] = {0, 0, 1, 0, 2, 1}, PB[6] = {0, 1, 0, 2, 0, 1};
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int p = 0; p < 6; p++)
#pragma unroll
    for (int s = 0; s < 8; s++) {
      const unsigned a = a0 + PA[p] * A_BYTES + s * 256;
      const unsigned b = b0 + PB[p] * B_BYTES + s * 256;
      mma(dtmem, sdesc(a), sdesc(b), (p | s) != 0);
    }
  commit(bar);
}

// bounded wait on the MMA barrier (uniform across the CTA)
__device__ __forceinline__ bool wait_mma(uint64_t *bar, unsigned parity) {
  bool ok = false;
  for (long i = 0; i < (1L << 22); i++)
    if (try_wait(bar, parity)) {
      ok = true;
      break;
    }
  return __syncthreads_and(ok);
}

}  // namespace tc

// tabs: [A_hi | A_mid | A_lo (32 KB each, canonical) | W_4096^r as float2 (cos, sin) x 4096]
__global__ void __launch_bounds__(tc::NT, 1) fft_tc4096_kernel(const __grid_constant__ fftz_pass_t P, int64_t ntiles) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t s_taddr;
  __shared__ int64_t s_in[TPC], s_out[TPC], s_col[TPC];
  unsigned char *base = smem_raw + ((1024u - (saddr(smem_raw) & 1023u)) & 1023u);
  unsigned char *a_hi = base;                // A terms hi, mid, lo
  unsigned char *b_hi = base + 3 * A_BYTES;  // B terms hi, mid, lo
  float2 *obuf = (float2 *)b_hi;  // TPC x 4096 results (64 KB), after the stage-2 MMAs
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const unsigned char *gtab = (const unsigned char *)P.tw;
  const float2 *wtab = (const float2 *)(gtab + 3 * A_BYTES);
  // DFT-64 operand (both halves) once per CTA
  for (int i = t; i < 3 * A_BYTES / 16; i += NT) ((uint4 *)a_hi)[i] = __ldg((const uint4 *)gtab + i);
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&s_taddr)),
                 "r"(NCOL)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t dt = s_taddr;
  const bool cj_in = (P.flags & FFTZ_F_CONJ_IN) != 0, cj_out = (P.flags & FFTZ_F_CONJ_OUT) != 0;
  const int q = warp & 3, h = warp >> 2;  // TMEM lane quarter and column half of this warp
  const int m = 32 * q + lane;           // accumulator row = TMEM lane
  unsigned phase = 0;
  bool failed = false;
  for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    if (t < TPC) batch_offsets(P, tile * TPC + t, s_in + t, s_out + t, s_col + t);
    __syncthreads();
    // stage-1 operand: B1[(t, j2)][2 j1 + ri] = x_t[64 j1 + j2]
    for (int i = t; i < TPC * 4096; i += NT) {
      const int tt = i >> 12, e = i & 4095;
      float2 x = make_float2(0.f, 0.f);
      if (s_col[tt] >= 0) x = ((const float2 *)P.in)[s_in[tt] + e];
      if (cj_in) x.y = -x.y;
      const int n = tt * 64 + (e & 63), j1 = e >> 6;
      split_store(b_hi, canon(n, 2 * j1), x.x);
      split_store(b_hi, canon(n, 2 * j1 + 1), x.y);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) stage_mma(dt, saddr(a_hi), saddr(b_hi), &bar);
    if (!wait_mma(&bar, phase)) {
      failed = true;
      break;
    }
    phase ^= 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // twiddle, then stage-2 operand B2[(t, k1)][2 j2 + ri]
    const int k1 = m >> 1, ri = m & 1;
#pragma unroll 1
    for (int c = 0; c < NCOL / 2; c += 16) {
      float v[16];
      tc::ld16(dt + ((uint32_t)(32 * q) << 16) + (uint32_t)(h * (NCOL / 2) + c), v);
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int n = h * (NCOL / 2) + c + u, tt = n >> 6, j2 = n & 63;
        const float other = __shfl_xor_sync(0xffffffffu, v[u], 1);
        const float re = ri ? other : v[u], im = ri ? v[u] : other;
        const float2 w = __ldg(wtab + ((j2 * k1) & 4095));  // (cos, sin) of 2 pi j2 k1 / 4096
        const float r = ri ? fmaf(im, w.x, -re * w.y) : fmaf(re, w.x, im * w.y);
        split_store(b_hi, canon(tt * 64 + k1, 2 * j2 + ri), r);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) stage_mma(dt, saddr(a_hi), saddr(b_hi), &bar);
    if (!wait_mma(&bar, phase)) {
      failed = true;
      break;
    }
    phase ^= 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // results X_t[k1 + 64 k2] (row m = 2 k2 + ri, column (t, k1)) into shared memory
    {
      const int k2 = m >> 1;
#pragma unroll 1
      for (int c = 0; c < NCOL / 2; c += 16) {
        float v[16];
        tc::ld16(dt + ((uint32_t)(32 * q) << 16) + (uint32_t)(h * (NCOL / 2) + c), v);
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int n = h * (NCOL / 2) + c + u, tt = n >> 6, kk1 = n & 63;
          float *o = (float *)(obuf + (size_t)tt * 4096 + kk1 + 64 * k2);
          o[ri] = (ri && cj_out) ? -v[u] : v[u];
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // coalesced HBM stores: lanes along elements (row outputs) or along lines (column outputs)
    for (int i = t; i < TPC * 4096; i += NT) {
      int tt, k;
      if (P.out_mode == 0) {
        tt = i >> 12;
        k = i & 4095;
      } else {
        tt = i & (TPC - 1);
        k = i / TPC;
      }
      if (s_col[tt] < 0) continue;
      ((float2 *)P.out)[s_out[tt] + (int64_t)k * P.oes] = obuf[(size_t)tt * 4096 + k];
    }
    __syncthreads();
  }
  if (failed) {
    if (t == 0) atomicExch(&g_tc_wait_failed, 1);
    // give the outstanding MMAs a last bounded chance before releasing TMEM
    for (long i = 0; i < (1L << 20); i++)
      if (tc::try_wait(&bar, phase)) break;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(dt), "r"(NCOL) : "memory");
  }
}

}  // namespace fftz

extern "C" {

/* Shared memory and threads of the tensor-core 4096-point kernel. */
int fftz_tc_smem_bytes(void) { return fftz::tc::SMEM; }

/* Launches a pass of variant FFTZ_VAR_TC (n = 4096, float, rows of unit
 * element stride, tpc = 2); returns a cudaError_t. */
int fftz_launch_pass_tc(const fftz_pass_t *p, void *stream) {
  if (p->n != 4096 || p->dtype != 0 || p->tpc != fftz::tc::TPC || p->ies != 1) return (int)cudaErrorInvalidValue;
  const void *fn = (const void *)&fftz::fft_tc4096_kernel;
  static int opted[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!opted[dev]) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, fftz::tc::SMEM);
    if (e != cudaSuccess) return (int)e;
    opted[dev] = 1;
  }
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int64_t ntiles = (p->ntf + fftz::tc::TPC - 1) / fftz::tc::TPC;
  const unsigned grid = (unsigned)(ntiles < nsm ? ntiles : (nsm > 0 ? nsm : 148));
  void *args[2] = {(void *)p, (void *)&ntiles};
  return (int)cudaLaunchKernel(fn, dim3(grid), dim3(fftz::tc::NT), args, (size_t)fftz::tc::SMEM,
                               (cudaStream_t)stream);
}

/* 1 if a tensor-core tile gave up waiting for its MMAs since the last call. */
int fftz_tc_wait_failed(void) {
  int v = 0, z = 0;
  if (cudaMemcpyFromSymbol(&v, fftz::g_tc_wait_failed, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (v) cudaMemcpyToSymbol(fftz::g_tc_wait_failed, &z, sizeof(int));
  return v;
}

}  // extern "C"
