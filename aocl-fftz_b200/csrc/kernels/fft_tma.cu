// Tensor-memory-accelerator (TMA) input path of the compile-time FFT kernel.
//
// The one-tile-per-CTA kernel of fft_fast.cuh fetches its tile with ordinary
// per-thread loads fused into the first stage. Column passes (lanes along
// neighbouring transforms) read only tpc * element-size contiguous bytes per
// row, so the load path issues many narrow requests. Here one thread issues
// cp.async.bulk.tensor copies of the whole tile -- boxes of (tpc columns x 256
// rows) for column passes, (256 elements x 1 row) for row passes -- into the
// shared-memory tile, completion is tracked by an mbarrier transaction count,
// and the first stage reads the dense staged tile instead of HBM (the stage
// code is the same template with its STG flag). Stores are unchanged.
//
// Eligibility is decided per launch on the host (the tensor map encodes the
// buffer address): complex input, plain or four-step-twiddle variant, at most
// two batch dimensions, tiles that do not straddle the outer batch dimension,
// 16-byte aligned base and strides. Anything else takes the ordinary kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_fast.cuh"

namespace fftz {

__device__ int g_tma_wait_failed;  // set when a tile's copies did not arrive in time

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

// Stores of the persistent kernels' outputs do not allocate in L1 (128 KB of
// output per tile would evict the twiddle tables), and twiddle loads are kept
// in L1 with the evict-last priority.
__device__ __forceinline__ void st_na(float2 *p, float2 v) {
  asm volatile("st.global.L1::no_allocate.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void st_na(double2 *p, double2 v) {
  asm volatile("st.global.L1::no_allocate.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ float2 ld_tw(const float2 *p) {
  float2 v;
  asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_tw(const double2 *p) {
  double2 v;
  asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

// One tile per CTA. MODE 1: column pass (tile = tpc adjacent columns, staged
// [e][p]); MODE 0: row pass (tile = tpc rows, staged [p][e]).
template <typename T, int N, int FEAT, int MODE>
__global__ void __launch_bounds__(ct_lb<T>()) fft_tma_kernel(const __grid_constant__ fftz_pass_t P,
                                                            const __grid_constant__ CUtensorMap tmap) {
  typedef typename Cplx<T>::type T2;
  constexpr int BOXE = N < 256 ? N : 256;   // elements of one box along the transform
  constexpr int CE = sizeof(T2) / 8;        // 8-byte units per complex element
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  // 128-byte aligned tile (the host adds 128 bytes of slack)
  unsigned char *base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  T2 *sdata = (T2 *)base;
  int64_t *s_in = (int64_t *)(sdata + (size_t)P.tpc * P.sstride);
  int64_t *s_out = s_in + P.tpc;
  int64_t *s_col = s_out + P.tpc;
  const int64_t tf0 = (int64_t)blockIdx.x * P.tpc;
  const int tpc = P.tpc;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar, (unsigned)(N * tpc * sizeof(T2) + P.test_tx_short));
    const int64_t b0 = P.bdim[0];
    const int c0 = (int)(tf0 % b0);
    const int z = (int)(tf0 / b0);
    if (MODE == 1) {
      for (int k = 0; k < N / BOXE; k++)
        tma_load_3d(sdata + (size_t)k * BOXE * tpc, &tmap, c0 * CE, k * BOXE, z, &bar);
    } else {
      for (int q = 0; q < tpc; q++)
        for (int k = 0; k < N / BOXE; k++) tma_load_3d(sdata + (size_t)q * N + k * BOXE, &tmap, k * BOXE * CE, c0 + q, z, &bar);
    }
  }
  for (int p = threadIdx.x; p < tpc; p += blockDim.x) {
    int64_t io;
    batch_offsets(P, tf0 + p, &io, s_out + p, s_col + p);
    s_in[p] = MODE == 1 ? p : (int64_t)p * N;
  }
  // bounded wait for the tile (about a second of polling); a wait that gives
  // up leaves the tile unwritten and flags the failure for the host
  bool ok = false;
  for (long i = 0; i < (1L << 22); i++)
    if (mbar_try_wait(&bar, 0)) {
      ok = true;
      break;
    }
  if (!__syncthreads_and(ok)) {  // every thread takes the same branch
    if (threadIdx.x == 0) atomicExch(&g_tma_wait_failed, 1);
    return;
  }
  T2 *twb = nullptr;
  if (P.smem_tw) {
    twb = (T2 *)(((uintptr_t)(s_col + tpc) + 15) & ~(uintptr_t)15);
    const T2 *g = (const T2 *)P.tw;
    for (int i = threadIdx.x; i < ct_tw_total(N); i += blockDim.x) twb[i] = __ldg(g + i);
    __syncthreads();
  }
  FastStages<T, N, 0, ct_nstages(N), 0, 1, FEAT, true, 1>::run(P, sdata, s_in, s_out, s_col,
                                                                   MODE == 1 ? tpc : 1, twb);
}

// Persistent variant: CTA b runs tiles b, b + grid, ...; while the stages of
// tile i run, TMA copies bring the half e < N/2 of tile i + 1 into a staging
// area beside the exchange buffer (there is not room for a whole second
// tile); the first stage of tile i + 1 takes that half from shared memory and
// the other half from HBM.
template <typename T, int N, int FEAT, int MODE>
__global__ void __launch_bounds__(ct_lb<T>(), 1) fft_tma_pipe_kernel(const __grid_constant__ fftz_pass_t P,
                                                                     const __grid_constant__ CUtensorMap tmap,
                                                                     int64_t ntiles) {
  typedef typename Cplx<T>::type T2;
  constexpr int H = N / 2;
  constexpr int HB = H < 256 ? H : 256;  // box extent along the transform
  constexpr int CE = sizeof(T2) / 8;
  constexpr int NST = ct_nstages(N);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  unsigned char *base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  const int tpc = P.tpc;
  T2 *sdata = (T2 *)base;
  const size_t xbytes = ((size_t)tpc * P.sstride * sizeof(T2) + 127) & ~(size_t)127;
  T2 *stg = (T2 *)(base + xbytes);
  int64_t *s_in = (int64_t *)(stg + (size_t)tpc * H);
  int64_t *s_out = s_in + tpc;
  int64_t *s_col = s_out + tpc;
  int64_t *s_stg = s_col + tpc;
  const int64_t b0 = P.bdim[0];
  auto issue = [&](int64_t tile) {
    const int64_t tf0 = tile * tpc;
    const int c0 = (int)(tf0 % b0);
    const int z = (int)(tf0 / b0);
    mbar_expect_tx(&bar, (unsigned)(H * tpc * sizeof(T2) + P.test_tx_short));
    if (MODE == 1) {
      for (int k = 0; k < H / HB; k++) tma_load_3d(stg + (size_t)k * HB * tpc, &tmap, c0 * CE, k * HB, z, &bar);
    } else {
      for (int q = 0; q < tpc; q++)
        for (int k = 0; k < H / HB; k++) tma_load_3d(stg + (size_t)q * H + k * HB, &tmap, k * HB * CE, c0 + q, z, &bar);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  int64_t tile = blockIdx.x;
  if (threadIdx.x == 0 && tile < ntiles) issue(tile);
  for (unsigned it = 0; tile < ntiles; it++, tile += gridDim.x) {
    for (int p = threadIdx.x; p < tpc; p += blockDim.x) {
      batch_offsets(P, tile * tpc + p, s_in + p, s_out + p, s_col + p);
      s_stg[p] = MODE == 1 ? p : (int64_t)p * H;
    }
    bool ok = false;
    for (long i = 0; i < (1L << 22); i++)
      if (mbar_try_wait(&bar, it & 1u)) {
        ok = true;
        break;
      }
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) atomicExch(&g_tma_wait_failed, 1);
      return;
    }
    fast_stage<T, N, 0, FEAT, true, NST == 1, true, false, 2>(P, sdata, s_in, s_out, s_col, MODE == 1 ? tpc : 1, stg,
                                                              s_stg);
    if (NST == 1) __syncthreads();
    // every thread has read its staged half: refill the staging area
    if (threadIdx.x == 0 && tile + gridDim.x < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(tile + gridDim.x);
    }
    FastStages<T, N, 1, NST, 0, 1, FEAT, true, 0>::run(P, sdata, s_in, s_out, s_col);
    __syncthreads();
  }
}

// ---------------------------------------------------------------- streaming
//
// Persistent row kernel for passes over contiguous lines (unit element
// stride, 16-byte aligned lines): CTA b runs tiles b, b + G, b + 2 G, ...
// (G = the grid), each tile's lines copied by one 1-D bulk copy per line into
// one of two slots. The copies of the next tile are in flight while the
// current one is computed, its stages run in place in its slot (the first
// stage reads the dense staged lines with the HBM lane map, later stages use
// the padded layout), the last stage writes HBM, and once every thread is done
// with the slot it is refilled with the tile two steps ahead. Several CTAs
// share an SM, so the SM has several tiles' copies in flight at once.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

template <typename T, int N, int FEAT>
__global__ void __launch_bounds__(ct_lb<T>()) fft_tma_stream_kernel(const __grid_constant__ fftz_pass_t P,
                                                                   int64_t ntiles) {
  typedef typename Cplx<T>::type T2;
  constexpr int NST = ct_nstages(N);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  unsigned char *base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  const int tpc = P.tpc;
  const size_t slot_bytes = ((size_t)tpc * P.sstride * sizeof(T2) + 127) & ~(size_t)127;
  int64_t *s_in = (int64_t *)(base + 2 * slot_bytes);
  int64_t *s_out = s_in + tpc;
  int64_t *s_col = s_out + tpc;
  // one thread: the lines of `tile` into slot sl (line p at p * N, dense)
  auto issue = [&](int64_t tile, int sl) {
    mbar_expect_tx(&bar[sl], (unsigned)(tpc * N * sizeof(T2) + P.test_tx_short));
    for (int p = 0; p < tpc; p++) {
      int64_t io, oo, col;
      batch_offsets(P, tile * tpc + p, &io, &oo, &col);
      bulk_load((T2 *)(base + sl * slot_bytes) + (size_t)p * N, (const T2 *)P.in + io, (unsigned)(N * sizeof(T2)),
                &bar[sl]);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  int64_t tile = blockIdx.x;
  if (threadIdx.x == 0) {
    if (tile < ntiles) issue(tile, 0);
    if (tile + gridDim.x < ntiles) issue(tile + gridDim.x, 1);
  }
  for (unsigned it = 0; tile < ntiles; it++, tile += gridDim.x) {
    const int sl = (int)(it & 1u);
    for (int p = threadIdx.x; p < tpc; p += blockDim.x) {
      int64_t io;
      batch_offsets(P, tile * tpc + p, &io, s_out + p, s_col + p);
      s_in[p] = (int64_t)p * N;
    }
    // bounded wait for this slot's copies (about a second of polling)
    bool ok = false;
    for (long i = 0; i < (1L << 22); i++)
      if (mbar_try_wait(&bar[sl], (it >> 1) & 1u)) {
        ok = true;
        break;
      }
    if (!__syncthreads_and(ok)) {  // every thread takes the same branch
      if (threadIdx.x == 0) {
        atomicExch(&g_tma_wait_failed, 1);
        // give the copies still in flight (this slot's, and the other slot's
        // if it was filled) a bounded time to land before the CTA exits
        for (long i = 0; i < (1L << 22); i++)
          if (mbar_try_wait(&bar[sl], (it >> 1) & 1u)) break;
        if (tile + gridDim.x < ntiles)
          for (long i = 0; i < (1L << 22); i++)
            if (mbar_try_wait(&bar[sl ^ 1], ((it + 1) >> 1) & 1u)) break;
      }
      return;
    }
    FastStages<T, N, 0, NST, 0, 1, FEAT, true, 1>::run(P, (T2 *)(base + sl * slot_bytes), s_in, s_out, s_col, 1,
                                                       nullptr);
    // every thread is done with the slot and the offsets: refill the slot
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0 && tile + 2 * (int64_t)gridDim.x < ntiles) issue(tile + 2 * (int64_t)gridDim.x, sl);
  }
}

// ------------------------------------------------------- register-resident
//
// Persistent 4096-point float kernel whose whole next tile is in flight while
// the current one is computed. Between stages the tile lives in registers
// (16 complex values a thread); a stage-to-stage exchange goes through a
// buffer holding ONE real component of the tile (x parts, then y parts), so
// the exchange buffer (4 x 4228 floats) plus a full staged tile (4 x 4096
// complex) fit in one SM's shared memory (199 KB). Per tile: wait for the
// staged tile, read it into registers, run stage 0 and exchange 1 (its y
// parts through the consumed staging area, so one barrier between writes and
// reads), let one thread issue the TMA copies of the next tile into the
// staging area, then run stage 1, exchange 2 (x then y through the exchange
// buffer) and stage 2, which stores to HBM with the pass's epilogue.

// Exchange 1's buffer layout (one pad word per 2^SH words, transforms SSF
// words apart): SH = 5 with the transforms 4228 (= 4 mod 32) words apart puts
// every access of both lane maps (rows: one transform per warp; columns: four
// transforms per warp) on 32 distinct banks with compile-time per-value
// offsets (checked by a simulation of every access). (Tiles of two transforms
// would let two CTAs share an SM, but their 16-byte column runs made both
// passes 1.4-2.5x slower on B200.)
template <int SH> __device__ __forceinline__ int rr_phys(int i) { return i + (i >> SH); }
constexpr int kRrSh1 = 5, kRrSsf1 = 4228;

template <int TPT> __device__ __forceinline__ void rr_lane(int mode, int tpc, int &p, int &j) {
  const int t = threadIdx.x;
  if (mode == 0) {
    p = t / TPT;
    j = t - p * TPT;
  } else {
    p = t % tpc;
    j = t / tpc;
  }
}

// Twiddles and butterflies of stage S on the thread's values (j under the
// stage's lane map).
template <typename T, int N, int S>
__device__ __forceinline__ void rr_butterflies(const fftz_pass_t &P, typename Cplx<T>::type (&v)[16], int j) {
  typedef typename Cplx<T>::type T2;
  constexpr int NS = ct_ns(N, S);
  static_assert(ct_radix(N, S) == 16, "radix-16 stages only");
  if (NS > 1) {
    const T2 *tw = (const T2 *)P.tw + P.tw_off[S];
    const int k = j & (NS - 1);
#pragma unroll
    for (int r = 1; r < 16; r++) v[r] = cmul(v[r], ld_tw(tw + (r - 1) * NS + k));
  }
  Dft<16>::template apply<T, T2>(v);
}

// Stage S outputs (lane map mw) -> stage S + 1 inputs (lane map mr) with the
// x parts in X and the y parts in Y (both in layout SH, SSF): one barrier
// between the writes and the reads. TRAIL: wait for every reader before
// returning (the buffers are written again after it).
template <typename T, int N, int S, int SH, int SSF, bool TRAIL>
__device__ __forceinline__ void rr_exchange2(T *X, T *Y, typename Cplx<T>::type (&v)[16], int mw, int mr, int tpc) {
  constexpr int NS = ct_ns(N, S);
  constexpr int TPT = ct_tpt(N);
  constexpr int NBF1 = N / 16;
  static_assert(NS == 1 ? 16 <= (1 << SH) : NS % (1 << SH) == 0, "stride vs pad");
  static_assert(NBF1 % (1 << SH) == 0, "stride vs pad");
  constexpr int WST = NS == 1 ? 1 : NS + (NS >> SH);
  constexpr int RST = NBF1 + (NBF1 >> SH);
  int p, j, p1, j1;
  rr_lane<TPT>(mw, tpc, p, j);
  rr_lane<TPT>(mr, tpc, p1, j1);
  const int k = j & (NS - 1);
  const int d0 = (j - k) * 16 + k;
  const int wo = p * SSF + rr_phys<SH>(d0), ro = p1 * SSF + rr_phys<SH>(j1);
#pragma unroll
  for (int r = 0; r < 16; r++) {
    X[wo + r * WST] = v[r].x;
    Y[wo + r * WST] = v[r].y;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; r++) {
    v[r].x = X[ro + r * RST];
    v[r].y = Y[ro + r * RST];
  }
  if (TRAIL) __syncthreads();
}

// Exchange 2 (stage 1, row map, outputs d0 + 16 r -> stage 2 inputs j1 + 256 r)
// through X in an unpadded layout: element i of transform p at p * 4096 +
// (i ^ (bit 8 of i) << 4 ^ 8 p), bank-conflict-free for row and column read
// maps (64 KB for four transforms instead of the padded layout's 68 KB, which
// keeps the CTA under the 196 KB shared-memory carveout and leaves L1 60 KB
// for the twiddle tables). Each thread needs two base offsets (even and odd
// r) with compile-time steps.
template <typename T, int N>
__device__ __forceinline__ void rr_exchange_x(T *X, typename Cplx<T>::type (&v)[16], int mr, int tpc) {
  static_assert(N == 4096 && ct_ns(N, 1) == 16, "4096 = 16 x 16 x 16");
  constexpr int TPT = ct_tpt(N);
  int p, j, p1, j1;
  rr_lane<TPT>(0, tpc, p, j);
  rr_lane<TPT>(mr, tpc, p1, j1);
  // writes: i = 256 a + c + 16 r (a = j / 16, c = j % 16); bit 8 of i is a & 1
  const int key = (((j >> 4) & 1) << 4) ^ (8 * p);
  const int kb = key >> 4 & 1;
  const int wb = p * 4096 + ((((j >> 4) << 8) + (j & 15)) ^ (key & 8));
  const int we = wb + 16 * kb, wo = wb - 16 * kb;
  // reads: i = j1 + 256 r; bit 8 of i is r & 1
  const int re = p1 * 4096 + (j1 ^ (8 * p1)), ro = re ^ 16;
  T tmp[16];
#pragma unroll
  for (int r = 0; r < 16; r++) X[((r & 1) ? wo : we) + 16 * r] = v[r].x;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; r++) tmp[r] = X[((r & 1) ? ro : re) + 256 * r];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; r++) X[((r & 1) ? wo : we) + 16 * r] = v[r].y;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; r++) {
    v[r].x = tmp[r];
    v[r].y = X[((r & 1) ? ro : re) + 256 * r];
  }
}

// Two table entries whose product is W^{(col * k) mod n} (the four-step
// twiddle of tw4 in fft_common.cuh), fetched without multiplying them so that
// the loads can be issued long before the product is needed.
template <typename T>
__device__ __forceinline__ void tw4_parts(const fftz_pass_t &P, int64_t col, int64_t k, typename Cplx<T>::type &hi,
                                          typename Cplx<T>::type &lo) {
  typedef typename Cplx<T>::type T2;
  const int64_t N = P.tw4_n, L = P.tw4_l;
  int64_t h, l;
  if (((N & (N - 1)) == 0) && N <= 0x80000000LL && ((L & (L - 1)) == 0)) {
    const unsigned r = ((unsigned)col * (unsigned)k) & (unsigned)(N - 1);
    h = r >> (31 - __clz((int)L));
    l = r & (unsigned)(L - 1);
  } else {
    const int64_t r = (col * k) % N;
    h = r / L;
    l = r - h * L;
  }
  hi = ld_tw((const T2 *)P.tw4_hi + h);
  lo = ld_tw((const T2 *)P.tw4_lo + l);
}

// Last stage's outputs to HBM (lane map out_mode) with the pass epilogue. In
// the last radix-16 stage of 4096 points (NS = 256) thread j owns outputs
// j + 256 r, so the four-step factor is W^{col j} (W^{256 col})^r: the
// product hi * lo of the parts fetched at the start of the tile, then a chain
// of products by the column's step (held in shared memory), restarted at
// r = 8 from W^{col j} W^{2048 col}.
template <typename T, int N, int S, int FEAT>
__device__ __forceinline__ void rr_store(const fftz_pass_t &P, const typename Cplx<T>::type (&v)[16], int j,
                                         int64_t obase, int64_t col, typename Cplx<T>::type hi,
                                         typename Cplx<T>::type lo, typename Cplx<T>::type stp,
                                         typename Cplx<T>::type stp8) {
  typedef typename Cplx<T>::type T2;
  constexpr int NS = ct_ns(N, S);
  static_assert(NS * 16 == N, "last stage");
  if (col < 0) return;
  const int64_t oes = P.oes;
  // blocked intermediate: output k of column col at (k / 4) * 4 oes + 4 col + k % 4
  // (the column base obase already holds col; outputs j + 256 r keep the stride)
  const int64_t jo = (P.flags & FFTZ_F_BLK4_OUT) ? (int64_t)(j >> 2) * 4 * oes + (j & 3) + 3 * col
                                                 : (int64_t)j * oes;
  T2 *ob = (T2 *)P.out + obase + jo;
  const int64_t st = (int64_t)NS * oes;
  const bool cj = (P.flags & FFTZ_F_CONJ_OUT) != 0;
  T2 w0 = zero2<T2>(), w = zero2<T2>();
  if constexpr ((FEAT & FEAT_TW4) != 0) {
    w0 = cmul(hi, lo);
    w = w0;
  }
#pragma unroll
  for (int r = 0; r < 16; r++) {
    T2 y = v[r];
    if constexpr ((FEAT & FEAT_TW4) != 0) {
      if (r == 8) w = cmul(w0, stp8);
      y = cmul(y, w);
      if (r != 7 && r != 15) w = cmul(w, stp);
    }
    if (cj) y.y = -y.y;
    st_na(ob + r * st, y);
  }
}

template <typename T, int N, int FEAT, int MODE>
__global__ void __launch_bounds__(ct_lb<T>(), 1) fft_tma_rr_kernel(const __grid_constant__ fftz_pass_t P,
                                                                   const __grid_constant__ CUtensorMap tmap,
                                                                   int64_t ntiles) {
  static_assert(N == 4096 && sizeof(T) == 4, "4096-point float tiles");
  typedef typename Cplx<T>::type T2;
  constexpr int TPT = ct_tpt(N);
  constexpr int NBF = N / 16;
  constexpr int BOXE = 256;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  unsigned char *base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  const int tpc = P.tpc;
  T2 *stg = (T2 *)base;                               // staged tile, TMA box layout
  T *X = (T *)(base + (size_t)tpc * N * sizeof(T2));  // one-component exchange buffer
  int64_t *offs = (int64_t *)(X + (size_t)tpc * kRrSsf1);  // 2 sets of {out, col} by tile parity
  T2 *steps = (T2 *)(offs + 4 * tpc);                        // 2 sets of {W^{256 col}, W^{2048 col}}
  const int64_t b0 = P.bdim[0];
  auto issue = [&](int64_t tile) {
    const int64_t tf0 = tile * tpc;
    const int c0 = (int)(tf0 % b0);
    const int z = (int)(tf0 / b0);
    mbar_expect_tx(&bar, (unsigned)(N * tpc * sizeof(T2) + P.test_tx_short));
    if (MODE == 1) {
      for (int k = 0; k < N / BOXE; k++) tma_load_3d(stg + (size_t)k * BOXE * tpc, &tmap, c0, k * BOXE, z, &bar);
    } else {
      for (int q = 0; q < tpc; q++)
        for (int k = 0; k < N / BOXE; k++) tma_load_3d(stg + (size_t)q * N + k * BOXE, &tmap, k * BOXE, c0 + q, z, &bar);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  int64_t tile = blockIdx.x;
  if (threadIdx.x == 0 && tile < ntiles) issue(tile);
  for (unsigned it = 0; tile < ntiles; it++, tile += gridDim.x) {
    int64_t *s_out = offs + (size_t)(it & 1u) * 2 * tpc;
    int64_t *s_col = s_out + tpc;
    T2 *s_stp = steps + (size_t)(it & 1u) * 2 * tpc;
    for (int p = threadIdx.x; p < tpc; p += blockDim.x) {
      int64_t io;
      batch_offsets(P, tile * tpc + p, &io, s_out + p, s_col + p);
      if constexpr ((FEAT & FEAT_TW4) != 0) {
        s_stp[p] = tw4<T>(P, s_col[p], N / 16);
        s_stp[tpc + p] = tw4<T>(P, s_col[p], N / 2);
      }
    }
    // bounded wait for the staged tile; a wait that gives up flags the
    // failure for the host and ends the CTA (every thread takes one branch)
    bool ok = false;
    for (long i = 0; i < (1L << 22); i++)
      if (mbar_try_wait(&bar, it & 1u)) {
        ok = true;
        break;
      }
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) atomicExch(&g_tma_wait_failed, 1);
      return;
    }
    T2 v[16];
    int p, j;
    rr_lane<TPT>(MODE, tpc, p, j);
    {
      const bool cj = (P.flags & FFTZ_F_CONJ_IN) != 0;
#pragma unroll
      for (int r = 0; r < 16; r++) {
        const int e = j + r * NBF;
        T2 x = MODE == 1 ? stg[(size_t)e * tpc + p] : stg[(size_t)p * N + e];
        if (cj) x.y = -x.y;
        v[r] = x;
      }
    }
    // the four-step factor's table entries for this thread's last-stage
    // outputs: fetched now, used after two stages
    T2 hi = zero2<T2>(), lo = zero2<T2>();
    if constexpr ((FEAT & FEAT_TW4) != 0) {
      int p2, j2;
      rr_lane<TPT>(P.out_mode, tpc, p2, j2);
      tw4_parts<T>(P, s_col[p2], j2, hi, lo);
    }
    __syncthreads();  // the staged tile is consumed: its space holds exchange 1's y parts
    rr_butterflies<T, N, 0>(P, v, j);
    rr_exchange2<T, N, 0, kRrSh1, kRrSsf1, true>(X, (T *)stg, v, MODE, 0, tpc);
    // the staging area is free again: bring in the next tile
    if (threadIdx.x == 0 && tile + gridDim.x < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(tile + gridDim.x);
    }
    rr_lane<TPT>(0, tpc, p, j);
    rr_butterflies<T, N, 1>(P, v, j);
    rr_exchange_x<T, N>(X, v, P.out_mode, tpc);
    rr_lane<TPT>(P.out_mode, tpc, p, j);
    rr_butterflies<T, N, 2>(P, v, j);
    rr_store<T, N, 2, FEAT>(P, v, j, s_out[p], s_col[p], hi, lo, s_stp[p], s_stp[tpc + p]);
  }
}

// ------------------------------------------------------------- 16 x 256 split
//
// Persistent 4096-point float kernel, one CTA of 1024 threads per SM, tiles of
// four transforms. The line is split as n = n0 + 16 m, k = k' + 256 k2:
//   X[k' + 256 k2] = sum_n0 W16^{n0 k2} W4096^{n0 k'} Z_n0[k'],
//   Z_n0[k'] = sum_m x[n0 + 16 m] W256^{m k'}.
// The 64 sub-transforms Z_n0 of a tile (4 transforms x 16 n0) run one per
// 16-lane group: each lane holds m = l + 16 s (s = 0..15), a radix-16 stage
// over s, the W256 twiddle, a 16 x 16 transpose among the group's lanes and a
// second radix-16 stage leave Z_n0[l + 16 k_hi] in lane l. One exchange across
// the CTA then gives thread (transform p, k') its 16 values Z_n0[k'], and a
// last radix-16 stage with the W4096 twiddle produces outputs k' + 256 r,
// stored with the pass epilogue like the register-resident kernel's last
// stage. Compared with three stages and two CTA-wide exchanges, the sub-
// transforms need no CTA barrier: only the one exchange does (two rounds of
// full complex values through a 64 KB buffer, half of the warps reading in
// each round).
//
// Staging: the tile arrives as 16 TMA boxes (box s = elements [256 s, 256 s +
// 256) of the four transforms), each box laid out [n0][m_l][transform] by the
// tensor map's dimension order (column tiles, 32-byte swizzle) or
// [transform][m_l][n0] (row tiles, 128-byte swizzle); a warp's groups read
// their 16 values from one 256-byte slice of every box, bank-conflict-free.
// The transpose of the sub-transforms reuses the warp's own slice (so it needs
// no other buffer and no CTA barrier); the last warp to finish with its slice
// issues the next tile's 16 boxes into the staging area. All index maps are
// restated and checked on the CPU by tests/test_split_layouts.py.

// staging, exchange, offsets, steps, mbarrier + counters; XM 1 adds the 32 KB stash
constexpr int kSplitSmem = 16384 * 8 + 8192 * 8 + 16 * 8 + 16 * 8 + 16;
constexpr int kSplitStash = 512 * 8 * 8;

__device__ __forceinline__ void nb_sync(int id) { asm volatile("bar.sync %0, 1024;" ::"r"(id) : "memory"); }
__device__ __forceinline__ void nb_arrive(int id) { asm volatile("bar.arrive %0, 1024;" ::"r"(id) : "memory"); }

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_addr(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5, %6}], [%7];" ::"r"(smem_addr(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
      : "memory");
}

// Slice offset of the transpose slot for difference d = writer lane ^ reader
// lane (XOR-linear in d): column tiles ([n0][m_l][col], 32-byte swizzle) and
// row tiles ([row][m_l][n0], 128-byte swizzle).
template <int MODE> __host__ __device__ constexpr int split_f(int d) {
  return MODE == 1 ? (((d & 7) << 2) | (((d >> 2) & 1) << 1) | ((d >> 3) & 1))
                   : (((d & 7) << 4) | ((d & 7) << 1) | ((d >> 3) & 1));
}

// Tensor-memory stash (XM 2): a warp's 32 lanes keep 16 words each in their
// own TMEM lanes (the warp's lane quarter), 16 columns per warp.
__device__ __forceinline__ void tm_st16(uint32_t taddr, const float2 (&v)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0].x)), "r"(__float_as_uint(v[0].y)), "r"(__float_as_uint(v[1].x)),
      "r"(__float_as_uint(v[1].y)), "r"(__float_as_uint(v[2].x)), "r"(__float_as_uint(v[2].y)),
      "r"(__float_as_uint(v[3].x)), "r"(__float_as_uint(v[3].y)), "r"(__float_as_uint(v[4].x)),
      "r"(__float_as_uint(v[4].y)), "r"(__float_as_uint(v[5].x)), "r"(__float_as_uint(v[5].y)),
      "r"(__float_as_uint(v[6].x)), "r"(__float_as_uint(v[6].y)), "r"(__float_as_uint(v[7].x)),
      "r"(__float_as_uint(v[7].y))
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_ld8(uint32_t taddr, float2 (&v)[4]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 4; i++) v[i] = make_float2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
}

template <typename T, int N, int FEAT, int MODE, int OMODE, int XM>
__global__ void __launch_bounds__(1024, 1) fft_tma_split_kernel(const __grid_constant__ fftz_pass_t P,
                                                                const __grid_constant__ CUtensorMap tmap,
                                                                int64_t ntiles) {
  static_assert(N == 4096 && sizeof(T) == 4, "4096-point float tiles");
  typedef typename Cplx<T>::type T2;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
  T2 *stg = (T2 *)base;                      // 16 boxes of 1024 complex
  T2 *X = stg + 16384;                       // one exchange round: 8192 complex
  int64_t *offs = (int64_t *)(X + 8192);     // 2 sets of {out[4], col[4]} by tile parity
  T2 *steps = (T2 *)(offs + 16);             // 2 sets of {W^{256 col}[4], W^{2048 col}[4]}
  uint64_t *bar = (uint64_t *)(steps + 16);
  unsigned *cnt = (unsigned *)(bar + 1);      // warps done with the staging area (32 a tile)
  volatile int *abort_flag = (volatile int *)(cnt + 1);
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int g = (lane >> 3) & 1, l = (lane & 7) | ((lane >> 4) << 3);
  // MODE 2 (a blocked intermediate read in 4-row slabs) stages like a column tile
  constexpr int SMODE = MODE == 2 ? 1 : MODE;
  // the group's sub-transform (transform pw, subsequence n0w) and its slice
  int pw, n0w, wb, c, rd0;
  if (SMODE == 1) {
    const int a = w & 1;
    n0w = w >> 1;
    pw = 2 * a + g;
    wb = n0w * 64;
    c = (33 * g) ^ (2 * a);
    rd0 = wb + ((l * 4 + 2 * ((l >> 2) & 1) + g) ^ (2 * a));
  } else {
    const int b = w & 7;
    pw = w >> 3;
    n0w = 2 * b + g;
    wb = pw * 256;
    c = (129 * g) ^ (2 * b);
    rd0 = wb + ((l * 16 + 2 * (l & 7) + g) ^ (2 * b));
  }
  const int u = split_f<SMODE>(l) ^ c;
  const int xw = (pw * 16 + n0w) * 128 + (l ^ (4 * ((pw >> 1) & 1) + 8 * ((pw ^ n0w) & 1)));
  // exchange reader: thread (pr, kr) of the output lane map
  const int pr = OMODE == 1 ? (tid & 3) : (tid >> 8);
  const int kr = OMODE == 1 ? (tid >> 2) : (tid & 255);
  const int rround = kr >> 7, kl = kr & 127;
  const int xr_e = pr * 2048 + (kl ^ (4 * ((pr >> 1) & 1) + 8 * (pr & 1)));
  const int xr_o = pr * 2048 + (kl ^ (4 * ((pr >> 1) & 1) + 8 * ((pr & 1) ^ 1)));
  // one-component layout: float (p * 16 + n0) * 256 + (k' ^ S), S = 8 (p >> 1 & 1) + 16 ((p ^ n0) & 1);
  // writers take even/odd k_hi bases, readers even/odd n0 bases
  const int sw1 = 8 * ((pw >> 1) & 1) + 16 * ((pw ^ n0w) & 1);
  const int xfw = (pw * 16 + n0w) * 256 + (l ^ (sw1 & 15)), s4 = 16 * (sw1 >> 4);
  const int xfw_e = xfw + s4, xfw_o = xfw - s4;
  const int xfr_e = pr * 4096 + (kr ^ (8 * ((pr >> 1) & 1) + 16 * (pr & 1)));
  const int xfr_o = pr * 4096 + (kr ^ (8 * ((pr >> 1) & 1) + 16 * ((pr & 1) ^ 1)));
  // stash slot of a round-1 reader (XM 1): 512 threads, [value][thread]
  const int si = OMODE == 1 ? (tid & 511) : ((w >> 3) * 128 + (w & 3) * 32 + lane);
  const int64_t b0 = P.bdim[0];
  const T2 *tw1 = (const T2 *)P.tw + P.tw_off[1];
  const T2 *tw2 = (const T2 *)P.tw + P.tw_off[2];
  const bool cjin = (P.flags & FFTZ_F_CONJ_IN) != 0;
  auto issue = [&](int64_t tile) {
    const int64_t tf0 = tile * 4;
    const int c0 = (int)(tf0 % b0);
    const int z = (int)(tf0 / b0);
    mbar_expect_tx(bar, (unsigned)(N * 4 * sizeof(T2) + P.test_tx_short));
#pragma unroll 1
    for (int s = 0; s < 16; s++) {
      if (MODE == 2)  // dims (row in slab, m, n0, slab, line)
        tma_load_5d(stg + s * 1024, &tmap, 0, 16 * s, 0, c0 >> 2, z, bar);
      else if (MODE == 1)
        tma_load_4d(stg + s * 1024, &tmap, c0, 16 * s, 0, z, bar);
      else
        tma_load_4d(stg + s * 1024, &tmap, 0, 16 * s, c0, z, bar);
    }
  };
  uint32_t *s_taddr = (uint32_t *)(abort_flag + 1);
  if (tid == 0) {
    mbar_init(bar, 1);
    *cnt = 0;
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (XM == 2 && w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_addr(s_taddr))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (XM == 2) asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (XM == 2) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // this warp's stash columns (round-1 reader warps, four per lane quarter)
  const uint32_t tstash = XM == 2 ? *s_taddr + ((uint32_t)(32 * (w & 3)) << 16) +
                                        (uint32_t)(16 * (OMODE == 1 ? (w >> 2) : (w >> 3)))
                                  : 0u;
  int64_t tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) issue(tile);
  unsigned it = 0;
  for (; tile < ntiles; it++, tile += gridDim.x) {
    int64_t *s_out = offs + (size_t)(it & 1u) * 8;
    int64_t *s_col = s_out + 4;
    T2 *s_stp = steps + (size_t)(it & 1u) * 8;
    if (tid < 4) {
      int64_t io;
      batch_offsets(P, tile * 4 + tid, &io, s_out + tid, s_col + tid);
      if constexpr ((FEAT & FEAT_TW4) != 0) {
        s_stp[tid] = tw4<T>(P, s_col[tid], N / 16);
        s_stp[4 + tid] = tw4<T>(P, s_col[tid], N / 2);
      }
    }
    // bounded wait for the staged tile; a wait that gives up flags the
    // failure for the host and stops further copies (the CTA still passes
    // every barrier, computing on whatever the staging area holds)
    if (!*abort_flag) {
      bool ok = false;
      for (long i = 0; i < (1L << 22); i++)
        if (mbar_try_wait(bar, it & 1u)) {
          ok = true;
          break;
        }
      if (!ok) {
        *abort_flag = (int)it + 1;
        if (lane == 0) atomicExch(&g_tma_wait_failed, 1);
      }
    }
    T2 v[16];
#pragma unroll
    for (int s = 0; s < 16; s++) {
      T2 x = stg[s * 1024 + rd0];
      if (cjin) x.y = -x.y;
      v[s] = x;
    }
    Dft<16>::template apply<T, T2>(v);
#pragma unroll
    for (int k = 1; k < 16; k++) v[k] = cmul(v[k], ld_tw(tw1 + (k - 1) * 16 + l));
    __syncwarp();  // every lane of the warp has read its staged values
    {
      T2 *wbase = stg + l * 1024 + wb;
#pragma unroll
      for (int k = 0; k < 16; k++) wbase[u ^ split_f<SMODE>(k)] = v[k];
      __syncwarp();
#pragma unroll
      for (int x = 0; x < 16; x++) v[x] = stg[x * 1024 + wb + (u ^ split_f<SMODE>(x))];
    }
    Dft<16>::template apply<T, T2>(v);  // lane l now holds Z[l + 16 k_hi], k_hi = 0..15
    // release the slice; the last warp issues the next tile's copies
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      const unsigned old = atomicAdd(cnt, 1u);
      if ((old & 31u) == 31u && tile + gridDim.x < ntiles && !*abort_flag) {
        __threadfence_block();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(tile + gridDim.x);
      }
    }
    T2 y[16];
    if constexpr (XM == 0) {
      // exchange of one real component at a time (x parts, then y parts)
      // through X viewed as 16384 floats: no thread holds more than 16
      // complex values at once
      T *Xf = (T *)X;
      nb_sync(4);  // the previous tile's readers are done with X
#pragma unroll
      for (int k = 0; k < 16; k++) Xf[((k & 1) ? xfw_o : xfw_e) + 16 * k] = v[k].x;
      nb_sync(1);
#pragma unroll
      for (int n0 = 0; n0 < 16; n0++) y[n0].x = Xf[((n0 & 1) ? xfr_o : xfr_e) + n0 * 256];
      nb_sync(2);
#pragma unroll
      for (int k = 0; k < 16; k++) Xf[((k & 1) ? xfw_o : xfw_e) + 16 * k] = v[k].y;
      nb_sync(3);
#pragma unroll
      for (int n0 = 0; n0 < 16; n0++) y[n0].y = Xf[((n0 & 1) ? xfr_o : xfr_e) + n0 * 256];
    } else {
      // two rounds of full complex values: round 1 k' < 128 (k_hi < 8),
      // round 2 the rest; the round-1 readers keep their round-2 values in
      // a stash instead of registers while they read
      T2 *stash = (T2 *)(abort_flag + 1) + si;
      nb_sync(4);  // the previous tile's round-2 readers are done with X
#pragma unroll
      for (int kh = 0; kh < 8; kh++) X[xw + 16 * kh] = v[kh];
      if (rround == 0) {
        if constexpr (XM == 2) {
          T2 hv[8];
#pragma unroll
          for (int kh = 0; kh < 8; kh++) hv[kh] = v[8 + kh];
          tm_st16(tstash, hv);
        } else {
#pragma unroll
          for (int kh = 0; kh < 8; kh++) stash[kh * 512] = v[8 + kh];
        }
        nb_sync(1);
#pragma unroll
        for (int n0 = 0; n0 < 16; n0++) y[n0] = X[((n0 & 1) ? xr_o : xr_e) + n0 * 128];
        nb_sync(2);  // round-1 reads done
        if constexpr (XM == 2) {
#pragma unroll
          for (int hq = 0; hq < 2; hq++) {
            T2 hv[4];
            tm_ld8(tstash + 8 * hq, hv);
#pragma unroll
            for (int kh = 0; kh < 4; kh++) X[xw + 16 * (4 * hq + kh)] = hv[kh];
          }
        } else {
#pragma unroll
          for (int kh = 0; kh < 8; kh++) X[xw + 16 * kh] = stash[kh * 512];
        }
        nb_arrive(3);
      } else {
        nb_arrive(1);
        nb_sync(2);
#pragma unroll
        for (int kh = 0; kh < 8; kh++) X[xw + 16 * kh] = v[8 + kh];
        nb_sync(3);
#pragma unroll
        for (int n0 = 0; n0 < 16; n0++) y[n0] = X[((n0 & 1) ? xr_o : xr_e) + n0 * 128];
      }
    }
    T2 hi = zero2<T2>(), lo = zero2<T2>();
    if constexpr ((FEAT & FEAT_TW4) != 0) tw4_parts<T>(P, s_col[pr], kr, hi, lo);
#pragma unroll
    for (int n0 = 1; n0 < 16; n0++) y[n0] = cmul(y[n0], ld_tw(tw2 + (n0 - 1) * 256 + kr));
    Dft<16>::template apply<T, T2>(y);
    rr_store<T, N, 2, FEAT>(P, y, kr, s_out[pr], s_col[pr], hi, lo, s_stp[pr], s_stp[4 + pr]);
  }
  // after a wait that gave up, give copies still in flight a bounded time to
  // land before the CTA's shared memory is released
  const int af = *abort_flag;
  if (af && tid == 0) {
    for (long i = 0; i < (1L << 22); i++)
      if (mbar_try_wait(bar, (unsigned)(af - 1) & 1u)) break;
  }
  if constexpr (XM == 2) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(*s_taddr) : "memory");
    }
  }
}

}  // namespace fftz

// ------------------------------------------------------------------- host

namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
int g_encode_state = 0;  // 0 unknown, 1 ready, -1 unavailable

bool encoder() {
  if (g_encode_state == 0) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess && fn) {
      g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
      g_encode_state = 1;
    } else {
      cudaGetLastError();
      g_encode_state = -1;
    }
  }
  return g_encode_state == 1;
}

template <typename T, int FEAT, int MODE>
const void *pick(int n) {
  switch (n) {
    case 256: return (const void *)&fftz::fft_tma_kernel<T, 256, FEAT, MODE>;
    case 512: return (const void *)&fftz::fft_tma_kernel<T, 512, FEAT, MODE>;
    case 1024: return (const void *)&fftz::fft_tma_kernel<T, 1024, FEAT, MODE>;
    case 2048: return (const void *)&fftz::fft_tma_kernel<T, 2048, FEAT, MODE>;
    case 4096: return (const void *)&fftz::fft_tma_kernel<T, 4096, FEAT, MODE>;
  }
  return nullptr;
}

template <typename T, int FEAT, int MODE>
const void *pick_pipe(int n) {
  switch (n) {
    case 512: return (const void *)&fftz::fft_tma_pipe_kernel<T, 512, FEAT, MODE>;
    case 1024: return (const void *)&fftz::fft_tma_pipe_kernel<T, 1024, FEAT, MODE>;
    case 2048: return (const void *)&fftz::fft_tma_pipe_kernel<T, 2048, FEAT, MODE>;
    case 4096: return (const void *)&fftz::fft_tma_pipe_kernel<T, 4096, FEAT, MODE>;
  }
  return nullptr;
}

const void *tma_pipe_kernel(int dtype, int n, int tw4, int mode) {
  if (dtype == 0)
    return tw4 ? (mode ? pick_pipe<float, 1, 1>(n) : pick_pipe<float, 1, 0>(n))
               : (mode ? pick_pipe<float, 0, 1>(n) : pick_pipe<float, 0, 0>(n));
  return tw4 ? (mode ? pick_pipe<double, 1, 1>(n) : pick_pipe<double, 1, 0>(n))
             : (mode ? pick_pipe<double, 0, 1>(n) : pick_pipe<double, 0, 0>(n));
}

const void *tma_rr_kernel(int dtype, int n, int tw4, int mode) {
  if (dtype != 0 || n != 4096) return nullptr;
  if (tw4) return mode ? (const void *)&fftz::fft_tma_rr_kernel<float, 4096, 1, 1>
                       : (const void *)&fftz::fft_tma_rr_kernel<float, 4096, 1, 0>;
  return mode ? (const void *)&fftz::fft_tma_rr_kernel<float, 4096, 0, 1>
              : (const void *)&fftz::fft_tma_rr_kernel<float, 4096, 0, 0>;
}


const void *tma_stream_kernel(int dtype, int n) {
  using fftz::fft_tma_stream_kernel;
  if (dtype == 0) switch (n) {
      case 256: return (const void *)&fft_tma_stream_kernel<float, 256, 0>;
      case 512: return (const void *)&fft_tma_stream_kernel<float, 512, 0>;
      case 1024: return (const void *)&fft_tma_stream_kernel<float, 1024, 0>;
      case 2048: return (const void *)&fft_tma_stream_kernel<float, 2048, 0>;
      case 4096: return (const void *)&fft_tma_stream_kernel<float, 4096, 0>;
      case 8192: return (const void *)&fft_tma_stream_kernel<float, 8192, 0>;
    }
  else switch (n) {
      case 256: return (const void *)&fft_tma_stream_kernel<double, 256, 0>;
      case 512: return (const void *)&fft_tma_stream_kernel<double, 512, 0>;
      case 1024: return (const void *)&fft_tma_stream_kernel<double, 1024, 0>;
      case 2048: return (const void *)&fft_tma_stream_kernel<double, 2048, 0>;
      case 4096: return (const void *)&fft_tma_stream_kernel<double, 4096, 0>;
    }
  return nullptr;
}

/* The streaming row kernel: plain row passes (no epilogue features) over
 * 16-byte aligned contiguous lines; -1 when the pass does not qualify. */
int launch_stream(const fftz_pass_t *p, void *stream) {
  if (p->variant != FFTZ_VAR_FAST || p->in_mode != 0 || p->ies != 1 || p->smem_tw || p->ind_in) return -1;
  const int64_t esz = p->dtype == 0 ? 8 : 16;
  if (p->tpc < 1 || p->ntf % p->tpc || ((uintptr_t)p->in & 15) || (p->n * esz) % 16) return -1;
  for (int d = 0; d < p->nbdims; d++)
    if ((p->ibs[d] * esz) % 16) return -1;
  const void *fn = tma_stream_kernel(p->dtype, (int)p->n);
  if (!fn) return -1;
  const size_t slot = ((size_t)p->tpc * p->sstride * esz + 127) & ~(size_t)127;
  const size_t smem = 2 * slot + 3 * 8 * (size_t)p->tpc + 128;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  static const void *opted[64][16];
  static int nopted[64], maxdyn[64][16];
  int s = -1;
  for (int i = 0; i < nopted[dev]; i++)
    if (opted[dev][i] == fn) s = i;
  if (s < 0) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return (int)cudaGetLastError();
    const int md = (int)(fftz_smem_limit() - (int64_t)fa.sharedSizeBytes);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
    if (e != cudaSuccess) return (int)e;
    if (nopted[dev] < 16) {
      s = nopted[dev]++;
      opted[dev][s] = fn;
      maxdyn[dev][s] = md;
    }
  }
  if (s < 0 || smem > (size_t)maxdyn[dev][s]) return -1;
  const dim3 block((unsigned)(p->tpc * p->tpt));
  int64_t ntiles = p->ntf / p->tpc;
  if (ntiles <= 0) return 0;
  static int nsm[64];
  if (!nsm[dev]) cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, (int)block.x, smem) != cudaSuccess || occ < 1) {
    cudaGetLastError();
    occ = 1;
  }
  const int64_t cap = (int64_t)occ * (nsm[dev] > 0 ? nsm[dev] : 148);
  const dim3 grid((unsigned)(ntiles < cap ? ntiles : cap));
  void *args[2] = {(void *)p, (void *)&ntiles};
  return (int)cudaLaunchKernel(fn, grid, block, args, smem, (cudaStream_t)stream);
}

template <int XM> const void *split_pick(int tw4, int mode, int omode) {
  using fftz::fft_tma_split_kernel;
  if (mode == 2)  // blocked input: the four-step's row pass (plain, transposed store)
    return (XM == 0 && !tw4 && omode == 1) ? (const void *)&fft_tma_split_kernel<float, 4096, 0, 2, 1, 0> : nullptr;
  if (tw4)
    return mode ? (omode ? (const void *)&fft_tma_split_kernel<float, 4096, 1, 1, 1, XM>
                         : (const void *)&fft_tma_split_kernel<float, 4096, 1, 1, 0, XM>)
                : (omode ? (const void *)&fft_tma_split_kernel<float, 4096, 1, 0, 1, XM>
                         : (const void *)&fft_tma_split_kernel<float, 4096, 1, 0, 0, XM>);
  return mode ? (omode ? (const void *)&fft_tma_split_kernel<float, 4096, 0, 1, 1, XM>
                       : (const void *)&fft_tma_split_kernel<float, 4096, 0, 1, 0, XM>)
              : (omode ? (const void *)&fft_tma_split_kernel<float, 4096, 0, 0, 1, XM>
                       : (const void *)&fft_tma_split_kernel<float, 4096, 0, 0, 0, XM>);
}

/* Launches a 4096-point float pass through the 16 x 256 split kernel; -1
 * (nothing launched) when the pass or its buffers do not qualify. */
int launch_split(const fftz_pass_t *p, void *stream) {
  if (p->n != 4096 || p->dtype != 0 || p->tpc != 4 || p->tpt != 256) return -1;
  if (p->variant != FFTZ_VAR_FAST && p->variant != FFTZ_VAR_FAST_TW4) return -1;
  if (p->in_kind != FFTZ_IN_COMPLEX || p->out_kind != FFTZ_OUT_COMPLEX) return -1;
  if ((p->flags & ~(FFTZ_F_CONJ_IN | FFTZ_F_CONJ_OUT | FFTZ_F_TW4 | FFTZ_F_BLK4_IN | FFTZ_F_BLK4_OUT)) != 0) return -1;
  if (p->nbdims < 1 || p->nbdims > 2 || p->ind_in || p->ind_out) return -1;
  const int64_t b0 = p->bdim[0], b1 = p->nbdims == 2 ? p->bdim[1] : 1;
  if (b0 % 4 || p->ntf != b0 * b1 || b0 > 0x7fffffff || b1 > 0x7fffffff) return -1;
  if (((uintptr_t)p->in & 15) != 0 || !encoder()) return -1;
  const int blk_in = (p->flags & FFTZ_F_BLK4_IN) != 0;
  const int mode = blk_in ? 2 : p->in_mode, omode = p->out_mode;
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
  CUtensorMapSwizzle swz;
  int rank = 4;
  if (mode == 2) {
    /* blocked rows: element e = n0 + 16 m of row 4 K + r at K * 4 n + 4 e + r
     * past the line: dims (r, m, n0, K, line) */
    if (p->ies != 1 || p->ibs[0] != 4096) return -1;
    dims[0] = 4;
    dims[1] = 256;
    dims[2] = 16;
    dims[3] = (cuuint64_t)(b0 / 4);
    strides[0] = 64 * 8;
    strides[1] = 4 * 8;
    strides[2] = (cuuint64_t)4 * 4096 * 8;
    box[0] = 4;
    box[1] = 16;
    box[2] = 16;
    box[3] = 1;
    swz = CU_TENSOR_MAP_SWIZZLE_32B;
    rank = 5;
  } else if (mode == 1) {
    /* element e = n0 + 16 m of column c: dims (c, m, n0, outer batch) */
    if (p->ibs[0] != 1 || p->ies <= 0) return -1;
    dims[0] = (cuuint64_t)b0;
    dims[1] = 256;
    dims[2] = 16;
    strides[0] = (cuuint64_t)(16 * p->ies * 8);
    strides[1] = (cuuint64_t)(p->ies * 8);
    box[0] = 4;
    box[1] = 16;
    box[2] = 16;
    swz = CU_TENSOR_MAP_SWIZZLE_32B;
  } else {
    /* element e = n0 + 16 m of row r: dims (n0, m, r, outer batch) */
    if (p->ies != 1 || p->ibs[0] <= 0) return -1;
    dims[0] = 16;
    dims[1] = 256;
    dims[2] = (cuuint64_t)b0;
    strides[0] = 128;
    strides[1] = (cuuint64_t)(p->ibs[0] * 8);
    box[0] = 16;
    box[1] = 16;
    box[2] = 4;
    swz = CU_TENSOR_MAP_SWIZZLE_128B;
  }
  if (mode == 2) {
    dims[4] = (cuuint64_t)b1;
    box[4] = 1;
    strides[3] = p->nbdims == 2 ? (cuuint64_t)(p->ibs[1] * 8) : (cuuint64_t)b0 * 4096 * 8;
  } else {
    dims[3] = (cuuint64_t)b1;
    box[3] = 1;
    strides[2] = p->nbdims == 2 ? (cuuint64_t)(p->ibs[1] * 8) : (cuuint64_t)(4096 * 8 * (mode == 1 ? p->ies : 1));
  }
  if (p->nbdims == 2 && p->ibs[1] <= 0) return -1;
  for (int i = 0; i < rank - 1; i++)
    if (strides[i] % 16 || strides[i] >= (1ULL << 40)) return -1;
  CUtensorMap map;
  if (g_encode(&map, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)rank, (void *)p->in, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return -1;
  const int xm = p->use_tma == 5 ? 1 : p->use_tma == 6 ? 2 : 0;
  const int tw4 = p->variant == FFTZ_VAR_FAST_TW4;
  const void *fn = xm == 1 ? split_pick<1>(tw4, mode, omode)
                 : xm == 2 ? split_pick<2>(tw4, mode, omode)
                           : split_pick<0>(tw4, mode, omode);
  if (!fn) return -1;
  const size_t smem = (size_t)fftz::kSplitSmem + (xm == 1 ? fftz::kSplitStash : 16) + 1024;
  static const void *opted[64][32];
  static int nopted[64], nsm[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  int seen = 0;
  for (int i = 0; i < nopted[dev]; i++)
    if (opted[dev][i] == fn) seen = 1;
  if (!seen) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    if (nopted[dev] < 32) opted[dev][nopted[dev]++] = fn;
  }
  if (!nsm[dev]) cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
  int64_t ntiles = p->ntf / 4;
  const int64_t cap = nsm[dev] > 0 ? nsm[dev] : 148;
  const dim3 grid((unsigned)(ntiles < cap ? ntiles : cap)), block(1024);
  void *args[3] = {(void *)p, (void *)&map, (void *)&ntiles};
  return (int)cudaLaunchKernel(fn, grid, block, args, smem, (cudaStream_t)stream);
}

const void *tma_kernel(int dtype, int n, int tw4, int mode) {
  if (dtype == 0)
    return tw4 ? (mode ? pick<float, 1, 1>(n) : pick<float, 1, 0>(n))
               : (mode ? pick<float, 0, 1>(n) : pick<float, 0, 0>(n));
  return tw4 ? (mode ? pick<double, 1, 1>(n) : pick<double, 1, 0>(n))
             : (mode ? pick<double, 0, 1>(n) : pick<double, 0, 0>(n));
}

}  // namespace

extern "C" {

/* Launches pass p through the TMA kernel. Returns -1 (nothing launched) when
 * the pass or its buffers do not qualify, else a cudaError_t value. */
int fftz_launch_pass_tma(const fftz_pass_t *p, void *stream) {
  if (p->variant != FFTZ_VAR_FAST && p->variant != FFTZ_VAR_FAST_TW4) return -1;
  if (p->in_kind != FFTZ_IN_COMPLEX || p->nbdims < 1 || p->nbdims > 2 || p->ind_in) return -1;
  const int mode = p->in_mode;
  const int64_t esz = p->dtype == 0 ? 8 : 16, ce = esz / 8;
  const int64_t b0 = p->bdim[0], b1 = p->nbdims == 2 ? p->bdim[1] : 1;
  if (p->tpc < 1 || b0 % p->tpc || p->ntf != b0 * b1) return -1;
  if (((uintptr_t)p->in & 15) != 0) return -1;
  if (p->use_tma == 7) return launch_stream(p, stream);
  if (p->use_tma >= 4) {
    const int e = launch_split(p, stream);
    if (e >= 0) return e;
  }
  /* only the split kernels read or write the blocked intermediate (the host
   * drops the layout for an execute that cannot take them) */
  if (p->flags & (FFTZ_F_BLK4_IN | FFTZ_F_BLK4_OUT)) return (int)cudaErrorNotSupported;
  const int tw4 = p->variant == FFTZ_VAR_FAST_TW4;
  int rr = p->use_tma >= 3 && p->tpc * p->tpt <= 1024;
  const void *fn = rr ? tma_rr_kernel(p->dtype, p->n, tw4, mode) : nullptr;
  if (!fn) rr = 0;
  int pipe = !rr && p->use_tma == 2;
  if (pipe) fn = tma_pipe_kernel(p->dtype, p->n, tw4, mode);
  if (!fn) {
    pipe = 0;
    fn = tma_kernel(p->dtype, p->n, tw4, mode);
  }
  if (!fn || !encoder()) return -1;
  const int64_t n = p->n;
  const int64_t ext = pipe ? n / 2 : n, boxe = ext < 256 ? ext : 256;
  cuuint64_t dims[3], strides[2];
  cuuint32_t box[3], estr[3] = {1, 1, 1};
  if (mode == 1) {
    /* columns: element e at e * ies, column c at c (contiguous), outer batch at ibs[1] */
    if (p->ibs[0] != 1 || (p->tpc * esz) % 16) return -1;
    dims[0] = (cuuint64_t)(b0 * ce);
    dims[1] = (cuuint64_t)n;
    strides[0] = (cuuint64_t)(p->ies * esz);
    box[0] = (cuuint32_t)(p->tpc * ce);
    box[1] = (cuuint32_t)boxe;
  } else {
    /* rows: element e contiguous, row r at ibs[0] */
    if (p->ies != 1) return -1;
    dims[0] = (cuuint64_t)(n * ce);
    dims[1] = (cuuint64_t)b0;
    strides[0] = (cuuint64_t)(p->ibs[0] * esz);
    box[0] = (cuuint32_t)(boxe * ce);
    box[1] = 1;
  }
  dims[2] = (cuuint64_t)b1;
  strides[1] = p->nbdims == 2 ? (cuuint64_t)(p->ibs[1] * esz) : (cuuint64_t)((strides[0] * dims[1] + 15) & ~15ULL);
  box[2] = 1;
  if (strides[0] % 16 || strides[1] % 16 || strides[0] >= (1ULL << 40) || strides[1] >= (1ULL << 40)) return -1;
  CUtensorMap map;
  if (g_encode(&map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, (void *)p->in, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return -1;
  static const void *opted[64][64];
  static int nopted[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  static int maxdyn[64][64];
  const size_t smem =
      rr ? ((size_t)p->tpc * n * esz + (size_t)p->tpc * fftz::kRrSsf1 * (esz / 2) + 8 * (size_t)p->tpc * 8 + 128)
      : pipe ? ((((size_t)p->tpc * p->sstride * esz + 127) & ~(size_t)127) + (size_t)p->tpc * (n / 2) * esz +
              4 * (size_t)p->tpc * 8 + 128)
           : (size_t)fftz_pass_smem_bytes(p) + 128;
  int slot = -1;
  for (int i = 0; i < nopted[dev]; i++)
    if (opted[dev][i] == fn) slot = i;
  if (slot < 0) {
    /* the kernel's static shared memory (its mbarrier) counts against the limit */
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return (int)cudaGetLastError();
    const int md = (int)(fftz_smem_limit() - (int64_t)fa.sharedSizeBytes);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
    if (e != cudaSuccess) return (int)e;
    if (nopted[dev] < 64) {
      slot = nopted[dev]++;
      opted[dev][slot] = fn;
      maxdyn[dev][slot] = md;
    }
  }
  if (slot < 0 || smem > (size_t)maxdyn[dev][slot]) return -1;
  const dim3 block((unsigned)(p->tpc * p->tpt));
  int64_t ntiles = p->ntf / p->tpc;
  dim3 grid((unsigned)ntiles);
  if (pipe || rr) {
    /* persistent: as many CTAs as are resident at once */
    static int nsm[64];
    if (!nsm[dev]) cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, (int)block.x, smem) != cudaSuccess || occ < 1) {
      cudaGetLastError();
      occ = 1;
    }
    const int64_t cap = (int64_t)occ * (nsm[dev] > 0 ? nsm[dev] : 148);
    grid.x = (unsigned)(ntiles < cap ? ntiles : cap);
  }
  void *args[3] = {(void *)p, (void *)&map, (void *)&ntiles};
  return (int)cudaLaunchKernel(fn, grid, block, args, smem, (cudaStream_t)stream);
}

/* 1 if some TMA tile gave up waiting for its copies since the last call (and
 * clears the flag); 0 otherwise. */
int fftz_tma_wait_failed(void) {
  int v = 0, z = 0;
  if (cudaMemcpyFromSymbol(&v, fftz::g_tma_wait_failed, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (v) cudaMemcpyToSymbol(fftz::g_tma_wait_failed, &z, sizeof(int));
  return v;
}

}  // extern "C"
