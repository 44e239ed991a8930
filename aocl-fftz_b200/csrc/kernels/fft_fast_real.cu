// Compile-time power-of-two kernel for real lines (packed r2c / c2r).
//
// A real line of n0 = 2N points is transformed as the N-point complex FFT of
// its packed pairs plus a Hermitian recombine (r2c), or a Hermitian separate
// plus the N-point complex FFT (c2r): the reference's packed real solver
// (core/solvers/real/packed_solver_rdft.c:154-226, recombine and separate in
// core/kernels/non_dft/real_packed/packed_rdft_common.h:42-340). The load and
// store phases are the generic kernel's (every real element kind, the
// recombine and separate with the half-length twiddles of P.rtw); between
// them the N-point FFT runs as the compile-time radix-16/8/4/2 stages of the
// power-of-two kernels, entirely in shared memory (no stage reads or writes
// HBM), instead of the generic kernel's runtime radix loop.
#include "fft_fast.cuh"
#include "fft_generic.cuh"

namespace fftz {

// Row-mapped phases with the length known at compile time: one line of the
// tile after the other with the threads along its elements (line pointers
// and checks hoisted), the one element a line has beyond a multiple of the
// power-of-two length (the Nyquist bin of r2c, the middle pair of c2r) for
// all lines in one extra step, pairs moved as one vector access when the
// line is aligned, the half spectrum stored directly when the pass has no
// epilogue tables. Same arithmetic as the generic load_phase / store_phase.

// r2c load: real pairs (x[2e], x[2e+1]) -> Z[e]
template <typename T, int N>
__device__ __forceinline__ void r2c_load(const fftz_pass_t &P, typename Cplx<T>::type *sdata, const int64_t *s_in,
                                         const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const bool cj = (P.flags & FFTZ_F_CONJ_IN) != 0;
  for (int p = 0; p < P.tpc; p++) {
    T2 *sd = sdata + (size_t)p * P.sstride;
    const bool ok = s_col[p] >= 0;
    const T *g = (const T *)P.in + s_in[p];
    const bool vec = P.ies == 1 && ((uintptr_t)g & (sizeof(T2) - 1)) == 0;
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
      T2 x = zero2<T2>();
      if (ok) {
        if (vec) {
          x = ((const T2 *)g)[e];
        } else {
          x.x = g[(int64_t)(2 * e) * P.ies];
          x.y = g[(int64_t)(2 * e + 1) * P.ies];
        }
        if (cj) x.y = -x.y;
      }
      sd[phys<SH>(e)] = x;
    }
  }
  __syncthreads();
}

// r2c store: X_k = (Z_k + conj Z_{N-k})/2 - (i/2) W^k (Z_k - conj Z_{N-k}), k = 0..N
template <typename T, int N>
__device__ __forceinline__ void r2c_out(const fftz_pass_t &P, const typename Cplx<T>::type *sd, int k, int64_t col,
                                        int64_t obase, bool plain) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const T2 zk = sd[phys<SH>(k == N ? 0 : k)];
  const T2 zm = sd[phys<SH>(k == 0 ? 0 : N - k)];
  const T2 w = __ldg((const T2 *)P.rtw + k);
  const T er = (T)0.5 * (zk.x + zm.x), ei = (T)0.5 * (zk.y - zm.y);
  const T orr = (T)0.5 * (zk.y + zm.y), oi = (T)0.5 * (zm.x - zk.x);
  T2 x;
  x.x = er + (w.x * orr - w.y * oi);
  x.y = ei + (w.x * oi + w.y * orr);
  if (plain)
    ((T2 *)P.out)[obase + k] = x;
  else
    store_complex<T>(P, x, k, col, obase);
}

template <typename T, int N>
__device__ __forceinline__ void r2c_store(const fftz_pass_t &P, const typename Cplx<T>::type *sdata,
                                          const int64_t *s_out, const int64_t *s_col) {
  const bool plain = (P.flags & (FFTZ_F_TW4 | FFTZ_F_CONJ_OUT | FFTZ_F_POST_TAB | FFTZ_F_SCALE)) == 0 &&
                     P.post_n == 0 && P.oes == 1;
  for (int p = 0; p < P.tpc; p++) {
    const int64_t col = s_col[p];
    if (col < 0) continue;
    const int64_t ob = s_out[p];
    for (int k = threadIdx.x; k < N; k += blockDim.x) r2c_out<T, N>(P, sdata + (size_t)p * P.sstride, k, col, ob, plain);
  }
  for (int p = threadIdx.x; p < P.tpc; p += blockDim.x)  // the Nyquist bins
    if (s_col[p] >= 0) r2c_out<T, N>(P, sdata + (size_t)p * P.sstride, N, s_col[p], s_out[p], plain);
}

// c2r load with the Hermitian separate fused: pair (k, N-k) of X[0..N] ->
// 2 conj(Z[k]), 2 conj(Z[N-k]) (the backward conjugation included)
template <typename T, int N>
__device__ __forceinline__ void c2r_pair(const fftz_pass_t &P, typename Cplx<T>::type *sd,
                                         const typename Cplx<T>::type *g, int k, bool ok) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const int km = (k == 0) ? N : N - k;
  T2 zk = zero2<T2>(), zm = zero2<T2>();
  if (ok) {
    const T2 xk = g[(int64_t)k * P.ies];
    const T2 xm = g[(int64_t)km * P.ies];
    const T2 w = __ldg((const T2 *)P.rtw + k);  // e^{-2 pi i k / 2N}
    const T dr = xk.x - xm.x, di = xk.y + xm.y;
    const T er = w.x * dr + w.y * di, ei = w.x * di - w.y * dr;  // conj(w) (X_k - conj X_m)
    zk.x = (xk.x + xm.x) - ei;
    zk.y = -((xk.y - xm.y) + er);
    const T dr2 = xm.x - xk.x, di2 = xm.y + xk.y;
    const T er2 = -(w.x * dr2 - w.y * di2), ei2 = -(w.x * di2 + w.y * dr2);  // -w (X_m - conj X_k)
    zm.x = (xm.x + xk.x) - ei2;
    zm.y = -((xm.y - xk.y) + er2);
  }
  if (k != 0 && km != k) sd[phys<SH>(km)] = zm;
  sd[phys<SH>(k)] = zk;
}

template <typename T, int N>
__device__ __forceinline__ void c2r_load(const fftz_pass_t &P, typename Cplx<T>::type *sdata, const int64_t *s_in,
                                         const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  for (int p = 0; p < P.tpc; p++) {
    const bool ok = s_col[p] >= 0;
    const T2 *g = (const T2 *)P.in + s_in[p];
    for (int k = threadIdx.x; k < N / 2; k += blockDim.x) c2r_pair<T, N>(P, sdata + (size_t)p * P.sstride, g, k, ok);
  }
  for (int p = threadIdx.x; p < P.tpc; p += blockDim.x)  // the middle pairs (k = N/2)
    c2r_pair<T, N>(P, sdata + (size_t)p * P.sstride, (const T2 *)P.in + s_in[p], N / 2, s_col[p] >= 0);
  __syncthreads();
}

// c2r store: Z[k] -> real pairs (with the output conjugation and scale)
template <typename T, int N>
__device__ __forceinline__ void c2r_store(const fftz_pass_t &P, const typename Cplx<T>::type *sdata,
                                          const int64_t *s_out, const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const bool cj = (P.flags & FFTZ_F_CONJ_OUT) != 0, sc = (P.flags & FFTZ_F_SCALE) != 0;
  for (int p = 0; p < P.tpc; p++) {
    if (s_col[p] < 0) continue;
    const T2 *sd = sdata + (size_t)p * P.sstride;
    T *g = (T *)P.out + s_out[p];
    const bool vec = P.oes == 1 && ((uintptr_t)g & (sizeof(T2) - 1)) == 0;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
      T2 v = sd[phys<SH>(k)];
      if (cj) v.y = -v.y;
      if (sc) {
        v.x = (T)(v.x * P.scale);
        v.y = (T)(v.y * P.scale);
      }
      if (vec) {
        ((T2 *)g)[k] = v;
      } else {
        g[(int64_t)(2 * k) * P.oes] = v.x;
        g[(int64_t)(2 * k + 1) * P.oes] = v.y;
      }
    }
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(ct_lb<T>()) fft_fast_real_kernel(const __grid_constant__ fftz_pass_t P) {
  typedef typename Cplx<T>::type T2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *sdata = (T2 *)smem_raw;
  int64_t *s_in = (int64_t *)(sdata + (size_t)P.tpc * P.sstride);
  int64_t *s_out = s_in + P.tpc;
  int64_t *s_col = s_out + P.tpc;
  tile_offsets(P, (int64_t)blockIdx.x * P.tpc, s_in, s_out, s_col);
  __syncthreads();
  const bool rows = P.in_mode == 0 && P.out_mode == 0;
  const bool r2c = P.in_kind == FFTZ_IN_REAL_PAIRS;
  if (rows && r2c)
    r2c_load<T, N>(P, sdata, s_in, s_col);
  else if (rows && P.in_kind == FFTZ_IN_HERM_SEPARATE)
    c2r_load<T, N>(P, sdata, s_in, s_col);
  else
    load_phase<T>(P, sdata, s_in, s_col);  // ends with a barrier (after the c2r separate)
  // sweep 0 of 2: every stage reads and writes shared memory
  FastStages<T, N, 0, ct_nstages(N), 0, 2, 0, false>::run(P, sdata, s_in, s_out, s_col);
  if (rows && r2c)
    r2c_store<T, N>(P, sdata, s_out, s_col);
  else if (rows && P.out_kind == FFTZ_OUT_REAL_PAIRS)
    c2r_store<T, N>(P, sdata, s_out, s_col);
  else
    store_phase<T>(P, sdata, s_out, s_col);
}

}  // namespace fftz

namespace {

template <typename T> const void *pick_real(int log2n) {
  switch (log2n) {
    case 3: return (const void *)&fftz::fft_fast_real_kernel<T, 8>;
    case 4: return (const void *)&fftz::fft_fast_real_kernel<T, 16>;
    case 5: return (const void *)&fftz::fft_fast_real_kernel<T, 32>;
    case 6: return (const void *)&fftz::fft_fast_real_kernel<T, 64>;
    case 7: return (const void *)&fftz::fft_fast_real_kernel<T, 128>;
    case 8: return (const void *)&fftz::fft_fast_real_kernel<T, 256>;
    case 9: return (const void *)&fftz::fft_fast_real_kernel<T, 512>;
    case 10: return (const void *)&fftz::fft_fast_real_kernel<T, 1024>;
    case 11: return (const void *)&fftz::fft_fast_real_kernel<T, 2048>;
    case 12: return (const void *)&fftz::fft_fast_real_kernel<T, 4096>;
  }
  return nullptr;
}

}  // namespace

/* The compile-time real-line kernel for complex length 2^log2n (real length
 * 2^(log2n + 1)), 8 <= 2^log2n <= 4096, or NULL. */
extern "C" const void *fftz_fast_real_kernel(int dtype, int log2n) {
  return dtype == 0 ? pick_real<float>(log2n) : pick_real<double>(log2n);
}
