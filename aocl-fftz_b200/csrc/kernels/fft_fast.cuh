// Compile-time power-of-two shared-memory FFT kernel family.
//
// Same algorithm as the generic kernel (Stockham radix stages in registers with
// shared-memory exchanges), but N and the radix list are template parameters,
// so every stride, modulus and loop bound folds to a constant and each
// instantiation holds only the registers its own radices need. The radix list
// follows the reference's balanced power-of-two split: the fewest stages with
// radix <= 16, exponents spread evenly, largest first
// (core/common/pow2_radix_decompose.c:122-150), e.g. 4096 = 16*16*16,
// 2048 = 16*16*8.
//
// Loads come straight from HBM in the first stage and stores go straight to
// HBM from the last stage (complex elements only), with the lane map chosen per
// side: mode 0 runs lanes along elements (rows), mode 1 runs lanes along
// neighbouring transforms (columns). Feature bits (template FEAT) add:
//   FEAT_TW4   output k of column c times W_{tw4_n}^{c k} (four-step twiddle,
//              FP64 factors);
//   FEAT_TABS  load-side bound and table product (Bluestein pre-chirp and zero
//              padding) and store-side table product, bound and scale;
//   FEAT_SWEEP2 two sweeps of the stages with v = conj(v) * mid_tab[e] between
//              them (the spectrum product of a one-kernel Bluestein transform).
#pragma once
#include "fft_common.cuh"

namespace fftz {

__host__ __device__ constexpr int ct_log2(int n) {
  int k = 0;
  while ((1 << k) < n) k++;
  return k;
}
__host__ __device__ constexpr int ct_nstages(int n) { return n <= 1 ? 0 : ((ct_log2(n) + 3) / 4); }
__host__ __device__ constexpr int ct_radix(int n, int s) {
  return 1 << (ct_log2(n) / ct_nstages(n) + (s < ct_log2(n) % ct_nstages(n) ? 1 : 0));
}
__host__ __device__ constexpr int ct_ns(int n, int s) {
  int p = 1;
  for (int i = 0; i < s; i++) p *= ct_radix(n, i);
  return p;
}
__host__ __device__ constexpr int ct_tpt(int n) { return n >= 16 ? n / 16 : 1; }
// Block-size bound of an instantiation: room for several columns per CTA
// (1024 threads for float, 512 for double keeps the double kernels at <= 128
// registers).
template <typename T> __host__ __device__ constexpr int ct_lb() { return sizeof(T) == 4 ? 1024 : 512; }

enum { FEAT_TW4 = 1, FEAT_TABS = 2, FEAT_SWEEP2 = 4 };

template <typename T, int FEAT>
__device__ __forceinline__ void store_fast(const fftz_pass_t &P, typename Cplx<T>::type v, int kk, int64_t col,
                                           int64_t obase) {
  typedef typename Cplx<T>::type T2;
  if (FEAT & FEAT_TABS) {
    store_complex<T>(P, v, kk, col, obase);
    return;
  }
  if (FEAT & FEAT_TW4) v = cmul(v, tw4<T>(P, col, kk));
  if (P.flags & FFTZ_F_CONJ_OUT) v.y = -v.y;
  ((T2 *)P.out)[obase + (int64_t)kk * P.oes] = v;
}

template <typename T, int FEAT>
__device__ __forceinline__ typename Cplx<T>::type load_fast(const fftz_pass_t &P, const typename Cplx<T>::type *gin,
                                                            int e, int64_t col, bool valid) {
  typedef typename Cplx<T>::type T2;
  T2 x = zero2<T2>();
  if (FEAT & FEAT_TABS) {
    const int64_t li = (int64_t)e * P.pre_es + col * P.pre_cs;
    if (valid && (P.pre_n == 0 || li < P.pre_n)) {
      x = gin[(int64_t)e * P.ies];
      if (P.flags & FFTZ_F_CONJ_IN) x.y = -x.y;
      if (P.flags & FFTZ_F_PRE_TAB) x = cmul(x, __ldg((const T2 *)P.pre_tab + li));
    }
  } else {
    if (valid) x = gin[(int64_t)e * P.ies];
    if (P.flags & FFTZ_F_CONJ_IN) x.y = -x.y;
  }
  return x;
}

template <typename T, int N, int S, int FEAT, bool FIRST, bool LAST>
__device__ __forceinline__ void fast_stage(const fftz_pass_t &P, typename Cplx<T>::type *sdata,
                                           const int64_t *s_in, const int64_t *s_out, const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  constexpr int R = ct_radix(N, S);
  constexpr int NS = ct_ns(N, S);
  constexpr int NB = kMaxE / R;
  constexpr int NBF = N / R;
  constexpr int TPT = ct_tpt(N);
  constexpr bool ALLV = (NB * TPT == NBF);
  constexpr int SH = Cplx<T>::PADSH;
  const int t = threadIdx.x;
  const int mode = FIRST ? P.in_mode : (LAST ? P.out_mode : 0);
  int p, j;
  if (mode == 0) {
    p = t / TPT;
    j = t - p * TPT;
  } else {
    p = t % P.tpc;
    j = t / P.tpc;
  }
  T2 *sd = sdata + (size_t)p * P.sstride;
  const int64_t col = s_col[p];
  const bool valid = col >= 0;
  T2 v[NB][R];
  if (FIRST) {
    const T2 *gin = (const T2 *)P.in + s_in[p];
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * TPT;
      if (ALLV || b < NBF) {
#pragma unroll
        for (int r = 0; r < R; r++) v[q][r] = load_fast<T, FEAT>(P, gin, b + r * NBF, col, valid);
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * TPT;
      if (ALLV || b < NBF) {
#pragma unroll
        for (int r = 0; r < R; r++) v[q][r] = sd[phys<SH>(b + r * NBF)];
      }
    }
    __syncthreads();
  }
  const T2 *tw = (const T2 *)P.tw + P.tw_off[S];
#pragma unroll
  for (int q = 0; q < NB; q++) {
    const int b = j + q * TPT;
    if (ALLV || b < NBF) {
      const int k = b & (NS - 1);
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], __ldg(tw + (r - 1) * NS + k));
      }
      Dft<R>::template apply<T, T2>(v[q]);
      const int d0 = (b - k) * R + k;
      if (LAST) {
        if (valid) {
#pragma unroll
          for (int r = 0; r < R; r++) store_fast<T, FEAT>(P, v[q][r], d0 + r * NS, col, s_out[p]);
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) sd[phys<SH>(d0 + r * NS)] = v[q][r];
      }
    }
  }
  if (!LAST) __syncthreads();
}

// Stage S of sweep SW out of NSW sweeps; HBM is touched only by the first
// stage of the first sweep and the last stage of the last sweep.
template <typename T, int N, int S, int NST, int SW, int NSW, int FEAT> struct FastStages {
  static __device__ __forceinline__ void run(const fftz_pass_t &P, typename Cplx<T>::type *sdata,
                                             const int64_t *s_in, const int64_t *s_out, const int64_t *s_col) {
    fast_stage<T, N, S, FEAT, (S == 0 && SW == 0), (S == NST - 1 && SW == NSW - 1)>(P, sdata, s_in, s_out, s_col);
    FastStages<T, N, S + 1, NST, SW, NSW, FEAT>::run(P, sdata, s_in, s_out, s_col);
  }
};
template <typename T, int N, int NST, int SW, int NSW, int FEAT> struct FastStages<T, N, NST, NST, SW, NSW, FEAT> {
  static __device__ __forceinline__ void run(const fftz_pass_t &, typename Cplx<T>::type *, const int64_t *,
                                             const int64_t *, const int64_t *) {}
};

template <typename T, int N, int FEAT>
__global__ void __launch_bounds__(ct_lb<T>()) fft_fast_kernel(const __grid_constant__ fftz_pass_t P) {
  typedef typename Cplx<T>::type T2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *sdata = (T2 *)smem_raw;
  int64_t *s_in = (int64_t *)(sdata + (size_t)P.tpc * P.sstride);
  int64_t *s_out = s_in + P.tpc;
  int64_t *s_col = s_out + P.tpc;
  const int64_t tf0 = (int64_t)blockIdx.x * P.tpc;
  for (int p = threadIdx.x; p < P.tpc; p += blockDim.x) {
    const int64_t b = tf0 + p;
    int64_t io = 0, oo = 0, col = -1;
    if (b < P.ntf) {
      int64_t r = b;
      col = 0;
      for (int d = 0; d < P.nbdims; d++) {
        const int64_t q = r / P.bdim[d];
        const int64_t i = r - q * P.bdim[d];
        if (d == 0) col = i;
        io += i * P.ibs[d];
        oo += i * P.obs[d];
        r = q;
      }
    }
    s_in[p] = io;
    s_out[p] = oo;
    s_col[p] = col;
  }
  __syncthreads();
  if (FEAT & FEAT_SWEEP2) {
    constexpr int SH = Cplx<T>::PADSH;
    FastStages<T, N, 0, ct_nstages(N), 0, 2, FEAT>::run(P, sdata, s_in, s_out, s_col);
    const T2 *mt = (const T2 *)P.mid_tab;
    for (int i = threadIdx.x; i < P.tpc * N; i += blockDim.x) {
      const int p = i / N;
      const int e = i - p * N;
      T2 *a = sdata + (size_t)p * P.sstride + phys<SH>(e);
      T2 v = *a;
      v.y = -v.y;
      *a = cmul(v, __ldg(mt + e));
    }
    __syncthreads();
    FastStages<T, N, 0, ct_nstages(N), 1, 2, FEAT>::run(P, sdata, s_in, s_out, s_col);
  } else {
    FastStages<T, N, 0, ct_nstages(N), 0, 1, FEAT>::run(P, sdata, s_in, s_out, s_col);
  }
}

}  // namespace fftz
