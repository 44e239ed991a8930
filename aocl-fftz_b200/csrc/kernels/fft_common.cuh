// Device helpers shared by the shared-memory FFT kernels (generic and
// compile-time power-of-two families).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "codelets.cuh"
#include "fftz_kernels.h"

namespace fftz {

template <typename T> struct Cplx;
template <> struct Cplx<float> {
  typedef float2 type;
  enum { PADSH = 4 };  // one pad slot per 16 complex (128 B) of shared memory
};
template <> struct Cplx<double> {
  typedef double2 type;
  enum { PADSH = 3 };  // one pad slot per 8 complex (128 B)
};

constexpr int kMaxE = 16;  // complex values a thread holds in one stage

template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

template <int SH> __device__ __forceinline__ int phys(int i) { return i + (i >> SH); }

template <typename T2> __device__ __forceinline__ T2 zero2() {
  T2 z;
  z.x = 0;
  z.y = 0;
  return z;
}

// Input / output element offsets and column index of transform b of a pass
// (col = index in bdim[0], -1 past the end). Batch dim ind_dim may be
// indirect: its index then selects ind_in / ind_out entries.
__device__ __forceinline__ void batch_offsets(const fftz_pass_t &P, int64_t b, int64_t *io_, int64_t *oo_,
                                              int64_t *col_) {
  int64_t io = 0, oo = 0, col = -1;
  if (b < P.ntf) {
    int64_t r = b;
    col = 0;
    for (int d = 0; d < P.nbdims; d++) {
      const int64_t q = r / P.bdim[d];
      const int64_t i = r - q * P.bdim[d];
      if (d == 0) col = i;
      const bool ind = d == P.ind_dim;
      io += (ind && P.ind_in) ? P.ind_in[i] : i * P.ibs[d];
      oo += (ind && P.ind_out) ? P.ind_out[i] : i * P.obs[d];
      r = q;
    }
  }
  *io_ = io;
  *oo_ = oo;
  *col_ = col;
}

// W_N^r for r = (col * k) mod N from two tables (factors formed in FP64, held
// in the working precision): W = hi[r / L] * lo[r % L]. Powers of two take a
// 32-bit path (r = col * k mod 2^32 reduced mod N is exact for N <= 2^31).
template <typename T>
__device__ __forceinline__ typename Cplx<T>::type tw4(const fftz_pass_t &P, int64_t col, int64_t k) {
  typedef typename Cplx<T>::type T2;
  const int64_t N = P.tw4_n, L = P.tw4_l;
  int64_t hi, lo;
  if (((N & (N - 1)) == 0) && N <= 0x80000000LL && ((L & (L - 1)) == 0)) {
    const unsigned r = ((unsigned)col * (unsigned)k) & (unsigned)(N - 1);
    hi = r >> (31 - __clz((int)L));
    lo = r & (unsigned)(L - 1);
  } else {
    const int64_t r = (col * k) % N;
    hi = r / L;
    lo = r - hi * L;
  }
  return cmul(__ldg((const T2 *)P.tw4_hi + hi), __ldg((const T2 *)P.tw4_lo + lo));
}

// Epilogue for one complex output element kk of a transform whose column
// index is col and whose output base offset is obase.
template <typename T>
__device__ __forceinline__ void store_complex(const fftz_pass_t &P, typename Cplx<T>::type v, int64_t kk,
                                              int64_t col, int64_t obase) {
  typedef typename Cplx<T>::type T2;
  const int f = P.flags;
  if (f & FFTZ_F_TW4) v = cmul(v, tw4<T>(P, col, kk));
  if (f & FFTZ_F_CONJ_OUT) v.y = -v.y;
  const int64_t li = kk * P.post_es + col * P.post_cs;
  if (P.post_n > 0 && li >= P.post_n) return;
  if (f & FFTZ_F_POST_TAB) v = cmul(v, __ldg((const T2 *)P.post_tab + li));
  if (f & FFTZ_F_SCALE) {
    v.x = (T)(v.x * P.scale);
    v.y = (T)(v.y * P.scale);
  }
  ((T2 *)P.out)[obase + kk * P.oes] = v;
}

}  // namespace fftz
