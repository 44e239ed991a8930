// Elementwise real-transform helpers for the lengths the one-pass real kernel
// does not cover (odd lengths with prime factors > 13, or half-lengths beyond
// one CTA). Each thread produces one output element of one line; lines are
// enumerated by the same batch-dimension decomposition as the FFT passes.
//
//   WIDEN_REAL   dense[e]   = (x[e*is], 0)                      e < n
//   WIDEN_PAIRS  dense[e]   = (x[2e*is], x[(2e+1)*is])          e < M
//   RECOMBINE    out[k*os]  = X_k from dense Z_k, Z_{M-k}        k <= M
//                (packed r2c, core/kernels/non_dft/real_packed/packed_rdft_common.h:42-63)
//   SEPARATE     dense[k]   = 2 Z_k from X_k, X_{M-k} at in     k < M
//                (packed c2r, packed_rdft_common.h:179-196)
//   HERM_EXPAND  dense[e]   = e <= n/2 ? X_e : conj(X_{n-e})     e < n
//   NARROW_HALF  out[k*os]  = dense[k]                           k <= n/2
//   REAL_OUT     out[e*os]  = re(dense[e])                       e < n
//   PAIRS_OUT    out[2e*os], out[(2e+1)*os] = dense[e]           e < M
// "dense" is a contiguous [line][len] complex scratch array.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fftz_kernels.h"

namespace fftz {

template <typename T> struct C2T;
template <> struct C2T<float> { typedef float2 type; };
template <> struct C2T<double> { typedef double2 type; };

template <typename T>
__global__ void __launch_bounds__(256) elem_kernel(const __grid_constant__ fftz_elem_t E) {
  typedef typename C2T<T>::type T2;
  const int64_t total = E.nlines * E.nout;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t line = g / E.nout;
    const int64_t e = g - line * E.nout;
    int64_t r = line, io = 0, oo = 0;
    for (int d = 0; d < E.nbdims; d++) {
      const int64_t q = r / E.bdim[d];
      const int64_t i = r - q * E.bdim[d];
      io += i * E.ibs[d];
      oo += i * E.obs[d];
      r = q;
    }
    const T *xr = (const T *)E.in + io;
    const T2 *xc = (const T2 *)E.in + io;
    T *yr = (T *)E.out + oo;
    T2 *yc = (T2 *)E.out + oo;
    const int64_t n = E.n;
    switch (E.mode) {
      case FFTZ_ELEM_WIDEN_REAL: {
        T2 v;
        v.x = xr[e * E.is];
        v.y = 0;
        yc[e * E.os] = v;
        break;
      }
      case FFTZ_ELEM_WIDEN_PAIRS: {
        T2 v;
        v.x = xr[2 * e * E.is];
        v.y = xr[(2 * e + 1) * E.is];
        yc[e * E.os] = v;
        break;
      }
      case FFTZ_ELEM_RECOMBINE: {
        const int64_t M = n;
        const T2 zk = xc[(e == M ? 0 : e) * E.is];
        const T2 zm = xc[(e == 0 ? 0 : M - e) * E.is];
        const T2 w = ((const T2 *)E.tab)[e];
        const T er = (T)0.5 * (zk.x + zm.x), ei = (T)0.5 * (zk.y - zm.y);
        const T orr = (T)0.5 * (zk.y + zm.y), oi = (T)0.5 * (zm.x - zk.x);
        T2 v;
        v.x = er + (w.x * orr - w.y * oi);
        v.y = ei + (w.x * oi + w.y * orr);
        yc[e * E.os] = v;
        break;
      }
      case FFTZ_ELEM_SEPARATE: {
        const int64_t M = n;
        const T2 xk = xc[e * E.is];
        const T2 xm = xc[(M - e) * E.is];
        const T2 w = ((const T2 *)E.tab)[e];  // e^{-2 pi i k / 2M}
        const T dr = xk.x - xm.x, di = xk.y + xm.y;
        const T er = w.x * dr + w.y * di, ei = w.x * di - w.y * dr;  // conj(w) * D
        T2 v;
        v.x = (xk.x + xm.x) - ei;
        v.y = (xk.y - xm.y) + er;
        yc[e * E.os] = v;
        break;
      }
      case FFTZ_ELEM_HERM_EXPAND: {
        const int64_t half = n / 2;
        T2 v = xc[(e <= half ? e : n - e) * E.is];
        if (e > half) v.y = -v.y;
        yc[e * E.os] = v;
        break;
      }
      case FFTZ_ELEM_NARROW_HALF:
        yc[e * E.os] = xc[e * E.is];
        break;
      case FFTZ_ELEM_REAL_OUT:
        yr[e * E.os] = xc[e * E.is].x;
        break;
      default: {  // FFTZ_ELEM_PAIRS_OUT
        const T2 v = xc[e * E.is];
        yr[2 * e * E.os] = v.x;
        yr[(2 * e + 1) * E.os] = v.y;
        break;
      }
    }
  }
}

}  // namespace fftz

extern "C" int fftz_launch_elem(const fftz_elem_t *e, void *stream) {
  const int64_t total = e->nlines * e->nout;
  if (total <= 0) return 0;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  void *args[1] = {(void *)e};
  const void *fn = e->dtype == 0 ? (const void *)&fftz::elem_kernel<float> : (const void *)&fftz::elem_kernel<double>;
  return (int)cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(256), args, 0, (cudaStream_t)stream);
}
