#pragma once
// Shared-memory FFT kernel for sm_100a (runtime radix list, every element kind).
//
// One CTA holds tf_per_cta whole transforms of length n in shared memory. The
// transform is a sequence of Stockham radix-R stages (R in {2,3,4,5,7,8,11,13,16},
// butterflies from codelets.cuh): each thread pulls its butterflies' R inputs
// at stride n/R, multiplies by the stage twiddles W_{Ns*R}^{k*r}, runs the
// register DFT and writes the R outputs at stride Ns into the auto-sorted
// position, so the result lands in natural order without a bit-reversal pass.
//
// The first stage can read straight from HBM (fuse_load) and the last stage can
// write straight to HBM (fuse_store): with lanes mapped along elements (mode 0)
// or along neighbouring transforms (mode 1), both accesses are coalesced for
// rows (unit element stride) and for columns (unit batch stride) respectively.
// Other element kinds go through a load/store phase with a separate thread map.
//
// The backward transform is conj(FFT(conj(x))): conjugation is fused into the
// load and the store, so only forward codelets and forward twiddles exist.
// The reference counterpart of this kernel is the pow2 iterative solver
// (core/solvers/complex/pow2_iterative_solver_dft.c:275-380) together with the
// radix and twiddle codelets it calls (core/kernels/dft/c2c, tw_c2c_fwd/bwd).
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_common.cuh"

namespace fftz {

// One Stockham stage of radix R over the transform this thread is mapped to.
// ROLE 0..3 fixes at compile time whether the stage reads HBM (bit 0) and
// writes HBM (bit 1), so that the shared-memory-only middle stages compile
// without the HBM load and epilogue code (measured on B200: float 5-15%
// faster); ROLE 4 takes both from the runtime flags (measured faster for
// double, whose per-role copies lose more to the call convention).
template <typename T, int R, int ROLE>
__device__ __noinline__ void run_stage(const fftz_pass_t &P, typename Cplx<T>::type *sdata, int s, int Ns,
                                          bool from_g_rt, bool to_g_rt, int mode, const int64_t *s_in,
                                          const int64_t *s_out, const int64_t *s_col) {
  const bool from_g = ROLE == 4 ? from_g_rt : (ROLE & 1) != 0;
  const bool to_g = ROLE == 4 ? to_g_rt : (ROLE & 2) != 0;
  typedef typename Cplx<T>::type T2;
  constexpr int NB = kMaxE / R;
  constexpr int SH = Cplx<T>::PADSH;
  const int n = P.n;
  const int nb = n / R;
  const int t = threadIdx.x;
  // blocks wider than the tile (the persistent ragged executor) idle the rest
  const bool active = t < P.tpc * P.tpt;
  const int nbe = active ? nb : 0;
  int p, j;
  if (mode == 0) {
    p = t / P.tpt;
    j = t - p * P.tpt;
  } else {
    p = t % P.tpc;
    j = t / P.tpc;
  }
  if (!active) p = 0;
  T2 *sd = sdata + (size_t)p * P.sstride;
  const int64_t col = s_col[p];
  const bool valid = col >= 0;
  T2 v[NB][R];
  if (from_g) {
    const T2 *gin = (const T2 *)P.in + s_in[p];
    const bool cj = (P.flags & FFTZ_F_CONJ_IN) != 0;
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * P.tpt;
      if (b < nbe) {
#pragma unroll
        for (int r = 0; r < R; r++) {
          T2 x = zero2<T2>();
          if (valid) x = gin[(int64_t)(b + r * nb) * P.ies];
          if (cj) x.y = -x.y;
          v[q][r] = x;
        }
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * P.tpt;
      if (b < nbe) {
#pragma unroll
        for (int r = 0; r < R; r++) v[q][r] = sd[phys<SH>(b + r * nb)];
      }
    }
    __syncthreads();
  }
  const T2 *tw = (const T2 *)P.tw + P.tw_off[s];
#pragma unroll
  for (int q = 0; q < NB; q++) {
    const int b = j + q * P.tpt;
    if (b < nbe) {
      const int k = (int)((unsigned)b % (unsigned)Ns);
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], __ldg(tw + (r - 1) * Ns + k));
      }
      Dft<R>::template apply<T, T2>(v[q]);
      const int d0 = (b - k) * R + k;
      if (to_g) {
        if (valid) {
#pragma unroll
          for (int r = 0; r < R; r++) store_complex<T>(P, v[q][r], d0 + r * Ns, col, s_out[p]);
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) sd[phys<SH>(d0 + r * Ns)] = v[q][r];
      }
    }
  }
  if (!to_g) __syncthreads();
}

template <typename T, int R>
__device__ __forceinline__ void stage_radix(const fftz_pass_t &P, typename Cplx<T>::type *sdata, int s, int Ns,
                                            bool from_g, bool to_g, int mode, const int64_t *s_in,
                                            const int64_t *s_out, const int64_t *s_col) {
  if constexpr (sizeof(T) != 4) {
    run_stage<T, R, 4>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col);
  } else if (from_g) {
    if (to_g)
      run_stage<T, R, 3>(P, sdata, s, Ns, true, true, mode, s_in, s_out, s_col);
    else
      run_stage<T, R, 1>(P, sdata, s, Ns, true, false, mode, s_in, s_out, s_col);
  } else {
    if (to_g)
      run_stage<T, R, 2>(P, sdata, s, Ns, false, true, mode, s_in, s_out, s_col);
    else
      run_stage<T, R, 0>(P, sdata, s, Ns, false, false, mode, s_in, s_out, s_col);
  }
}

template <typename T>
__device__ __forceinline__ void stage_dispatch(const fftz_pass_t &P, typename Cplx<T>::type *sdata, int s,
                                               int Ns, bool from_g, bool to_g, int mode, const int64_t *s_in,
                                               const int64_t *s_out, const int64_t *s_col) {
  switch (P.radix[s]) {
    case 2: stage_radix<T, 2>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    case 3: stage_radix<T, 3>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    case 4: stage_radix<T, 4>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    case 5: stage_radix<T, 5>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    case 7: stage_radix<T, 7>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    case 8: stage_radix<T, 8>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    case 11: stage_radix<T, 11>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    case 13: stage_radix<T, 13>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
    default: stage_radix<T, 16>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col); break;
  }
}

// Global -> shared load phase for every element kind (no stage fused).
template <typename T>
__device__ void load_phase(const fftz_pass_t &P, typename Cplx<T>::type *sdata, const int64_t *s_in,
                           const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const int total = P.tpc * P.nload;
  const int f = P.flags;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int p, e;
    if (P.in_mode == 0) {
      p = i / P.nload;
      e = i - p * P.nload;
    } else {
      e = i / P.tpc;
      p = i - e * P.tpc;
    }
    const int64_t col = s_col[p];
    T2 x = zero2<T2>();
    if (col >= 0) {
      switch (P.in_kind) {
        case FFTZ_IN_COMPLEX: {
          const int64_t li = (int64_t)e * P.pre_es + col * P.pre_cs;
          if (P.pre_n == 0 || li < P.pre_n) {
            x = ((const T2 *)P.in)[s_in[p] + (int64_t)e * P.ies];
            if (f & FFTZ_F_CONJ_IN) x.y = -x.y;
            if (f & FFTZ_F_PRE_TAB) x = cmul(x, __ldg((const T2 *)P.pre_tab + li));
          }
          break;
        }
        case FFTZ_IN_REAL_PAIRS: {
          const T *g = (const T *)P.in + s_in[p];
          x.x = g[(int64_t)(2 * e) * P.ies];
          x.y = g[(int64_t)(2 * e + 1) * P.ies];
          if (f & FFTZ_F_CONJ_IN) x.y = -x.y;
          break;
        }
        case FFTZ_IN_REAL: {
          const T *g = (const T *)P.in + s_in[p];
          x.x = g[(int64_t)e * P.ies];
          break;
        }
        case FFTZ_IN_HERM_FULL: {
          const int half = P.n / 2;
          const int idx = (e <= half) ? e : P.n - e;
          x = ((const T2 *)P.in)[s_in[p] + (int64_t)idx * P.ies];
          if (e > half) x.y = -x.y;
          if (f & FFTZ_F_CONJ_IN) x.y = -x.y;
          break;
        }
        default: {  // FFTZ_IN_HERM_SEPARATE: raw X[e], e <= M
          x = ((const T2 *)P.in)[s_in[p] + (int64_t)e * P.ies];
          break;
        }
      }
    }
    sdata[(size_t)p * P.sstride + phys<SH>(e)] = x;
  }
  __syncthreads();
  if (P.in_kind == FFTZ_IN_HERM_SEPARATE) {
    // 2 Z[k] = (X_k + conj X_{M-k}) + i e^{+2 pi i k/2M} (X_k - conj X_{M-k}); the
    // conjugation of the backward transform is applied here as well.
    const int M = P.n;
    const int npairs = M / 2 + 1;
    const T2 *rtw = (const T2 *)P.rtw;
    for (int i = threadIdx.x; i < P.tpc * npairs; i += blockDim.x) {
      const int p = i / npairs;
      const int k = i - p * npairs;
      T2 *sd = sdata + (size_t)p * P.sstride;
      const int km = (k == 0) ? M : M - k;
      const T2 xk = sd[phys<SH>(k)];
      const T2 xm = sd[phys<SH>(km)];
      const T2 w = __ldg(rtw + k);  // e^{-2 pi i k / 2M}
      // E = conj(w) applied to D = X_k - conj(X_m)
      const T dr = xk.x - xm.x, di = xk.y + xm.y;
      const T er = w.x * dr + w.y * di, ei = w.x * di - w.y * dr;  // conj(w) * D
      T2 zk;
      zk.x = (xk.x + xm.x) - ei;
      zk.y = -((xk.y - xm.y) + er);  // conjugated
      if (k != 0 && km != k) {
        // Z[M-k]: S' = X_m + conj X_k, D' = X_m - conj X_k, twiddle conj(w_{M-k}) = -w
        const T dr2 = xm.x - xk.x, di2 = xm.y + xk.y;
        const T er2 = -(w.x * dr2 - w.y * di2), ei2 = -(w.x * di2 + w.y * dr2);  // -w * D'
        T2 zm;
        zm.x = (xm.x + xk.x) - ei2;
        zm.y = -((xm.y - xk.y) + er2);
        sd[phys<SH>(km)] = zm;
      }
      sd[phys<SH>(k)] = zk;
    }
    __syncthreads();
  }
}

// Shared -> global store phase for every element kind (no stage fused).
template <typename T>
__device__ void store_phase(const fftz_pass_t &P, typename Cplx<T>::type *sdata, const int64_t *s_out,
                            const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const int total = P.tpc * P.nstore;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int p, k;
    if (P.out_mode == 0) {
      p = i / P.nstore;
      k = i - p * P.nstore;
    } else {
      k = i / P.tpc;
      p = i - k * P.tpc;
    }
    const int64_t col = s_col[p];
    if (col < 0) continue;
    const T2 *sd = sdata + (size_t)p * P.sstride;
    switch (P.out_kind) {
      case FFTZ_OUT_COMPLEX:
      case FFTZ_OUT_HALF:
        store_complex<T>(P, sd[phys<SH>(k)], k, col, s_out[p]);
        break;
      case FFTZ_OUT_HALF_RECOMBINE: {
        // X_k = (Z_k + conj Z_{M-k})/2 - (i/2) W^k (Z_k - conj Z_{M-k}), Z_M = Z_0
        const int M = P.n;
        const T2 zk = sd[phys<SH>(k == M ? 0 : k)];
        const T2 zm = sd[phys<SH>(k == 0 ? 0 : M - k)];
        const T2 w = __ldg((const T2 *)P.rtw + k);
        const T er = (T)0.5 * (zk.x + zm.x), ei = (T)0.5 * (zk.y - zm.y);
        const T orr = (T)0.5 * (zk.y + zm.y), oi = (T)0.5 * (zm.x - zk.x);
        T2 x;
        x.x = er + (w.x * orr - w.y * oi);
        x.y = ei + (w.x * oi + w.y * orr);
        store_complex<T>(P, x, k, col, s_out[p]);
        break;
      }
      case FFTZ_OUT_REAL_PAIRS: {
        T2 v = sd[phys<SH>(k)];
        if (P.flags & FFTZ_F_CONJ_OUT) v.y = -v.y;
        if (P.flags & FFTZ_F_SCALE) {
          v.x = (T)(v.x * P.scale);
          v.y = (T)(v.y * P.scale);
        }
        T *g = (T *)P.out + s_out[p];
        g[(int64_t)(2 * k) * P.oes] = v.x;
        g[(int64_t)(2 * k + 1) * P.oes] = v.y;
        break;
      }
      default: {  // FFTZ_OUT_REAL
        T2 v = sd[phys<SH>(k)];
        T *g = (T *)P.out + s_out[p];
        g[(int64_t)k * P.oes] = (P.flags & FFTZ_F_SCALE) ? (T)(v.x * P.scale) : v.x;
        break;
      }
    }
  }
}

// One CTA-worth of a pass: transforms [blk * tpc, (blk + 1) * tpc).
template <typename T>
__device__ __forceinline__ void generic_tile(const fftz_pass_t &P, int64_t blk, unsigned char *smem_raw) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  T2 *sdata = (T2 *)smem_raw;
  int64_t *s_in = (int64_t *)(sdata + (size_t)P.tpc * P.sstride);
  int64_t *s_out = s_in + P.tpc;
  int64_t *s_col = s_out + P.tpc;
  const int64_t tf0 = blk * P.tpc;
  for (int p = threadIdx.x; p < P.tpc; p += blockDim.x) batch_offsets(P, tf0 + p, s_in + p, s_out + p, s_col + p);
  __syncthreads();

  const int nsweeps = (P.flags & FFTZ_F_MID_TAB) ? 2 : 1;
  if (!P.fuse_load) load_phase<T>(P, sdata, s_in, s_col);
  for (int sw = 0; sw < nsweeps; sw++) {
    int Ns = 1;
    for (int s = 0; s < P.nstages; s++) {
      const bool from_g = P.fuse_load && sw == 0 && s == 0;
      const bool to_g = P.fuse_store && sw == nsweeps - 1 && s == P.nstages - 1;
      const int mode = from_g ? P.in_mode : (to_g ? P.out_mode : 0);
      stage_dispatch<T>(P, sdata, s, Ns, from_g, to_g, mode, s_in, s_out, s_col);
      Ns *= P.radix[s];
    }
    if (sw == 0 && nsweeps == 2) {
      // between the sweeps: v = conj(v) * mid_tab[e] (spectrum product of Bluestein)
      const T2 *mt = (const T2 *)P.mid_tab;
      for (int i = threadIdx.x; i < P.tpc * P.n; i += blockDim.x) {
        const int p = i / P.n;
        const int e = i - p * P.n;
        const int64_t c = s_col[p];
        if (c < 0) continue;
        T2 *a = sdata + (size_t)p * P.sstride + phys<SH>(e);
        T2 v = *a;
        v.y = -v.y;
        *a = cmul(v, __ldg(mt + e + c * P.mid_cs));
      }
      __syncthreads();
    }
  }
  if (!P.fuse_store) store_phase<T>(P, sdata, s_out, s_col);
}

// ------------------------------------------------------------ ping-pong tile
//
// Runtime-radix stages over two shared-memory buffers per transform (stage s
// reads one, writes the other): every stage is a loop in which a thread takes
// one radix-R butterfly at a time, so only R values are live, and the
// butterflies of all the CTA's transforms are spread over all its threads
// (item i -> transform p and butterfly bf by multiply-high division with
// per-stage reciprocals, no runtime / or %). One barrier per stage. Used when
// both buffers fit shared memory; longer lines keep the in-place tile above.

// m = ceil(2^32 / d) for d > 1 (0 for d = 1): x / d = umulhi(x, m) exactly
// while x * d < 2^32, which holds for every index here (x * d < 2^31)
__host__ __device__ __forceinline__ uint32_t pp_magic(uint32_t d) {
  return d <= 1 ? 0u : (uint32_t)((0xFFFFFFFFull + d) / d);
}
__device__ __forceinline__ int pp_div(int x, uint32_t m) { return m ? (int)__umulhi((uint32_t)x, m) : x; }

// One stage of radix R. MAP (first / last fused stage): 0 lanes along
// elements (rows), 1 lanes along transforms (columns).
template <typename T, int R, bool FROMG, bool TOG, int MAP>
__device__ __forceinline__ void pp_stage(const fftz_pass_t &P, const typename Cplx<T>::type *src,
                                         typename Cplx<T>::type *dst, int s, int Ns, uint32_t mNs, int nbf,
                                         uint32_t mnbf, uint32_t mtpc, const int64_t *s_in, const int64_t *s_out,
                                         const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const int tpc = P.tpc, sst = P.sstride;
  const int total = tpc * nbf;
  const T2 *tw = (const T2 *)P.tw + P.tw_off[s];
  const bool cjin = FROMG && (P.flags & FFTZ_F_CONJ_IN) != 0;
  // stores with at most a conjugation take the direct path
  const bool plain_out =
      TOG && (P.flags & (FFTZ_F_TW4 | FFTZ_F_POST_TAB | FFTZ_F_SCALE)) == 0 && P.post_n == 0;
  const bool cjout = TOG && (P.flags & FFTZ_F_CONJ_OUT) != 0;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int p, bf;
    if (MAP == 1) {
      bf = pp_div(i, mtpc);
      p = i - bf * tpc;
    } else {
      p = pp_div(i, mnbf);
      bf = i - p * nbf;
    }
    T2 v[R];
    if (FROMG) {
      const int64_t col = s_col[p];
      const T2 *gin = (const T2 *)P.in + s_in[p];
#pragma unroll
      for (int r = 0; r < R; r++) {
        T2 x = zero2<T2>();
        if (col >= 0) x = gin[(int64_t)(bf + r * nbf) * P.ies];
        if (cjin) x.y = -x.y;
        v[r] = x;
      }
    } else {
      const T2 *sp = src + (size_t)p * sst;
#pragma unroll
      for (int r = 0; r < R; r++) v[r] = sp[phys<SH>(bf + r * nbf)];
    }
    const int g = pp_div(bf, mNs);
    const int k = bf - g * Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; r++) v[r] = cmul(v[r], __ldg(tw + (r - 1) * Ns + k));
    }
    Dft<R>::template apply<T, T2>(v);
    const int d0 = g * Ns * R + k;
    if (TOG) {
      const int64_t col = s_col[p];
      if (col >= 0) {
        if (plain_out) {
          T2 *gout = (T2 *)P.out + s_out[p];
          const int64_t oes = P.oes;
#pragma unroll
          for (int r = 0; r < R; r++) {
            T2 y = v[r];
            if (cjout) y.y = -y.y;
            gout[(int64_t)(d0 + r * Ns) * oes] = y;
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) store_complex<T>(P, v[r], d0 + r * Ns, col, s_out[p]);
        }
      }
    } else {
      T2 *dp = dst + (size_t)p * sst;
#pragma unroll
      for (int r = 0; r < R; r++) dp[phys<SH>(d0 + r * Ns)] = v[r];
    }
  }
}

template <typename T, int R>
__device__ __forceinline__ void pp_stage_role(const fftz_pass_t &P, const typename Cplx<T>::type *src,
                                              typename Cplx<T>::type *dst, int s, int Ns, uint32_t mNs, int nbf,
                                              uint32_t mnbf, uint32_t mtpc, bool from_g, bool to_g,
                                              const int64_t *s_in, const int64_t *s_out, const int64_t *s_col) {
  if (from_g && to_g) {
    if (P.in_mode == 1)
      pp_stage<T, R, true, true, 1>(P, src, dst, s, Ns, mNs, nbf, mnbf, mtpc, s_in, s_out, s_col);
    else
      pp_stage<T, R, true, true, 0>(P, src, dst, s, Ns, mNs, nbf, mnbf, mtpc, s_in, s_out, s_col);
  } else if (from_g) {
    if (P.in_mode == 1)
      pp_stage<T, R, true, false, 1>(P, src, dst, s, Ns, mNs, nbf, mnbf, mtpc, s_in, s_out, s_col);
    else
      pp_stage<T, R, true, false, 0>(P, src, dst, s, Ns, mNs, nbf, mnbf, mtpc, s_in, s_out, s_col);
  } else if (to_g) {
    if (P.out_mode == 1)
      pp_stage<T, R, false, true, 1>(P, src, dst, s, Ns, mNs, nbf, mnbf, mtpc, s_in, s_out, s_col);
    else
      pp_stage<T, R, false, true, 0>(P, src, dst, s, Ns, mNs, nbf, mnbf, mtpc, s_in, s_out, s_col);
  } else {
    pp_stage<T, R, false, false, 0>(P, src, dst, s, Ns, mNs, nbf, mnbf, mtpc, s_in, s_out, s_col);
  }
}

// Shared memory of a ping-pong tile: two buffers of tpc * sstride complex,
// then in / out offsets and columns, then two reciprocals per stage.
template <typename T>
__device__ __forceinline__ void generic_tile_pp(const fftz_pass_t &P, int64_t blk, unsigned char *smem_raw) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  T2 *buf0 = (T2 *)smem_raw;
  T2 *buf1 = buf0 + (size_t)P.tpc * P.sstride;
  int64_t *s_in = (int64_t *)(buf1 + (size_t)P.tpc * P.sstride);
  int64_t *s_out = s_in + P.tpc;
  int64_t *s_col = s_out + P.tpc;
  uint32_t *s_mag = (uint32_t *)(s_col + P.tpc);  // [s]: Ns, n / R
  const int64_t tf0 = blk * P.tpc;
  for (int p = threadIdx.x; p < P.tpc; p += blockDim.x) batch_offsets(P, tf0 + p, s_in + p, s_out + p, s_col + p);
  if (threadIdx.x < P.nstages) {
    int Ns = 1;
    for (int s = 0; s < (int)threadIdx.x; s++) Ns *= P.radix[s];
    s_mag[2 * threadIdx.x] = pp_magic((uint32_t)Ns);
    s_mag[2 * threadIdx.x + 1] = pp_magic((uint32_t)(P.n / P.radix[threadIdx.x]));
  }
  __syncthreads();
  const uint32_t mtpc = pp_magic((uint32_t)P.tpc);
  const int nsweeps = (P.flags & FFTZ_F_MID_TAB) ? 2 : 1;
  T2 *cur = buf0, *nxt = buf1;
  if (!P.fuse_load) load_phase<T>(P, cur, s_in, s_col);
  for (int sw = 0; sw < nsweeps; sw++) {
    int Ns = 1;
    for (int s = 0; s < P.nstages; s++) {
      const bool from_g = P.fuse_load && sw == 0 && s == 0;
      const bool to_g = P.fuse_store && sw == nsweeps - 1 && s == P.nstages - 1;
      const int R = P.radix[s];
      const int nbf = P.n / R;
      const uint32_t mNs = s_mag[2 * s], mnbf = s_mag[2 * s + 1];
      switch (R) {
        case 2: pp_stage_role<T, 2>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        case 3: pp_stage_role<T, 3>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        case 4: pp_stage_role<T, 4>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        case 5: pp_stage_role<T, 5>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        case 7: pp_stage_role<T, 7>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        case 8: pp_stage_role<T, 8>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        case 11: pp_stage_role<T, 11>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        case 13: pp_stage_role<T, 13>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
        default: pp_stage_role<T, 16>(P, cur, nxt, s, Ns, mNs, nbf, mnbf, mtpc, from_g, to_g, s_in, s_out, s_col); break;
      }
      if (!to_g) {
        __syncthreads();
        T2 *t = cur;
        cur = nxt;
        nxt = t;
      }
      Ns *= R;
    }
    if (sw == 0 && nsweeps == 2) {
      // between the sweeps: v = conj(v) * mid_tab[e] (spectrum product of Bluestein)
      const T2 *mt = (const T2 *)P.mid_tab;
      for (int i = threadIdx.x; i < P.tpc * P.n; i += blockDim.x) {
        const int p = i / P.n;
        const int e = i - p * P.n;
        const int64_t c = s_col[p];
        if (c < 0) continue;
        T2 *a = cur + (size_t)p * P.sstride + phys<SH>(e);
        T2 v = *a;
        v.y = -v.y;
        *a = cmul(v, __ldg(mt + e + c * P.mid_cs));
      }
      __syncthreads();
    }
  }
  if (!P.fuse_store) store_phase<T>(P, cur, s_out, s_col);
}

// 256 threads; float 80 registers (3 CTAs per SM), double 128 (2 CTAs): the
// bounds at which the inlined radix paths keep their spills to a few bytes
// (a float build bounded to 4 CTAs per SM measured 8% slower on mixed1000)
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) fft_pp_kernel(const __grid_constant__ fftz_pass_t P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  generic_tile_pp<T>(P, (int64_t)blockIdx.x, smem_raw);
}

// float: at most 80 registers (3 CTAs of 256 threads per SM) -- measured on
// B200 1.6-2.8x faster than the unbounded build for mixed-radix lines
// (n = 1000 ... 44100); double keeps the plain thread bound (a minimum-blocks
// bound of 1 measured 1.7x slower for it)
template <typename T>
__global__ void __launch_bounds__(256, 3) fft_smem_kernel_occ3(const __grid_constant__ fftz_pass_t P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  generic_tile<T>(P, (int64_t)blockIdx.x, smem_raw);
}

template <typename T>
__global__ void __launch_bounds__(256) fft_smem_kernel(const __grid_constant__ fftz_pass_t P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  generic_tile<T>(P, (int64_t)blockIdx.x, smem_raw);
}

}  // namespace fftz

