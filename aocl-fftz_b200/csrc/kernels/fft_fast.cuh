// Compile-time power-of-two shared-memory FFT kernel families.
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
// Two kernel shapes share the stage code:
//   fft_fast_kernel  one tile of transforms per CTA; the first stage reads HBM
//                    directly and the last stage writes HBM directly.
//   fft_pipe_kernel  persistent CTAs looping over tiles with two shared-memory
//                    slots: while the stages run on one slot, cp.async copies
//                    of the next tile stream into the other, so HBM traffic
//                    overlaps the arithmetic even at one CTA per SM.
// Lanes map along elements (mode 0, rows) or along neighbouring transforms
// (mode 1, columns) on the HBM side, which keeps both row and column accesses
// coalesced. Feature bits (template FEAT) add:
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
// Entries of the stage-twiddle table (entry 0 unused, stage s >= 1 holds
// (R_s - 1) * Ns entries).
__host__ __device__ constexpr int ct_tw_total(int n) {
  int t = 1, ns = 1;
  for (int s = 0; s < ct_nstages(n); s++) {
    if (s > 0) t += (ct_radix(n, s) - 1) * ns;
    ns *= ct_radix(n, s);
  }
  return t;
}
// Block-size bound of an instantiation: room for several columns per CTA
// (1024 threads for float, 512 for double keeps the double kernels at <= 128
// registers).
template <typename T> __host__ __device__ constexpr int ct_lb() { return sizeof(T) == 4 ? 1024 : 512; }

// The persistent kernels run few transforms per CTA: 512 threads (128
// registers a thread) unless one transform needs more.
__host__ __device__ constexpr int ct_pipe_lb(int n) { return ct_tpt(n) > 512 ? ct_tpt(n) : 512; }

enum { FEAT_TW4 = 1, FEAT_TABS = 2, FEAT_SWEEP2 = 4 };

// Epilogue of one output element kk (the destination pointer already points
// at it).
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
  T2 *o = (T2 *)P.out + obase;
  if (P.oes == 1)
    o[kk] = v;
  else
    o[(int64_t)kk * P.oes] = v;
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
    if (valid) x = (P.ies == 1) ? gin[e] : gin[(int64_t)e * P.ies];
    if (P.flags & FFTZ_F_CONJ_IN) x.y = -x.y;
  }
  return x;
}

// One Stockham stage. FROMG: the stage reads its inputs from HBM (otherwise
// from shared memory). LAST: it writes its outputs to HBM. MAPFIRST /
// MAPLAST select the HBM-side lane map (in_mode / out_mode). STG: the first
// stage's inputs were staged densely in sdata by the tensor-memory
// accelerator (transform p at s_in[p], element e at e * stg_es); the stage
// reads them with the HBM lane map and waits for every thread before it
// overwrites the staging area with its own outputs.
// STG == 2: the half e < N/2 of every transform was staged in stg (transform
// p at stg_off[p], element e at e * stg_es); the other half is read from HBM.
template <typename T, int N, int S, int FEAT, bool FROMG, bool LAST, bool MAPFIRST, bool CONJ0 = false,
          int STG = 0>
__device__ __forceinline__ void fast_stage(const fftz_pass_t &P, typename Cplx<T>::type *sdata,
                                           const int64_t *s_in, const int64_t *s_out, const int64_t *s_col,
                                           int stg_es = 1, const typename Cplx<T>::type *stg = nullptr,
                                           const int64_t *stg_off = nullptr,
                                           const typename Cplx<T>::type *twb = nullptr) {
  typedef typename Cplx<T>::type T2;
  constexpr int R = ct_radix(N, S);
  constexpr int NS = ct_ns(N, S);
  constexpr int NB = kMaxE / R;
  constexpr int NBF = N / R;
  constexpr int TPT = ct_tpt(N);
  constexpr bool ALLV = (NB * TPT == NBF);
  constexpr int SH = Cplx<T>::PADSH;
  constexpr int PAD = 1 << SH;
  const int t = threadIdx.x;
  const int mode = MAPFIRST ? P.in_mode : (LAST ? P.out_mode : 0);
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
  if (FROMG && STG == 2) {
    const T2 *gin = (const T2 *)P.in + s_in[p];
    const T2 *src = stg + stg_off[p];
    const bool cj = (P.flags & FFTZ_F_CONJ_IN) != 0;
    const int64_t ies = P.ies;
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * TPT;
      if (ALLV || b < NBF) {
#pragma unroll
        for (int r = 0; r < R; r++) {
          T2 x = zero2<T2>();
          if (r < R / 2)
            x = src[(b + r * NBF) * stg_es];  // e < N/2: staged
          else if (valid)
            x = gin[(int64_t)(b + r * NBF) * ies];
          if (cj) x.y = -x.y;
          v[q][r] = x;
        }
      }
    }
  } else if (FROMG && STG) {
    const T2 *src = sdata + s_in[p];
    const bool cj = (P.flags & FFTZ_F_CONJ_IN) != 0;
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * TPT;
      if (ALLV || b < NBF) {
        const T2 *sb = src + b * stg_es;
        const int st = NBF * stg_es;
#pragma unroll
        for (int r = 0; r < R; r++) {
          T2 x = sb[r * st];
          if (cj) x.y = -x.y;
          v[q][r] = x;
        }
      }
    }
    __syncthreads();
  } else if (FROMG) {
    const T2 *gin = (const T2 *)P.in + s_in[p];
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * TPT;
      if (ALLV || b < NBF) {
        if constexpr ((FEAT & FEAT_TABS) != 0) {
#pragma unroll
          for (int r = 0; r < R; r++) v[q][r] = load_fast<T, FEAT>(P, gin, b + r * NBF, col, valid);
        } else {
          // one 64-bit product per butterfly, constant multiples after it
          const int64_t ies = P.ies;
          const T2 *gb = gin + (int64_t)b * ies;
          const int64_t st = (int64_t)NBF * ies;
          const bool cj = (P.flags & FFTZ_F_CONJ_IN) != 0;
#pragma unroll
          for (int r = 0; r < R; r++) {
            T2 x = zero2<T2>();
            if (valid) x = gb[r * st];
            if (cj) x.y = -x.y;
            v[q][r] = x;
          }
        }
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < NB; q++) {
      const int b = j + q * TPT;
      if (ALLV || b < NBF) {
        if constexpr (NBF % PAD == 0) {
          const T2 *src = sd + phys<SH>(b);
#pragma unroll
          for (int r = 0; r < R; r++) v[q][r] = src[r * (NBF + NBF / PAD)];
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) v[q][r] = sd[phys<SH>(b + r * NBF)];
        }
      }
    }
    if (CONJ0 && (P.flags & FFTZ_F_CONJ_IN)) {
#pragma unroll
      for (int q = 0; q < NB; q++)
#pragma unroll
        for (int r = 0; r < R; r++) v[q][r].y = -v[q][r].y;
    }
    __syncthreads();
  }
  // stage twiddles from the shared-memory copy when the tile made one
  const T2 *tw = (twb ? twb : (const T2 *)P.tw) + P.tw_off[S];
#pragma unroll
  for (int q = 0; q < NB; q++) {
    const int b = j + q * TPT;
    if (ALLV || b < NBF) {
      const int k = b & (NS - 1);
      if (NS > 1) {
        if (twb) {
#pragma unroll
          for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], tw[(r - 1) * NS + k]);
        } else {
#pragma unroll
          for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], __ldg(tw + (r - 1) * NS + k));
        }
      }
      Dft<R>::template apply<T, T2>(v[q]);
      const int d0 = (b - k) * R + k;
      if (LAST) {
        if (valid) {
          if constexpr ((FEAT & FEAT_TABS) != 0) {
#pragma unroll
            for (int r = 0; r < R; r++) store_fast<T, FEAT>(P, v[q][r], d0 + r * NS, col, s_out[p]);
          } else {
            const int64_t oes = P.oes;
            T2 *ob = (T2 *)P.out + s_out[p] + (int64_t)d0 * oes;
            const int64_t st = (int64_t)NS * oes;
            const bool cj = (P.flags & FFTZ_F_CONJ_OUT) != 0;
            // four-step factor of output d0 + r NS: W^{col d0} (W^{col NS})^r,
            // two table products per chain start and one for the step, then
            // a chain of at most CH - 1 products (CH = 8 for radix 16)
            constexpr int CH = R > 8 ? R / 2 : R;
            T2 w = zero2<T2>(), stp = zero2<T2>();
            if constexpr ((FEAT & FEAT_TW4) != 0) {
              stp = tw4<T>(P, col, NS);
              w = tw4<T>(P, col, d0);
            }
#pragma unroll
            for (int r = 0; r < R; r++) {
              T2 y = v[q][r];
              if constexpr ((FEAT & FEAT_TW4) != 0) {
                if (r > 0 && r % CH == 0) w = tw4<T>(P, col, d0 + r * NS);
                y = cmul(y, w);
                if ((r + 1) % CH != 0) w = cmul(w, stp);
              }
              if (cj) y.y = -y.y;
              ob[r * st] = y;
            }
          }
        }
      } else if constexpr (NS % PAD == 0) {
        T2 *dst = sd + phys<SH>(d0);
#pragma unroll
        for (int r = 0; r < R; r++) dst[r * (NS + NS / PAD)] = v[q][r];
      } else if constexpr (NS * R == PAD) {
        T2 *dst = sd + phys<SH>(d0 - k) + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[r * NS] = v[q][r];
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) sd[phys<SH>(d0 + r * NS)] = v[q][r];
      }
    }
  }
  if (!LAST) __syncthreads();
}

// Stage S of sweep SW out of NSW sweeps. GLOBALIN: the very first stage reads
// HBM (fast kernel); the pipelined kernel has already staged the tile.
template <typename T, int N, int S, int NST, int SW, int NSW, int FEAT, bool GLOBALIN, int STG = 0>
struct FastStages {
  static __device__ __forceinline__ void run(const fftz_pass_t &P, typename Cplx<T>::type *sdata,
                                             const int64_t *s_in, const int64_t *s_out, const int64_t *s_col,
                                             int stg_es = 1, const typename Cplx<T>::type *twb = nullptr) {
    constexpr bool FIRSTG = (S == 0 && SW == 0);
    fast_stage<T, N, S, FEAT, GLOBALIN && FIRSTG, (S == NST - 1 && SW == NSW - 1), GLOBALIN && FIRSTG,
               !GLOBALIN && FIRSTG, FIRSTG ? STG : 0>(P, sdata, s_in, s_out, s_col, stg_es, nullptr, nullptr, twb);
    FastStages<T, N, S + 1, NST, SW, NSW, FEAT, GLOBALIN, STG>::run(P, sdata, s_in, s_out, s_col, stg_es, twb);
  }
};
template <typename T, int N, int NST, int SW, int NSW, int FEAT, bool GLOBALIN, int STG>
struct FastStages<T, N, NST, NST, SW, NSW, FEAT, GLOBALIN, STG> {
  static __device__ __forceinline__ void run(const fftz_pass_t &, typename Cplx<T>::type *, const int64_t *,
                                             const int64_t *, const int64_t *, int = 1,
                                             const typename Cplx<T>::type * = nullptr) {}
};

// Base offsets and column index of the transforms of one tile.
__device__ __forceinline__ void tile_offsets(const fftz_pass_t &P, int64_t tf0, int64_t *s_in, int64_t *s_out,
                                             int64_t *s_col) {
  for (int p = threadIdx.x; p < P.tpc; p += blockDim.x) batch_offsets(P, tf0 + p, s_in + p, s_out + p, s_col + p);
}

// One tile of a pass: transforms [tf0, tf0 + tpc) with blockDim == tpc * tpt.
template <typename T, int N, int FEAT>
__device__ __forceinline__ void fast_tile(const fftz_pass_t &P, int64_t tf0, unsigned char *smem_raw) {
  typedef typename Cplx<T>::type T2;
  T2 *sdata = (T2 *)smem_raw;
  int64_t *s_in = (int64_t *)(sdata + (size_t)P.tpc * P.sstride);
  int64_t *s_out = s_in + P.tpc;
  int64_t *s_col = s_out + P.tpc;
  tile_offsets(P, tf0, s_in, s_out, s_col);
  T2 *twb = nullptr;
  if (P.smem_tw) {
    // stage twiddles copied next to the tile: shared-memory loads in the stages
    twb = (T2 *)(((uintptr_t)(s_col + P.tpc) + 15) & ~(uintptr_t)15);
    const T2 *g = (const T2 *)P.tw;
    for (int i = threadIdx.x; i < ct_tw_total(N); i += blockDim.x) twb[i] = __ldg(g + i);
  }
  __syncthreads();
  if (FEAT & FEAT_SWEEP2) {
    constexpr int SH = Cplx<T>::PADSH;
    FastStages<T, N, 0, ct_nstages(N), 0, 2, FEAT, true>::run(P, sdata, s_in, s_out, s_col, 1, twb);
    const T2 *mt = (const T2 *)P.mid_tab;
    for (int i = threadIdx.x; i < P.tpc * N; i += blockDim.x) {
      const int p = i / N;
      const int e = i - p * N;
      const int64_t c = s_col[p];
      if (c < 0) continue;
      T2 *a = sdata + (size_t)p * P.sstride + phys<SH>(e);
      T2 v = *a;
      v.y = -v.y;
      *a = cmul(v, __ldg(mt + e + c * P.mid_cs));
    }
    __syncthreads();
    FastStages<T, N, 0, ct_nstages(N), 1, 2, FEAT, true>::run(P, sdata, s_in, s_out, s_col, 1, twb);
  } else {
    FastStages<T, N, 0, ct_nstages(N), 0, 1, FEAT, true>::run(P, sdata, s_in, s_out, s_col, 1, twb);
  }
}

template <typename T, int N, int FEAT>
__global__ void __launch_bounds__(ct_lb<T>()) fft_fast_kernel(const __grid_constant__ fftz_pass_t P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fast_tile<T, N, FEAT>(P, (int64_t)blockIdx.x * P.tpc, smem_raw);
}

// ---------------------------------------------------------------- pipelined

template <typename T> __device__ __forceinline__ void cp_async_elem(void *sdst, const void *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  if (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
  else
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Issue the asynchronous copies of one tile (tpc transforms of length N) into
// a shared-memory slot, in the padded layout the stages read.
template <typename T, int N>
__device__ __forceinline__ void issue_tile(const fftz_pass_t &P, typename Cplx<T>::type *slot, const int64_t *s_in,
                                           const int64_t *s_col) {
  typedef typename Cplx<T>::type T2;
  constexpr int SH = Cplx<T>::PADSH;
  const int total = P.tpc * N;
  const T2 *gin = (const T2 *)P.in;
  const bool unit = P.ies == 1;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int p, e;
    if (P.in_mode == 0) {
      p = i / N;
      e = i & (N - 1);
    } else {
      p = i % P.tpc;
      e = i / P.tpc;
    }
    if (s_col[p] < 0) continue;
    const T2 *src = gin + s_in[p] + (unit ? (int64_t)e : (int64_t)e * P.ies);
    cp_async_elem<T>(slot + (size_t)p * P.sstride + phys<SH>(e), src);
  }
}

// Persistent double-buffered kernel: CTA b handles tiles b, b + grid, ...;
// the copies of tile i+1 are in flight while the stages of tile i run.
template <typename T, int N, int FEAT>
__global__ void __launch_bounds__(ct_pipe_lb(N), 1) fft_pipe_kernel(const __grid_constant__ fftz_pass_t P) {
  typedef typename Cplx<T>::type T2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T2 *slot0 = (T2 *)smem_raw;
  const size_t slot_elems = (size_t)P.tpc * P.sstride;
  T2 *slot1 = slot0 + slot_elems;
  int64_t *offs = (int64_t *)(slot0 + 2 * slot_elems);  // 3 rotating sets of {in, out, col}
  const int64_t ntiles = (P.ntf + P.tpc - 1) / P.tpc;
  int64_t tile = blockIdx.x;
  if (tile >= ntiles) return;
#define FZ_OFF(bf, a) (offs + (size_t)((bf)*3 + (a)) * P.tpc)
  tile_offsets(P, tile * P.tpc, FZ_OFF(0, 0), FZ_OFF(0, 1), FZ_OFF(0, 2));
  __syncthreads();
  issue_tile<T, N>(P, slot0, FZ_OFF(0, 0), FZ_OFF(0, 2));
  cp_async_commit();
  for (int64_t it = 0;; it++) {
    const int64_t next = tile + gridDim.x;
    const bool has_next = next < ntiles;
    const int ob = (int)(it % 3), nob = (int)((it + 1) % 3);
    T2 *cur = (it & 1) ? slot1 : slot0;
    T2 *nxt = (it & 1) ? slot0 : slot1;
    if (has_next) tile_offsets(P, next * P.tpc, FZ_OFF(nob, 0), FZ_OFF(nob, 1), FZ_OFF(nob, 2));
    __syncthreads();  // the slot about to be refilled is no longer read
    if (has_next) issue_tile<T, N>(P, nxt, FZ_OFF(nob, 0), FZ_OFF(nob, 2));
    cp_async_commit();
    cp_async_wait1();  // this thread's copies of the current tile have landed
    __syncthreads();   // ... and everyone else's
    FastStages<T, N, 0, ct_nstages(N), 0, 1, FEAT, false>::run(P, cur, FZ_OFF(ob, 0), FZ_OFF(ob, 1), FZ_OFF(ob, 2));
    if (!has_next) break;
    tile = next;
  }
#undef FZ_OFF
}

}  // namespace fftz
