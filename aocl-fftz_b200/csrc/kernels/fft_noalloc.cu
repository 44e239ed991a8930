// No-allocation execute: single-precision complex four-step transforms whose
// intermediate lives in a file-scope static device array instead of memory
// taken from cudaMalloc at set-up.
//
// Who needs it. Some callers cannot allocate device memory when they want a
// transform:
//   * processes where another allocator owns the device's memory (a serving
//     engine or a framework's caching allocator that reserves almost all of
//     HBM up front): a plan's cudaMalloc there can fail, or takes memory out
//     of a budget that the owner accounts for itself;
//   * latency-critical loops, where cudaFree's implicit device-wide
//     synchronisation would stall every other stream;
//   * code that must not fail for lack of memory once it has started (error
//     handlers, watchdog paths).
// Such callers cannot use aoclfftz_setup_f, which allocates tables and scratch
// per plan. This entry point needs no plan: it runs the same two kernels as a
// plan's four-step path (column FFTs with the twiddle epilogue, then row FFTs
// with the transposed store) on a scratch array and twiddle tables that are
// static device variables of this file.
//
// Limits: n a power of two, 2^15 <= n <= 2^22, and n * howmany <= 2^22
// complex elements (the scratch array is 2^22 float2 = 32 MiB; every GPU on
// which this library's module is loaded holds it until the process exits).
//
// Set-up: the first call on each device (that device current) looks up the
// two arrays with cudaGetSymbolAddress - in host code their names are only
// host-side stand-ins, not device addresses - fills the twiddle tables with a
// few small kernels and waits for them on the caller's stream. Make that first
// call before any stream capture begins: made while the stream is being
// captured, it is refused with AOCLFFTZ_SETUP_FAILURE. Later calls only
// validate and launch.
//
// Sharing: every call on a device uses the same scratch array, which keeps
// whatever the last call left in it. Nothing in it needs to start at zero
// (the column pass writes every element that the row pass then reads), but
// two calls whose kernels overlap on the GPU - on different streams, or from
// different threads without ordering - race on the scratch and both results
// are undefined. Order such calls on one stream.
//
// No cudaMalloc, cudaFree or other allocating routine is called, at set-up or
// afterwards.
#include <cuda_runtime.h>
#include <pthread.h>
#include <stdint.h>
#include <string.h>

#include "aoclfftz_gpu.h"
#include "fftz_kernels.h"

extern "C" void fz_set_error(const char *fmt, ...);

#define FZ_NA_MAX_ELEMS (1 << 22) /* complex float elements of the scratch array (32 MiB) */
#define FZ_NA_LOG_MIN 15          /* smallest log2(n): shorter lines run as one single-pass kernel */
#define FZ_NA_LOG_MAX 22
#define FZ_NA_LINE_MIN 7 /* log2 of the shortest column / row length (n = 2^15 -> 256 x 128) */
#define FZ_NA_LINE_MAX 11
#define FZ_NA_TAB_ELEMS (1 << 15) /* twiddle table capacity (complex float); the layout needs < 20000 */
#define FZ_NA_MAX_DEV 64

static __device__ __align__(256) float2 g_na_scratch[FZ_NA_MAX_ELEMS];
static __device__ __align__(256) float2 g_na_tables[FZ_NA_TAB_ELEMS];

namespace {

// W_M^e = exp(-2 pi i e / M) in double, rounded once to float. Stage
// segments (mode 0): entry i is W_M^{r k} with r = i / ns + 1, k = i % ns.
// Plain segments (mode 1): entry i is W_M^{i * mul}.
__global__ void na_fill(float2 *dst, int64_t count, int64_t M, int64_t ns, int64_t mul, int mode) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  int64_t e = mode == 0 ? (i / ns + 1) * (i % ns) : i * mul;
  e %= M;
  double s, c;
  sincospi(2.0 * (double)e / (double)M, &s, &c);
  dst[i] = make_float2((float)c, 0.0f - (float)s);
}

// Offsets (complex elements) of every table in g_na_tables; the same on every
// device, computed once.
struct Layout {
  int ready;
  int32_t nst[FZ_NA_LINE_MAX + 1];
  int32_t radix[FZ_NA_LINE_MAX + 1][FFTZ_MAX_STAGES];
  int32_t tw_off[FZ_NA_LINE_MAX + 1][FFTZ_MAX_STAGES];
  int64_t stage_off[FZ_NA_LINE_MAX + 1];
  int64_t L[FZ_NA_LOG_MAX + 1], hi_off[FZ_NA_LOG_MAX + 1], lo_off[FZ_NA_LOG_MAX + 1];
  int64_t total;
};

struct DevState {
  int ready;
  float2 *scratch;
  float2 *tables;
};

Layout g_layout;
DevState g_devs[FZ_NA_MAX_DEV];
pthread_mutex_t g_na_mu = PTHREAD_MUTEX_INITIALIZER;

int64_t align32(int64_t x) { return (x + 31) & ~(int64_t)31; } /* 256-byte table starts */

// Stage tables in the layout the compile-time kernels read: entry 0 unused,
// stage s >= 1 holds W_{Ns*R}^{k*r} at tw_off[s] + (r-1)*Ns + k.
void make_layout(Layout *t) {
  int64_t off = 0;
  for (int g = FZ_NA_LINE_MIN; g <= FZ_NA_LINE_MAX; g++) {
    t->nst[g] = fftz_fast_radices(1 << g, t->radix[g]);
    int64_t total = 1, ns = 1;
    for (int s = 0; s < t->nst[g]; s++) {
      t->tw_off[g][s] = (int32_t)total;
      if (s > 0) total += (int64_t)(t->radix[g][s] - 1) * ns;
      ns *= t->radix[g][s];
    }
    t->stage_off[g] = off;
    off = align32(off + total);
  }
  for (int l = FZ_NA_LOG_MIN; l <= FZ_NA_LOG_MAX; l++) {
    const int64_t N = (int64_t)1 << l;
    int64_t L = 1;
    while (L * L < N) L *= 2;
    t->L[l] = L;
    t->hi_off[l] = off;
    off = align32(off + N / L);
    t->lo_off[l] = off;
    off = align32(off + L);
  }
  t->total = off;
  t->ready = 1;
}

int launch_fill(float2 *dst, int64_t count, int64_t M, int64_t ns, int64_t mul, int mode, cudaStream_t st) {
  if (count <= 0) return 0;
  na_fill<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(dst, count, M, ns, mul, mode);
  return (int)cudaGetLastError();
}

int fill_tables(const Layout *t, float2 *tab, cudaStream_t st) {
  int e = 0;
  for (int g = FZ_NA_LINE_MIN; g <= FZ_NA_LINE_MAX && !e; g++) {
    float2 *seg = tab + t->stage_off[g];
    e = launch_fill(seg, 1, 1, 1, 0, 1, st); /* entry 0: the unused stage-0 slot */
    int64_t ns = t->radix[g][0];
    for (int s = 1; s < t->nst[g] && !e; s++) {
      const int64_t R = t->radix[g][s];
      e = launch_fill(seg + t->tw_off[g][s], (R - 1) * ns, ns * R, ns, 0, 0, st);
      ns *= R;
    }
  }
  for (int l = FZ_NA_LOG_MIN; l <= FZ_NA_LOG_MAX && !e; l++) {
    const int64_t N = (int64_t)1 << l, L = t->L[l];
    e = launch_fill(tab + t->hi_off[l], N / L, N, 1, L, 1, st); /* W_N^{j L} */
    if (!e) e = launch_fill(tab + t->lo_off[l], L, N, 1, 1, 1, st); /* W_N^{j} */
  }
  return e;
}

// Once per device, with that device current: symbol addresses and tables.
aoclfftz_error_type setup_device(int dev, cudaStream_t st, DevState **out) {
  pthread_mutex_lock(&g_na_mu);
  aoclfftz_error_type rc = AOCLFFTZ_SUCCESS;
  DevState *d = &g_devs[dev];
  if (!d->ready) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      fz_set_error("no-allocation execute: the first call on device %d sets up its tables and must not be made "
                   "while the stream is being captured",
                   dev);
      rc = AOCLFFTZ_SETUP_FAILURE;
    } else {
      if (!g_layout.ready) make_layout(&g_layout);
      void *scr = NULL, *tab = NULL;
      e = cudaGetSymbolAddress(&scr, g_na_scratch);
      if (e == cudaSuccess) e = cudaGetSymbolAddress(&tab, g_na_tables);
      if (e != cudaSuccess) {
        fz_set_error("no-allocation execute: cudaGetSymbolAddress failed on device %d: %s", dev,
                     cudaGetErrorString(e));
        cudaGetLastError();
        rc = AOCLFFTZ_SETUP_FAILURE;
      } else if (g_layout.total > FZ_NA_TAB_ELEMS) {
        fz_set_error("no-allocation execute: twiddle layout of %lld entries exceeds the table array",
                     (long long)g_layout.total);
        rc = AOCLFFTZ_SETUP_FAILURE;
      } else {
        int fe = fill_tables(&g_layout, (float2 *)tab, st);
        if (!fe) fe = (int)cudaStreamSynchronize(st);
        if (fe) {
          fz_set_error("no-allocation execute: table set-up failed on device %d: %s", dev,
                       cudaGetErrorString((cudaError_t)fe));
          cudaGetLastError();
          rc = AOCLFFTZ_SETUP_FAILURE;
        } else {
          d->scratch = (float2 *)scr;
          d->tables = (float2 *)tab;
          d->ready = 1;
        }
      }
    }
  }
  pthread_mutex_unlock(&g_na_mu);
  *out = d;
  return rc;
}

// One pass of the compile-time kernel over cols * howmany transforms of
// length 2^g: element e of transform (c, b) at c * cs + b * dist + e * es on
// each side. The launch shape (transforms per CTA, shared-memory stride) is
// the planner's default for the same pass.
int line_pass(fftz_pass_t *k, int g, int64_t ies, int64_t oes, int64_t cols, int64_t ics, int64_t ocs,
              int64_t howmany, int64_t idist, int64_t odist, int flags, int variant, const Layout *t,
              const float2 *tab) {
  memset(k, 0, sizeof(*k));
  const int n = 1 << g;
  k->n = n;
  k->ies = ies;
  k->oes = oes;
  k->flags = flags;
  k->in_kind = FFTZ_IN_COMPLEX;
  k->out_kind = FFTZ_OUT_COMPLEX;
  k->nload = n;
  k->nstore = n;
  k->dtype = 0;
  k->scale = 1.0;
  k->variant = variant;
  k->fuse_load = 1;
  k->fuse_store = 1;
  k->nbdims = 1;
  k->bdim[0] = cols;
  k->ibs[0] = ics;
  k->obs[0] = ocs;
  if (howmany > 1) {
    k->nbdims = 2;
    k->bdim[1] = howmany;
    k->ibs[1] = idist;
    k->obs[1] = odist;
  }
  k->ntf = cols * howmany;
  k->in_mode = ics < ies ? 1 : 0;
  k->out_mode = ocs < oes ? 1 : 0;
  k->nstages = t->nst[g];
  for (int s = 0; s < k->nstages; s++) {
    k->radix[s] = t->radix[g][s];
    k->tw_off[s] = t->tw_off[g][s];
  }
  k->tpt = fftz_fast_tpt(n);
  if (k->nstages == 1 && k->in_mode != k->out_mode) k->out_mode = k->in_mode;
  const int colmap = k->in_mode == 1 || k->out_mode == 1;
  k->sstride = fftz_smem_stride(0, n);
  int by_thr = 1024 / k->tpt;
  if (by_thr < 1) by_thr = 1;
  const int64_t by_smem = fftz_smem_limit() / (((int64_t)k->sstride + 16) * 8 + 24);
  int tpc = colmap ? 8 : (int)((4096 + n - 1) / n);
  if (!colmap && tpc * k->tpt < 128) tpc = (128 + k->tpt - 1) / k->tpt;
  if (tpc > by_thr) tpc = by_thr;
  if (tpc > by_smem) tpc = (int)by_smem;
  if (tpc > k->ntf) tpc = (int)k->ntf;
  if (tpc < 1) tpc = 1;
  k->tpc = tpc;
  if (colmap) k->sstride = fftz_smem_stride_cols(0, n, tpc);
  k->tw = tab + t->stage_off[g];
  return fftz_pass_smem_bytes(k) <= fftz_smem_limit() ? 0 : -1;
}

int device_pointer(const void *p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (a.type == cudaMemoryTypeManaged) return 1;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" aoclfftz_error_type aoclfftz_gpu_execute_noalloc_c2c_f(const FFTZ_VOID *in, FFTZ_VOID *out,
                                                                  FFTZ_INT64 n, FFTZ_INT64 howmany,
                                                                  FFTZ_INT32 direction, FFTZ_VOID *stream) {
  if (!in || !out) {
    fz_set_error("no-allocation execute: in and out must be device pointers");
    return AOCLFFTZ_INVALID_INPUT;
  }
  if (direction != 0 && direction != 1) {
    fz_set_error("no-allocation execute: direction must be 0 (forward) or 1 (backward)");
    return AOCLFFTZ_INVALID_INPUT;
  }
  int l = 0;
  while (l < 62 && ((int64_t)1 << l) < n) l++;
  if (n <= 0 || ((int64_t)1 << l) != n || l < FZ_NA_LOG_MIN || l > FZ_NA_LOG_MAX) {
    fz_set_error("no-allocation execute: n = %lld must be a power of two in [2^%d, 2^%d]", (long long)n,
                 FZ_NA_LOG_MIN, FZ_NA_LOG_MAX);
    return AOCLFFTZ_INVALID_INPUT;
  }
  if (howmany < 1 || howmany > FZ_NA_MAX_ELEMS / n) {
    fz_set_error("no-allocation execute: n * howmany = %lld x %lld exceeds the static scratch of %d complex "
                 "elements (32 MiB)",
                 (long long)n, (long long)howmany, FZ_NA_MAX_ELEMS);
    return AOCLFFTZ_INVALID_INPUT;
  }
  if (((uintptr_t)in & 7) || ((uintptr_t)out & 7)) {
    fz_set_error("no-allocation execute: in and out must be 8-byte aligned");
    return AOCLFFTZ_INVALID_INPUT;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= FZ_NA_MAX_DEV) {
    cudaGetLastError();
    fz_set_error("no-allocation execute: no usable current device");
    return AOCLFFTZ_EXECUTION_FAILURE;
  }
  if (!device_pointer(in, dev) || !device_pointer(out, dev)) {
    fz_set_error("no-allocation execute: in and out must be memory of the current device (%d)", dev);
    return AOCLFFTZ_INVALID_INPUT;
  }
  cudaStream_t st = (cudaStream_t)stream;
  DevState *d = NULL;
  aoclfftz_error_type rc = setup_device(dev, st, &d);
  if (rc != AOCLFFTZ_SUCCESS) return rc;
  const Layout *t = &g_layout;
  const int g1 = (l + 1) / 2, g2 = l / 2; /* n1 >= n2, the planner's balanced split */
  const int64_t n1 = (int64_t)1 << g1, n2 = (int64_t)1 << g2;
  const int conj_in = direction == 1 ? FFTZ_F_CONJ_IN : 0, conj_out = direction == 1 ? FFTZ_F_CONJ_OUT : 0;
  fftz_pass_t a, b;
  /* pass A: column j2 of the n1 x n2 view -> scratch[line][k1][j2], times W_n^{j2 k1} */
  if (line_pass(&a, g1, n2, n2, n2, 1, 1, howmany, n, n, conj_in | FFTZ_F_TW4, FFTZ_VAR_FAST_TW4, t, d->tables)) {
    fz_set_error("no-allocation execute: column pass of length %lld does not fit shared memory", (long long)n1);
    return AOCLFFTZ_SETUP_FAILURE;
  }
  a.tw4_n = n;
  a.tw4_l = t->L[l];
  a.tw4_hi = d->tables + t->hi_off[l];
  a.tw4_lo = d->tables + t->lo_off[l];
  a.in = in;
  a.out = d->scratch;
  /* pass B: row k1 (contiguous j2) -> out[k1 + n1 k2] */
  if (line_pass(&b, g2, 1, n1, n1, n2, 1, howmany, n, n, conj_out, FFTZ_VAR_FAST, t, d->tables)) {
    fz_set_error("no-allocation execute: row pass of length %lld does not fit shared memory", (long long)n2);
    return AOCLFFTZ_SETUP_FAILURE;
  }
  b.in = d->scratch;
  b.out = out;
  int e = fftz_launch_pass(&a, st);
  if (!e) e = fftz_launch_pass(&b, st);
  if (e) {
    fz_set_error("no-allocation execute: launch failed: %s", cudaGetErrorString((cudaError_t)e));
    return AOCLFFTZ_EXECUTION_FAILURE;
  }
  return AOCLFFTZ_SUCCESS;
}
