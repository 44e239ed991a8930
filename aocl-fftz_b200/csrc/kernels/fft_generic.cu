// Launch side of the shared-memory FFT kernels: the generic runtime-radix
// kernel, dispatch to the compile-time families, shared-memory sizing.
#include "fft_generic.cuh"
#include "fft_fast.cuh"

extern "C" {

const void *fftz_fast_f32_a(int log2n, int feat);
const void *fftz_fast_f32_b(int log2n, int feat);
const void *fftz_fast_f64_a(int log2n, int feat);
const void *fftz_fast_f64_b(int log2n, int feat);
const void *fftz_fast_f32_c(int log2n, int feat);
const void *fftz_fast_f64_c(int log2n, int feat);
const void *fftz_fast_real_kernel(int dtype, int log2n);

static const void *fast_kernel(int dtype, int log2n, int variant) {
  int feat;
  switch (variant) {
    case FFTZ_VAR_FAST: feat = 0; break;
    case FFTZ_VAR_FAST_TW4: feat = fftz::FEAT_TW4; break;
    case FFTZ_VAR_FAST_TABS: feat = fftz::FEAT_TABS; break;
    case FFTZ_VAR_FAST_TW4_TABS: feat = fftz::FEAT_TW4 | fftz::FEAT_TABS; break;
    case FFTZ_VAR_FAST_BLUE: feat = fftz::FEAT_TABS | fftz::FEAT_SWEEP2; break;
    case FFTZ_VAR_PIPE: feat = 16; break;
    case FFTZ_VAR_PIPE_TW4: feat = 16 | fftz::FEAT_TW4; break;
    case FFTZ_VAR_FAST_REAL: return fftz_fast_real_kernel(dtype, log2n);
    default: return 0;
  }
  if (feat >= 16) return dtype == 0 ? fftz_fast_f32_c(log2n, feat) : fftz_fast_f64_c(log2n, feat);
  const void *f = dtype == 0 ? fftz_fast_f32_a(log2n, feat) : fftz_fast_f64_a(log2n, feat);
  if (!f) f = dtype == 0 ? fftz_fast_f32_b(log2n, feat) : fftz_fast_f64_b(log2n, feat);
  return f;
}

int fftz_max_smem_n(int dtype) { return dtype == 0 ? 16384 : 8192; }
int fftz_fast_max_n(int dtype) { return dtype == 0 ? 16384 : 8192; }
int fftz_fast_tpt(int n) { return fftz::ct_tpt(n); }
int fftz_generic_max_threads(void) { return 256; }
int fftz_pipe_max_threads(int n) { return fftz::ct_pipe_lb(n); }

int fftz_fast_radices(int n, int32_t *radix) {
  const int S = fftz::ct_nstages(n);
  for (int s = 0; s < S; s++) radix[s] = fftz::ct_radix(n, s);
  return S;
}

int32_t fftz_smem_stride(int dtype, int32_t nslots) {
  const int sh = dtype == 0 ? (int)fftz::Cplx<float>::PADSH : (int)fftz::Cplx<double>::PADSH;
  if (nslots < 1) nslots = 1;
  int32_t s = (nslots - 1) + ((nslots - 1) >> sh) + 1;
  const int32_t m = 1 << sh;
  while ((s & (m - 1)) != 1) s++;  // neighbouring transforms start on neighbouring banks
  return s;
}

int32_t fftz_smem_stride_cols(int dtype, int32_t nslots, int32_t tpc) {
  const int sh = dtype == 0 ? (int)fftz::Cplx<float>::PADSH : (int)fftz::Cplx<double>::PADSH;
  const int32_t w = 1 << sh;  // complex slots per 128-byte bank row
  if (tpc <= 1 || tpc > w || (tpc & (tpc - 1))) return fftz_smem_stride(dtype, nslots);
  if (nslots < 1) nslots = 1;
  int32_t s = (nslots - 1) + ((nslots - 1) >> sh) + 1;
  const int32_t want = w / tpc;  // transforms p and p+1 land w/tpc slots apart
  while ((s & (w - 1)) != want) s++;
  return s;
}

static int is_pipe(const fftz_pass_t *p) { return p->variant == FFTZ_VAR_PIPE || p->variant == FFTZ_VAR_PIPE_TW4; }

int fftz_threads_per_transform(int dtype, int n, int nstages, const int32_t *radix) {
  (void)dtype;
  int tpt = 1;
  for (int s = 0; s < nstages; s++) {
    const int R = radix[s];
    const int per = fftz::kMaxE / R;
    if (per < 1 || n % R) return 0;
    const int nb = n / R;
    const int need = (nb + per - 1) / per;
    if (need > tpt) tpt = need;
  }
  return tpt;
}

int64_t fftz_smem_limit(void) { return 227 * 1024; }

int32_t fftz_fast_tw_entries(int n) {
  switch (n) {
    case 2: return fftz::ct_tw_total(2);
    case 4: return fftz::ct_tw_total(4);
    case 8: return fftz::ct_tw_total(8);
    case 16: return fftz::ct_tw_total(16);
    case 32: return fftz::ct_tw_total(32);
    case 64: return fftz::ct_tw_total(64);
    case 128: return fftz::ct_tw_total(128);
    case 256: return fftz::ct_tw_total(256);
    case 512: return fftz::ct_tw_total(512);
    case 1024: return fftz::ct_tw_total(1024);
    case 2048: return fftz::ct_tw_total(2048);
    case 4096: return fftz::ct_tw_total(4096);
    case 8192: return fftz::ct_tw_total(8192);
    case 16384: return fftz::ct_tw_total(16384);
  }
  return 0;
}

int64_t fftz_pass_smem_bytes(const fftz_pass_t *p) {
  if (p->variant == FFTZ_VAR_TC) return fftz_tc_smem_bytes();
  const int64_t esz = p->dtype == 0 ? 8 : 16;
  if (p->variant == FFTZ_VAR_GENERIC_PP)
    return 2 * (int64_t)p->tpc * p->sstride * esz + 3 * 8 * (int64_t)p->tpc + 8 * FFTZ_MAX_STAGES;
  if (is_pipe(p)) return 2 * (int64_t)p->tpc * p->sstride * esz + 9 * 8 * (int64_t)p->tpc;
  int64_t b = (int64_t)p->tpc * p->sstride * esz + 3 * 8 * (int64_t)p->tpc;
  if (p->smem_tw) b += 16 + (int64_t)fftz_fast_tw_entries(p->n) * esz;  // shared copy of the stage twiddles
  return b;
}

int fftz_launch_pass(const fftz_pass_t *p, void *stream) {
  if (p->variant == FFTZ_VAR_TC) return fftz_launch_pass_tc(p, stream);
  if (p->use_tma) {
    const int e = fftz_launch_pass_tma(p, stream);
    if (e >= 0) return e;
  }
  // one opt-in of the large dynamic shared memory size per kernel and device
  static const void *opted[64][96];
  static int nopted[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  const int64_t nblk = (p->ntf + p->tpc - 1) / p->tpc;
  if (nblk <= 0) return 0;
  if (nblk > 0x7fffffffLL) return (int)cudaErrorInvalidConfiguration;
  const void *fn = 0;
  if (p->variant == FFTZ_VAR_GENERIC) {
    fn = p->dtype == 0 ? (const void *)&fftz::fft_smem_kernel_occ3<float>
                       : (const void *)&fftz::fft_smem_kernel<double>;
  } else if (p->variant == FFTZ_VAR_GENERIC_PP) {
    fn = p->dtype == 0 ? (const void *)&fftz::fft_pp_kernel<float> : (const void *)&fftz::fft_pp_kernel<double>;
  } else {
    fn = fast_kernel(p->dtype, fftz::ct_log2(p->n), p->variant);
  }
  if (!fn) return (int)cudaErrorInvalidDeviceFunction;
  int seen = 0;
  for (int i = 0; i < nopted[dev]; i++)
    if (opted[dev][i] == fn) seen = 1;
  if (!seen) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fftz_smem_limit());
    if (e != cudaSuccess) return (int)e;
    if (nopted[dev] < 96) opted[dev][nopted[dev]++] = fn;
  }
  const dim3 block(p->variant == FFTZ_VAR_GENERIC_PP ? 256u : (unsigned)(p->tpc * p->tpt));
  const size_t smem = (size_t)fftz_pass_smem_bytes(p);
  dim3 grid((unsigned)nblk);
  if (is_pipe(p)) {
    // persistent: as many CTAs as fit on the device at once
    static const void *occ_fn[64][32];
    static size_t occ_smem[64][32];
    static int occ_val[64][32], nocc[64], nsm[64];
    int occ = 0;
    for (int i = 0; i < nocc[dev]; i++)
      if (occ_fn[dev][i] == fn && occ_smem[dev][i] == smem) occ = occ_val[dev][i];
    if (!occ) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, (int)block.x, smem) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        occ = 1;
      }
      if (!nsm[dev]) cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
      if (nocc[dev] < 32) {
        occ_fn[dev][nocc[dev]] = fn;
        occ_smem[dev][nocc[dev]] = smem;
        occ_val[dev][nocc[dev]++] = occ;
      }
    }
    if (!nsm[dev]) cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
    const int64_t cap = (int64_t)occ * (nsm[dev] > 0 ? nsm[dev] : 148);
    grid.x = (unsigned)(nblk < cap ? nblk : cap);
  }
  void *args[1] = {(void *)p};
  return (int)cudaLaunchKernel(fn, grid, block, args, smem, (cudaStream_t)stream);
}

}  // extern "C"
