/* Planner: problem descriptor -> flat list of GPU kernel passes (C99).
 *
 * The reference's selector walks a rule tree (selector/selector.c:509-789):
 * pow2 iterative for in-cache powers of two, four-step beyond the cache
 * (:603-633), batched / N-D row-column (:660-694), Bluestein when no kernel
 * radix divides N (:701-717), Cooley-Tukey otherwise (:772-786), and the
 * packed real path for even real lengths (:858-874). The same decisions are
 * made here against the GPU's limits instead of the CPU's caches:
 *
 *   line of length n fits one CTA's shared memory
 *       -> one pass (compile-time kernel for powers of two, generic otherwise)
 *   n too long for one CTA, all factors in {2,3,5,7,11,13}
 *       -> four-step n = n1 * n2 in two passes through scratch
 *          (column FFTs with the W_n^{j2 k1} twiddle fused into their store,
 *           then row FFTs whose store performs the transpose)
 *   any prime factor > 13
 *       -> Bluestein over a power-of-two convolution length m >= 2n - 1, in one
 *          kernel when m fits shared memory, in three passes otherwise
 *   N-D -> one line pass per dimension (dims[0] first, the rest in place)
 *   real, dims[0] even -> packed: n0/2-point complex FFT with the Hermitian
 *          recombination fused into the store (r2c) or the separation fused
 *          into the load (c2r); odd n0 -> full-length complex line.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fz_internal.h"

static int is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

static int ilog2i(int64_t n)
{
    int k = 0;
    while (((int64_t)1 << k) < n) k++;
    return k;
}

static int smooth13(int64_t n)
{
    static const int64_t pr[] = {2, 3, 5, 7, 11, 13};
    for (int i = 0; i < 6; i++)
        while (n % pr[i] == 0) n /= pr[i];
    return n == 1;
}

/* radix list of the generic kernel: balanced power-of-two part (<= 16 per
 * stage, largest first) followed by the odd prime factors */
static int generic_radices(int64_t n, int32_t *radix)
{
    int s = 0;
    int k = 0;
    while ((n & 1) == 0)
    {
        n >>= 1;
        k++;
    }
    if (k > 0)
    {
        int st = (k + 3) / 4;
        int base = k / st, extra = k % st;
        for (int i = 0; i < st; i++)
        {
            if (s >= FFTZ_MAX_STAGES) return -1;
            radix[s++] = 1 << (base + (i < extra ? 1 : 0));
        }
    }
    static const int64_t odd[] = {13, 11, 7, 5, 3};
    for (int i = 0; i < 5; i++)
        while (n % odd[i] == 0)
        {
            if (s >= FFTZ_MAX_STAGES) return -1;
            radix[s++] = (int32_t)odd[i];
            n /= odd[i];
        }
    return n == 1 ? s : -1;
}

static fz_pass *push_pass(fz_plan *pl)
{
    if (pl->npass == pl->cap)
    {
        int nc = pl->cap ? pl->cap * 2 : 8;
        fz_pass *np = (fz_pass *)realloc(pl->pass, sizeof(fz_pass) * (size_t)nc);
        if (!np) return NULL;
        pl->pass = np;
        pl->cap = nc;
    }
    fz_pass *p = &pl->pass[pl->npass++];
    memset(p, 0, sizeof(*p));
    p->off_tw = p->off_tw4hi = p->off_tw4lo = p->off_pre = p->off_post = p->off_mid = p->off_rtw = -1;
    p->k.dtype = pl->dtype;
    p->k.scale = 1.0;
    return p;
}

static int64_t absl(int64_t x) { return x < 0 ? -x : x; }

/* every pass on the generic kernel (the persistent executor runs only that) */
static int generic_only(const fz_plan *pl) { return pl->hints.kernel_family == 3; }

/* kernel_family 4: passes for the persistent ragged executor, whose CTAs have
 * 256 threads: compile-time kernels up to length 4096, never the pipelined
 * family */
static int ragged_mode(const fz_plan *pl) { return pl->hints.kernel_family == 4; }
static int64_t fast_max_n(const fz_plan *pl)
{
    const int64_t m = fftz_fast_max_n(pl->dtype);
    return ragged_mode(pl) && m > 4096 ? 4096 : m;
}
static int fast_max_threads(const fz_plan *pl) { return ragged_mode(pl) ? 256 : (pl->dtype == 0 ? 1024 : 512); }

/* Batch dims: optionally sorted by stride (smallest first, so that bdim[0]
 * is the one lanes may run along), then adjacent dims merged when they form
 * one arithmetic progression on both sides (the reference's fuse_vecs,
 * selector/selector.c:1861-1912). keep_first pins b[0] as the column dim. */
static int set_batch(fftz_pass_t *k, const fz_dim *b, int nb, int keep_first)
{
    fz_dim d[32];
    int m = 0;
    for (int i = 0; i < nb && m < 32; i++)
        if (b[i].n != 1) d[m++] = b[i];
    if (m == 0 && keep_first && nb > 0) d[m++] = b[0];
    int start = keep_first ? 1 : 0;
    for (int i = start + 1; i < m; i++)
        for (int j = i; j > start; j--)
        {
            int64_t sj = absl(d[j].is) < absl(d[j].os) ? absl(d[j].is) : absl(d[j].os);
            int64_t sp = absl(d[j - 1].is) < absl(d[j - 1].os) ? absl(d[j - 1].is) : absl(d[j - 1].os);
            if (sj < sp)
            {
                fz_dim t = d[j];
                d[j] = d[j - 1];
                d[j - 1] = t;
            }
        }
    /* merge neighbours that continue one another on both sides; a pinned
     * column dim stays separate because its index is the column number */
    int w = 0;
    for (int i = 0; i < m; i++)
    {
        if (w > 0 && !(keep_first && w == 1) && d[i].is == d[w - 1].is * d[w - 1].n &&
            d[i].os == d[w - 1].os * d[w - 1].n)
        {
            d[w - 1].n *= d[i].n;
            continue;
        }
        d[w++] = d[i];
    }
    if (w > FFTZ_MAX_BDIMS)
    {
        fz_set_error("too many independent batch dimensions (%d > %d)", w, FFTZ_MAX_BDIMS);
        return -1;
    }
    k->nbdims = w;
    k->ntf = 1;
    for (int i = 0; i < w; i++)
    {
        k->bdim[i] = d[i].n;
        k->ibs[i] = d[i].is;
        k->obs[i] = d[i].os;
        k->ntf *= d[i].n;
    }
    return 0;
}

/* shared memory of one ping-pong tile holding one line of n */
static int64_t pp_one_line_bytes(int dtype, int64_t n)
{
    const int64_t esz = dtype == 0 ? 8 : 16;
    return 2 * (int64_t)fftz_smem_stride(dtype, (int32_t)n) * esz + 24 + 8 * FFTZ_MAX_STAGES;
}

/* transforms per CTA: enough columns for coalesced column access, enough
 * work per CTA for short rows, bounded by threads and shared memory (two
 * slots for the double-buffered kernels) */
static int is_pipe_variant(int v) { return v == FFTZ_VAR_PIPE || v == FFTZ_VAR_PIPE_TW4; }

static void finish_launch_shape(fz_plan *pl, fftz_pass_t *k, int nslots, int maxthr)
{
    const int64_t esz = pl->dtype == 0 ? 8 : 16;
    const int pipe = is_pipe_variant(k->variant);
    const int colmap = (k->in_mode == 1 || k->out_mode == 1);
    k->sstride = fftz_smem_stride(pl->dtype, nslots);
    int by_thr = maxthr / k->tpt;
    if (by_thr < 1) by_thr = 1;
    const int64_t per_tf = (pipe ? 2 : 1) * ((int64_t)k->sstride + 16) * esz + (pipe ? 72 : 24);
    int64_t by_smem = fftz_smem_limit() / per_tf;
    int want;
    if (colmap)
    {
        /* column segments: 8 float columns (64 bytes); double columns 8 wide
         * (128 bytes) when whole tiles cover the columns, else 4 (measured on
         * B200, fp64 512^3 outer-dimension pass: 0.537 -> 0.442 ms with 8;
         * 257 columns: 0.572 ms with 4, 0.588 ms with 8) */
        want = pipe ? 2 : (pl->dtype == 0 ? 8 : (k->nbdims > 0 && k->bdim[0] % 8 == 0 ? 8 : 4));
    }
    else
    {
        int64_t per = pipe ? 4096 : (pl->dtype == 0 ? 4096 : 2048); /* complex elements per CTA */
        want = (int)((per + k->n - 1) / k->n);
        if (want * k->tpt < 128) want = (128 + k->tpt - 1) / k->tpt;
        /* double real lines in the compile-time real kernel: two lines per CTA
         * (measured on B200, fp64 512^3 real: r2c 0.95 -> 0.79 ms, c2r 0.79 ->
         * 0.70 ms against eight lines of 256 points; 1024-point lines equal) */
        if (k->variant == FFTZ_VAR_FAST_REAL && pl->dtype == 1) want = 2;
    }
    if (colmap && pl->hints.tpc_col > 0) want = pl->hints.tpc_col;
    if (!colmap && pl->hints.tpc_row > 0) want = pl->hints.tpc_row;
    int tpc = want;
    if (tpc > by_thr) tpc = by_thr;
    if (tpc > by_smem) tpc = (int)by_smem;
    if (tpc > k->ntf) tpc = (int)k->ntf;
    if (tpc > 1024) tpc = 1024;
    if (tpc < 1) tpc = 1;
    k->tpc = tpc;
    if (colmap) k->sstride = fftz_smem_stride_cols(pl->dtype, nslots, tpc);
}

static void set_modes(fftz_pass_t *k)
{
    k->in_mode = (k->nbdims > 0 && absl(k->ibs[0]) < absl(k->ies)) ? 1 : 0;
    k->out_mode = (k->nbdims > 0 && absl(k->obs[0]) < absl(k->oes)) ? 1 : 0;
}

/* one complex line pass in the shared-memory kernel; returns the pass */
static fz_pass *line_pass(fz_plan *pl, int64_t n, int64_t ies, int64_t oes, const fz_dim *b, int nb,
                          int keep_first, int src, int dst, int flags, int variant_bits)
{
    fz_pass *p = push_pass(pl);
    if (!p) return NULL;
    fftz_pass_t *k = &p->k;
    k->n = (int32_t)n;
    k->ies = ies;
    k->oes = oes;
    k->flags = flags;
    k->in_kind = FFTZ_IN_COMPLEX;
    k->out_kind = FFTZ_OUT_COMPLEX;
    k->nload = (int32_t)n;
    k->nstore = (int32_t)n;
    p->src = src;
    p->dst = dst;
    if (set_batch(k, b, nb, keep_first)) return NULL;
    set_modes(k);
    const int fast = !generic_only(pl) && is_pow2(n) && n >= 2 && n <= fast_max_n(pl);
    int maxthr;
    if (fast)
    {
        k->nstages = fftz_fast_radices((int)n, k->radix);
        k->tpt = fftz_fast_tpt((int)n);
        maxthr = fast_max_threads(pl);
        if (k->nstages == 1 && k->in_mode != k->out_mode) k->out_mode = k->in_mode;
        int tabs = (variant_bits & 2) != 0, tw4 = (flags & FFTZ_F_TW4) != 0;
        const int fam = pl->hints.kernel_family;
        const int pipe_ok = n >= 64 && !tabs && !(variant_bits & 4);
        /* the persistent double-buffered kernel is a tuning option (hint
         * kernel_family = 2); measured on B200 the one-tile-per-CTA kernel is
         * faster for both dtypes and both lane maps, so it is the default */
        const int pipe_default = 0;
        if (pipe_ok && (fam == 2 || (fam == 0 && pipe_default)))
            k->variant = tw4 ? FFTZ_VAR_PIPE_TW4 : FFTZ_VAR_PIPE;
        else if (variant_bits & 4)
            k->variant = FFTZ_VAR_FAST_BLUE;
        else if (tabs && tw4)
            k->variant = FFTZ_VAR_FAST_TW4_TABS;
        else if (tabs)
            k->variant = FFTZ_VAR_FAST_TABS;
        else if (tw4)
            k->variant = FFTZ_VAR_FAST_TW4;
        else
            k->variant = FFTZ_VAR_FAST;
        /* TMA-fed tiles: by default for column passes (measured on B200: pass A
         * of the 2^24 four-step 3% faster, row passes 13% slower), for every
         * qualifying pass with kernel_family 5, never with kernel_family 1 */
        k->use_tma = (k->variant == FFTZ_VAR_FAST || k->variant == FFTZ_VAR_FAST_TW4) &&
                     (fam == 5 || fam == 6 || (fam == 0 && k->in_mode == 1));
        if (k->use_tma && fam == 6) k->use_tma = 2; /* persistent, next tile half-prefetched */
        /* persistent register-resident tiles with the next tile prefetched
         * (4096-point float passes): by default where a column lane map
         * makes the tile four transforms wide (measured on B200: the 2^24
         * four-step's column pass 0.424 -> 0.324 ms, its row pass with the
         * transposed store 0.325 -> 0.303 ms; plain rows 9% slower, so they
         * keep the one-tile kernel), for every 4096-point float pass with
         * kernel_family = 8 */
        if ((k->variant == FFTZ_VAR_FAST || k->variant == FFTZ_VAR_FAST_TW4) && pl->dtype == 0 && n == 4096 &&
            (fam == 8 || (fam == 0 && (k->in_mode == 1 || k->out_mode == 1))))
            k->use_tma = 3;
        /* 16 x 256 split tiles (persistent, one exchange across the CTA per
         * tile): by default where the register-resident kernel was (measured
         * on B200, 2^24 four-step: column pass 0.300 -> 0.290 ms, row pass
         * with the transposed store 0.301 -> 0.251 ms), for every 4096-point
         * float pass with kernel_family 9 (one real component per exchange
         * round) or 10 (full complex values in two rounds, round-1 readers'
         * values stashed in shared memory: 0.326 / 0.282 ms) */
        if ((k->variant == FFTZ_VAR_FAST || k->variant == FFTZ_VAR_FAST_TW4) && pl->dtype == 0 && n == 4096 &&
            (fam == 9 || fam == 10 || fam == 11 || (fam == 0 && (k->in_mode == 1 || k->out_mode == 1))))
            k->use_tma = fam == 10 ? 5 : fam == 11 ? 6 : 4;
        /* persistent streaming row tiles, whole lines by 1-D bulk copies with
         * the next tile in flight (kernel_family 13) */
        if (k->variant == FFTZ_VAR_FAST && k->in_mode == 0 && fam == 13) k->use_tma = 7;
        /* stage twiddles copied to shared memory by each CTA (hint twiddles = 2) */
        k->smem_tw = pl->hints.twiddles == 2 && !ragged_mode(pl) && n >= 512;
        if ((tw4 || tabs) && n < 32 && !(variant_bits & 4))
        {
            /* small feature kernels are not instantiated: use the generic one */
            goto generic;
        }
        if (is_pipe_variant(k->variant)) maxthr = fftz_pipe_max_threads((int)n);
        k->fuse_load = 1;
        k->fuse_store = 1;
    }
    else
    {
    generic:
        k->variant = FFTZ_VAR_GENERIC;
        k->nstages = n > 1 ? generic_radices(n, k->radix) : 0;
        if (k->nstages < 0)
        {
            fz_set_error("length %lld has no radix decomposition", (long long)n);
            return NULL;
        }
        k->tpt = k->nstages ? fftz_threads_per_transform(pl->dtype, (int)n, k->nstages, k->radix) : 1;
        maxthr = fftz_generic_max_threads();
        /* lines longer than the in-place tile's thread budget run as ping-pong
         * tiles (chosen below) */
        if (k->tpt > maxthr && pl->hints.kernel_family != 12 && pp_one_line_bytes(pl->dtype, n) <= fftz_smem_limit())
            k->tpt = maxthr;
        if (k->tpt > maxthr)
        {
            fz_set_error("length %lld exceeds the generic kernel's thread budget", (long long)n);
            return NULL;
        }
        k->fuse_load = 0;
        k->fuse_store = 0;
    }
    int nslots = (int)n;
    if (k->nload > nslots) nslots = k->nload;
    finish_launch_shape(pl, k, nslots, maxthr);
    /* split tiles hold four transforms: row passes take four per CTA too when
     * whole tiles cover the first batch dimension */
    const int split = k->use_tma >= 4 && k->use_tma <= 6;
    if (split && k->tpc < 4 && pl->hints.tpc_row == 0 && k->nbdims > 0 && k->bdim[0] % 4 == 0) k->tpc = 4;
    if (split && k->tpc != 4) k->use_tma = 3; /* no whole tiles: register-resident kernel */
    if (is_pipe_variant(k->variant) && fftz_pass_smem_bytes(k) > fftz_smem_limit())
    {
        /* two slots do not fit: the one-tile-per-CTA kernel of the same shape */
        k->variant = k->variant == FFTZ_VAR_PIPE_TW4 ? FFTZ_VAR_FAST_TW4 : FFTZ_VAR_FAST;
        maxthr = fast_max_threads(pl);
        finish_launch_shape(pl, k, nslots, maxthr);
    }
    if (k->smem_tw && fftz_pass_smem_bytes(k) > fftz_smem_limit()) k->smem_tw = 0;
    /* runtime-radix lines: the ping-pong kernel (two shared-memory buffers,
     * one butterfly per thread at a time, 256 threads) when both buffers fit;
     * kernel_family 12 keeps the in-place kernel */
    if (k->variant == FFTZ_VAR_GENERIC && pl->hints.kernel_family != 12)
    {
        const int esz = pl->dtype == 0 ? 8 : 16;
        const int32_t sst = fftz_smem_stride(pl->dtype, nslots);
        const int colm = (k->in_mode == 1 || k->out_mode == 1);
        /* about 4096 float (2048 double) elements per CTA: measured on B200,
         * mixed1000 (N = 1000, batch 32768) 0.618 ms per step with two lines
         * per CTA, 0.498 with four, 0.732 with eight (one CTA per SM) */
        int64_t want = (pl->dtype == 0 ? 4096 : 2048) / n;
        if (colm && want < (pl->dtype == 0 ? 8 : 4)) want = pl->dtype == 0 ? 8 : 4;
        if (colm && pl->hints.tpc_col > 0) want = pl->hints.tpc_col;
        if (!colm && pl->hints.tpc_row > 0) want = pl->hints.tpc_row;
        if (want < 1) want = 1;
        if (want > 64) want = 64;
        if (want > k->ntf) want = k->ntf;
        while (want > 1 && 2 * want * sst * esz + 24 * want + 8 * FFTZ_MAX_STAGES > fftz_smem_limit()) want--;
        if (2 * want * (int64_t)sst * esz + 24 * want + 8 * FFTZ_MAX_STAGES <= fftz_smem_limit())
        {
            k->variant = FFTZ_VAR_GENERIC_PP;
            k->tpc = (int32_t)want;
            k->sstride = sst;
            k->tpt = (int32_t)(256 / want > 0 ? 256 / want : 1);
            /* complex lines read HBM in their first stage and write it in
             * their last (the load / store phases stay for the other kinds
             * and for load-side tables) */
            k->fuse_load = k->nstages > 0 && k->in_kind == FFTZ_IN_COMPLEX && k->nload == n &&
                           !(flags & FFTZ_F_PRE_TAB);
            k->fuse_store = k->nstages > 0 && k->out_kind == FFTZ_OUT_COMPLEX && k->nstore == n;
        }
    }
    if (fftz_pass_smem_bytes(k) > fftz_smem_limit())
    {
        fz_set_error("length %lld does not fit shared memory", (long long)n);
        return NULL;
    }
    /* kernel_family 7: 4096-point float rows as two radix-64 tensor-core GEMM
     * stages (three-term BF16 operands, FP32 accuracy; on request only) */
    if (pl->hints.kernel_family == 7 && k->variant == FFTZ_VAR_FAST && n == 4096 && pl->dtype == 0 &&
        k->in_mode == 0 && ies == 1 && k->ntf % 2 == 0 && (flags & ~(FFTZ_F_CONJ_IN | FFTZ_F_CONJ_OUT)) == 0)
    {
        k->variant = FFTZ_VAR_TC;
        k->tpc = 2;
        k->use_tma = 0;
        k->smem_tw = 0;
        p->off_tw = fz_tc64_tables(&pl->blob);
        if (p->off_tw < 0) return NULL;
        snprintf(p->what, sizeof(p->what), "tc n=%lld x%lld", (long long)n, (long long)k->ntf);
        return p;
    }
    if (k->nstages > 0)
    {
        p->off_tw = fz_stage_twiddles(&pl->blob, pl->dtype, (int)n, k->nstages, k->radix, k->tw_off);
        if (p->off_tw < 0) return NULL;
    }
    snprintf(p->what, sizeof(p->what), "%s n=%lld x%lld",
             k->variant == FFTZ_VAR_GENERIC ? "generic"
             : k->variant == FFTZ_VAR_GENERIC_PP ? "generic-pp"
                                                 : (is_pipe_variant(k->variant) ? "pipe" : "fast"),
             (long long)n, (long long)k->ntf);
    return p;
}

static int single_pass_ok(const fz_plan *pl, int64_t n)
{
    if (n == 1) return 1;
    if (!generic_only(pl) && is_pow2(n) && n <= fast_max_n(pl)) return 1;
    int32_t r[FFTZ_MAX_STAGES];
    int s = generic_radices(n, r);
    if (s < 0 || n > (1 << 20)) return 0;
    /* the executor's tiles (ragged batches) are ping-pong tiles within its cap */
    if (ragged_mode(pl)) return pp_one_line_bytes(pl->dtype, n) <= fz_ragged_smem_cap(pl->dtype);
    if (pl->hints.kernel_family != 12 && pp_one_line_bytes(pl->dtype, n) <= fftz_smem_limit()) return 1;
    int tpt = fftz_threads_per_transform(pl->dtype, (int)n, s, r);
    if (tpt < 1 || tpt > fftz_generic_max_threads()) return 0;
    int64_t esz = pl->dtype == 0 ? 8 : 16;
    return (int64_t)fftz_smem_stride(pl->dtype, (int32_t)n) * esz + 24 <= fftz_smem_limit();
}

/* n = n1 * n2 with both single-pass lengths; prefers powers of two and a
 * balanced split with n1 >= n2 (the reference's pow2_balanced_split,
 * core/common/pow2_radix_decompose.c:15-35) */
static int splittable(const fz_plan *pl, int64_t n)
{
    const int64_t m = fast_max_n(pl);
    return single_pass_ok(pl, n) || (smooth13(n) && n <= m * m);
}

static int choose_split(const fz_plan *pl, int64_t n, int64_t *n1, int64_t *n2)
{
    int64_t best1 = 0, best2 = 0;
    double bestscore = 1e300;
    int64_t h1 = pl->depth == 0 ? pl->hints.fourstep_n1 : 0;
    if (h1 > 1 && n % h1 == 0 && n / h1 > 1 && single_pass_ok(pl, h1) && splittable(pl, n / h1))
    {
        *n1 = h1;
        *n2 = n / h1;
        return 0;
    }
    for (int64_t a = 2; a * 2 <= n && a <= 1 << 20; a++)
    {
        if (n % a) continue;
        int64_t b = n / a;
        if (b < 2 || !single_pass_ok(pl, a) || !single_pass_ok(pl, b)) continue;
        double score = (a > b ? (double)a / b : (double)b / a) + (is_pow2(a) ? 0 : 0.5) + (is_pow2(b) ? 0 : 0.5) +
                       (a < b ? 0.25 : 0);
        if (score < bestscore)
        {
            bestscore = score;
            best1 = a;
            best2 = b;
        }
    }
    if (!best1) return -1;
    *n1 = best1;
    *n2 = best2;
    return 0;
}

static int64_t lines_of(const fz_dim *b, int nb)
{
    int64_t t = 1;
    for (int i = 0; i < nb; i++) t *= b[i].n;
    return t;
}

/* a new plan-owned scratch array of elems complex elements; returns its
 * buffer id, or -1 when the plan already holds the maximum number */
static int new_scratch(fz_plan *pl, int64_t elems)
{
    if (pl->nscratch >= FZ_MAX_SCRATCH)
    {
        fz_set_error("plan needs more than %d scratch arrays", FZ_MAX_SCRATCH);
        return -1;
    }
    pl->scratch_elems[pl->nscratch] = elems;
    return FZ_BUF_SCR0 + pl->nscratch++;
}

/* Four-step split of one line of length n = n1 * n2 (logical j = n2 j1 + j2,
 * k = k1 + n1 k2), the reference's pow2 four-step solver
 * (core/solvers/complex/pow2_fourstep_solver_dft.c:700-763) with its fused
 * twiddle+transpose (core/kernels/non_dft/fused_twiddle_transpose) folded into
 * the two passes' stores. */
static int fourstep(fz_plan *pl, int64_t n, int64_t ies, int64_t oes, const fz_dim *b, int nb, int src, int dst,
                    int flags);

static int fourstep_lines(fz_plan *pl, int64_t n, int64_t n1, int64_t n2, int64_t ies, int64_t oes, const fz_dim *b,
                          int nb, int src, int dst, int flags, int64_t in_off, int64_t out_off, int64_t hi,
                          int64_t lo, int64_t L, int S)
{
    fz_dim bb[FFTZ_MAX_BDIMS + 2];
    /* pass A: columns j2 of the n1 x n2 view; scratch layout [line][k1][j2] */
    bb[0].n = n2;
    bb[0].is = ies;
    bb[0].os = 1;
    int64_t so = n;
    for (int i = 0; i < nb; i++)
    {
        bb[i + 1] = b[i];
        bb[i + 1].os = so;
        so *= b[i].n;
    }
    fz_pass *pa = line_pass(pl, n1, n2 * ies, n2, bb, nb + 1, 1, src, S, (flags & FFTZ_F_CONJ_IN) | FFTZ_F_TW4, 0);
    if (!pa) return -1;
    pa->k.tw4_n = n;
    pa->k.tw4_l = L;
    pa->off_tw4hi = hi;
    pa->off_tw4lo = lo;
    pa->in_off = in_off;
    /* pass B: rows k1 (contiguous j2) -> X[k1 + n1 k2] */
    bb[0].n = n1;
    bb[0].is = n2;
    bb[0].os = oes;
    so = n;
    for (int i = 0; i < nb; i++)
    {
        bb[i + 1] = b[i];
        bb[i + 1].is = so;
        so *= b[i].n;
    }
    if (!single_pass_ok(pl, n2))
    {
        /* the rows are themselves split: a nested four-step over length n2 */
        if (out_off) return -1;
        pl->depth++;
        int rc = fourstep(pl, n2, 1, n1 * oes, bb, nb + 1, S, dst, flags & FFTZ_F_CONJ_OUT);
        pl->depth--;
        return rc;
    }
    fz_pass *pb = line_pass(pl, n2, 1, n1 * oes, bb, nb + 1, 1, S, dst, flags & FFTZ_F_CONJ_OUT, 0);
    if (!pb) return -1;
    pb->out_off = out_off;
    /* 4096 x 4096 on split tiles both ways: the intermediate in 4 x 4 blocks,
     * so that the column pass writes whole 128-byte lines and the row pass
     * reads its four rows as one contiguous slab */
    if (n1 == 4096 && n2 == 4096 && pl->dtype == 0 && pa->k.use_tma == 4 && pb->k.use_tma == 4 &&
        pa->k.tpc == 4 && pb->k.tpc == 4 && pb->k.in_mode == 0 && pb->k.out_mode == 1 && pb->k.ibs[0] == n2)
    {
        pa->k.flags |= FFTZ_F_BLK4_OUT;
        pb->k.flags |= FFTZ_F_BLK4_IN;
    }
    return 0;
}

/* Four-step split of one line of length n = n1 * n2 (logical j = n2 j1 + j2,
 * k = k1 + n1 k2), the reference's pow2 four-step solver
 * (core/solvers/complex/pow2_fourstep_solver_dft.c:700-763) with its fused
 * twiddle+transpose (core/kernels/non_dft/fused_twiddle_transpose) folded into
 * the two passes' stores. With a batch chunk, the two passes run per chunk of
 * lines so that the intermediate of a chunk can stay in L2. */
static int fourstep(fz_plan *pl, int64_t n, int64_t ies, int64_t oes, const fz_dim *b, int nb, int src, int dst,
                    int flags)
{
    int64_t n1, n2;
    if (choose_split(pl, n, &n1, &n2)) return -1;
    int64_t L, hi, lo;
    if (fz_tw4_tables(&pl->blob, pl->dtype, n, &L, &hi, &lo)) return -1;
    int64_t lines = lines_of(b, nb);
    int64_t chunk = pl->hints.batch_chunk;
    int nbig = 0;
    for (int i = 0; i < nb; i++)
        if (b[i].n > 1) nbig++;
    if (chunk > 0 && chunk < lines && nbig == 1)
    {
        const int64_t esz = pl->dtype == 0 ? 8 : 16;
        fz_dim one;
        for (int i = 0; i < nb; i++)
            if (b[i].n > 1) one = b[i];
        int S = new_scratch(pl, n * chunk);
        if (S < 0 || !single_pass_ok(pl, n2)) return -1;
        for (int64_t c0 = 0; c0 < lines; c0 += chunk)
        {
            fz_dim cb = one;
            cb.n = (lines - c0 < chunk) ? lines - c0 : chunk;
            if (fourstep_lines(pl, n, n1, n2, ies, oes, &cb, 1, src, dst, flags, c0 * one.is * esz,
                               c0 * one.os * esz, hi, lo, L, S))
                return -1;
        }
        return 0;
    }
    int S = new_scratch(pl, n * lines);
    if (S < 0) return -1;
    return fourstep_lines(pl, n, n1, n2, ies, oes, b, nb, src, dst, flags, 0, 0, hi, lo, L, S);
}

/* Bluestein (chirp-z) over a power-of-two m >= 2n - 1 (the reference pads to
 * a 13-smooth m, core/common/bluestein_utils.c:39-67; a power of two keeps
 * every sub-transform on the compile-time kernels). */
static int bluestein(fz_plan *pl, int64_t n, int64_t ies, int64_t oes, const fz_dim *b, int nb, int src, int dst)
{
    int64_t m = 1;
    while (m < 2 * n - 1) m *= 2;
    int64_t pre, post, mid;
    if (fz_bluestein_tables(&pl->blob, pl->dtype, n, m, pl->direction, &pre, &post, &mid)) return -1;
    const int bwd = pl->direction == 1;
    if (m >= 4 && single_pass_ok(pl, m))
    {
        fz_pass *p = line_pass(pl, m, ies, oes, b, nb, 0, src, dst,
                               (bwd ? FFTZ_F_CONJ_IN : FFTZ_F_CONJ_OUT) | FFTZ_F_PRE_TAB | FFTZ_F_POST_TAB |
                                   FFTZ_F_MID_TAB,
                               2 | 4);
        if (!p) return -1;
        p->k.pre_n = n;
        p->k.pre_es = 1;
        p->k.post_n = n;
        p->k.post_es = 1;
        p->off_pre = pre;
        p->off_post = post;
        p->off_mid = mid;
        snprintf(p->what, sizeof(p->what), "bluestein n=%lld m=%lld x%lld", (long long)n, (long long)m,
                 (long long)p->k.ntf);
        return 0;
    }
    /* three passes through S0 / S1: A (column FFTs of the chirped, padded
     * input), M (row FFTs, spectrum product, row FFTs of the second FFT_m),
     * D (row FFTs of the second FFT_m, output chirp) */
    int64_t n1, n2;
    if (choose_split(pl, m, &n1, &n2)) return -1;
    int64_t lines = lines_of(b, nb);
    const int S0 = new_scratch(pl, m * lines), S1 = new_scratch(pl, m * lines);
    if (S0 < 0 || S1 < 0) return -1;
    int64_t L, hi, lo;
    if (fz_tw4_tables(&pl->blob, pl->dtype, m, &L, &hi, &lo)) return -1;
    fz_dim bb[FFTZ_MAX_BDIMS + 2];
    int64_t so;
    /* A: src -> S0, column FFTs of the padded chirped input */
    bb[0].n = n2;
    bb[0].is = ies;
    bb[0].os = 1;
    so = m;
    for (int i = 0; i < nb; i++)
    {
        bb[i + 1] = b[i];
        bb[i + 1].os = so;
        so *= b[i].n;
    }
    fz_pass *pa = line_pass(pl, n1, n2 * ies, n2, bb, nb + 1, 1, src, S0,
                            (bwd ? FFTZ_F_CONJ_IN : 0) | FFTZ_F_PRE_TAB | FFTZ_F_TW4, 2);
    if (!pa) return -1;
    pa->k.pre_n = n;
    pa->k.pre_es = n2;
    pa->k.pre_cs = 1;
    pa->k.tw4_n = m;
    pa->k.tw4_l = L;
    pa->off_tw4hi = hi;
    pa->off_tw4lo = lo;
    pa->off_pre = pre;
    /* M: S0 -> S1, one pass per row k1 (contiguous j2): forward FFT over j2
     * (the second half of FFT_m of the chirped input, spectrum index
     * k = k1 + n1 k2), v = conj(v) * conj(Bhat)[k] (table rows made contiguous),
     * then the first half of the second FFT_m with the split swapped
     * (n2 x n1): the FFT over k2 for this k1, times W_m^{k1 k1'}, stored
     * transposed as S1[k1'][k1]. Three passes through scratch instead of four. */
    const int64_t midT = fz_blob_permute(&pl->blob, pl->dtype, mid, n1, n2);
    if (midT < 0) return -1;
    bb[0].n = n1;
    bb[0].is = n2;
    bb[0].os = 1;
    so = m;
    for (int i = 0; i < nb; i++)
    {
        bb[i + 1] = b[i];
        bb[i + 1].is = so;
        bb[i + 1].os = so;
        so *= b[i].n;
    }
    fz_pass *pm = line_pass(pl, n2, 1, n1, bb, nb + 1, 1, S0, S1, FFTZ_F_MID_TAB | FFTZ_F_TW4, 2 | 4);
    if (!pm) return -1;
    pm->k.mid_cs = n2;
    pm->off_mid = midT;
    pm->k.tw4_n = m;
    pm->k.tw4_l = L;
    pm->off_tw4hi = hi;
    pm->off_tw4lo = lo;
    snprintf(pm->what, sizeof(pm->what), "bluestein-mid n=%lld m=%lld x%lld", (long long)n, (long long)m,
             (long long)pm->k.ntf);
    /* D: S1 -> dst, rows k1' (contiguous k1): FFT over k1 -> k2', output
     * k' = k1' + n2 k2' in natural order, X_k' = chirp_k' * conv_k' / m for k' < n */
    bb[0].n = n2;
    bb[0].is = n1;
    bb[0].os = oes;
    so = m;
    for (int i = 0; i < nb; i++)
    {
        bb[i + 1] = b[i];
        bb[i + 1].is = so;
        so *= b[i].n;
    }
    fz_pass *pd = line_pass(pl, n1, 1, n2 * oes, bb, nb + 1, 1, S1, dst,
                            (bwd ? 0 : FFTZ_F_CONJ_OUT) | FFTZ_F_POST_TAB, 2);
    if (!pd) return -1;
    pd->k.post_n = n;
    pd->k.post_es = n2;
    pd->k.post_cs = 1;
    pd->off_post = post;
    return 0;
}

/* one complex line transform of length n over batch b */
static int add_line(fz_plan *pl, int64_t n, int64_t ies, int64_t oes, const fz_dim *b, int nb, int src, int dst)
{
    const int flags = pl->direction ? (FFTZ_F_CONJ_IN | FFTZ_F_CONJ_OUT) : 0;
    const int algo = pl->hints.algorithm;
    if (n == 1 && src == dst) return 0;
    if (algo == 3 && n > 1) return bluestein(pl, n, ies, oes, b, nb, src, dst);
    if (algo != 2 && single_pass_ok(pl, n))
    {
        /* a column-mapped pass over a column count that whole tiles do not
         * cover (the n0/2 + 1 half-spectrum columns of a real N-D transform)
         * cannot take TMA-fed tiles: the largest multiple of 8 columns runs as
         * one pass, the rest as a second (measured on B200, fp64 512^3 real:
         * the 257-column pass 0.571 ms in one, 0.483 + 0.019 ms in two) */
        int c = -1;
        for (int i = 0; i < nb; i++)
            if (c < 0 || absl(b[i].is) < absl(b[c].is)) c = i;
        int merged8 = 0; /* the column dim continues into another one: whole tiles cover the merged run */
        for (int i = 0; c >= 0 && i < nb; i++)
            if (i != c && b[i].is == b[c].n * b[c].is && b[i].os == b[c].n * b[c].os && (b[c].n * b[i].n) % 8 == 0)
                merged8 = 1;
        if (c >= 0 && !merged8 && nb <= 16 && !ragged_mode(pl) && is_pow2(n) && n <= fast_max_n(pl) &&
            b[c].n > 8 && b[c].n % 8 != 0 && absl(b[c].is) < absl(ies) && absl(b[c].os) < absl(oes))
        {
            const int64_t esz = pl->dtype == 0 ? 8 : 16;
            fz_dim bm[16];
            memcpy(bm, b, sizeof(fz_dim) * (size_t)nb);
            const int64_t m = b[c].n - b[c].n % 8;
            bm[c].n = m;
            if (!line_pass(pl, n, ies, oes, bm, nb, 0, src, dst, flags, 0)) return -1;
            bm[c].n = b[c].n - m;
            fz_pass *r = line_pass(pl, n, ies, oes, bm, nb, 0, src, dst, flags, 0);
            if (!r) return -1;
            r->in_off = m * b[c].is * esz;
            r->out_off = m * b[c].os * esz;
            return 0;
        }
        return line_pass(pl, n, ies, oes, b, nb, 0, src, dst, flags, 0) ? 0 : -1;
    }
    if (smooth13(n) && n <= fast_max_n(pl) * fast_max_n(pl))
    {
        if (src == dst)
        {
            /* in place: the four-step reads all of src before the row pass writes dst */
        }
        if (fourstep(pl, n, ies, oes, b, nb, src, dst, flags) == 0) return 0;
    }
    return bluestein(pl, n, ies, oes, b, nb, src, dst);
}

/* batch list for the line along dimension d: all other dims, then vecs */
static int other_dims(const fz_dim *dims, int rank, int d, const fz_dim *vecs, int vrank, fz_dim *out, int use_out)
{
    int m = 0;
    for (int i = 0; i < rank; i++)
        if (i != d)
        {
            out[m] = dims[i];
            if (use_out) out[m].is = out[m].os;
            m++;
        }
    for (int i = 0; i < vrank; i++)
    {
        out[m] = vecs[i];
        if (use_out) out[m].is = out[m].os;
        m++;
    }
    return m;
}

static int plan_c2c(fz_plan *pl, int rank, const fz_dim *dims, int vrank, const fz_dim *vecs)
{
    fz_dim b[64];
    for (int d = 0; d < rank; d++)
    {
        int first = d == 0;
        int nb = other_dims(dims, rank, d, vecs, vrank, b, !first);
        int src = first ? FZ_BUF_IN : FZ_BUF_OUT;
        int64_t ies = first ? dims[d].is : dims[d].os;
        if (add_line(pl, dims[d].n, ies, dims[d].os, b, nb, src, FZ_BUF_OUT)) return -1;
    }
    return 0;
}

/* real line along dims[0]: r2c (forward) or c2r (backward) in one generic pass */
static fz_pass *real_pass(fz_plan *pl, int64_t n0, int64_t ies, int64_t oes, const fz_dim *b, int nb, int src,
                          int dst)
{
    fz_pass *p = push_pass(pl);
    if (!p) return NULL;
    fftz_pass_t *k = &p->k;
    const int packed = (n0 % 2 == 0) && n0 >= 2;
    const int64_t n = packed ? n0 / 2 : n0;
    k->n = (int32_t)n;
    k->ies = ies;
    k->oes = oes;
    p->src = src;
    p->dst = dst;
    if (pl->direction == 0)
    {
        k->in_kind = packed ? FFTZ_IN_REAL_PAIRS : FFTZ_IN_REAL;
        k->out_kind = packed ? FFTZ_OUT_HALF_RECOMBINE : FFTZ_OUT_HALF;
        k->nload = (int32_t)n;
        k->nstore = (int32_t)(n0 / 2 + 1);
    }
    else
    {
        k->in_kind = packed ? FFTZ_IN_HERM_SEPARATE : FFTZ_IN_HERM_FULL;
        k->out_kind = packed ? FFTZ_OUT_REAL_PAIRS : FFTZ_OUT_REAL;
        k->nload = (int32_t)(packed ? n + 1 : n);
        k->nstore = (int32_t)n;
        k->flags = packed ? FFTZ_F_CONJ_OUT : FFTZ_F_CONJ_IN;
    }
    if (set_batch(k, b, nb, 0)) return NULL;
    /* element stride of the real side is doubled for pairs */
    int64_t es_in = (k->in_kind == FFTZ_IN_REAL_PAIRS) ? 2 * ies : ies;
    int64_t es_out = (k->out_kind == FFTZ_OUT_REAL_PAIRS) ? 2 * oes : oes;
    k->in_mode = (k->nbdims > 0 && absl(k->ibs[0]) < absl(es_in)) ? 1 : 0;
    k->out_mode = (k->nbdims > 0 && absl(k->obs[0]) < absl(es_out)) ? 1 : 0;
    /* power-of-two packed lines: compile-time stages between the generic
     * load and store phases (measured on B200, fp64 512^3 r2c: the 512-point
     * row pass at 1.14 TB/s with the generic kernel) */
    const int fast = packed && !generic_only(pl) && is_pow2(n) && n <= fast_max_n(pl) &&
                     !(k->flags & FFTZ_F_CONJ_IN) && fftz_fast_real_kernel(pl->dtype, ilog2i(n)) != NULL;
    int maxthr = fftz_generic_max_threads();
    if (fast)
    {
        k->variant = FFTZ_VAR_FAST_REAL;
        k->nstages = fftz_fast_radices((int)n, k->radix);
        k->tpt = fftz_fast_tpt((int)n);
        maxthr = fast_max_threads(pl);
    }
    else
    {
        k->variant = FFTZ_VAR_GENERIC;
        k->nstages = n > 1 ? generic_radices(n, k->radix) : 0;
        if (k->nstages < 0)
        {
            fz_set_error("real length %lld has no radix decomposition", (long long)n0);
            return NULL;
        }
        k->tpt = k->nstages ? fftz_threads_per_transform(pl->dtype, (int)n, k->nstages, k->radix) : 1;
    }
    if (k->tpt < 1 || k->tpt > maxthr)
    {
        fz_set_error("real length %lld exceeds the one-pass real kernel", (long long)n0);
        return NULL;
    }
    int nslots = k->nload > n ? k->nload : (int)n;
    finish_launch_shape(pl, k, nslots, maxthr);
    if (fftz_pass_smem_bytes(k) > fftz_smem_limit())
    {
        fz_set_error("real length %lld does not fit shared memory", (long long)n0);
        return NULL;
    }
    if (k->nstages > 0)
    {
        p->off_tw = fz_stage_twiddles(&pl->blob, pl->dtype, (int)n, k->nstages, k->radix, k->tw_off);
        if (p->off_tw < 0) return NULL;
    }
    if (packed)
    {
        p->off_rtw = fz_real_twiddles(&pl->blob, pl->dtype, n);
        if (p->off_rtw < 0) return NULL;
    }
    snprintf(p->what, sizeof(p->what), "%s n=%lld x%lld", pl->direction ? "c2r" : "r2c", (long long)n0,
             (long long)k->ntf);
    return p;
}

static int real_pass_ok(const fz_plan *pl, int64_t n0)
{
    const int packed = (n0 % 2 == 0) && n0 >= 2;
    const int64_t n = packed ? n0 / 2 : n0;
    if (n == 1) return 1;
    int32_t r[FFTZ_MAX_STAGES];
    int s = generic_radices(n, r);
    if (s < 0) return 0;
    int tpt = fftz_threads_per_transform(pl->dtype, (int)n, s, r);
    if (tpt < 1 || tpt > fftz_generic_max_threads()) return 0;
    int64_t esz = pl->dtype == 0 ? 8 : 16;
    return (int64_t)fftz_smem_stride(pl->dtype, (int32_t)(n + 1)) * esz + 24 <= fftz_smem_limit();
}

static fz_pass *elem_pass(fz_plan *pl, int mode, int64_t n, int64_t nout, int64_t is, int64_t os, const fz_dim *b,
                          int nb, int src, int dst)
{
    fz_pass *p = push_pass(pl);
    if (!p) return NULL;
    p->is_elem = 1;
    fftz_elem_t *e = &p->e;
    e->mode = mode;
    e->dtype = pl->dtype;
    e->n = n;
    e->nout = nout;
    e->is = is;
    e->os = os;
    e->nlines = 1;
    int m = 0;
    for (int i = 0; i < nb; i++)
    {
        if (b[i].n == 1) continue;
        if (m >= FFTZ_MAX_BDIMS)
        {
            fz_set_error("too many batch dimensions for a real line");
            return NULL;
        }
        e->bdim[m] = b[i].n;
        e->ibs[m] = b[i].is;
        e->obs[m] = b[i].os;
        e->nlines *= b[i].n;
        m++;
    }
    e->nbdims = m;
    p->src = src;
    p->dst = dst;
    static const char *names[] = {"widen", "widen-pairs", "recombine", "separate", "herm-expand", "narrow-half",
                                  "real-out", "pairs-out"};
    snprintf(p->what, sizeof(p->what), "elem %s n=%lld x%lld", names[mode], (long long)n, (long long)e->nlines);
    return p;
}

/* Real line of length n0 along dims[0] that one CTA cannot hold: widen into a
 * dense complex scratch line (R), run any complex line algorithm on it, then
 * recombine / narrow into the destination. Packed (even n0) lines use the
 * n0/2-point complex transform as the reference's packed solver does. */
static int real_line_multipass(fz_plan *pl, int64_t n0, int64_t ies, int64_t oes, const fz_dim *b, int nb, int src,
                               int dst)
{
    const int packed = (n0 % 2 == 0);
    const int64_t len = packed ? n0 / 2 : n0;
    fz_dim side_in[32], side_out[32], dense[32];
    int64_t ds = len;
    for (int i = 0; i < nb; i++)
    {
        dense[i] = b[i];
        dense[i].is = dense[i].os = ds;
        ds *= b[i].n;
        side_in[i] = b[i];
        side_in[i].os = dense[i].os;
        side_out[i] = b[i];
        side_out[i].is = dense[i].is;
    }
    const int RB = new_scratch(pl, ds);
    if (RB < 0) return -1;
    int64_t rtw = -1;
    if (packed && (rtw = fz_real_twiddles(&pl->blob, pl->dtype, len)) < 0) return -1;
    fz_pass *p;
    if (pl->direction == 0)
    {
        p = elem_pass(pl, packed ? FFTZ_ELEM_WIDEN_PAIRS : FFTZ_ELEM_WIDEN_REAL, len, len, ies, 1, side_in, nb, src,
                      RB);
        if (!p) return -1;
        if (add_line(pl, len, 1, 1, dense, nb, RB, RB)) return -1;
        p = elem_pass(pl, packed ? FFTZ_ELEM_RECOMBINE : FFTZ_ELEM_NARROW_HALF, len, n0 / 2 + 1, 1, oes, side_out, nb,
                      RB, dst);
        if (!p) return -1;
        p->off_rtw = rtw;
        return 0;
    }
    p = elem_pass(pl, packed ? FFTZ_ELEM_SEPARATE : FFTZ_ELEM_HERM_EXPAND, len, len, ies, 1, side_in, nb, src,
                  RB);
    if (!p) return -1;
    p->off_rtw = rtw;
    if (add_line(pl, len, 1, 1, dense, nb, RB, RB)) return -1;
    p = elem_pass(pl, packed ? FFTZ_ELEM_PAIRS_OUT : FFTZ_ELEM_REAL_OUT, len, len, 1, oes, side_out, nb, RB,
                  dst);
    return p ? 0 : -1;
}

static int real_line(fz_plan *pl, int64_t n0, int64_t ies, int64_t oes, const fz_dim *b, int nb, int src, int dst)
{
    if (real_pass_ok(pl, n0)) return real_pass(pl, n0, ies, oes, b, nb, src, dst) ? 0 : -1;
    return real_line_multipass(pl, n0, ies, oes, b, nb, src, dst);
}

static int plan_real(fz_plan *pl, int rank, const fz_dim *dims, int vrank, const fz_dim *vecs)
{
    const int64_t n0 = dims[0].n;
    const int64_t h0 = n0 / 2 + 1;
    fz_dim b[64];
    if (pl->direction == 0)
    {
        /* r2c along dims[0] (real in -> half-complex out), then c2c in place */
        int nb = other_dims(dims, rank, 0, vecs, vrank, b, 0);
        if (real_line(pl, n0, dims[0].is, dims[0].os, b, nb, FZ_BUF_IN, FZ_BUF_OUT)) return -1;
        fz_dim hd[16];
        for (int i = 0; i < rank; i++)
        {
            hd[i] = dims[i];
            hd[i].is = hd[i].os;
        }
        hd[0].n = h0;
        for (int d = 1; d < rank; d++)
        {
            int m = other_dims(hd, rank, d, vecs, vrank, b, 1);
            if (add_line(pl, dims[d].n, dims[d].os, dims[d].os, b, m, FZ_BUF_OUT, FZ_BUF_OUT)) return -1;
        }
        return 0;
    }
    /* c2r: outer dims first on the half-complex array, then c2r along dims[0].
     * Out-of-place keeps the input intact: the c2c passes work in scratch W. */
    int src = FZ_BUF_IN;
    fz_dim hd[16];
    for (int i = 0; i < rank; i++) hd[i] = dims[i];
    hd[0].n = h0;
    fz_dim hv[16];
    for (int i = 0; i < vrank; i++) hv[i] = vecs[i];
    if (rank > 1)
    {
        int work = FZ_BUF_IN;
        if (pl->placement != 0)
        {
            int64_t tot = 1;
            for (int i = 0; i < rank; i++) tot *= hd[i].n;
            for (int i = 0; i < vrank; i++) tot *= hv[i].n;
            work = new_scratch(pl, tot);
            if (work < 0) return -1;
        }
        fz_dim sd[16], sv[16];
        int64_t st = 1;
        for (int i = 0; i < rank; i++)
        {
            sd[i] = hd[i];
            if (work != FZ_BUF_IN)
            {
                sd[i].os = st;
                st *= hd[i].n;
            }
            else
                sd[i].os = hd[i].is;
        }
        for (int i = 0; i < vrank; i++)
        {
            sv[i] = hv[i];
            if (work != FZ_BUF_IN)
            {
                sv[i].os = st;
                st *= hv[i].n;
            }
            else
                sv[i].os = hv[i].is;
        }
        for (int d = rank - 1; d >= 1; d--)
        {
            int first = d == rank - 1;
            int m = other_dims(sd, rank, d, sv, vrank, b, !first);
            int64_t ies = first ? sd[d].is : sd[d].os;
            if (add_line(pl, dims[d].n, ies, sd[d].os, b, m, first ? FZ_BUF_IN : work, work)) return -1;
        }
        src = work;
        for (int i = 0; i < rank; i++) hd[i].is = sd[i].os;
        for (int i = 0; i < vrank; i++) hv[i].is = sv[i].os;
    }
    int nb = other_dims(hd, rank, 0, hv, vrank, b, 0);
    return real_line(pl, n0, hd[0].is, dims[0].os, b, nb, src, FZ_BUF_OUT);
}

int fz_plan_build(fz_plan *pl, int rank, const fz_dim *dims_in, int vrank, const fz_dim *vecs_in)
{
    fz_dim dims[16], vecs[16];
    int r = 0, v = 0;
    if (rank > 16 || vrank > 16)
    {
        fz_set_error("rank above 16");
        return -1;
    }
    for (int i = 0; i < vrank; i++)
    {
        if (vecs_in[i].n == 0) pl->nop = 1;
        if (vecs_in[i].n != 1) vecs[v++] = vecs_in[i];
    }
    if (pl->nop) return 0;
    if (pl->fft_type == 1)
    {
        /* real: dims[0] is the real/half-complex dimension, keep it */
        dims[r++] = dims_in[0];
        for (int i = 1; i < rank; i++)
            if (dims_in[i].n != 1) dims[r++] = dims_in[i];
        return plan_real(pl, r, dims, v, vecs);
    }
    /* drop size-one dims (the reference's SHRINK_DIM_RANK, selector/selector.h:194-214) */
    for (int i = 0; i < rank; i++)
        if (dims_in[i].n != 1) dims[r++] = dims_in[i];
    if (r == 0) dims[r++] = dims_in[0];
    return plan_c2c(pl, r, dims, v, vecs);
}
