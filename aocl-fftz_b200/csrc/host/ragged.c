/* Ragged batches (C99 host layer): many 1-D c2c transforms of different
 * lengths -- powers of two, smooth composites, primes -- executed in ONE
 * persistent launch, captured once in a CUDA graph.
 *
 * The reference has no ragged API: its callers run one plan per length
 * back to back (AOCL-FFTZ executes each plan's solver tree,
 * core/executor.c:17-44). Here the transforms are grouped by length; each
 * group is planned once by the ordinary planner (in its executor mode:
 * 256-thread tiles, compile-time kernels up to length 4096) as a batch whose
 * transform dimension is indirect, so the group's transforms keep their own
 * offsets in the packed buffers. The passes are flattened into a table of CTA
 * tiles (pass, tile, predecessor pass) and the persistent executor
 * (kernels/fft_ragged.cu) runs the whole table. Tiles are ordered by pass
 * depth, then by decreasing length (largest first balances the tail).
 */
#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "aoclfftz_gpu.h"
#include "fz_internal.h"

#define FZ_MAX_PASSES_RG 64

typedef struct
{
    fftz_ritem_t it;
    int depth;
    int chain; /* passes of its plan from this one to the last */
    int64_t cost;
} fz_item_sort;

static int item_cmp(const void *a, const void *b)
{
    const fz_item_sort *x = (const fz_item_sort *)a, *y = (const fz_item_sort *)b;
    if (x->depth != y->depth) return x->depth < y->depth ? -1 : 1;
    if (x->chain != y->chain) return x->chain > y->chain ? -1 : 1;
    if (x->cost != y->cost) return x->cost > y->cost ? -1 : 1;
    if (x->it.pass != y->it.pass) return x->it.pass < y->it.pass ? -1 : 1;
    return x->it.blk < y->it.blk ? -1 : (x->it.blk > y->it.blk);
}

void fz_ragged_free(fz_ragged *rg)
{
    if (!rg) return;
    if (rg->graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)rg->graph_exec);
    if (rg->graph) cudaGraphDestroy((cudaGraph_t)rg->graph);
    if (rg->cap_stream) cudaStreamDestroy((cudaStream_t)rg->cap_stream);
    cudaFree(rg->d_passes);
    cudaFree(rg->d_items);
    cudaFree(rg->d_done);
    cudaFree(rg->d_queue);
    cudaFree(rg->d_err);
    cudaFree(rg->d_ind);
    free(rg);
}

/* byte offset of a sub-plan buffer id inside the launch's in / out / scratch */
static void resolve(int id, int64_t io_off_bytes, const int64_t *soff, int32_t *buf, int64_t *off)
{
    if (id == FZ_BUF_IN)
    {
        *buf = FFTZ_RBUF_IN;
        *off = io_off_bytes;
    }
    else if (id == FZ_BUF_OUT)
    {
        *buf = FFTZ_RBUF_OUT;
        *off = io_off_bytes;
    }
    else
    {
        *buf = FFTZ_RBUF_SCRATCH;
        *off = soff[id - FZ_BUF_SCR0];
    }
}

#define RG_THREADS 256

/* The executor's shared memory per CTA is the largest of its passes', so
 * every tile shape stays within 44 KB (float: five CTAs per SM, the
 * executor's register bound) or 100 KB (double: two CTAs per SM). Measured on
 * B200 (4096 float transforms): float ping-pong tiles of up to 72 KB made the
 * whole launch 1.353 -> 1.688 ms although their own class got faster. */
int64_t fz_ragged_smem_cap(int dtype) { return dtype == 0 ? 44 * 1024 : 100 * 1024; }

/* Launch shape of one pass inside the executor (256-thread CTAs): a
 * compile-time tile with tpc * tpt == 256 where the executor has one,
 * otherwise the generic tile with as many transforms as fit (loads and stores
 * through the generic phases, which know every table and bound). */
static int ragged_shape(fftz_pass_t *k, int dtype, int64_t smem_cap)
{
    const int nslots = k->n > k->nload ? k->n : k->nload;
    const int colmap = k->in_mode == 1 || k->out_mode == 1;
    const int fastv = k->variant == FFTZ_VAR_FAST || k->variant == FFTZ_VAR_FAST_TW4 ||
                      k->variant == FFTZ_VAR_FAST_TABS || k->variant == FFTZ_VAR_FAST_TW4_TABS ||
                      k->variant == FFTZ_VAR_FAST_BLUE;
    if (fastv && fftz_ragged_fast_ok(k->n, k->variant) && k->tpt <= RG_THREADS && RG_THREADS % k->tpt == 0)
    {
        fftz_pass_t t = *k;
        t.tpc = RG_THREADS / t.tpt;
        t.sstride = colmap ? fftz_smem_stride_cols(dtype, nslots, t.tpc) : fftz_smem_stride(dtype, nslots);
        if (fftz_pass_smem_bytes(&t) <= smem_cap)
        {
            *k = t;
            return 0;
        }
    }
    /* everything else runs as a ping-pong tile (the same radix list and
     * twiddle table; tables and other element kinds through its load / store
     * phases): as many lines as fit the cap, up to about 4096 elements */
    if (k->variant != FFTZ_VAR_GENERIC_PP)
    {
        k->variant = FFTZ_VAR_GENERIC_PP;
        k->fuse_load = k->nstages > 0 && k->in_kind == FFTZ_IN_COMPLEX && k->nload == k->n &&
                       !(k->flags & FFTZ_F_PRE_TAB);
        k->fuse_store = k->nstages > 0 && k->out_kind == FFTZ_OUT_COMPLEX && k->nstore == k->n;
    }
    int tpc = (int)((dtype == 0 ? 4096 : 2048) / k->n);
    if (colmap && tpc < (dtype == 0 ? 8 : 4)) tpc = dtype == 0 ? 8 : 4;
    if (tpc < 1) tpc = 1;
    if (tpc > 64) tpc = 64;
    if (tpc > k->ntf) tpc = (int)k->ntf;
    for (; tpc >= 1; tpc--)
    {
        k->tpc = tpc;
        k->sstride = fftz_smem_stride(dtype, nslots);
        k->tpt = RG_THREADS / tpc > 0 ? RG_THREADS / tpc : 1;
        if (fftz_pass_smem_bytes(k) <= smem_cap) return 0;
    }
    return -1;
}

typedef struct
{
    fz_plan *pl;
    int dtype, direction;
    int64_t csz, smem_cap;
    int64_t npass, cap_pass, cap_aux, nitem, cap_item, scratch_total, nind, cap_ind;
    fftz_pass_t *passes;
    int64_t (*toff)[7];  /* per pass: table offsets in the merged blob */
    int64_t (*indpos)[2]; /* per pass: positions of its in / out offset lists, -1 if none */
    int64_t *ind;         /* host copy of every offset list */
    fz_item_sort *items;
} rg_build;

static int grow(void **p, int64_t *cap, int64_t need, size_t esz, int64_t first)
{
    if (need <= *cap) return 0;
    int64_t nc = *cap ? *cap : first;
    while (nc < need) nc *= 2;
    void *np = realloc(*p, esz * (size_t)nc);
    if (!np) return -1;
    *p = np;
    *cap = nc;
    return 0;
}

/* Plans c transforms of length n whose element offsets are tin[] / tout[] and
 * appends their passes and tiles. With c >= 2 the transform dimension of the
 * plan becomes the indirect batch dimension of each pass that reads the input
 * or writes the output. Returns 1 when the plan's passes do not expose that
 * dimension (the caller then plans the transforms one by one), -1 on error. */
static int add_group(rg_build *B, int64_t n, int64_t c, const int64_t *tin, const int64_t *tout)
{
    const int64_t big = 2 * n + 1; /* a batch stride no other dimension can continue */
    fz_plan sub;
    memset(&sub, 0, sizeof(sub));
    sub.dtype = B->dtype;
    sub.direction = B->direction;
    sub.placement = 1;
    sub.hints.kernel_family = 4;
    fz_dim d = {n, 1, 1}, v = {c, c > 1 ? big : n, c > 1 ? big : n};
    if (fz_plan_build(&sub, 1, &d, 1, &v))
    {
        free(sub.pass);
        free(sub.blob.p);
        return -1;
    }
    int rc = 0;
    int32_t inddim[FZ_MAX_PASSES_RG];
    if (sub.npass > FZ_MAX_PASSES_RG) rc = 1;
    /* every pass must be plain c2c, and the indirect dimension must be found */
    for (int j = 0; j < sub.npass && rc == 0; j++)
    {
        fz_pass *sp = &sub.pass[j];
        if (sp->is_elem)
        {
            rc = 1;
            break;
        }
        inddim[j] = -1;
        if (c < 2) continue;
        const fftz_pass_t *k = &sp->k;
        const int need_in = sp->src == FZ_BUF_IN, need_out = sp->dst == FZ_BUF_OUT;
        if (!need_in && !need_out) continue;
        for (int q = 0; q < k->nbdims; q++)
            if (k->bdim[q] == c && (!need_in || k->ibs[q] == big) && (!need_out || k->obs[q] == big)) inddim[j] = q;
        if (inddim[j] < 0) rc = 1;
    }
    if (rc)
    {
        free(sub.pass);
        free(sub.blob.p);
        return rc;
    }
    int64_t boff = 0;
    if (sub.blob.len)
    {
        boff = fz_blob_add(&B->pl->blob, sub.blob.p, sub.blob.len);
        if (boff < 0) rc = -1;
    }
    int64_t soff[FZ_MAX_SCRATCH];
    for (int q = 0; q < sub.nscratch; q++)
    {
        soff[q] = B->scratch_total;
        B->scratch_total += (sub.scratch_elems[q] * B->csz + 255) & ~(int64_t)255;
    }
    /* offset lists of this group */
    int64_t pin = -1, pout = -1;
    if (rc == 0 && c > 1)
    {
        if (grow((void **)&B->ind, &B->cap_ind, B->nind + 2 * c, sizeof(int64_t), 4096))
            rc = -1;
        else
        {
            pin = B->nind;
            memcpy(B->ind + pin, tin, sizeof(int64_t) * (size_t)c);
            pout = pin + c;
            memcpy(B->ind + pout, tout, sizeof(int64_t) * (size_t)c);
            B->nind += 2 * c;
        }
    }
    int64_t prev_nblk = 0;
    for (int j = 0; j < sub.npass && rc == 0; j++)
    {
        fz_pass *sp = &sub.pass[j];
        if (grow((void **)&B->passes, &B->cap_pass, B->npass + 1, sizeof(fftz_pass_t), 1024))
        {
            rc = -1;
            break;
        }
        if (B->cap_aux < B->cap_pass)
        {
            void *a = realloc(B->toff, sizeof(int64_t) * 7 * (size_t)B->cap_pass);
            if (a) B->toff = (int64_t(*)[7])a;
            void *b = a ? realloc(B->indpos, sizeof(int64_t) * 2 * (size_t)B->cap_pass) : NULL;
            if (b) B->indpos = (int64_t(*)[2])b;
            if (!a || !b)
            {
                rc = -1;
                break;
            }
            B->cap_aux = B->cap_pass;
        }
        fftz_pass_t k = sp->k;
        const int64_t io = c > 1 ? 0 : tin[0] * B->csz, oo = c > 1 ? 0 : tout[0] * B->csz;
        int64_t ioff, ooff;
        resolve(sp->src, io + sp->in_off, soff, &k.src_buf, &ioff);
        resolve(sp->dst, oo + sp->out_off, soff, &k.dst_buf, &ooff);
        if (k.src_buf == FFTZ_RBUF_SCRATCH) ioff += sp->in_off;
        if (k.dst_buf == FFTZ_RBUF_SCRATCH) ooff += sp->out_off;
        k.in = (const void *)(size_t)ioff;
        k.out = (void *)(size_t)ooff;
        k.ind_dim = inddim[j] >= 0 ? inddim[j] : 0;
        k.ind_in = NULL;
        k.ind_out = NULL;
        if (ragged_shape(&k, B->dtype, B->smem_cap))
        {
            fz_set_error("ragged setup: a pass of length %d does not fit the executor", k.n);
            rc = -1;
            break;
        }
        const int64_t o7[7] = {sp->off_tw, sp->off_tw4hi, sp->off_tw4lo, sp->off_pre, sp->off_post, sp->off_mid,
                               sp->off_rtw};
        for (int t = 0; t < 7; t++) B->toff[B->npass][t] = o7[t] >= 0 ? boff + o7[t] : -1;
        B->indpos[B->npass][0] = (inddim[j] >= 0 && sp->src == FZ_BUF_IN) ? pin : -1;
        B->indpos[B->npass][1] = (inddim[j] >= 0 && sp->dst == FZ_BUF_OUT) ? pout : -1;
        B->passes[B->npass] = k;
        const int64_t nblk = (k.ntf + k.tpc - 1) / k.tpc;
        /* the tile's work, about tpc lines of n log2 n: longest first */
        int64_t lg = 1;
        while ((1LL << lg) < k.n) lg++;
        const int64_t tile_work = (int64_t)k.tpc * k.n * lg;
        if (grow((void **)&B->items, &B->cap_item, B->nitem + nblk, sizeof(fz_item_sort), 4096))
        {
            rc = -1;
            break;
        }
        for (int64_t b = 0; b < nblk; b++)
        {
            fz_item_sort *it = &B->items[B->nitem++];
            it->it.pass = (int32_t)B->npass;
            it->it.dep = j > 0 ? (int32_t)(B->npass - 1) : -1;
            it->it.blk = b;
            it->it.dep_count = j > 0 ? prev_nblk : 0;
            it->it.signal = j + 1 < sub.npass;
            it->it.pad_ = 0;
            it->depth = j;
            it->chain = sub.npass - j;
            it->cost = tile_work;
        }
        prev_nblk = nblk;
        B->npass++;
    }
    free(sub.pass);
    free(sub.blob.p);
    return rc;
}

typedef struct
{
    int64_t n, idx;
} rg_size;

static int size_cmp(const void *a, const void *b)
{
    const rg_size *x = (const rg_size *)a, *y = (const rg_size *)b;
    if (x->n != y->n) return x->n < y->n ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

FFTZ_VOID *aoclfftz_gpu_ragged_setup(FFTZ_INT32 dtype, FFTZ_INT32 direction, FFTZ_INT64 count,
                                     const FFTZ_INT64 *sizes, const FFTZ_INT64 *in_offsets,
                                     const FFTZ_INT64 *out_offsets)
{
    if ((dtype != 0 && dtype != 1) || (direction != 0 && direction != 1) || count <= 0 || !sizes)
    {
        fz_set_error("ragged setup: invalid arguments");
        return NULL;
    }
    rg_build B;
    memset(&B, 0, sizeof(B));
    fz_plan *pl = (fz_plan *)calloc(1, sizeof(fz_plan));
    fz_ragged *rg = (fz_ragged *)calloc(1, sizeof(fz_ragged));
    rg_size *ord = (rg_size *)malloc(sizeof(rg_size) * (size_t)count);
    int64_t *tin = (int64_t *)malloc(sizeof(int64_t) * (size_t)count);
    int64_t *tout = (int64_t *)malloc(sizeof(int64_t) * (size_t)count);
    int64_t *gin = (int64_t *)malloc(sizeof(int64_t) * (size_t)count);
    int64_t *gout = (int64_t *)malloc(sizeof(int64_t) * (size_t)count);
    fftz_ritem_t *flat = NULL;
    if (!pl || !rg || !ord || !tin || !tout || !gin || !gout) goto fail_mem;
    pl->magic = FZ_MAGIC;
    pl->dtype = dtype;
    pl->direction = direction;
    pl->placement = 1;
    pl->rg = rg;
    rg->count = count;
    if (cudaGetDevice(&pl->device) != cudaSuccess)
    {
        fz_set_error("no CUDA device available");
        goto fail;
    }
    B.pl = pl;
    B.dtype = dtype;
    B.direction = direction;
    B.csz = dtype == 0 ? 8 : 16;
    B.smem_cap = fz_ragged_smem_cap(dtype);
    int64_t next_in = 0, next_out = 0;
    for (int64_t i = 0; i < count; i++)
    {
        const int64_t n = sizes[i];
        if (n < 1)
        {
            fz_set_error("ragged setup: transform %lld has length %lld", (long long)i, (long long)n);
            goto fail;
        }
        tin[i] = in_offsets ? in_offsets[i] : next_in;
        tout[i] = out_offsets ? out_offsets[i] : next_out;
        next_in = tin[i] + n;
        next_out = tout[i] + n;
        if (tin[i] + n > rg->in_elems) rg->in_elems = tin[i] + n;
        if (tout[i] + n > rg->out_elems) rg->out_elems = tout[i] + n;
        ord[i].n = n;
        ord[i].idx = i;
    }
    /* one batched plan per distinct length */
    qsort(ord, (size_t)count, sizeof(rg_size), size_cmp);
    for (int64_t g0 = 0; g0 < count;)
    {
        int64_t g1 = g0;
        while (g1 < count && ord[g1].n == ord[g0].n) g1++;
        const int64_t c = g1 - g0;
        for (int64_t q = 0; q < c; q++)
        {
            gin[q] = tin[ord[g0 + q].idx];
            gout[q] = tout[ord[g0 + q].idx];
        }
        int rc = add_group(&B, ord[g0].n, c, gin, gout);
        if (rc > 0 && c > 1)
            for (int64_t q = 0; q < c && rc >= 0; q++) rc = add_group(&B, ord[g0].n, 1, gin + q, gout + q);
        if (rc > 0)
        {
            fz_set_error("ragged setup: length %lld has no executor plan", (long long)ord[g0].n);
            goto fail;
        }
        if (rc < 0) goto fail;
        rg->ngroups++;
        g0 = g1;
    }
    qsort(B.items, (size_t)B.nitem, sizeof(fz_item_sort), item_cmp);
    /* device state: tables, offset lists, pass table, item table, counters, scratch */
    if (pl->blob.len &&
        (fz_dev_malloc(&pl->dtab, pl->blob.len) ||
         cudaMemcpy(pl->dtab, pl->blob.p, pl->blob.len, cudaMemcpyHostToDevice) != cudaSuccess))
        goto fail_cuda;
    if (B.nind &&
        (fz_dev_malloc(&rg->d_ind, sizeof(int64_t) * (size_t)B.nind) ||
         cudaMemcpy(rg->d_ind, B.ind, sizeof(int64_t) * (size_t)B.nind, cudaMemcpyHostToDevice) != cudaSuccess))
        goto fail_cuda;
    int64_t smem = 0;
    for (int64_t i = 0; i < B.npass; i++)
    {
        unsigned char *base = (unsigned char *)pl->dtab;
        const void **ptrs[7] = {&B.passes[i].tw, &B.passes[i].tw4_hi, &B.passes[i].tw4_lo, &B.passes[i].pre_tab,
                                &B.passes[i].post_tab, &B.passes[i].mid_tab, &B.passes[i].rtw};
        for (int t = 0; t < 7; t++) *ptrs[t] = B.toff[i][t] >= 0 ? base + B.toff[i][t] : NULL;
        if (B.indpos[i][0] >= 0) B.passes[i].ind_in = (const int64_t *)rg->d_ind + B.indpos[i][0];
        if (B.indpos[i][1] >= 0) B.passes[i].ind_out = (const int64_t *)rg->d_ind + B.indpos[i][1];
        int64_t b = fftz_pass_smem_bytes(&B.passes[i]);
        if (b > smem) smem = b;
    }
    flat = (fftz_ritem_t *)malloc(sizeof(fftz_ritem_t) * (size_t)B.nitem);
    if (!flat) goto fail_mem;
    for (int64_t i = 0; i < B.nitem; i++) flat[i] = B.items[i].it;
    if (fz_inj_ragged_dep > 0) /* injected: the first dependency cannot complete */
        for (int64_t i = 0; i < B.nitem; i++)
            if (flat[i].dep >= 0)
            {
                flat[i].dep_count += fz_inj_ragged_dep;
                break;
            }
    int ok = !fz_dev_malloc(&rg->d_passes, sizeof(fftz_pass_t) * (size_t)B.npass) &&
             cudaMemcpy(rg->d_passes, B.passes, sizeof(fftz_pass_t) * (size_t)B.npass, cudaMemcpyHostToDevice) ==
                 cudaSuccess &&
             !fz_dev_malloc(&rg->d_items, sizeof(fftz_ritem_t) * (size_t)B.nitem) &&
             cudaMemcpy(rg->d_items, flat, sizeof(fftz_ritem_t) * (size_t)B.nitem, cudaMemcpyHostToDevice) ==
                 cudaSuccess &&
             !fz_dev_malloc(&rg->d_done, sizeof(int) * (size_t)B.npass) &&
             !fz_dev_malloc(&rg->d_queue, sizeof(unsigned long long)) &&
             !fz_dev_malloc(&rg->d_err, sizeof(int)) &&
             cudaMemset(rg->d_err, 0, sizeof(int)) == cudaSuccess &&
             (B.scratch_total == 0 || !fz_dev_malloc(&pl->scratch, (size_t)B.scratch_total)) &&
             cudaStreamCreateWithFlags((cudaStream_t *)&rg->cap_stream, cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) goto fail_cuda;
    pl->scratch_bytes = B.scratch_total;
    rg->npasses = B.npass;
    rg->nitems = B.nitem;
    rg->smem = (int)(smem < 1024 ? 1024 : smem);
    rg->grid = fftz_ragged_grid(dtype, rg->smem);
    if (rg->grid > B.nitem) rg->grid = (int)B.nitem;
    snprintf(rg->summary, sizeof(rg->summary),
             "ragged: %lld transforms in %lld length groups, %lld passes, %lld tiles, grid %d x %d, %d B smem",
             (long long)count, (long long)rg->ngroups, (long long)B.npass, (long long)B.nitem, rg->grid, RG_THREADS,
             rg->smem);
    pl->in_bytes = rg->in_elems * B.csz;
    pl->out_bytes = rg->out_elems * B.csz;
    pl->nlaunch = 1;
    goto done;
fail_cuda:
    cudaGetLastError();
    fz_set_error("ragged setup: device allocation failed");
    goto fail;
fail_mem:
    fz_set_error("ragged setup: out of host memory");
fail:
    if (pl)
    {
        pl->rg = rg;
        fz_plan_free(pl);
    }
    else
        free(rg);
    pl = NULL;
done:
    free(flat);
    free(B.passes);
    free(B.toff);
    free(B.indpos);
    free(B.ind);
    free(B.items);
    free(ord);
    free(tin);
    free(tout);
    free(gin);
    free(gout);
    return pl;
}

/* capture: reset counters, one launch of the executor */
static int ragged_capture(fz_plan *pl, const void *in, void *out)
{
    fz_ragged *rg = pl->rg;
    cudaStream_t cs = (cudaStream_t)rg->cap_stream;
    if (rg->graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)rg->graph_exec);
    if (rg->graph) cudaGraphDestroy((cudaGraph_t)rg->graph);
    rg->graph_exec = rg->graph = NULL;
    fftz_ragged_t r;
    memset(&r, 0, sizeof(r));
    r.passes = (const fftz_pass_t *)rg->d_passes;
    r.items = (const fftz_ritem_t *)rg->d_items;
    r.nitems = rg->nitems;
    r.queue = (unsigned long long *)rg->d_queue;
    r.done = (int *)rg->d_done;
    r.err = (int *)rg->d_err;
    r.in = in;
    r.out = out;
    r.scratch = pl->scratch;
    /* about 10 s of polling at the executor's sleep, unless a test set a limit */
    const int64_t spin = fz_inj_ragged_wait > 0 ? fz_inj_ragged_wait : 1LL << 26;
    r.spin_limit = spin;
    r.dtype = pl->dtype;
    r.smem_bytes = rg->smem;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1;
    int e = cudaMemsetAsync(rg->d_done, 0, sizeof(int) * (size_t)rg->npasses, cs) == cudaSuccess &&
            cudaMemsetAsync(rg->d_queue, 0, sizeof(unsigned long long), cs) == cudaSuccess &&
            fftz_launch_ragged(&r, rg->grid, cs) == 0;
    cudaGraph_t g = NULL;
    cudaError_t ce = cudaStreamEndCapture(cs, &g);
    if (!e || ce != cudaSuccess || !g)
    {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return -1;
    }
    cudaGraphExec_t ge = NULL;
    if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
    {
        cudaGraphDestroy(g);
        cudaGetLastError();
        return -1;
    }
    rg->graph = g;
    rg->graph_exec = ge;
    rg->g_in = in;
    rg->g_out = out;
    rg->g_spin = spin;
    return 0;
}

aoclfftz_error_type aoclfftz_gpu_ragged_execute(FFTZ_VOID *handle, FFTZ_VOID *in, FFTZ_VOID *out)
{
    fz_plan *pl = (fz_plan *)handle;
    if (!pl || pl->magic != FZ_MAGIC || !pl->rg || !in || !out || in == out) return AOCLFFTZ_EXECUTION_FAILURE;
    fz_ragged *rg = pl->rg;
    struct cudaPointerAttributes a, b;
    if (cudaPointerGetAttributes(&a, in) != cudaSuccess || cudaPointerGetAttributes(&b, out) != cudaSuccess ||
        (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) ||
        (b.type != cudaMemoryTypeDevice && b.type != cudaMemoryTypeManaged))
    {
        cudaGetLastError();
        fz_set_error("ragged execute takes device buffers");
        return AOCLFFTZ_INVALID_INPUT;
    }
    const int64_t spin = fz_inj_ragged_wait > 0 ? fz_inj_ragged_wait : 1LL << 26;
    if (!rg->graph_exec || rg->g_in != in || rg->g_out != out || rg->g_spin != spin)
        if (ragged_capture(pl, in, out))
        {
            fz_set_error("ragged execute: graph capture failed");
            return AOCLFFTZ_EXECUTION_FAILURE;
        }
    if (cudaGraphLaunch((cudaGraphExec_t)rg->graph_exec, (cudaStream_t)pl->stream) != cudaSuccess)
    {
        cudaGetLastError();
        fz_set_error("ragged execute: graph launch failed");
        return AOCLFFTZ_EXECUTION_FAILURE;
    }
    return AOCLFFTZ_SUCCESS;
}
