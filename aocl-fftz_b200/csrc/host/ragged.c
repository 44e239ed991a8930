/* Ragged batches (C99 host layer): many 1-D c2c transforms of different
 * lengths -- powers of two, smooth composites, primes -- executed in ONE
 * persistent launch, captured once in a CUDA graph.
 *
 * The reference has no ragged API: its callers run one plan per length
 * back to back (AOCL-FFTZ executes each plan's solver tree,
 * core/executor.c:17-44). Here every transform is planned with the ordinary
 * planner restricted to the generic kernel, its passes are flattened into a
 * table of CTA tiles (pass, tile, predecessor pass), and the persistent
 * executor (kernels/fft_ragged.cu) runs the whole table. Tiles are ordered by
 * pass depth, then by decreasing length (largest first balances the tail).
 */
#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "aoclfftz_gpu.h"
#include "fz_internal.h"

typedef struct
{
    fftz_ritem_t it;
    int depth;
    int64_t cost;
} fz_item_sort;

static int item_cmp(const void *a, const void *b)
{
    const fz_item_sort *x = (const fz_item_sort *)a, *y = (const fz_item_sort *)b;
    if (x->depth != y->depth) return x->depth < y->depth ? -1 : 1;
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

FFTZ_VOID *aoclfftz_gpu_ragged_setup(FFTZ_INT32 dtype, FFTZ_INT32 direction, FFTZ_INT64 count,
                                     const FFTZ_INT64 *sizes, const FFTZ_INT64 *in_offsets,
                                     const FFTZ_INT64 *out_offsets)
{
    if ((dtype != 0 && dtype != 1) || (direction != 0 && direction != 1) || count <= 0 || !sizes)
    {
        fz_set_error("ragged setup: invalid arguments");
        return NULL;
    }
    fz_plan *pl = (fz_plan *)calloc(1, sizeof(fz_plan));
    fz_ragged *rg = (fz_ragged *)calloc(1, sizeof(fz_ragged));
    int64_t npass = 0, cap_pass = 0, nitem = 0, cap_item = 0, scratch_total = 0;
    fftz_pass_t *passes = NULL;
    int64_t(*toff)[7] = NULL; /* per pass: table offsets in the merged blob */
    fz_item_sort *items = NULL;
    if (!pl || !rg) goto fail_mem;
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
    const int64_t csz = dtype == 0 ? 8 : 16;
    int64_t next_in = 0, next_out = 0;
    for (int64_t i = 0; i < count; i++)
    {
        const int64_t n = sizes[i];
        if (n < 1)
        {
            fz_set_error("ragged setup: transform %lld has length %lld", (long long)i, (long long)n);
            goto fail;
        }
        const int64_t io = in_offsets ? in_offsets[i] : next_in;
        const int64_t oo = out_offsets ? out_offsets[i] : next_out;
        next_in = io + n;
        next_out = oo + n;
        if (io + n > rg->in_elems) rg->in_elems = io + n;
        if (oo + n > rg->out_elems) rg->out_elems = oo + n;
        fz_plan sub;
        memset(&sub, 0, sizeof(sub));
        sub.dtype = dtype;
        sub.direction = direction;
        sub.placement = 1;
        sub.hints.kernel_family = 3;
        fz_dim d = {n, 1, 1}, v = {1, n, n};
        if (fz_plan_build(&sub, 1, &d, 1, &v))
        {
            free(sub.pass);
            free(sub.blob.p);
            goto fail;
        }
        int64_t boff = 0;
        if (sub.blob.len)
        {
            boff = fz_blob_add(&pl->blob, sub.blob.p, sub.blob.len);
            if (boff < 0)
            {
                free(sub.pass);
                free(sub.blob.p);
                goto fail_mem;
            }
        }
        int64_t soff[FZ_MAX_SCRATCH];
        for (int k = 0; k < sub.nscratch; k++)
        {
            soff[k] = scratch_total;
            scratch_total += (sub.scratch_elems[k] * csz + 255) & ~(int64_t)255;
        }
        int64_t prev_nblk = 0;
        for (int j = 0; j < sub.npass; j++)
        {
            fz_pass *sp = &sub.pass[j];
            if (sp->is_elem)
            {
                fz_set_error("ragged setup: unexpected elementwise pass");
                free(sub.pass);
                free(sub.blob.p);
                goto fail;
            }
            if (npass == cap_pass)
            {
                cap_pass = cap_pass ? 2 * cap_pass : 1024;
                fftz_pass_t *np = (fftz_pass_t *)realloc(passes, sizeof(fftz_pass_t) * (size_t)cap_pass);
                int64_t(*nt)[7] = (int64_t(*)[7])realloc(toff, sizeof(int64_t) * 7 * (size_t)cap_pass);
                if (!np || !nt)
                {
                    free(np ? np : passes);
                    passes = NULL;
                    free(nt ? (void *)nt : (void *)toff);
                    toff = NULL;
                    free(sub.pass);
                    free(sub.blob.p);
                    goto fail_mem;
                }
                passes = np;
                toff = nt;
            }
            fftz_pass_t k = sp->k;
            int64_t ioff, ooff;
            resolve(sp->src, io * csz + sp->in_off, soff, &k.src_buf, &ioff);
            resolve(sp->dst, oo * csz + sp->out_off, soff, &k.dst_buf, &ooff);
            if (k.src_buf == FFTZ_RBUF_SCRATCH) ioff += sp->in_off;
            if (k.dst_buf == FFTZ_RBUF_SCRATCH) ooff += sp->out_off;
            k.in = (const void *)(size_t)ioff;
            k.out = (void *)(size_t)ooff;
            const int64_t o7[7] = {sp->off_tw, sp->off_tw4hi, sp->off_tw4lo, sp->off_pre, sp->off_post, sp->off_mid,
                                   sp->off_rtw};
            for (int t = 0; t < 7; t++) toff[npass][t] = o7[t] >= 0 ? boff + o7[t] : -1;
            passes[npass] = k;
            const int64_t nblk = (k.ntf + k.tpc - 1) / k.tpc;
            for (int64_t b = 0; b < nblk; b++)
            {
                if (nitem == cap_item)
                {
                    cap_item = cap_item ? 2 * cap_item : 4096;
                    fz_item_sort *ni = (fz_item_sort *)realloc(items, sizeof(fz_item_sort) * (size_t)cap_item);
                    if (!ni)
                    {
                        free(sub.pass);
                        free(sub.blob.p);
                        goto fail_mem;
                    }
                    items = ni;
                }
                fz_item_sort *it = &items[nitem++];
                it->it.pass = (int32_t)npass;
                it->it.dep = j > 0 ? (int32_t)(npass - 1) : -1;
                it->it.blk = b;
                it->it.dep_count = j > 0 ? prev_nblk : 0;
                it->depth = j;
                it->cost = n;
            }
            prev_nblk = nblk;
            npass++;
        }
        free(sub.pass);
        free(sub.blob.p);
    }
    qsort(items, (size_t)nitem, sizeof(fz_item_sort), item_cmp);
    /* device state: tables, pass table, item table, counters, scratch */
    if (pl->blob.len &&
        (cudaMalloc(&pl->dtab, pl->blob.len) != cudaSuccess ||
         cudaMemcpy(pl->dtab, pl->blob.p, pl->blob.len, cudaMemcpyHostToDevice) != cudaSuccess))
        goto fail_cuda;
    int64_t smem = 0;
    for (int64_t i = 0; i < npass; i++)
    {
        unsigned char *base = (unsigned char *)pl->dtab;
        const void **ptrs[7] = {&passes[i].tw, &passes[i].tw4_hi, &passes[i].tw4_lo, &passes[i].pre_tab,
                                &passes[i].post_tab, &passes[i].mid_tab, &passes[i].rtw};
        for (int t = 0; t < 7; t++) *ptrs[t] = toff[i][t] >= 0 ? base + toff[i][t] : NULL;
        int64_t b = fftz_pass_smem_bytes(&passes[i]);
        if (b > smem) smem = b;
    }
    fftz_ritem_t *flat = (fftz_ritem_t *)malloc(sizeof(fftz_ritem_t) * (size_t)nitem);
    if (!flat) goto fail_mem;
    for (int64_t i = 0; i < nitem; i++) flat[i] = items[i].it;
    int ok = cudaMalloc(&rg->d_passes, sizeof(fftz_pass_t) * (size_t)npass) == cudaSuccess &&
             cudaMemcpy(rg->d_passes, passes, sizeof(fftz_pass_t) * (size_t)npass, cudaMemcpyHostToDevice) ==
                 cudaSuccess &&
             cudaMalloc(&rg->d_items, sizeof(fftz_ritem_t) * (size_t)nitem) == cudaSuccess &&
             cudaMemcpy(rg->d_items, flat, sizeof(fftz_ritem_t) * (size_t)nitem, cudaMemcpyHostToDevice) ==
                 cudaSuccess &&
             cudaMalloc(&rg->d_done, sizeof(int) * (size_t)npass) == cudaSuccess &&
             cudaMalloc(&rg->d_queue, sizeof(unsigned long long)) == cudaSuccess &&
             cudaMalloc(&rg->d_err, sizeof(int)) == cudaSuccess &&
             cudaMemset(rg->d_err, 0, sizeof(int)) == cudaSuccess &&
             (scratch_total == 0 || cudaMalloc(&pl->scratch, (size_t)scratch_total) == cudaSuccess) &&
             cudaStreamCreateWithFlags((cudaStream_t *)&rg->cap_stream, cudaStreamNonBlocking) == cudaSuccess;
    free(flat);
    if (!ok) goto fail_cuda;
    pl->scratch_bytes = scratch_total;
    rg->npasses = npass;
    rg->nitems = nitem;
    rg->smem = (int)(smem < 1024 ? 1024 : smem);
    rg->grid = fftz_ragged_grid(dtype, rg->smem);
    if (rg->grid > nitem) rg->grid = (int)nitem;
    snprintf(rg->summary, sizeof(rg->summary), "ragged: %lld transforms, %lld passes, %lld tiles, grid %d x 256, %d B smem",
             (long long)count, (long long)npass, (long long)nitem, rg->grid, rg->smem);
    pl->in_bytes = rg->in_elems * csz;
    pl->out_bytes = rg->out_elems * csz;
    pl->nlaunch = 1;
    free(passes);
    free(toff);
    free(items);
    return pl;
fail_cuda:
    cudaGetLastError();
    fz_set_error("ragged setup: device allocation failed");
    goto fail;
fail_mem:
    fz_set_error("ragged setup: out of host memory");
fail:
    free(passes);
    free(toff);
    free(items);
    if (pl)
    {
        pl->rg = rg;
        fz_plan_free(pl);
    }
    else
        free(rg);
    return NULL;
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
    r.spin_limit = 1LL << 26; /* about 10 s of polling at the executor's sleep */
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
    if (!rg->graph_exec || rg->g_in != in || rg->g_out != out)
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
