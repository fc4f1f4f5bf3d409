// cg_graph.cu -- the CG iterations of gpair_cg_run as one CUDA graph with
// conditional nodes, so that a run of any length is a single graph launch:
// no host round trip per line-search trial.
//
//   WHILE (h_iter)                               one CG iteration per pass
//     [pre ] criterion + gradient of the current image, beta, descent
//            direction, wolfe1                    (gpair1/trunk/gpair.c:688-806)
//     WHILE (h_ls)                               line-search trials
//       [crit] trial image max(I + s d, minval), criterion, controller
//       IF (h_grad)
//         [grad] gradient of the trial image, controller
//     [post] image update with the accepted step, gradient backup, trace
//
// The controller kernel (k_cg_ctrl_g) holds every decision of the reference's
// line search (gpair1/trunk/gpair.c:832-903, gpair1/trunk/gpu.c:1947-2065) and
// sets the three conditions with cudaGraphSetConditional. Loops are bounded:
// the iteration count by run_limit, the trials by the controller's bracket
// and zoom caps.
//
// With the batched line search (GPAIR_LS_BATCH) the inner loop body is one
// batched evaluation of GPAIR_LS_TRIALS trial images and there is no gradient
// branch:
//
//   WHILE (h_iter)
//     [pre ] as above
//     WHILE (h_ls)
//       [batch] trial images, batched forward DFT, chi2 of each, controller
//     [post] as above
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gpair_internal.cuh"

int gp_eval_criterion(gpair_ctx *c, int which, int trial);
int gp_eval_gradient(gpair_ctx *c, int which, float alpha);

struct CgGraph {
    cudaGraph_t g;
    cudaGraphExec_t exec;
    int precision;
    int ls_mode;
    int lbfgs;  // direction by the projected L-BFGS passes (method 4) instead of the CG update
    double *trace;
    int trace_cap;
    int n_pre, n_crit, n_grad, n_post;  // kernel launches per sequence
    unsigned int buf_gen;                // the context's buffer generation at capture
};

enum { SEQ_PRE = 0, SEQ_CRIT = 1, SEQ_GRAD = 2, SEQ_POST = 3 };

static int emit(gpair_ctx *c, CgGraph *G, int seq, cudaGraphConditionalHandle hi, cudaGraphConditionalHandle hl,
                cudaGraphConditionalHandle hg)
{
    // the controller runs in the last block of the reduction kernel that precedes it;
    // it steers the graph when it has handles (a lockstep batch steers by routers)
    c->fuse_handles = hi != 0;
    c->fh_iter = hi;
    c->fh_ls = hl;
    c->fh_grad = hg;
    int rc;
    switch (seq) {
    case SEQ_PRE:
        if ((rc = gp_eval_criterion(c, GPAIR_IMG_CURR, 0))) break;
        c->fuse_ctrl = CTRL_BEGIN;
        if ((rc = gp_eval_gradient(c, GPAIR_IMG_CURR, -1.f))) break;  // alpha from the device state
        c->fuse_ctrl = CTRL_AFTER_DIR;
        rc = G->lbfgs ? gp_lbfgs_direction(c) : gp_descent_dir(c, 1, 0.0);
        break;
    case SEQ_CRIT:
        if (G->ls_mode == GPAIR_LS_BATCH) {
            c->fuse_ctrl = CTRL_AFTER_BATCH;
            rc = gp_eval_batch(c);
        } else {
            c->fuse_ctrl = CTRL_AFTER_CRIT;
            rc = gp_eval_criterion(c, GPAIR_IMG_TEMP, 1);
        }
        break;
    case SEQ_GRAD:
        c->fuse_ctrl = CTRL_AFTER_GRAD;
        rc = gp_eval_gradient(c, GPAIR_IMG_TEMP, -1.f);
        break;
    default:
        if ((rc = gp_update_image(c, 1, 0.0, 1e-8, 1))) break;
        rc = gp_cg_kernel_graph(c, CTRL_END, hi, hl, hg, G->trace, G->trace_cap);
        break;
    }
    c->fuse_ctrl = -1;
    c->fuse_handles = 0;
    return rc;
}

static int capture(gpair_ctx *c, CgGraph *G, int seq, cudaGraphConditionalHandle hi, cudaGraphConditionalHandle hl,
                   cudaGraphConditionalHandle hg, cudaGraph_t *out, int *nlaunch)
{
    const long long l0 = c->launches;
    const int st = c->stage_timing;
    c->stage_timing = 0;
    GP_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = emit(c, G, seq, hi, hl, hg);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->stage_timing = st;
    *nlaunch = (int)(c->launches - l0);
    c->launches = l0;
    if (rc || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        if (!rc) snprintf(c->last_error, sizeof(c->last_error), "stream capture failed: %s", cudaGetErrorString(e));
        return rc ? rc : GPAIR_ERR_CUDA;
    }
    *out = g;
    return GPAIR_OK;
}

static void graph_free_one(gpair_ctx *c, int mode)
{
    CgGraph *G = (CgGraph *)c->cg_graph[mode];
    if (!G) return;
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->g) cudaGraphDestroy(G->g);
    if (G->trace) cudaFree(G->trace);
    free(G);
    c->cg_graph[mode] = nullptr;
}

void gp_cg_graph_free(gpair_ctx *c)
{
    graph_free_one(c, 0);
    graph_free_one(c, 1);
}

static cudaGraphNode_t add_conditional(gpair_ctx *c, cudaGraph_t parent, cudaGraphConditionalHandle h,
                                       cudaGraphConditionalNodeType type, cudaGraph_t *body, int *rc)
{
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};  // remaining members zero
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t n = nullptr;
    cudaError_t e = cudaGraphAddNode(&n, parent, nullptr, 0, &p);
    if (e != cudaSuccess) {
        snprintf(c->last_error, sizeof(c->last_error), "cudaGraphAddNode(conditional): %s", cudaGetErrorString(e));
        *rc = GPAIR_ERR_CUDA;
        return nullptr;
    }
    *body = p.conditional.phGraph_out[0];
    return n;
}

// Adds one context's whole CG loop (the WHILE node and its bodies) to `parent`.
// G carries the loop's line-search mode, trace buffer and launch counts.
static int add_loop(gpair_ctx *c, CgGraph *G, cudaGraph_t parent)
{
    if (c->precision != GPAIR_PREC_FP32) {
        int rc = gp_tc_prepare(c);  // operand buffers must exist before capture
        if (rc) return rc;
    }
    if (G->ls_mode == GPAIR_LS_BATCH) {
        int rc = gp_batch_alloc(c);
        if (rc) return rc;
    }
    if (G->lbfgs) {
        int rc = gp_lbfgs_alloc(c);  // no allocation inside a capture
        if (rc) return rc;
    }
    int rc = GPAIR_OK;
    cudaGraphConditionalHandle h_iter, h_ls, h_grad;
    GP_CUDA(c, cudaGraphConditionalHandleCreate(&h_iter, parent, 1, cudaGraphCondAssignDefault));
    cudaGraph_t B1, B2, B3;
    add_conditional(c, parent, h_iter, cudaGraphCondTypeWhile, &B1, &rc);
    if (rc) return rc;
    GP_CUDA(c, cudaGraphConditionalHandleCreate(&h_ls, B1, 0, 0));
    cudaGraphNode_t n_ls = add_conditional(c, B1, h_ls, cudaGraphCondTypeWhile, &B2, &rc);
    if (rc) return rc;
    const bool wolfe = G->ls_mode != GPAIR_LS_BATCH;
    cudaGraphNode_t n_if = nullptr;
    h_grad = 0;
    if (wolfe) {
        GP_CUDA(c, cudaGraphConditionalHandleCreate(&h_grad, B2, 0, 0));
        n_if = add_conditional(c, B2, h_grad, cudaGraphCondTypeIf, &B3, &rc);
        if (rc) return rc;
    }
    cudaGraph_t S[4] = {nullptr, nullptr, nullptr, nullptr};
    int *counts[4] = {&G->n_pre, &G->n_crit, &G->n_grad, &G->n_post};
    for (int q = 0; q < 4 && !rc; q++) {
        if (q == SEQ_GRAD && !wolfe) continue;
        rc = capture(c, G, q, h_iter, h_ls, h_grad, &S[q], counts[q]);
    }
    if (!rc) {
        cudaGraphNode_t n_pre, n_post, n_crit, n_grad;
        cudaError_t e = cudaGraphAddChildGraphNode(&n_pre, B1, nullptr, 0, S[SEQ_PRE]);
        if (e == cudaSuccess) e = cudaGraphAddChildGraphNode(&n_post, B1, nullptr, 0, S[SEQ_POST]);
        if (e == cudaSuccess) e = cudaGraphAddDependencies(B1, &n_pre, &n_ls, 1);
        if (e == cudaSuccess) e = cudaGraphAddDependencies(B1, &n_ls, &n_post, 1);
        if (e == cudaSuccess) e = cudaGraphAddChildGraphNode(&n_crit, B2, nullptr, 0, S[SEQ_CRIT]);
        if (wolfe) {
            if (e == cudaSuccess) e = cudaGraphAddDependencies(B2, &n_crit, &n_if, 1);
            if (e == cudaSuccess) e = cudaGraphAddChildGraphNode(&n_grad, B3, nullptr, 0, S[SEQ_GRAD]);
        }
        if (e != cudaSuccess) {
            snprintf(c->last_error, sizeof(c->last_error), "CG graph assembly: %s", cudaGetErrorString(e));
            rc = GPAIR_ERR_CUDA;
        }
    }
    for (int q = 0; q < 4; q++)
        if (S[q]) cudaGraphDestroy(S[q]);
    return rc;
}

static int build(gpair_ctx *c, int trace_cap, int ls_mode)
{
    graph_free_one(c, ls_mode);
    CgGraph *G = (CgGraph *)calloc(1, sizeof(CgGraph));
    if (!G) return GPAIR_ERR_ALLOC;
    c->cg_graph[ls_mode] = G;
    G->precision = c->precision;
    G->ls_mode = ls_mode;
    G->lbfgs = c->cg_method == 4;
    G->trace_cap = trace_cap;
    GP_CUDA(c, cudaMalloc(&G->trace, sizeof(double) * 5 * (size_t)trace_cap));
    GP_CUDA(c, cudaGraphCreate(&G->g, 0));
    int rc = add_loop(c, G, G->g);
    if (!rc) {
        cudaError_t e = cudaGraphInstantiate(&G->exec, G->g, 0);
        if (e != cudaSuccess) {
            snprintf(c->last_error, sizeof(c->last_error), "CG graph instantiate: %s", cudaGetErrorString(e));
            rc = GPAIR_ERR_CUDA;
        }
    }
    if (rc) graph_free_one(c, ls_mode);
    return rc;
}

// ------------------------------------------------ many contexts, one graph
//
// One graph holding every context's whole CG loop as an independent branch
// (each a WHILE node with its own conditional handles), so that one launch
// runs all the reconstructions and the device schedules their kernels side
// by side.
struct BatchGraph {
    int n;
    cudaGraph_t g;
    cudaGraphExec_t exec;
    CgGraph *loops;  // per context: mode, trace buffer, launch counts (no graph of its own)
    // lockstep batch with grouped forwards (instances in lockstep order: by class)
    int grouped;
    int ngrp;
    void **grps;                      // one grouped forward per class of tensor instances (umma_dft.cu)
    unsigned int *gerr;               // device: wait failures of the grouped forwards
    int *flags;                       // device: act[n], ls[n], lockstep order
    cudaGraphConditionalHandle *hd;   // device: h_pre[n], h_post[n], lockstep order
    DevScalars **scs;                 // device: every instance's scalars, lockstep order
    // staged lockstep: every stage grouped (per class: the image forward and the adjoint)
    int staged;
    void **grps_img, **grps_adj;
    int nadj;  // grouped adjoints (classes without the forward operand kind)
    int prep_passes;  // passes of rows per block of the grouped trial prep
    void *stg_args[GS_COUNT];  // device: argument structs of every instance, lockstep order
    int *stg_start[GS_COUNT];  // device: block starts [n + 1]
    int stg_total[GS_COUNT];
    // staged batches built with stage stamps: device timer after every launch of
    // the last iteration (GP_NSTAMPS values, overwritten by every iteration)
    unsigned long long *stamps;
};

// Stamp positions of a staged iteration: the pre-phase (start, then after the
// prep, forwards, V2/T3/chi2, c_k, W, adjoints, gradient, direction, router),
// a batched evaluation (start, then after the trial prep, trial forwards,
// trial chi2, router) and the post-phase (start, then after the update,
// controller, router). The buffer holds the last value of every stamp
// [0, GP_NSTAMPS), the time since the stamp before it summed over the whole
// run [GP_NSTAMPS, 2 GP_NSTAMPS) (0 for the three segment starts) and the
// number of batched evaluations [2 GP_NSTAMPS].
#define GP_NSTAMPS 19
#define GP_STAMP_WORDS (2 * GP_NSTAMPS + 1)

__global__ void k_stamp(unsigned long long *__restrict__ t, int i)
{
    if (threadIdx.x == 0) {
        unsigned long long v;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
        if (i != 0 && i != 10 && i != 15) t[GP_NSTAMPS + i] += v - t[i - 1];
        if (i == 10) t[2 * GP_NSTAMPS] += 1ull;
        t[i] = v;
    }
}

void gp_batch_graph_free(void *bg)
{
    BatchGraph *B = (BatchGraph *)bg;
    if (!B) return;
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->g) cudaGraphDestroy(B->g);
    if (B->loops) {
        for (int i = 0; i < B->n; i++)
            if (B->loops[i].trace) cudaFree(B->loops[i].trace);
        free(B->loops);
    }
    for (int k = 0; k < B->ngrp; k++) {
        gp_tc_group_free(B->grps[k]);
        if (B->grps_img) gp_tc_group_free(B->grps_img[k]);
    }
    for (int k = 0; k < B->nadj; k++)
        if (B->grps_adj) gp_tc_group_free(B->grps_adj[k]);
    free(B->grps);
    free(B->grps_img);
    free(B->grps_adj);
    for (int s = 0; s < GS_COUNT; s++) {
        if (B->stg_args[s]) cudaFree(B->stg_args[s]);
        if (B->stg_start[s]) cudaFree(B->stg_start[s]);
    }
    if (B->stamps) cudaFree(B->stamps);
    if (B->gerr) cudaFree(B->gerr);
    if (B->flags) cudaFree(B->flags);
    if (B->hd) cudaFree(B->hd);
    if (B->scs) cudaFree(B->scs);
    free(B);
}

// ----------------------------------------- lockstep batches, grouped forward
//
// With the batched line search the instances can advance in lockstep, so that
// the batched-trial forwards of all of them run as one grouped tcgen05 launch
// per class of tensor instances (same operand kind, product count and tile
// layout; gp_tc_group_forward); instances on the CUDA cores keep their own
// batched evaluation. In lockstep order (instances sorted by class):
//
//   [route INIT]   act[i] = 1
//   WHILE (h_any_iter)
//     [route BEGIN]  h_pre[i] = h_post[i] = act[i]
//     IF (h_pre[i])  criterion + gradient + direction of instance i   (each i, side by side)
//     [route LS0]    ls[i] = act[i] and the line search of i goes on; h_any_ls
//     WHILE (h_any_ls)
//       trial images + operands of instance i, if ls[i]              (each tensor i)
//       one grouped forward per class over its instances with ls[i]
//       chi2 of the trials + controller of instance i, if ls[i]      (each tensor i)
//       the whole batched evaluation of instance i, if ls[i]         (each CUDA-core i)
//       [route LSN]  ls[i] = ls[i] and the line search of i goes on; h_any_ls
//     IF (h_post[i]) image update + end of the iteration of instance i
//     [route END]    act[i] = act[i] and the run of i goes on; h_any_iter
//
// Each instance runs the kernels of its own graph with the same arguments
// (its controllers steer nothing; the routers read their decisions), so its
// results are bitwise those of a separate run.
// GR_LS0S: LS0 of a staged batch, whose criterion and gradient contractions are
// grouped too: a wait failure of those stops every active instance
enum { GR_INIT = 0, GR_BEGIN = 1, GR_LS0 = 2, GR_LSN = 3, GR_END = 4, GR_LS0S = 5 };

__global__ void k_lockstep_route(int what, DevScalars *const *__restrict__ scs, int n, int *__restrict__ act,
                                 int *__restrict__ ls, const cudaGraphConditionalHandle *__restrict__ h_pre,
                                 const cudaGraphConditionalHandle *__restrict__ h_post,
                                 cudaGraphConditionalHandle h_any, unsigned int *__restrict__ gerr)
{
    gp_pdl_enter();
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        DevScalars *sc = scs[i];
        int v = 0;
        switch (what) {
        case GR_INIT:
            act[i] = 1;
            if (i == 0) *gerr = 0u;  // wait failures of this launch's grouped forwards
            break;
        case GR_BEGIN:
            cudaGraphSetConditional(h_pre[i], act[i] ? 1u : 0u);
            cudaGraphSetConditional(h_post[i], act[i] ? 1u : 0u);
            break;
        case GR_LS0:
            v = act[i] && sc->cg.action != CG_DONE;
            ls[i] = v;
            break;
        case GR_LS0S:
            if (act[i] && *gerr) sc->tc_err |= *gerr;
            v = act[i] && sc->cg.action != CG_DONE && !sc->tc_err;
            ls[i] = v;
            break;
        case GR_LSN:
            // a bounded wait of a grouped forward gave up: every instance stops
            if (ls[i] && *gerr) sc->tc_err |= *gerr;
            v = ls[i] && sc->cg.action != CG_DONE && !sc->tc_err;
            ls[i] = v;
            break;
        default:  // GR_END
            v = act[i] && cg_run_goes_on(sc);
            act[i] = v;
            break;
        }
        if (v) atomicOr(&any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0 && what >= GR_LS0) cudaGraphSetConditional(h_any, any ? 1u : 0u);
}

template <typename F>
static int capture_fn(gpair_ctx *c, F f, cudaGraph_t *out, int *nlaunch)
{
    const long long l0 = c->launches;
    const int st = c->stage_timing;
    c->stage_timing = 0;
    GP_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = f();
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->stage_timing = st;
    if (nlaunch) *nlaunch = (int)(c->launches - l0);
    c->launches = l0;
    if (rc || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        if (!rc) snprintf(c->last_error, sizeof(c->last_error), "stream capture failed: %s", cudaGetErrorString(e));
        return rc ? rc : GPAIR_ERR_CUDA;
    }
    *out = g;
    return GPAIR_OK;
}

// adds `child` (destroyed here) to `parent` after the nodes `deps`
static int add_child(gpair_ctx *c, cudaGraph_t parent, cudaGraph_t child, const cudaGraphNode_t *deps, size_t ndeps,
                     cudaGraphNode_t *node)
{
    cudaError_t e = cudaGraphAddChildGraphNode(node, parent, deps, ndeps, child);
    cudaGraphDestroy(child);
    if (e != cudaSuccess) {
        snprintf(c->last_error, sizeof(c->last_error), "lockstep graph assembly: %s", cudaGetErrorString(e));
        return GPAIR_ERR_CUDA;
    }
    return GPAIR_OK;
}

static int lockstep_route(BatchGraph *B, gpair_ctx *c, int what, cudaGraphConditionalHandle h_any, cudaGraph_t parent,
                          const cudaGraphNode_t *deps, size_t ndeps, cudaGraphNode_t *node)
{
    const int n = B->n;
    cudaGraph_t g = nullptr;
    int rc = capture_fn(
        c,
        [&]() {
            GP_LAUNCH(c, gp_launch(c, k_lockstep_route, dim3(1), dim3(256), 0, what, B->scs, n, B->flags,
                                   B->flags + n, B->hd, B->hd + n, h_any, B->gerr));
            return GPAIR_OK;
        },
        &g, nullptr);
    if (rc) return rc;
    return add_child(c, parent, g, deps, ndeps, node);
}

// GPAIR_ERR_STATE: no instance can take part in a grouped forward (the caller
// builds the independent branches instead)
static int build_lockstep(gpair_ctx **ctx_in, int n, BatchGraph *B)
{
    // lockstep order: tensor instances by class (stable), then the CUDA-core ones
    std::vector<int> key((size_t)n), order((size_t)n);
    for (int i = 0; i < n; i++) {
        key[i] = gp_tc_group_key(ctx_in[i]);
        order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const int ka = key[a] < 0 ? 1 << 30 : key[a], kb = key[b] < 0 ? 1 << 30 : key[b];
        return ka < kb;
    });
    if (key[order[0]] < 0 || n > 4096) return GPAIR_ERR_STATE;
    std::vector<gpair_ctx *> ctx((size_t)n);
    for (int k = 0; k < n; k++) ctx[k] = ctx_in[order[k]];
    gpair_ctx *c0 = ctx[0];
    GP_CUDA(c0, cudaMalloc(&B->flags, sizeof(int) * 2 * (size_t)n));
    GP_CUDA(c0, cudaMemset(B->flags, 0, sizeof(int) * 2 * (size_t)n));
    GP_CUDA(c0, cudaMalloc(&B->gerr, sizeof(unsigned int)));
    GP_CUDA(c0, cudaMemset(B->gerr, 0, sizeof(unsigned int)));
    // classes: [cls_begin[q], cls_begin[q + 1]) in lockstep order; grouped launches hold
    // at most 256 instances, a larger class is split
    std::vector<int> cls_begin;
    for (int k = 0; k < n; k++) {
        if (key[order[k]] < 0) break;
        if (cls_begin.empty() || key[order[k]] != key[order[k - 1]] || k - cls_begin.back() == 256)
            cls_begin.push_back(k);
    }
    int ntc = 0;
    while (ntc < n && key[order[ntc]] >= 0) ntc++;
    cls_begin.push_back(ntc);
    B->ngrp = (int)cls_begin.size() - 1;
    B->grps = (void **)calloc((size_t)B->ngrp, sizeof(void *));
    if (!B->grps) return GPAIR_ERR_ALLOC;
    int rc = GPAIR_OK;
    for (int q = 0; q < B->ngrp && !rc; q++) {
        const int k0 = cls_begin[q], k1 = cls_begin[q + 1];
        rc = gp_tc_group_build(&ctx[k0], k1 - k0, B->flags + n + k0, B->gerr, &B->grps[q]);
    }
    for (int k = ntc; k < n && !rc; k++) rc = gp_batch_alloc(ctx[k]);  // no allocation inside a capture
    if (rc) return rc == GPAIR_ERR_STATE ? GPAIR_ERR_CUDA : rc;  // the instances were eligible
    GP_CUDA(c0, cudaMalloc(&B->hd, sizeof(cudaGraphConditionalHandle) * 2 * (size_t)n));
    GP_CUDA(c0, cudaMalloc(&B->scs, sizeof(DevScalars *) * (size_t)n));
    std::vector<DevScalars *> hs((size_t)n);
    for (int k = 0; k < n; k++) hs[k] = ctx[k]->sc;
    GP_CUDA(c0, cudaMemcpy(B->scs, hs.data(), sizeof(DevScalars *) * (size_t)n, cudaMemcpyHostToDevice));

    // loops and their handles
    cudaGraphConditionalHandle h_iter, h_ls;
    GP_CUDA(c0, cudaGraphConditionalHandleCreate(&h_iter, B->g, 1, cudaGraphCondAssignDefault));
    cudaGraph_t B1, B2;
    cudaGraphNode_t n_init;
    if ((rc = lockstep_route(B, c0, GR_INIT, h_iter, B->g, nullptr, 0, &n_init))) return rc;
    cudaGraphNode_t n_loop = add_conditional(c0, B->g, h_iter, cudaGraphCondTypeWhile, &B1, &rc);
    if (rc) return rc;
    GP_CUDA(c0, cudaGraphAddDependencies(B->g, &n_init, &n_loop, 1));
    GP_CUDA(c0, cudaGraphConditionalHandleCreate(&h_ls, B1, 0, 0));
    std::vector<cudaGraphConditionalHandle> hh(2 * (size_t)n);
    for (size_t i = 0; i < hh.size(); i++) GP_CUDA(c0, cudaGraphConditionalHandleCreate(&hh[i], B1, 0, 0));
    GP_CUDA(c0, cudaMemcpy(B->hd, hh.data(), sizeof(cudaGraphConditionalHandle) * hh.size(), cudaMemcpyHostToDevice));

    // B1: BEGIN, IF(pre_k), LS0, WHILE(ls), IF(post_k), END
    cudaGraphNode_t n_begin, n_ls0, n_lsw, n_end;
    std::vector<cudaGraphNode_t> pre((size_t)n), post((size_t)n);
    if ((rc = lockstep_route(B, c0, GR_BEGIN, h_iter, B1, nullptr, 0, &n_begin))) return rc;
    for (int k = 0; k < n && !rc; k++) {
        CgGraph *G = &B->loops[order[k]];
        cudaGraph_t body, s = nullptr;
        pre[k] = add_conditional(ctx[k], B1, hh[k], cudaGraphCondTypeIf, &body, &rc);
        if (rc) return rc;
        GP_CUDA(c0, cudaGraphAddDependencies(B1, &n_begin, &pre[k], 1));
        if ((rc = capture(ctx[k], G, SEQ_PRE, 0, 0, 0, &s, &G->n_pre))) return rc;
        cudaGraphNode_t nn;
        if ((rc = add_child(ctx[k], body, s, nullptr, 0, &nn))) return rc;
    }
    if ((rc = lockstep_route(B, c0, GR_LS0, h_ls, B1, pre.data(), pre.size(), &n_ls0))) return rc;
    n_lsw = add_conditional(c0, B1, h_ls, cudaGraphCondTypeWhile, &B2, &rc);
    if (rc) return rc;
    GP_CUDA(c0, cudaGraphAddDependencies(B1, &n_ls0, &n_lsw, 1));
    for (int k = 0; k < n && !rc; k++) {
        CgGraph *G = &B->loops[order[k]];
        cudaGraph_t body, s = nullptr;
        post[k] = add_conditional(ctx[k], B1, hh[n + k], cudaGraphCondTypeIf, &body, &rc);
        if (rc) return rc;
        GP_CUDA(c0, cudaGraphAddDependencies(B1, &n_lsw, &post[k], 1));
        if ((rc = capture(ctx[k], G, SEQ_POST, 0, 0, 0, &s, &G->n_post))) return rc;
        cudaGraphNode_t nn;
        if ((rc = add_child(ctx[k], body, s, nullptr, 0, &nn))) return rc;
    }
    if ((rc = lockstep_route(B, c0, GR_END, h_iter, B1, post.data(), post.size(), &n_end))) return rc;

    // B2: per class, the trial prep of its instances, its grouped forward, their
    // chi2 + controller; the CUDA-core instances' whole evaluations; LSN after all
    std::vector<cudaGraphNode_t> last;  // what LSN waits for
    for (int q = 0; q < B->ngrp && !rc; q++) {
        const int k0 = cls_begin[q], k1 = cls_begin[q + 1];
        std::vector<cudaGraphNode_t> bprep;
        for (int k = k0; k < k1 && !rc; k++) {
            gpair_ctx *c = ctx[k];
            CgGraph *G = &B->loops[order[k]];
            const int *gate = B->flags + n + k;
            cudaGraph_t s = nullptr;
            cudaGraphNode_t nd;
            rc = capture_fn(
                c,
                [&]() {
                    c->gate = gate;
                    int r = gp_eval_batch_part(c, 1);
                    c->gate = nullptr;
                    return r;
                },
                &s, &G->n_crit);
            if (rc || (rc = add_child(c, B2, s, nullptr, 0, &nd))) return rc;
            bprep.push_back(nd);
        }
        cudaGraphNode_t n_gemm;
        {
            gpair_ctx *c = ctx[k0];
            cudaGraph_t s = nullptr;
            rc = capture_fn(c, [&]() { return gp_tc_group_forward(B->grps[q], c); }, &s, nullptr);
            if (rc || (rc = add_child(c, B2, s, bprep.data(), bprep.size(), &n_gemm))) return rc;
        }
        for (int k = k0; k < k1 && !rc; k++) {
            gpair_ctx *c = ctx[k];
            CgGraph *G = &B->loops[order[k]];
            const int *gate = B->flags + n + k;
            cudaGraph_t s = nullptr;
            int n2 = 0;
            cudaGraphNode_t nd;
            rc = capture_fn(
                c,
                [&]() {
                    c->gate = gate;
                    c->fuse_ctrl = CTRL_AFTER_BATCH;
                    c->fuse_handles = 0;
                    int r = gp_eval_batch_part(c, 2);
                    c->fuse_ctrl = -1;
                    c->gate = nullptr;
                    return r;
                },
                &s, &n2);
            if (rc || (rc = add_child(c, B2, s, &n_gemm, 1, &nd))) return rc;
            G->n_crit += n2;
            last.push_back(nd);
        }
    }
    for (int k = ntc; k < n && !rc; k++) {
        gpair_ctx *c = ctx[k];
        CgGraph *G = &B->loops[order[k]];
        const int *gate = B->flags + n + k;
        cudaGraph_t s = nullptr;
        cudaGraphNode_t nd;
        rc = capture_fn(
            c,
            [&]() {
                c->gate = gate;
                c->fuse_ctrl = CTRL_AFTER_BATCH;
                c->fuse_handles = 0;
                int r = gp_eval_batch(c);
                c->fuse_ctrl = -1;
                c->gate = nullptr;
                return r;
            },
            &s, &G->n_crit);
        if (rc || (rc = add_child(c, B2, s, nullptr, 0, &nd))) return rc;
        last.push_back(nd);
    }
    cudaGraphNode_t n_lsn;
    return lockstep_route(B, c0, GR_LSN, h_ls, B2, last.data(), last.size(), &n_lsn);
}

// --------------------------------- staged lockstep batches (every stage grouped)
//
// With every instance on the tensor path (one operand element type, (u, v)
// given), every stage of an iteration is ONE launch over all instances
// (group.cuh), and every contraction one grouped tcgen05 launch per class:
//
//   [route INIT]   act[i] = 1
//   WHILE (h_any_iter)
//     prep | forward (per class) | V2/T3/chi2 | c_k | W | adjoint (per class)
//       | gradient, CTRL_BEGIN | direction, CTRL_AFTER_DIR           (gate act[i])
//     [route LS0S]   ls[i] = act[i] and the line search of i goes on; h_any_ls
//     WHILE (h_any_ls)
//       trial prep | trial forward (per class) | trial chi2, CTRL_AFTER_BATCH   (gate ls[i])
//       [route LSN]
//     image update | CTRL_END                                          (gate act[i])
//     [route END]    act[i] = act[i] and the run of i goes on; h_any_iter
//
// An instance's part of every launch has the arguments and the block grid of
// its own single launch, so its results are bitwise those of a separate run.

// argument structs and block starts of one stage over the instances ctx[0..n-1]
static int stage_table(BatchGraph *B, gpair_ctx **ctx, int n, int stage, double *const *trace, int *op_out,
                       int prep_passes)
{
    const bool tc = stage == GS_PREP_IMAGE || stage == GS_PREP_TRIALS || stage == GS_BUILD_W;
    const size_t sz = tc ? gp_tc_stage_args_size(stage) : gp_stage_args_size(stage);
    std::vector<unsigned char> h(sz * (size_t)n);
    std::vector<int> start((size_t)n + 1, 0);
    int op0 = -1;
    for (int k = 0; k < n; k++) {
        int nb = 0, op = -1, rc;
        if (tc) {
            rc = gp_tc_stage_args(ctx[k], stage, h.data() + sz * k, &nb, &op, prep_passes);
            if (!rc && op0 >= 0 && op != op0) rc = GPAIR_ERR_STATE;  // one operand element type per launch
            op0 = op;
        } else {
            rc = gp_stage_args(ctx[k], stage, trace[k], h.data() + sz * k, &nb);
        }
        if (rc) return rc;
        if (nb < 1 || (long long)start[k] + nb > (1LL << 30)) return GPAIR_ERR_STATE;
        start[k + 1] = start[k] + nb;
    }
    gpair_ctx *c0 = ctx[0];
    GP_CUDA(c0, cudaMalloc(&B->stg_args[stage], sz * (size_t)n));
    GP_CUDA(c0, cudaMemcpy(B->stg_args[stage], h.data(), sz * (size_t)n, cudaMemcpyHostToDevice));
    GP_CUDA(c0, cudaMalloc(&B->stg_start[stage], sizeof(int) * ((size_t)n + 1)));
    GP_CUDA(c0, cudaMemcpy(B->stg_start[stage], start.data(), sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice));
    B->stg_total[stage] = start[(size_t)n];
    if (op_out) *op_out = op0;
    return GPAIR_OK;
}

// GPAIR_ERR_STATE: the instances cannot run fully staged (the caller builds the
// lockstep with grouped trial forwards only, or independent branches)
static int build_lockstep_staged(gpair_ctx **ctx_in, int n, BatchGraph *B, int with_stamps, int prep_passes_req)
{
    if (n > 4096) return GPAIR_ERR_STATE;
    std::vector<int> key((size_t)n), order((size_t)n);
    for (int i = 0; i < n; i++) {
        key[i] = gp_tc_group_key(ctx_in[i]);
        if (key[i] < 0 || !ctx_in[i]->have_uv) return GPAIR_ERR_STATE;
        order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<gpair_ctx *> ctx((size_t)n);
    for (int k = 0; k < n; k++) ctx[k] = ctx_in[order[k]];
    gpair_ctx *c0 = ctx[0];
    // classes of the contractions, at most 256 instances per grouped launch
    std::vector<int> cls_begin;
    for (int k = 0; k < n; k++)
        if (cls_begin.empty() || key[order[k]] != key[order[k - 1]] || k - cls_begin.back() == 256)
            cls_begin.push_back(k);
    cls_begin.push_back(n);
    const int ngrp = (int)cls_begin.size() - 1;
    // adjoint classes: the same without the forward operand kind (key >> 3), contiguous in key order
    std::vector<int> acls_begin;
    for (int k = 0; k < n; k++)
        if (acls_begin.empty() || (key[order[k]] >> 3) != (key[order[k - 1]] >> 3) || k - acls_begin.back() == 256)
            acls_begin.push_back(k);
    acls_begin.push_back(n);
    const int nadj = (int)acls_begin.size() - 1;
    // every instance's tensor state and batch buffers (no allocation inside a capture)
    for (int k = 0; k < n; k++) {
        int rc = gp_batch_alloc(ctx[k]);
        if (!rc) rc = gp_tc_stage_sizes(ctx[k], &ctx[k]->mt, &ctx[k]->splits);
        if (rc) return rc == GPAIR_ERR_STATE ? GPAIR_ERR_CUDA : rc;
    }
    // the prep and W stages need one operand element type for all instances
    int op_prep = -1;
    {
        std::vector<unsigned char> tmp(gp_tc_stage_args_size(GS_PREP_IMAGE));
        for (int k = 0; k < n; k++) {
            int nb = 0, op = -1;
            int rc = gp_tc_stage_args(ctx[k], GS_PREP_IMAGE, tmp.data(), &nb, &op);
            if (rc) return rc == GPAIR_ERR_STATE ? GPAIR_ERR_CUDA : rc;
            if (op_prep >= 0 && op != op_prep) return GPAIR_ERR_STATE;
            op_prep = op;
        }
    }
    GP_CUDA(c0, cudaMalloc(&B->flags, sizeof(int) * 2 * (size_t)n));
    GP_CUDA(c0, cudaMemset(B->flags, 0, sizeof(int) * 2 * (size_t)n));
    GP_CUDA(c0, cudaMalloc(&B->gerr, sizeof(unsigned int)));
    GP_CUDA(c0, cudaMemset(B->gerr, 0, sizeof(unsigned int)));
    const int *act = B->flags, *lsg = B->flags + n;
    B->ngrp = ngrp;
    B->grps = (void **)calloc((size_t)ngrp, sizeof(void *));
    B->grps_img = (void **)calloc((size_t)ngrp, sizeof(void *));
    B->grps_adj = (void **)calloc((size_t)nadj, sizeof(void *));
    if (!B->grps || !B->grps_img || !B->grps_adj) return GPAIR_ERR_ALLOC;
    B->nadj = nadj;
    int rc = GPAIR_OK;
    for (int q = 0; q < ngrp && !rc; q++) {
        const int k0 = cls_begin[q], k1 = cls_begin[q + 1];
        rc = gp_tc_group_build_kind(&ctx[k0], k1 - k0, GP_TCG_TRIALS, lsg + k0, B->gerr, &B->grps[q]);
        if (!rc) rc = gp_tc_group_build_kind(&ctx[k0], k1 - k0, GP_TCG_IMAGE, act + k0, B->gerr, &B->grps_img[q]);
    }
    for (int q = 0; q < nadj && !rc; q++) {
        const int k0 = acls_begin[q], k1 = acls_begin[q + 1];
        rc = gp_tc_group_build_kind(&ctx[k0], k1 - k0, GP_TCG_ADJOINT, act + k0, B->gerr, &B->grps_adj[q]);
    }
    if (rc) return rc == GPAIR_ERR_STATE ? GPAIR_ERR_CUDA : rc;  // the instances were eligible
    std::vector<double *> trace((size_t)n);
    for (int k = 0; k < n; k++) trace[k] = B->loops[order[k]].trace;
    int op = -1;
    // the trial prep's trial sums are per image row where rows are one warp wide, so its
    // blocks can take several passes without changing a result
    const int prep_passes = prep_passes_req ? prep_passes_req : gp_tc_prep_trials_passes(ctx.data(), n, op_prep);
    B->prep_passes = prep_passes;
    for (int st = 0; st < GS_COUNT && !rc; st++)
        rc = stage_table(B, ctx.data(), n, st, trace.data(), &op, prep_passes);
    if (rc) return rc == GPAIR_ERR_STATE ? GPAIR_ERR_CUDA : rc;
    GP_CUDA(c0, cudaMalloc(&B->scs, sizeof(DevScalars *) * (size_t)n));
    std::vector<DevScalars *> hs((size_t)n);
    for (int k = 0; k < n; k++) hs[k] = ctx[k]->sc;
    GP_CUDA(c0, cudaMemcpy(B->scs, hs.data(), sizeof(DevScalars *) * (size_t)n, cudaMemcpyHostToDevice));

    auto stage = [&](int st, const int *gate) {
        const bool tc = st == GS_PREP_IMAGE || st == GS_PREP_TRIALS || st == GS_BUILD_W;
        return tc ? gp_tc_stage_group_launch(c0, st, op_prep, B->stg_args[st], B->stg_start[st], n, B->stg_total[st],
                                             gate)
                  : gp_stage_group_launch(c0, st, B->stg_args[st], B->stg_start[st], n, B->stg_total[st], gate);
    };
    // grouped contractions: each class on c0's stream, with the wait budget of its first instance
    auto gemms = [&](void **grps, const std::vector<int> &cb) {
        for (size_t q = 0; q + 1 < cb.size(); q++) {
            int r = gp_tc_group_run(grps[q], ctx[cb[q]], c0->stream);
            if (r) return r;
        }
        return GPAIR_OK;
    };
    if (with_stamps) {
        GP_CUDA(c0, cudaMalloc(&B->stamps, sizeof(unsigned long long) * GP_STAMP_WORDS));
        GP_CUDA(c0, cudaMemset(B->stamps, 0, sizeof(unsigned long long) * GP_STAMP_WORDS));
    }
    // a device timer stamp (plain launch: it follows the complete kernel before it)
    auto stamp = [&](int i) {
        if (!B->stamps) return GPAIR_OK;
        k_stamp<<<1, 32, 0, c0->stream>>>(B->stamps, i);
        GP_LAUNCH_CHECK(c0);
        return GPAIR_OK;
    };
    auto route = [&](int what, cudaGraphConditionalHandle h) {
        GP_LAUNCH(c0, gp_launch(c0, k_lockstep_route, dim3(1), dim3(256), 0, what, B->scs, n, B->flags,
                                B->flags + n, (const cudaGraphConditionalHandle *)nullptr,
                                (const cudaGraphConditionalHandle *)nullptr, h, B->gerr));
        return GPAIR_OK;
    };

    cudaGraphConditionalHandle h_iter, h_ls;
    GP_CUDA(c0, cudaGraphConditionalHandleCreate(&h_iter, B->g, 1, cudaGraphCondAssignDefault));
    cudaGraph_t g_init = nullptr, B1, B2;
    if ((rc = capture_fn(c0, [&]() { return route(GR_INIT, h_iter); }, &g_init, nullptr))) return rc;
    cudaGraphNode_t n_init, n_loop, n_pre, n_lsw, n_post, n_ls;
    if ((rc = add_child(c0, B->g, g_init, nullptr, 0, &n_init))) return rc;
    n_loop = add_conditional(c0, B->g, h_iter, cudaGraphCondTypeWhile, &B1, &rc);
    if (rc) return rc;
    GP_CUDA(c0, cudaGraphAddDependencies(B->g, &n_init, &n_loop, 1));
    GP_CUDA(c0, cudaGraphConditionalHandleCreate(&h_ls, B1, 0, 0));

    // B1: pre-phase + LS0S, WHILE (h_ls), post-phase + END
    int npre = 0, nls = 0, npost = 0;
    cudaGraph_t g_pre = nullptr, g_post = nullptr, g_ls = nullptr;
    rc = capture_fn(
        c0,
        [&]() {
            int r;
            if ((r = stamp(0)) || (r = stage(GS_PREP_IMAGE, act)) || (r = stamp(1))) return r;
            if ((r = gemms(B->grps_img, cls_begin)) || (r = stamp(2))) return r;
            if ((r = stage(GS_VIS_DATA, act)) || (r = stamp(3))) return r;
            if ((r = stage(GS_ADJ_WEIGHTS, act)) || (r = stamp(4))) return r;
            if ((r = stage(GS_BUILD_W, act)) || (r = stamp(5))) return r;
            if ((r = gemms(B->grps_adj, acls_begin)) || (r = stamp(6))) return r;
            if ((r = stage(GS_GRAD_FINALIZE, act)) || (r = stamp(7))) return r;
            if ((r = stage(GS_DESCENT, act)) || (r = stamp(8))) return r;
            if ((r = route(GR_LS0S, h_ls))) return r;
            return stamp(9);
        },
        &g_pre, &npre);
    if (rc || (rc = add_child(c0, B1, g_pre, nullptr, 0, &n_pre))) return rc;
    n_lsw = add_conditional(c0, B1, h_ls, cudaGraphCondTypeWhile, &B2, &rc);
    if (rc) return rc;
    GP_CUDA(c0, cudaGraphAddDependencies(B1, &n_pre, &n_lsw, 1));
    rc = capture_fn(
        c0,
        [&]() {
            int r;
            if ((r = stamp(15)) || (r = stage(GS_UPDATE, act)) || (r = stamp(16))) return r;
            if ((r = stage(GS_CTRL_END, act)) || (r = stamp(17))) return r;
            if ((r = route(GR_END, h_iter))) return r;
            return stamp(18);
        },
        &g_post, &npost);
    if (rc || (rc = add_child(c0, B1, g_post, &n_lsw, 1, &n_post))) return rc;
    // B2: one batched evaluation of every searching instance
    rc = capture_fn(
        c0,
        [&]() {
            int r;
            if ((r = stamp(10)) || (r = stage(GS_PREP_TRIALS, lsg)) || (r = stamp(11))) return r;
            if ((r = gemms(B->grps, cls_begin)) || (r = stamp(12))) return r;
            if ((r = stage(GS_CHI2_BATCH, lsg)) || (r = stamp(13))) return r;
            if ((r = route(GR_LSN, h_ls))) return r;
            return stamp(14);
        },
        &g_ls, &nls);
    if (rc || (rc = add_child(c0, B2, g_ls, nullptr, 0, &n_ls))) return rc;
    // launches an instance takes part in (shared with the other instances)
    for (int i = 0; i < n; i++) {
        B->loops[i].n_pre = npre;
        B->loops[i].n_post = npost;
        B->loops[i].n_crit = nls;
        B->loops[i].n_grad = 0;
    }
    B->staged = 1;
    return GPAIR_OK;
}

int gp_batch_graph_build(gpair_ctx **ctx, int n, int ls_mode, int allow_group, void **out)
{
    *out = nullptr;
    BatchGraph *B = (BatchGraph *)calloc(1, sizeof(BatchGraph));
    if (!B) return GPAIR_ERR_ALLOC;
    B->n = n;
    B->loops = (CgGraph *)calloc((size_t)n, sizeof(CgGraph));
    if (!B->loops || cudaGraphCreate(&B->g, 0) != cudaSuccess) {
        gp_batch_graph_free(B);
        return GPAIR_ERR_ALLOC;
    }
    int rc = GPAIR_OK;
    for (int i = 0; i < n && !rc; i++) {
        CgGraph *G = &B->loops[i];
        G->precision = ctx[i]->precision;
        G->ls_mode = ls_mode;
        G->trace_cap = 1;  // one row; batch runs return no trace
        if (cudaMalloc(&G->trace, sizeof(double) * 5) != cudaSuccess) rc = GPAIR_ERR_ALLOC;
    }
    if (!rc && (allow_group & 3) >= 2 && ls_mode == GPAIR_LS_BATCH) {
        rc = build_lockstep_staged(ctx, n, B, allow_group & 4, (allow_group >> 8) & 63);
        if (rc == GPAIR_OK) {
            B->grouped = 2;
        } else if (rc == GPAIR_ERR_STATE) {
            // not every instance can take part in every grouped stage (nothing was
            // built yet): the lockstep with grouped forwards only
            rc = GPAIR_OK;
        }
    }
    if (!rc && !B->grouped && (allow_group & 3) && ls_mode == GPAIR_LS_BATCH) {
        rc = build_lockstep(ctx, n, B);
        if (rc == GPAIR_OK) {
            B->grouped = 1;
        } else if (rc == GPAIR_ERR_STATE) {
            // no instance on the tensor path: independent branches
            cudaGraphDestroy(B->g);
            B->g = nullptr;
            rc = cudaGraphCreate(&B->g, 0) == cudaSuccess ? GPAIR_OK : GPAIR_ERR_CUDA;
        }
    }
    for (int i = 0; i < n && !rc && !B->grouped; i++) rc = add_loop(ctx[i], &B->loops[i], B->g);
    for (int i = 0; i < n && !rc; i++) B->loops[i].buf_gen = ctx[i]->buf_gen;
    if (!rc) {
        cudaError_t e = cudaGraphInstantiate(&B->exec, B->g, 0);
        if (e != cudaSuccess) {
            snprintf(ctx[0]->last_error, sizeof(ctx[0]->last_error), "batch graph instantiate: %s",
                     cudaGetErrorString(e));
            rc = GPAIR_ERR_CUDA;
        }
    }
    if (rc) {
        gp_batch_graph_free(B);
        return rc;
    }
    *out = B;
    return GPAIR_OK;
}

int gp_batch_graph_launch(void *bg, cudaStream_t stream)
{
    BatchGraph *B = (BatchGraph *)bg;
    return cudaGraphLaunch(B->exec, stream) == cudaSuccess ? GPAIR_OK : GPAIR_ERR_CUDA;
}

int gp_batch_graph_precision(void *bg, int i) { return ((BatchGraph *)bg)->loops[i].precision; }
unsigned int gp_batch_graph_buf_gen(void *bg, int i) { return ((BatchGraph *)bg)->loops[i].buf_gen; }
int gp_batch_graph_grouped(void *bg) { return bg ? ((BatchGraph *)bg)->grouped : 0; }
int gp_batch_graph_prep_passes(void *bg) { return bg && ((BatchGraph *)bg)->staged ? ((BatchGraph *)bg)->prep_passes : 0; }

// the stage stamps of a staged batch (none recorded: 0); `reset` zeroes them
// afterwards (on st), so that the next run's sums start from zero
int gp_batch_graph_stamps(void *bg, unsigned long long *out, int max, cudaStream_t st, int reset)
{
    BatchGraph *B = (BatchGraph *)bg;
    if (!B || !B->stamps) return 0;
    const int n = max < GP_STAMP_WORDS ? max : GP_STAMP_WORDS;
    if (n > 0 && cudaMemcpyAsync(out, B->stamps, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, st) !=
                     cudaSuccess)
        return GPAIR_ERR_CUDA;
    if (reset && cudaMemsetAsync(B->stamps, 0, sizeof(unsigned long long) * GP_STAMP_WORDS, st) != cudaSuccess)
        return GPAIR_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GPAIR_ERR_CUDA;
    return GP_STAMP_WORDS;
}

long long gp_batch_graph_launches(void *bg, int i, int iterations_done, int criterion_evals, int grad_evals,
                                  int batches)
{
    const CgGraph *G = &((BatchGraph *)bg)->loops[i];
    long long base = (long long)iterations_done * (G->n_pre + G->n_post);
    if (G->ls_mode == GPAIR_LS_BATCH) return base + (long long)batches * G->n_crit;
    return base + (long long)(criterion_evals - iterations_done) * G->n_crit +
           (long long)(grad_evals - iterations_done) * G->n_grad;
}

// Launch `iterations` CG iterations as one graph. Returns the kernel launches
// it executed through *launches (from the controller's evaluation counters).
int gp_cg_graph_run(gpair_ctx *c, int iterations, int want_trace, int ls_mode, long long *launches)
{
    if (ls_mode < 0 || ls_mode > 1) return GPAIR_ERR_INVALID;
    c->cg_graph_mode = ls_mode;
    CgGraph *G = (CgGraph *)c->cg_graph[ls_mode];
    int cap = iterations > 4096 ? iterations : 4096;
    if (!G || G->precision != c->precision || G->lbfgs != (c->cg_method == 4) ||
        (want_trace && G->trace_cap < iterations)) {
        int rc = build(c, cap, ls_mode);
        if (rc) return rc;
        G = (CgGraph *)c->cg_graph[ls_mode];
    }
    if (iterations > 0) GP_CUDA(c, cudaGraphLaunch(G->exec, c->stream));
    *launches = 0;
    return GPAIR_OK;
}

int gp_cg_graph_trace(gpair_ctx *c, int iterations, double *tJ, double *tchi2, double *tS, double *tstep,
                      double *tbeta)
{
    CgGraph *G = (CgGraph *)c->cg_graph[c->cg_graph_mode];
    if (!G || iterations <= 0) return GPAIR_OK;
    int n = iterations < G->trace_cap ? iterations : G->trace_cap;
    double *h = (double *)malloc(sizeof(double) * 5 * (size_t)n);
    if (!h) return GPAIR_ERR_ALLOC;
    cudaError_t e = cudaMemcpyAsync(h, G->trace, sizeof(double) * 5 * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        free(h);
        snprintf(c->last_error, sizeof(c->last_error), "trace copy: %s", cudaGetErrorString(e));
        return GPAIR_ERR_CUDA;
    }
    for (int i = 0; i < n; i++) {
        if (tJ) tJ[i] = h[5 * i];
        if (tchi2) tchi2[i] = h[5 * i + 1];
        if (tS) tS[i] = h[5 * i + 2];
        if (tstep) tstep[i] = h[5 * i + 3];
        if (tbeta) tbeta[i] = h[5 * i + 4];
    }
    free(h);
    return GPAIR_OK;
}

// kernel launches a finished graph run executed
long long gp_cg_graph_launches(gpair_ctx *c, int iterations_done, int criterion_evals, int grad_evals, int batches)
{
    CgGraph *G = (CgGraph *)c->cg_graph[c->cg_graph_mode];
    if (!G) return 0;
    long long base = (long long)iterations_done * (G->n_pre + G->n_post);
    if (G->ls_mode == GPAIR_LS_BATCH) return base + (long long)batches * G->n_crit;
    long long trials_c = criterion_evals - iterations_done, trials_g = grad_evals - iterations_done;
    return base + trials_c * G->n_crit + trials_g * G->n_grad;
}
