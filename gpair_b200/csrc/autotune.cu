// autotune.cu -- per-problem choice of the precision path, the tensor-core tile
// and the adjoint's split-K tile length, by timing criterion + gradient
// evaluations of the loaded problem on the device (CUDA events on the
// context's stream).
//
// Candidates:
//   precision  FP32 (CUDA-core contractions), split-f16 and split-f16/E4M3
//              (tcgen05); all meet the accuracy bounds, the fastest depends on
//              the image width and the uv count (small problems leave the
//              tensor GEMM's tiles mostly empty)
//   tile       (tensor) 256 x 256 output tiles on CTA pairs or 128 x 256 on
//              single CTAs: pairs halve the operand traffic per MMA, single
//              CTAs pad the uv rows less and give small problems more tiles
//   splits     the adjoint's K-blocks per split (tensor) or split count
//              (CUDA cores): the heuristic's value, half and double of it,
//              within the FP32-accumulation cap and the partial-image buffer
// Objective: one criterion + gradient evaluation, or (GPAIR_TUNE_BATCHED) that
// plus two batched 8-trial evaluations, the work of a batched-line-search
// iteration. Choices are cached per (device, width, uv count to 1/8, objective,
// and the precision path and tile layout when those are not tuned).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "gpair_internal.cuh"

namespace {

struct Choice {
    int precision, tc_kb_per, simt_splits, tc_pair;
    double ms;
};

std::mutex g_mu;
std::map<std::tuple<int, int, int, int>, Choice> g_cache;

int uv_bucket(int nuv) { return nuv <= 0 ? 0 : (int)floor(log2((double)nuv) * 8.0); }

// average ms of one criterion + gradient evaluation of the current image, plus
// (batched) two evaluations of 8 trial images: the work of one iteration of the
// batched line search
int time_evals(gpair_ctx *c, int reps, int batched, double *ms)
{
    if (batched) {
        int rc = gp_batch_alloc(c);
        if (rc) return rc;
    }
    cudaEvent_t e0, e1;
    GP_CUDA(c, cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return GPAIR_ERR_CUDA;
    }
    int rc = GPAIR_OK;
    const int st = c->stage_timing;
    c->stage_timing = 0;
    c->fuse_ctrl = -1;
    // one untimed pass: first-use costs (operand tables, function attributes)
    rc = gp_eval_criterion(c, GPAIR_IMG_CURR, 0);
    if (!rc) rc = gp_eval_gradient(c, GPAIR_IMG_CURR, 1e-3f);
    if (!rc && batched) rc = gp_eval_batch(c);
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && !rc; r++) {
        rc = gp_eval_criterion(c, GPAIR_IMG_CURR, 0);
        if (!rc) rc = gp_eval_gradient(c, GPAIR_IMG_CURR, 1e-3f);
        for (int b = 0; b < 2 * batched && !rc; b++) rc = gp_eval_batch(c);  // no controller: fuse_ctrl = -1
    }
    cudaEventRecord(e1, c->stream);
    c->stage_timing = st;
    float t = 0.f;
    if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = GPAIR_ERR_CUDA;
    if (!rc) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!rc) rc = gp_sync_scalars(c);  // a bounded-wait timeout surfaces here
    *ms = t / reps;
    return rc;
}

int apply(gpair_ctx *c, const Choice &ch)
{
    if (c->tc_pair != ch.tc_pair) {
        int rc = gpair_set_tc_pair(c, ch.tc_pair);  // rebuilds the tensor state on the tensor path
        if (rc) return rc;
    }
    int rc = gpair_set_precision(c, ch.precision);
    if (rc) return rc;
    if (ch.precision != GPAIR_PREC_FP32) {
        if ((rc = gp_tc_prepare(c))) return rc;
        if ((rc = gp_tc_set_kb_per(c, ch.tc_kb_per))) return rc;
    }
    c->splits_simt = ch.simt_splits;
    gp_cg_graph_free(c);  // a captured CG graph holds the old configuration
    return GPAIR_OK;
}

}  // namespace

extern "C" int gpair_autotune(gpair_ctx *c, int flags, int reps, gpair_tune_result *res)
{
    if (!c || !c->have_problem || !c->have_image) return GPAIR_ERR_STATE;
    if (reps <= 0) reps = 3;
    GP_CUDA(c, cudaSetDevice(c->device));
    // the settings that are not tuned are part of the key: a choice made for another
    // fixed precision path or tile layout is not reused
    const int fixed = ((flags & GPAIR_TUNE_PRECISION) ? 0 : c->precision + 1) * 4 +
                      ((flags & GPAIR_TUNE_TILE) ? 0 : c->tc_pair + 1);
    const auto key = std::make_tuple(c->device, c->N,
                                     uv_bucket(c->nuv) * 4 + ((flags & GPAIR_TUNE_BATCHED) ? 1 : 0) +
                                         ((flags & GPAIR_TUNE_TILE) ? 2 : 0),
                                     fixed);
    if (res) memset(res, 0, sizeof(*res));
    if (flags & GPAIR_TUNE_CACHE) {
        Choice ch;
        bool hit = false;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            auto it = g_cache.find(key);
            if (it != g_cache.end()) {
                ch = it->second;
                hit = true;
            }
        }
        bool applied = false;
        if (hit) {
            // a cached split-K length can exceed this problem's partial-image buffer
            // (GPAIR_ERR_INVALID): then this problem is tuned afresh
            int rc = apply(c, ch);
            if (rc && rc != GPAIR_ERR_INVALID) return rc;
            applied = rc == GPAIR_OK;
        }
        if (applied) {
            if (res) {
                res->precision = ch.precision;
                res->adjoint_splits = ch.precision == GPAIR_PREC_FP32 ? ch.simt_splits : gp_tc_split_count(c, ch.tc_kb_per);
                res->ms_per_eval = ch.ms;
                res->from_cache = 1;
                res->tile_m = ch.precision == GPAIR_PREC_FP32 ? 0 : (ch.tc_pair ? 256 : 128);
            }
            return GPAIR_OK;
        }
    }
    std::vector<int> precs;
    if (flags & GPAIR_TUNE_PRECISION) {
        precs.push_back(GPAIR_PREC_SPLIT16);
        precs.push_back(GPAIR_PREC_SPLIT16F8);
        precs.push_back(GPAIR_PREC_FP32);
    } else {
        precs.push_back(c->precision);
    }
    const int simt0 = c->splits_simt > 0 ? c->splits_simt : 1;
    std::vector<Choice> cand;
    for (int prec : precs) {
        if (prec == GPAIR_PREC_FP32) {
            std::vector<int> ss = {simt0};
            if (flags & GPAIR_TUNE_SPLITS) {
                if (simt0 / 2 >= 1) ss.push_back(simt0 / 2);
                if (2 * simt0 <= c->gpart_cap && 2 * simt0 <= 64) ss.push_back(2 * simt0);
            }
            for (int s : ss) cand.push_back({prec, 0, s, c->tc_pair, 0.0});
        } else {
            std::vector<int> pairs = {c->tc_pair};
            if (flags & GPAIR_TUNE_TILE) pairs.push_back(!c->tc_pair);
            for (int pr : pairs) {
                int rc = gpair_set_tc_pair(c, pr);
                if (rc) return rc;
                if ((rc = gpair_set_precision(c, prec))) return rc;
                if ((rc = gp_tc_prepare(c))) return rc;
                const int k0 = gp_tc_kb_per(c);  // the heuristic's split for this tile
                if (k0 <= 0) return GPAIR_ERR_STATE;
                std::vector<int> ks = {k0};
                if (flags & GPAIR_TUNE_SPLITS) {
                    if (k0 / 2 >= 1) ks.push_back(k0 / 2);
                    if (2 * k0 <= gp_tc_kb_cap(c)) ks.push_back(2 * k0);
                }
                for (int k : ks) cand.push_back({prec, k, simt0, pr, 0.0});
            }
        }
    }
    if ((int)cand.size() > GPAIR_TUNE_MAX_CANDIDATES) cand.resize(GPAIR_TUNE_MAX_CANDIDATES);
    int best = -1;
    for (size_t i = 0; i < cand.size(); i++) {
        int rc = apply(c, cand[i]);
        if (rc == GPAIR_ERR_INVALID) {  // a split count beyond the partial-image buffer: skip it
            cand[i].ms = INFINITY;
            continue;
        }
        if (rc) return rc;
        if ((rc = time_evals(c, reps, (flags & GPAIR_TUNE_BATCHED) ? 1 : 0, &cand[i].ms))) return rc;
        if (best < 0 || cand[i].ms < cand[best].ms) best = (int)i;
    }
    if (best < 0) return GPAIR_ERR_STATE;
    int rc = apply(c, cand[best]);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_cache[key] = cand[best];
    }
    if (res) {
        res->precision = cand[best].precision;
        res->adjoint_splits = cand[best].precision == GPAIR_PREC_FP32 ? cand[best].simt_splits
                                                                       : gp_tc_split_count(c, cand[best].tc_kb_per);
        res->ms_per_eval = cand[best].ms;
        res->n_candidates = (int)cand.size();
        res->tile_m = cand[best].precision == GPAIR_PREC_FP32 ? 0 : (cand[best].tc_pair ? 256 : 128);
        for (size_t i = 0; i < cand.size(); i++) {
            res->cand_tile_m[i] = cand[i].precision == GPAIR_PREC_FP32 ? 0 : (cand[i].tc_pair ? 256 : 128);
            res->cand_precision[i] = cand[i].precision;
            res->cand_splits[i] = cand[i].precision == GPAIR_PREC_FP32 ? cand[i].simt_splits
                                                                      : gp_tc_split_count(c, cand[i].tc_kb_per);
            res->cand_ms[i] = cand[i].ms;
        }
    }
    return GPAIR_OK;
}
