// C-ABI: groups of independent H_eff plans applied and solved together (the batching form).
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/qcm_b200.h"
#include "capi_types.hpp"
#include "capi_util.hpp"
#include "dmrg_dev.hpp"
#include "heff.hpp"

struct qcm_heff_group {
    qcm_ctx* ctx = nullptr;
    std::unique_ptr<qcm::HeffPlan> g;
    std::vector<uint64_t> xo, xn;
    qcm::DBuf<double> x, y;  // arena staging for host-buffer calls
};

extern "C" {

int qcm_heff_group_create(qcm_ctx* ctx, qcm_heff* const* plans, int n, qcm_heff_group** out) {
    QCM_TRY
    if (!ctx || !plans || n < 1 || !out) return qcm::fail(QCM_ERR_ARG, "qcm_heff_group_create: bad arguments");
    std::vector<qcm::HeffPlan*> ps;
    for (int i = 0; i < n; ++i) {
        if (!plans[i] || plans[i]->ctx != ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_group_create: a plan of another context, or NULL");
        ps.push_back(plans[i]->p.get());
    }
    QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx->stream);
    auto g = std::make_unique<qcm_heff_group>();
    g->ctx = ctx;
    g->g = qcm::merge_plans(ps, g->xo, ctx->stream);
    for (auto* p : ps) g->xn.push_back(p->x_len);
    *out = g.release();
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_group_layout(const qcm_heff_group* g, uint64_t* arena_len, uint64_t* offsets, uint64_t* lengths) {
    if (!g) return qcm::fail(QCM_ERR_ARG, "qcm_heff_group_layout: NULL group");
    if (arena_len) *arena_len = g->g->x_len;
    for (std::size_t i = 0; i < g->xo.size(); ++i) {
        if (offsets) offsets[i] = g->xo[i];
        if (lengths) lengths[i] = g->xn[i];
    }
    return QCM_OK;
}

int qcm_heff_group_get_info(const qcm_heff_group* g, qcm_heff_info* info) {
    if (!g || !info) return qcm::fail(QCM_ERR_ARG, "qcm_heff_group_get_info: NULL argument");
    const qcm::HeffPlan& p = *g->g;
    std::memset(info, 0, sizeof(*info));
    info->vec_len = p.x_len;
    info->t_len = p.t_len;
    info->s_len = p.s_len;
    info->p_len = p.p_len;
    info->n_tjobs = p.tjobs.size();
    info->n_gtasks = p.units.size();
    info->n_alpha = p.n_alpha;
    info->n_segs = p.segs.size();
    info->n_outs = p.outs.size();
    info->launches = uint64_t(qcm::heff_launches_per_apply(p));
    info->flops = p.flops;
    info->flops_t = p.flops_t;
    info->flops_ls = p.flops_ls;
    info->flops_s = p.flops_s;
    info->flops_sexec = p.flops_sexec;
    return QCM_OK;
}

int qcm_heff_group_apply_device(qcm_heff_group* g, const double* x_dev, double* y_dev) {
    QCM_TRY
    if (!g || !x_dev || !y_dev) return qcm::fail(QCM_ERR_ARG, "qcm_heff_group_apply_device: NULL argument");
    qcm::heff_apply_device(*g->g, x_dev, y_dev);
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_group_apply(qcm_heff_group* g, const double* x, double* y) {
    QCM_TRY
    if (!g || !x || !y) return qcm::fail(QCM_ERR_ARG, "qcm_heff_group_apply: NULL argument");
    qcm::HeffPlan& p = *g->g;
    qcm::AllocStream scope(p.stream);
    if (g->x.size() < p.x_len) { g->x.alloc(p.x_len); g->y.alloc(p.x_len); }
    QCM_CUDA(cudaMemcpyAsync(g->x.get(), x, p.x_len * sizeof(double), cudaMemcpyHostToDevice, p.stream));
    qcm::heff_apply_device(p, g->x.get(), g->y.get());
    QCM_CUDA(cudaMemcpyAsync(y, g->y.get(), p.x_len * sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    QCM_CUDA(cudaStreamSynchronize(p.stream));
    return QCM_OK;
    QCM_CATCH
}

int qcm_jd_solve_batched(qcm_heff_group* g, const double* x0, double tol, int maxiter, int use_graphs, double* out,
                         double* evals, int* iters, int* applies) {
    QCM_TRY
    if (!g || !x0 || !out || !evals || !iters) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_batched: NULL argument");
    qcm::HeffPlan& p = *g->g;
    qcm::AllocStream scope(p.stream);
    if (g->x.size() < p.x_len) { g->x.alloc(p.x_len); g->y.alloc(p.x_len); }
    QCM_CUDA(cudaMemcpyAsync(g->x.get(), x0, p.x_len * sizeof(double), cudaMemcpyHostToDevice, p.stream));
    std::vector<double> ev;
    std::vector<int> it;
    qcm::jacobi_davidson_batched(p, g->xo, g->xn, g->x.get(), tol, maxiter, ev, it, use_graphs != 0, applies);
    QCM_CUDA(cudaMemcpyAsync(out, g->x.get(), p.x_len * sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    QCM_CUDA(cudaStreamSynchronize(p.stream));
    std::copy(ev.begin(), ev.end(), evals);
    std::copy(it.begin(), it.end(), iters);
    return QCM_OK;
    QCM_CATCH
}

void qcm_heff_group_free(qcm_heff_group* g) { delete g; }

}  // extern "C"
