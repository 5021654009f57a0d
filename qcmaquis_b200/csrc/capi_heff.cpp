// C-ABI: context, resident boundaries and the H_eff plan / apply (the H.psi callback).
#include <cstring>
#include <string>
#include <memory>
#include <vector>

#include "../../include/qcm_b200.h"
#include "capi_types.hpp"
#include "capi_util.hpp"
#include "device.hpp"
#include "heff.hpp"

namespace qcm {
const MPO& mpo_of(const qcm_mpo* m);
}


namespace {
qcm::Index to_index(uint32_t n, const qcm_sector* s) {
    qcm::Index r;
    for (uint32_t i = 0; i < n; ++i) r.d.push_back({qcm::Charge(s[i].a, s[i].b), s[i].size});
    for (std::size_t i = 1; i < r.d.size(); ++i)
        if (!(r.d[i - 1].first > r.d[i].first)) throw std::runtime_error("sector list must be in strictly descending charge order");
    return r;
}
}  // namespace

extern "C" {

int qcm_ctx_create(int device, qcm_ctx** out) {
    QCM_TRY
    if (!out) return qcm::fail(QCM_ERR_ARG, "qcm_ctx_create: out is NULL");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return qcm::fail(QCM_ERR_NODEV, "no CUDA device (no CPU fallback)");
    if (device < 0 || device >= n) return qcm::fail(QCM_ERR_ARG, "qcm_ctx_create: bad device index");
    QCM_CUDA(cudaSetDevice(device));
    auto c = std::make_unique<qcm_ctx>();
    c->device = device;
    // the allocation-free apply's array is loaded on this device now, not at its first call, so
    // that its memory is taken before a host allocator reserves the rest of HBM
    c->noalloc_scratch = qcm::noalloc_scratch_address();
    QCM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    qcm::register_stream(c->stream);
    *out = c.release();
    return QCM_OK;
    QCM_CATCH
}

void qcm_ctx_destroy(qcm_ctx* c) {
    if (!c) return;
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
        qcm::retire_stream(c->stream);
        cudaStreamDestroy(c->stream);
    }
    delete c;
}

int qcm_ctx_synchronize(qcm_ctx* c) {
    QCM_TRY
    QCM_CUDA(cudaStreamSynchronize(c->stream));
    return QCM_OK;
    QCM_CATCH
}

}  // extern "C"

namespace {
int boundary_make(qcm_ctx* ctx, const qcm_boundary_desc* d, qcm_boundary** out) {
    QCM_TRY
    if (!d || !out) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_upload: NULL argument");
    if (ctx) QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx ? ctx->stream : nullptr);
    auto b = std::make_unique<qcm_boundary>();
    b->ctx = ctx;
    qcm::BoundaryIndexH& x = b->b.idx;
    x.bra = to_index(d->n_bra, d->bra);
    x.ket = to_index(d->n_ket, d->ket);
    x.aux = d->aux_dim;
    const uint32_t nc = d->n_cohorts;
    x.cbra.assign(d->cohort_bra, d->cohort_bra + nc);
    x.cket.assign(d->cohort_ket, d->cohort_ket + nc);
    x.tr.assign(d->tr, d->tr + nc);
    x.offsets.assign(d->offsets, d->offsets + std::size_t(nc) * d->aux_dim);
    x.cscale.assign(d->cscale, d->cscale + std::size_t(nc) * d->aux_dim);
    x.lsz.resize(nc); x.rsz.resize(nc); x.nb.resize(nc);
    for (uint32_t ci = 0; ci < nc; ++ci) {
        if (x.cbra[ci] >= x.bra.size() || x.cket[ci] >= x.ket.size())
            return qcm::fail(QCM_ERR_ARG, "qcm_boundary_upload: cohort sector out of range");
        x.lsz[ci] = uint32_t(x.bra[x.cbra[ci]].second);
        x.rsz[ci] = uint32_t(x.ket[x.cket[ci]].second);
        if (d->n_blocks) x.nb[ci] = d->n_blocks[ci];
        else {
            uint32_t n = 0;
            for (uint32_t k = 0; k < d->aux_dim; ++k) n += x.offsets[std::size_t(ci) * d->aux_dim + k] > -1;
            x.nb[ci] = x.tr[ci] ? 0 : n;
        }
    }
    x.finish();
    if (!ctx) {
        *out = b.release();
        return QCM_OK;
    }
    b->b.data.alloc(x.total ? x.total : 1);
    QCM_CUDA(cudaMemsetAsync(b->b.data.get(), 0, (x.total ? x.total : 1) * sizeof(double), ctx->stream));
    if (d->data) {
        for (uint32_t ci = 0; ci < nc; ++ci) {
            uint64_t n = x.cohort_size(ci);
            if (n)
                QCM_CUDA(cudaMemcpyAsync(b->b.data.get() + x.data_off[ci], d->data + d->data_offset[ci], n * sizeof(double),
                                         cudaMemcpyHostToDevice, ctx->stream));
        }
    }
    QCM_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = b.release();
    return QCM_OK;
    QCM_CATCH
}
}  // namespace

extern "C" {

int qcm_boundary_upload(qcm_ctx* ctx, const qcm_boundary_desc* d, qcm_boundary** out) {
    if (!ctx) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_upload: ctx is NULL");
    return boundary_make(ctx, d, out);
}

int qcm_boundary_index_create(const qcm_boundary_desc* d, qcm_boundary** out) { return boundary_make(nullptr, d, out); }

void qcm_boundary_free(qcm_boundary* b) { delete b; }

int qcm_heff_plan_create(qcm_ctx* ctx, const qcm_boundary* L, const qcm_boundary* R, const qcm_mpo* ts_mpo, int site,
                         const qcm_mps_desc* twin, int flags, qcm_heff** out) {
    QCM_TRY
    const bool host_only = (flags & QCM_PLAN_HOST_ONLY) != 0;
    if ((!ctx && !host_only) || !L || !R || !ts_mpo || !twin || !out)
        return qcm::fail(QCM_ERR_ARG, "qcm_heff_plan_create: NULL argument");
    if (!host_only && (!L->ctx || !R->ctx)) return qcm::fail(QCM_ERR_ARG, "qcm_heff_plan_create: boundaries are not resident");
    const qcm::MPO& m = qcm::mpo_of(ts_mpo);
    if (!m.twosite) return qcm::fail(QCM_ERR_ARG, "qcm_heff_plan_create: expected a two-site MPO");
    if (site < 0 || std::size_t(site) >= m.t.size()) return qcm::fail(QCM_ERR_ARG, "qcm_heff_plan_create: site out of range");
    if (!host_only) QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(host_only ? nullptr : ctx->stream);
    auto h = std::make_unique<qcm_heff>();
    h->ctx = ctx;
    h->p = qcm::build_heff_plan(L->b, R->b, m.t[site], to_index(twin->n_phys, twin->phys), to_index(twin->n_left, twin->left),
                                to_index(twin->n_right, twin->right), (flags & QCM_PLAN_BOOKKEEPING) != 0);
    if (!host_only) {
        h->p->stream = ctx->stream;
        qcm::upload_plan(*h->p);
    }
    *out = h.release();
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_get_info(const qcm_heff* h, qcm_heff_info* info) {
    if (!h || !info) return qcm::fail(QCM_ERR_ARG, "qcm_heff_get_info: NULL argument");
    const qcm::HeffPlan& p = *h->p;
    info->vec_len = p.x_len;
    info->t_len = p.t_len;
    info->s_len = p.s_len;
    info->n_tjobs = p.tjobs.size();
    info->n_ttiles = 0;
    info->n_otiles = 0;
    info->n_kitems = 0;
    for (int sh = 0; sh < qcm::N_SHAPES; ++sh) {
        info->n_ttiles += p.ttiles[sh].size();
        info->n_otiles += p.otiles[sh].size();
        info->n_kitems += p.kitems[sh].size();
    }
    info->n_gtasks = p.units.size();
    info->n_alpha = p.n_alpha;
    info->n_segs = p.segs.size();
    info->n_outs = p.outs.size();
    info->launches = uint64_t(qcm::heff_launches_per_apply(p));
    info->w_len = p.w_len;
    info->flops_sexec = p.flops_sexec;
    info->flops = p.flops;
    info->flops_t = p.flops_t;
    info->flops_ls = p.flops_ls;
    info->flops_s = p.flops_s;
    info->g_elems = p.g_elems;
    info->g_reads = p.g_reads;
    info->flops_sdense = p.flops_sdense;
    info->l_len = p.L ? p.L->idx.total : 0;
    info->r_len = p.R ? p.R->idx.total : 0;
    info->p_len = p.p_len;
    return QCM_OK;
}

int qcm_heff_apply_device(qcm_heff* h, const double* x_dev, double* y_dev) {
    QCM_TRY
    if (!h || !x_dev || !y_dev) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device: host-only plan");
    qcm::heff_apply_device(*h->p, x_dev, y_dev);
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_stream_coefficients(qcm_heff* h, uint64_t max_bytes) {
    QCM_TRY
    if (!h) return qcm::fail(QCM_ERR_ARG, "qcm_heff_stream_coefficients: NULL argument");
    if (!h->ctx || !h->p->stream) return qcm::fail(QCM_ERR_ARG, "qcm_heff_stream_coefficients: a plan built for the host only");
    QCM_CUDA(cudaSetDevice(h->ctx->device));
    qcm::AllocStream scope(h->ctx->stream);
    qcm::HeffPlan& p = *h->p;
    qcm::release_plan_device(p);
    qcm::stream_coefficients(p, max_bytes / sizeof(double));
    p.stream = h->ctx->stream;
    qcm::upload_plan(p);
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_chunk_apply(qcm_heff* h, uint64_t max_bytes) {
    QCM_TRY
    if (!h) return qcm::fail(QCM_ERR_ARG, "qcm_heff_chunk_apply: NULL argument");
    if (!h->ctx || !h->p->stream) return qcm::fail(QCM_ERR_ARG, "qcm_heff_chunk_apply: a plan built for the host only");
    QCM_CUDA(cudaSetDevice(h->ctx->device));
    qcm::AllocStream scope(h->ctx->stream);
    qcm::HeffPlan& p = *h->p;
    qcm::release_plan_device(p);
    qcm::chunk_sectors(p, max_bytes / sizeof(double));
    p.stream = h->ctx->stream;
    qcm::upload_plan(p);
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_apply(qcm_heff* h, const double* x, double* y) {
    QCM_TRY
    if (!h || !x || !y) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply: host-only plan");
    qcm::HeffPlan& p = *h->p;
    qcm::AllocStream scope(p.stream);
    if (p.d_x.size() < p.x_len) { p.d_x.alloc(p.x_len); p.d_y.alloc(p.x_len); }
    QCM_CUDA(cudaMemcpyAsync(p.d_x.get(), x, p.x_len * sizeof(double), cudaMemcpyHostToDevice, p.stream));
    qcm::heff_apply_device(p, p.d_x.get(), p.d_y.get());
    QCM_CUDA(cudaMemcpyAsync(y, p.d_y.get(), p.x_len * sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    QCM_CUDA(cudaStreamSynchronize(p.stream));
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_bookkeeping(const qcm_heff* h, uint32_t* ints, double* alpha, uint64_t cap, uint64_t* n) {
    if (!h || !n) return qcm::fail(QCM_ERR_ARG, "qcm_heff_bookkeeping: NULL argument");
    const qcm::HeffPlan& p = *h->p;
    *n = p.bk_alpha.size();
    if (ints && alpha) {
        if (cap < *n) return qcm::fail(QCM_ERR_ARG, "qcm_heff_bookkeeping: buffer too small");
        std::memcpy(ints, p.bk_int.data(), p.bk_int.size() * sizeof(uint32_t));
        std::memcpy(alpha, p.bk_alpha.data(), p.bk_alpha.size() * sizeof(double));
    }
    return QCM_OK;
}

int qcm_heff_profile(qcm_heff* h, const double* x_dev, double* y_dev, float* ms) {
    QCM_TRY
    if (!h || !h->ctx || !x_dev || !y_dev || !ms) return qcm::fail(QCM_ERR_ARG, "qcm_heff_profile: bad argument");
    cudaEvent_t ev[4];
    for (auto& e : ev) QCM_CUDA(cudaEventCreate(&e));
    qcm::heff_apply_device(*h->p, x_dev, y_dev, ev);
    QCM_CUDA(cudaEventSynchronize(ev[3]));
    for (int i = 0; i < 3; ++i) QCM_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
    QCM_CUDA(cudaEventElapsedTime(&ms[3], ev[0], ev[3]));
    for (auto& e : ev) cudaEventDestroy(e);
    return QCM_OK;
    QCM_CATCH
}

namespace {
int check_mode(int precision, const char* who) {
    if (precision != QCM_PRECISION_FP64 && precision != QCM_PRECISION_MIXED && precision != QCM_PRECISION_MIXED_TC)
        return qcm::fail(QCM_ERR_ARG, std::string(who) + ": unknown precision mode");
    return QCM_OK;
}
void apply_mode(qcm::HeffPlan& p, const double* x, double* y, int precision, cudaEvent_t* ev = nullptr) {
    if (precision == QCM_PRECISION_FP64) qcm::heff_apply_device(p, x, y, ev);
    else qcm::heff_apply_device_mixed(p, x, y, ev, precision == QCM_PRECISION_MIXED_TC);
}
}  // namespace

int qcm_heff_apply_device_mode(qcm_heff* h, const double* x_dev, double* y_dev, int precision) {
    QCM_TRY
    if (!h || !x_dev || !y_dev) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_mode: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_mode: host-only plan");
    if (int rc = check_mode(precision, "qcm_heff_apply_device_mode")) return rc;
    apply_mode(*h->p, x_dev, y_dev, precision);
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_apply_mode(qcm_heff* h, const double* x, double* y, int precision) {
    QCM_TRY
    if (!h || !x || !y) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_mode: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_mode: host-only plan");
    if (int rc = check_mode(precision, "qcm_heff_apply_mode")) return rc;
    qcm::HeffPlan& p = *h->p;
    qcm::AllocStream scope(p.stream);
    if (p.d_x.size() < p.x_len) { p.d_x.alloc(p.x_len); p.d_y.alloc(p.x_len); }
    QCM_CUDA(cudaMemcpyAsync(p.d_x.get(), x, p.x_len * sizeof(double), cudaMemcpyHostToDevice, p.stream));
    apply_mode(p, p.d_x.get(), p.d_y.get(), precision);
    QCM_CUDA(cudaMemcpyAsync(y, p.d_y.get(), p.x_len * sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    QCM_CUDA(cudaStreamSynchronize(p.stream));
    if (precision != QCM_PRECISION_FP64) qcm::check_mixed(p);
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_adjoint_terms(const qcm_heff* h, uint64_t* n_terms) {
    if (!h || !h->p || !n_terms) return qcm::fail(QCM_ERR_ARG, "qcm_heff_adjoint_terms: NULL argument");
    *n_terms = qcm::heff_adjoint_terms(*h->p);
    return QCM_OK;
}

int qcm_heff_adjoint(qcm_heff* h, const double* x, const double* ybar, double* psi_bar, double* coeff_bar) {
    QCM_TRY
    if (!h || !ybar || (coeff_bar && !x)) return qcm::fail(QCM_ERR_ARG, "qcm_heff_adjoint: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_adjoint: host-only plan");
    qcm::HeffPlan& p = *h->p;
    qcm::AllocStream scope(p.stream);
    const uint64_t n = p.x_len, nt = qcm::heff_adjoint_terms(p);
    qcm::DBuf<double> dv(2 * n + 1), dpb(psi_bar ? n + 1 : 0), dcb(coeff_bar ? nt + 1 : 0);
    double* dx = dv.get();
    double* dyb = dv.get() + n;
    if (coeff_bar) QCM_CUDA(cudaMemcpyAsync(dx, x, n * sizeof(double), cudaMemcpyHostToDevice, p.stream));
    QCM_CUDA(cudaMemcpyAsync(dyb, ybar, n * sizeof(double), cudaMemcpyHostToDevice, p.stream));
    qcm::heff_adjoint_device(p, dx, dyb, psi_bar ? dpb.get() : nullptr, coeff_bar ? dcb.get() : nullptr);
    if (psi_bar) QCM_CUDA(cudaMemcpyAsync(psi_bar, dpb.get(), n * sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    if (coeff_bar && nt) QCM_CUDA(cudaMemcpyAsync(coeff_bar, dcb.get(), nt * sizeof(double), cudaMemcpyDeviceToHost, p.stream));
    QCM_CUDA(cudaStreamSynchronize(p.stream));
    return QCM_OK;
    QCM_CATCH
}

int qcm_heff_profile_mode(qcm_heff* h, const double* x_dev, double* y_dev, float* ms, int precision) {
    QCM_TRY
    if (!h || !h->ctx || !x_dev || !y_dev || !ms) return qcm::fail(QCM_ERR_ARG, "qcm_heff_profile_mode: bad argument");
    if (int rc = check_mode(precision, "qcm_heff_profile_mode")) return rc;
    cudaEvent_t ev[4];
    for (auto& e : ev) QCM_CUDA(cudaEventCreate(&e));
    apply_mode(*h->p, x_dev, y_dev, precision, ev);
    QCM_CUDA(cudaEventSynchronize(ev[3]));
    if (precision != QCM_PRECISION_FP64) qcm::check_mixed(*h->p);
    for (int i = 0; i < 3; ++i) QCM_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
    QCM_CUDA(cudaEventElapsedTime(&ms[3], ev[0], ev[3]));
    for (auto& e : ev) cudaEventDestroy(e);
    return QCM_OK;
    QCM_CATCH
}

void qcm_heff_free(qcm_heff* h) { delete h; }

}  // extern "C"
