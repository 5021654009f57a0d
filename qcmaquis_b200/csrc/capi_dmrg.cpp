#include <algorithm>
// C-ABI: Jacobi-Davidson solve, boundary steps, boundary download and the two-site sweep.
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/qcm_b200.h"
#include "capi_types.hpp"
#include "capi_util.hpp"
#include "dmrg_dev.hpp"

namespace qcm {
const MPO& mpo_of(const qcm_mpo* m);
}

struct qcm_dmrg {
    qcm_ctx* ctx = nullptr;
    std::unique_ptr<qcm::DevDMRG> e;
};

namespace {

qcm::Index to_index(uint32_t n, const qcm_sector* s) {
    qcm::Index r;
    for (uint32_t i = 0; i < n; ++i) r.d.push_back({qcm::Charge(s[i].a, s[i].b), s[i].size});
    for (std::size_t i = 1; i < r.d.size(); ++i)
        if (!(r.d[i - 1].first > r.d[i].first)) throw std::runtime_error("sector list must be in strictly descending charge order");
    return r;
}

// right-paired MPS tensor from packed host blocks (left-sector order, ls x stripe each)
qcm::DMPS upload_mps(qcm::Ctx& c, const qcm_mps_desc* d, const double* data) {
    qcm::DMPS t;
    t.phys = to_index(d->n_phys, d->phys);
    t.left = to_index(d->n_left, d->left);
    t.right = to_index(d->n_right, d->right);
    t.right_paired = true;
    t.b = qcm::layout_right_paired(t.phys, t.left, t.right);
    t.b.allocate(c.s, true);
    uint64_t h = 0;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        const uint64_t n = t.b.elems(k);
        QCM_CUDA(cudaMemcpyAsync(t.b.d.get() + t.b.off[k], data + h, n * sizeof(double), cudaMemcpyHostToDevice, c.s));
        h += n;
    }
    return t;
}

int boundary_step(qcm_ctx* ctx, const qcm_boundary* B, const qcm_mpo* mpo, int site, const qcm_mps_desc* mps,
                  const double* data_rp, int symmetric, bool left, qcm_boundary** out) {
    QCM_TRY
    if (!ctx || !B || !mpo || !mps || !data_rp || !out) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_step: NULL argument");
    if (!B->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_step: boundary is not resident");
    const qcm::MPO& m = qcm::mpo_of(mpo);
    if (m.twosite) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_step: expected a single-site MPO");
    if (site < 0 || std::size_t(site) >= m.t.size()) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_step: site out of range");
    const qcm::MPOTensor& W = m.t[site];
    if ((left ? W.rows : W.cols) != B->b.idx.aux)
        return qcm::fail(QCM_ERR_ARG, "qcm_boundary_step: MPO bond dimension does not match the boundary");
    QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx->stream);
    qcm::Ctx c;
    c.s = ctx->stream;
    qcm::DMPS ket = upload_mps(c, mps, data_rp);
    auto res = std::make_unique<qcm_boundary>();
    res->ctx = ctx;
    std::unique_ptr<qcm::DevBoundary> nb;
    if (left) {
        qcm::DMPS bra = qcm::right_paired_copy(c, ket);
        qcm::make_left_paired(c, bra);
        nb = qcm::boundary_step_left(c, B->b, ket, bra, W, symmetric != 0);
    } else {
        nb = qcm::boundary_step_right(c, B->b, ket, W, symmetric != 0);
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
    res->b.idx = std::move(nb->idx);
    res->b.data = std::move(nb->data);
    *out = res.release();
    return QCM_OK;
    QCM_CATCH
}

// "QSPB" v1 site-problem blob writer (the frozen-problem interchange format)
struct Blob {
    std::vector<uint8_t> b;
    template <class T> void put(T v) { const uint8_t* p = reinterpret_cast<const uint8_t*>(&v); b.insert(b.end(), p, p + sizeof(T)); }
    void idx(const qcm::Index& i) {
        put<uint32_t>(uint32_t(i.size()));
        for (auto& e : i.d) { put<int32_t>(e.first.a); put<int32_t>(e.first.b); put<uint32_t>(uint32_t(e.second)); }
    }
    void bnd(const qcm::DevBoundary& B, cudaStream_t s, bool with_data) {
        const qcm::BoundaryIndexH& x = B.idx;
        std::vector<double> h(with_data ? x.total : 0);
        if (with_data && x.total)
            QCM_CUDA(cudaMemcpyAsync(h.data(), B.data.get(), x.total * sizeof(double), cudaMemcpyDeviceToHost, s));
        QCM_CUDA(cudaStreamSynchronize(s));
        idx(x.bra); idx(x.ket);
        put<uint32_t>(x.n_cohorts()); put<uint32_t>(x.aux);
        for (uint32_t ci = 0; ci < x.n_cohorts(); ++ci) {
            put<uint32_t>(x.cbra[ci]); put<uint32_t>(x.cket[ci]); put<uint8_t>(x.tr[ci]);
            put<uint32_t>(x.lsz[ci]); put<uint32_t>(x.rsz[ci]); put<uint32_t>(x.nb[ci]);
            for (uint32_t b = 0; b < x.aux; ++b) put<int64_t>(x.offsets[std::size_t(ci) * x.aux + b]);
            for (uint32_t b = 0; b < x.aux; ++b) put<double>(x.cscale[std::size_t(ci) * x.aux + b]);
            const uint64_t n = with_data ? x.cohort_size(ci) : 0;
            put<uint64_t>(n);
            if (n) {
                const uint8_t* p = reinterpret_cast<const uint8_t*>(h.data() + x.data_off[ci]);
                b.insert(b.end(), p, p + n * sizeof(double));
            }
        }
    }
};

void fill_sectors(const qcm::Index& x, qcm_sector* out) {
    for (std::size_t i = 0; i < x.size(); ++i)
        out[i] = qcm_sector{x[i].first.a, x[i].first.b, uint32_t(x[i].second)};
}

}  // namespace

extern "C" {

int qcm_jd_solve(qcm_heff* h, const double* x0, double tol, int maxiter, double* out, double* eval, int* iters) {
    return qcm_jd_solve_mode(h, x0, tol, maxiter, QCM_PRECISION_FP64, out, eval, iters);
}

int qcm_jd_solve_mode(qcm_heff* h, const double* x0, double tol, int maxiter, int precision, double* out, double* eval,
                      int* iters) {
    QCM_TRY
    if (precision < QCM_PRECISION_FP64 || precision > QCM_PRECISION_MIXED_TC)
        return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_mode: unknown precision mode");
    if (!h || !x0 || !out || !eval) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve: host-only plan");
    if (maxiter < 1 || maxiter > 64) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve: maxiter must be in 1..64");
    qcm::HeffPlan& p = *h->p;
    qcm::AllocStream scope(p.stream);
    qcm::Ctx c;
    c.s = p.stream;
    qcm::DBuf<double> x(p.x_len ? p.x_len : 1);
    QCM_CUDA(cudaMemcpyAsync(x.get(), x0, p.x_len * sizeof(double), cudaMemcpyHostToDevice, c.s));
    int it = 0;
    *eval = qcm::jacobi_davidson(c, p, x.get(), tol, maxiter, it, precision);
    QCM_CUDA(cudaMemcpyAsync(out, x.get(), p.x_len * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
    if (iters) *iters = it;
    return QCM_OK;
    QCM_CATCH
}

int qcm_jd_solve_ex(qcm_heff* h, const double* x0, const double* const* ortho, int n_ortho, int gmres, double tol,
                    int maxiter, int precision, double* out, double* eval, int* iters, int* applies) {
    QCM_TRY
    if (precision < QCM_PRECISION_FP64 || precision > QCM_PRECISION_MIXED_TC)
        return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_ex: unknown precision mode");
    if (!h || !x0 || !out || !eval) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_ex: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_ex: host-only plan");
    if (maxiter < 1 || maxiter > 64) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_ex: maxiter must be in 1..64");
    if (gmres < 0 || gmres > qcm::JD_MAX_GMRES) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_ex: gmres must be in 0..64");
    if (n_ortho < 0 || (n_ortho > 0 && !ortho)) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_ex: bad ortho vectors");
    for (int i = 0; i < n_ortho; ++i)
        if (!ortho[i]) return qcm::fail(QCM_ERR_ARG, "qcm_jd_solve_ex: NULL ortho vector");
    qcm::HeffPlan& p = *h->p;
    qcm::AllocStream scope(p.stream);
    qcm::Ctx c;
    c.s = p.stream;
    const uint64_t n = p.x_len;
    qcm::DBuf<double> x(n ? n : 1);
    QCM_CUDA(cudaMemcpyAsync(x.get(), x0, n * sizeof(double), cudaMemcpyHostToDevice, c.s));
    qcm::DBuf<double> ov(n_ortho > 0 && n ? uint64_t(n_ortho) * n : 1);
    for (int i = 0; i < n_ortho; ++i)
        QCM_CUDA(cudaMemcpyAsync(ov.get() + uint64_t(i) * n, ortho[i], n * sizeof(double), cudaMemcpyHostToDevice, c.s));
    qcm::JDOptions o;
    o.gmres = gmres;
    o.ortho = ov.get();
    o.n_ortho = n_ortho;
    o.ortho_ld = n;
    int it = 0, na = 0;
    *eval = qcm::jacobi_davidson(c, p, x.get(), tol, maxiter, it, precision, &o, &na);
    QCM_CUDA(cudaMemcpyAsync(out, x.get(), n * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
    if (iters) *iters = it;
    if (applies) *applies = na;
    return QCM_OK;
    QCM_CATCH
}

int qcm_boundary_step_left(qcm_ctx* ctx, const qcm_boundary* L, const qcm_mpo* mpo, int site, const qcm_mps_desc* mps,
                           const double* data_rp, int symmetric, qcm_boundary** out) {
    return boundary_step(ctx, L, mpo, site, mps, data_rp, symmetric, true, out);
}

int qcm_boundary_step_right(qcm_ctx* ctx, const qcm_boundary* R, const qcm_mpo* mpo, int site, const qcm_mps_desc* mps,
                            const double* data_rp, int symmetric, qcm_boundary** out) {
    return boundary_step(ctx, R, mpo, site, mps, data_rp, symmetric, false, out);
}

int qcm_boundary_get_info(const qcm_boundary* b, qcm_boundary_info* info) {
    if (!b || !info) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_get_info: NULL argument");
    const qcm::BoundaryIndexH& x = b->b.idx;
    info->n_bra = uint32_t(x.bra.size());
    info->n_ket = uint32_t(x.ket.size());
    info->n_cohorts = x.n_cohorts();
    info->aux_dim = x.aux;
    info->total = x.total;
    info->resident = b->ctx ? 1 : 0;
    return QCM_OK;
}

int qcm_boundary_download(const qcm_boundary* b, qcm_sector* bra, qcm_sector* ket, uint32_t* cohort_bra,
                          uint32_t* cohort_ket, uint8_t* tr, uint32_t* n_blocks, int64_t* offsets, double* cscale,
                          uint64_t* data_offset, double* data) {
    QCM_TRY
    if (!b) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_download: NULL boundary");
    const qcm::BoundaryIndexH& x = b->b.idx;
    const std::size_t nc = x.n_cohorts(), na = std::size_t(nc) * x.aux;
    if (bra) fill_sectors(x.bra, bra);
    if (ket) fill_sectors(x.ket, ket);
    if (cohort_bra) std::memcpy(cohort_bra, x.cbra.data(), nc * sizeof(uint32_t));
    if (cohort_ket) std::memcpy(cohort_ket, x.cket.data(), nc * sizeof(uint32_t));
    if (tr) std::memcpy(tr, x.tr.data(), nc);
    if (n_blocks) std::memcpy(n_blocks, x.nb.data(), nc * sizeof(uint32_t));
    if (offsets) std::memcpy(offsets, x.offsets.data(), na * sizeof(int64_t));
    if (cscale) std::memcpy(cscale, x.cscale.data(), na * sizeof(double));
    if (data_offset) std::memcpy(data_offset, x.data_off.data(), nc * sizeof(uint64_t));
    if (data) {
        if (!b->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_boundary_download: boundary is not resident");
        QCM_CUDA(cudaSetDevice(b->ctx->device));
        qcm::AllocStream scope(b->ctx->stream);
        if (x.total)
            QCM_CUDA(cudaMemcpyAsync(data, b->b.data.get(), x.total * sizeof(double), cudaMemcpyDeviceToHost, b->ctx->stream));
        QCM_CUDA(cudaStreamSynchronize(b->ctx->stream));
    }
    return QCM_OK;
    QCM_CATCH
}

namespace {
// qcm_dmrg_params -> DMRGParams; returns an error message for values outside their ranges
const char* to_params(const qcm_dmrg_params& prm, qcm::DMRGParams& p) {
    if (prm.hpsi_precision < QCM_PRECISION_FP64 || prm.hpsi_precision > QCM_PRECISION_MIXED_TC)
        return "qcm_dmrg: unknown hpsi_precision";
    if (prm.optimization != QCM_OPTIMIZATION_TWOSITE && prm.optimization != QCM_OPTIMIZATION_SINGLESITE)
        return "qcm_dmrg: optimization must be QCM_OPTIMIZATION_TWOSITE or QCM_OPTIMIZATION_SINGLESITE";
    p.Mmax = prm.max_bond_dimension;
    p.init_bond_dimension = prm.init_bond_dimension;
    p.cutoff = prm.truncation_cutoff;
    p.jcd_tol = prm.jcd_tol;
    p.jcd_maxiter = prm.jcd_maxiter;
    p.jcd_gmres = prm.jcd_gmres;
    p.ecore = prm.ecore;
    p.heev = prm.twosite_truncation == 1;
    p.alpha_initial = prm.alpha_initial;
    p.alpha_main = prm.alpha_main;
    p.alpha_final = prm.alpha_final;
    p.ngrowsweeps = prm.ngrowsweeps;
    p.nmainsweeps = prm.nmainsweeps;
    p.precision = prm.hpsi_precision;
    p.single_site = prm.optimization == QCM_OPTIMIZATION_SINGLESITE;
    if (prm.mixed_fp64_refine < 0 || prm.mixed_fp64_refine > 64) return "qcm_dmrg: mixed_fp64_refine must be in 0..64";
    p.mixed_floor = prm.mixed_residual_floor > 0 ? prm.mixed_residual_floor : 0.0;
    p.mixed_refine = prm.mixed_fp64_refine;
    return nullptr;
}
}  // namespace

int qcm_dmrg_create(qcm_ctx* ctx, const qcm_mpo* mpo, int nup, int ndown, const qcm_dmrg_params* prm, qcm_dmrg** out) {
    QCM_TRY
    if (!ctx || !mpo || !prm || !out) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create: NULL argument");
    const qcm::MPO& m = qcm::mpo_of(mpo);
    if (m.twosite) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create: expected a single-site MPO");
    if (prm->jcd_maxiter < 1 || prm->jcd_maxiter > 64) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create: jcd_maxiter must be in 1..64");
    if (prm->jcd_gmres < 0 || prm->jcd_gmres > qcm::JD_MAX_GMRES)
        return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create: jcd_gmres must be in 0..64");
    if (prm->twosite_truncation != 0 && prm->twosite_truncation != 1)
        return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create: twosite_truncation must be 0 (svd) or 1 (heev)");
    if (prm->max_bond_dimension < 1 || prm->init_bond_dimension < 1)
        return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create: bond dimensions must be positive");
    QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx->stream);
    qcm::DMRGParams p;
    if (const char* err = to_params(*prm, p)) return qcm::fail(QCM_ERR_ARG, err);
    qcm::MPO ts = qcm::make_twosite_mpo(m);
    auto d = std::make_unique<qcm_dmrg>();
    d->ctx = ctx;
    d->e = std::make_unique<qcm::DevDMRG>(m.t, ts.t, nup, ndown, p, ctx->stream);
    *out = d.release();
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_create_from_mps(qcm_ctx* ctx, const qcm_mpo* mpo, const qcm_dmrg_params* prm, const qcm_mps_desc* sites,
                             const double* const* data, qcm_dmrg** out) {
    return qcm_dmrg_create_from_mps_at(ctx, mpo, prm, sites, data, 0, out);
}

int qcm_dmrg_create_from_mps_at(qcm_ctx* ctx, const qcm_mpo* mpo, const qcm_dmrg_params* prm, const qcm_mps_desc* sites,
                                const double* const* data, int initial_site, qcm_dmrg** out) {
    QCM_TRY
    if (!ctx || !mpo || !prm || !sites || !data || !out) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create_from_mps: NULL argument");
    const qcm::MPO& m = qcm::mpo_of(mpo);
    if (m.twosite) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create_from_mps: expected a single-site MPO");
    if (prm->jcd_maxiter < 1 || prm->jcd_maxiter > 64) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create_from_mps: jcd_maxiter must be in 1..64");
    if (prm->jcd_gmres < 0 || prm->jcd_gmres > qcm::JD_MAX_GMRES)
        return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create_from_mps: jcd_gmres must be in 0..64");
    QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx->stream);
    qcm::DMRGParams p;
    if (const char* err = to_params(*prm, p)) return qcm::fail(QCM_ERR_ARG, err);
    qcm::Ctx tmp;
    tmp.s = ctx->stream;
    std::vector<qcm::DMPS> ms;
    for (std::size_t i = 0; i < m.t.size(); ++i) {
        if (!data[i]) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_create_from_mps: NULL site data");
        ms.push_back(upload_mps(tmp, &sites[i], data[i]));
    }
    qcm::MPO ts = qcm::make_twosite_mpo(m);
    auto d = std::make_unique<qcm_dmrg>();
    d->ctx = ctx;
    d->e = std::make_unique<qcm::DevDMRG>(m.t, ts.t, std::move(ms), p, ctx->stream, initial_site);
    *out = d.release();
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_measure_1rdm(qcm_dmrg* d, double* gamma) {
    QCM_TRY
    if (!d || !gamma) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_measure_1rdm: NULL argument");
    qcm::DevDMRG& e = *d->e;
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    const int L = e.L;
    std::vector<double> h(std::size_t(L) * L, 0.0), V(std::size_t(L) * L * L * L, 0.0);
    for (int i = 0; i < L; ++i)
        for (int j = i; j < L; ++j) {
            // the one-body operator sum_s (a+_is a_js + a+_js a_is) as the QC MPO of h = e_ij + e_ji, V = 0
            std::fill(h.begin(), h.end(), 0.0);
            h[std::size_t(i) + std::size_t(j) * L] = 1.0;
            h[std::size_t(j) + std::size_t(i) * L] = 1.0;
            const qcm::MPO O = qcm::build_qc_mpo(L, h.data(), V.data(), 1e-20);
            const double x = e.expectation(O.t);
            const double g = i == j ? x : 0.5 * x;
            gamma[std::size_t(i) + std::size_t(j) * L] = g;
            gamma[std::size_t(j) + std::size_t(i) * L] = g;
        }
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_mpo_gradient(qcm_dmrg* d, const qcm_mpo* W, double* const* grad) {
    QCM_TRY
    if (!d || !W || !grad) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_mpo_gradient: NULL argument");
    const qcm::MPO& m = qcm::mpo_of(W);
    qcm::DevDMRG& e = *d->e;
    if (m.twosite || int(m.t.size()) != e.L)
        return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_mpo_gradient: expected a single-site MPO of the state's length");
    for (int k = 0; k < e.L; ++k)
        if (!grad[k] && !m.t[std::size_t(k)].b1.empty()) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_mpo_gradient: NULL gradient buffer");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    const auto g = e.mpo_gradient(m.t);
    for (int k = 0; k < e.L; ++k)
        if (!g[std::size_t(k)].empty()) std::memcpy(grad[k], g[std::size_t(k)].data(), g[std::size_t(k)].size() * sizeof(double));
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_integral_gradient(qcm_dmrg* d, const double* h, const double* V, double* dh, double* dV) {
    QCM_TRY
    if (!d || !h || !V || !dh) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_integral_gradient: NULL argument");
    qcm::DevDMRG& e = *d->e;
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    const int L = e.L;
    const uint64_t L2 = uint64_t(L) * L, n = L2 + L2 * L2;
    qcm::IntegralProvenance prov;
    const qcm::MPO W = qcm::build_qc_mpo(L, h, V, 0.0, &prov);
    const auto g = e.mpo_gradient(W.t);
    std::vector<double> dx(n, 0.0);
    qcm::integral_gradient(prov, g, dx.data(), n);
    std::memcpy(dh, dx.data(), L2 * sizeof(double));
    if (dV) std::memcpy(dV, dx.data() + L2, L2 * L2 * sizeof(double));
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_measure_2rdm_grad(qcm_dmrg* d, double* G) {
    QCM_TRY
    if (!d || !G) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_measure_2rdm_grad: NULL argument");
    qcm::DevDMRG& e = *d->e;
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    const int L = e.L;
    const std::size_t L2 = std::size_t(L) * L;
    auto at = [&](int p, int q, int r, int t) { return std::size_t(p) + std::size_t(q) * L + std::size_t(r) * L2 + std::size_t(t) * L2 * L; };
    std::vector<double> h(L2, 0.0), V(L2 * L2, 0.0);
    // one orbit of index quadruples per unique integral (pq|rs), p >= q, r >= s, (p,q) >= (r,s)
    for (int p = 0; p < L; ++p)
        for (int q = 0; q <= p; ++q)
            for (int r = 0; r <= p; ++r)
                for (int t = 0; t <= r; ++t) {
                    if (r == p && t > q) continue;
                    const int orb[8][4] = {{p, q, r, t}, {q, p, r, t}, {p, q, t, r}, {q, p, t, r},
                                           {r, t, p, q}, {t, r, p, q}, {r, t, q, p}, {t, r, q, p}};
                    std::vector<std::size_t> pos;
                    for (const auto& o : orb) {
                        const std::size_t k = at(o[0], o[1], o[2], o[3]);
                        if (std::find(pos.begin(), pos.end(), k) == pos.end()) pos.push_back(k);
                    }
                    std::fill(V.begin(), V.end(), 0.0);
                    for (std::size_t k : pos) V[k] = 1.0;
                    const qcm::MPO O = qcm::build_qc_mpo(L, h.data(), V.data(), 1e-20);
                    const double x = e.expectation(O.t) / double(pos.size());
                    for (std::size_t k : pos) G[k] = x;
                }
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_export_site(qcm_dmrg* d, int site, void* buf, size_t cap, size_t* len) {
    QCM_TRY
    if (!d || !len) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_export_site: NULL argument");
    qcm::DevDMRG& e = *d->e;
    if (site < 0 || site >= e.L) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_export_site: site out of range");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    const qcm::DMPS t = qcm::right_paired_copy(e.c, e.mps[std::size_t(site)]);
    std::vector<double> h(t.b.total);
    if (t.b.total)
        QCM_CUDA(cudaMemcpyAsync(h.data(), t.b.d.get(), t.b.total * sizeof(double), cudaMemcpyDeviceToHost, e.c.s));
    QCM_CUDA(cudaStreamSynchronize(e.c.s));
    std::vector<uint8_t> w;
    auto put = [&](const void* p, std::size_t n) { const uint8_t* b = static_cast<const uint8_t*>(p); w.insert(w.end(), b, b + n); };
    auto u32 = [&](uint32_t v) { put(&v, 4); };
    auto i32 = [&](int32_t v) { put(&v, 4); };
    auto idx = [&](const qcm::Index& i) {
        u32(uint32_t(i.size()));
        for (auto& x : i.d) { i32(x.first.a); i32(x.first.b); u32(uint32_t(x.second)); }
    };
    u32(0x53504D51u);  // "QMPS"
    u32(1);
    idx(t.phys); idx(t.left); idx(t.right);
    u32(uint32_t(t.b.n()));
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        i32(t.b.lc[k].a); i32(t.b.lc[k].b); u32(t.b.rows[k]); u32(t.b.cols[k]);
        put(h.data() + t.b.off[k], t.b.elems(k) * sizeof(double));
    }
    *len = w.size();
    if (buf) {
        if (cap < w.size()) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_export_site: buffer too small");
        std::memcpy(buf, w.data(), w.size());
    }
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_set_ortho(qcm_dmrg* d, int n_states, const qcm_mps_desc* sites, const double* const* data) {
    QCM_TRY
    if (!d || n_states < 0 || (n_states > 0 && (!sites || !data))) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_set_ortho: bad arguments");
    qcm::DevDMRG& e = *d->e;
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    std::vector<std::vector<qcm::DMPS>> st(static_cast<std::size_t>(n_states));
    for (int o = 0; o < n_states; ++o)
        for (int i = 0; i < e.L; ++i) {
            const std::size_t k = std::size_t(o) * e.L + i;
            if (!data[k]) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_set_ortho: NULL site data");
            st[o].push_back(upload_mps(e.c, &sites[k], data[k]));
        }
    e.set_ortho(std::move(st));
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_length(const qcm_dmrg* d) { return d ? d->e->L : -1; }

int qcm_dmrg_steps_per_sweep(const qcm_dmrg* d) { return d ? d->e->steps_per_sweep() : -1; }

int qcm_dmrg_run(qcm_dmrg* d, int stop_step, double* energies, qcm_trunc_result* trunc, int* n_steps) {
    QCM_TRY
    if (!d) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_run: NULL argument");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    std::vector<double> E;
    std::vector<qcm::TruncResults> T;
    d->e->run_until(stop_step, E, T);
    if (energies) std::memcpy(energies, E.data(), E.size() * sizeof(double));
    if (trunc)
        for (std::size_t i = 0; i < T.size(); ++i)
            trunc[i] = qcm_trunc_result{T[i].bond_dimension, T[i].truncated_weight, T[i].truncated_fraction, T[i].smallest_ev};
    if (n_steps) *n_steps = int(E.size());
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_next_step(const qcm_dmrg* d) { return d ? d->e->next_step : -1; }

int qcm_dmrg_pending_plan(qcm_dmrg* d, double* twin, uint64_t cap, qcm_heff** out) {
    QCM_TRY
    if (!d || !out) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_pending_plan: NULL argument");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    std::vector<double> x;
    auto h = std::make_unique<qcm_heff>();
    h->ctx = d->ctx;
    h->p = d->e->pending_plan(twin ? &x : nullptr, nullptr, nullptr, nullptr);
    h->p->stream = d->ctx->stream;
    qcm::upload_plan(*h->p);
    if (twin) {
        if (cap < x.size()) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_pending_plan: twin buffer too small");
        std::memcpy(twin, x.data(), x.size() * sizeof(double));
    }
    *out = h.release();
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_pending_twin(qcm_dmrg* d, double* twin, uint64_t cap, uint64_t* n) {
    QCM_TRY
    if (!d || !n) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_pending_twin: NULL argument");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    std::vector<double> x;
    d->e->pending_twin(x);
    *n = x.size();
    if (twin) {
        if (cap < x.size()) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_pending_twin: buffer too small");
        std::memcpy(twin, x.data(), x.size() * sizeof(double));
    }
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_pending_export(qcm_dmrg* d, int flags, void* buf, size_t cap, size_t* len) {
    QCM_TRY
    if (!d || !len) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_pending_export: NULL argument");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    qcm::DevDMRG& e = *d->e;
    std::vector<double> x;
    qcm::Index phys, left, right;
    auto plan = e.pending_plan(&x, &phys, &left, &right);
    int lr, site1, site2;
    e.step_sites(e.next_step, lr, site1, site2);
    Blob w;
    w.put<uint32_t>(0x42505351u);  // "QSPB"
    w.put<uint32_t>(1);
    w.idx(phys); w.idx(left); w.idx(right);
    const bool data = (flags & QCM_EXPORT_INDEX_ONLY) == 0;
    w.put<uint32_t>(uint32_t(left.size()));
    for (std::size_t lb = 0; lb < left.size(); ++lb) {
        w.put<int32_t>(left[lb].first.a); w.put<int32_t>(left[lb].first.b);
        w.put<uint32_t>(uint32_t(left[lb].second)); w.put<uint32_t>(data ? plan->x_cols[lb] : 0);
        if (!data) continue;
        const uint8_t* p = reinterpret_cast<const uint8_t*>(x.data() + plan->x_off[lb]);
        w.b.insert(w.b.end(), p, p + uint64_t(left[lb].second) * plan->x_cols[lb] * sizeof(double));
    }
    w.bnd(*e.left_[site1], e.c.s, data);
    w.bnd(*e.right_[site2 + 1], e.c.s, data);
    *len = w.b.size();
    if (buf) {
        if (cap < w.b.size()) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_pending_export: buffer too small");
        std::memcpy(buf, w.b.data(), w.b.size());
    }
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_sweep(qcm_dmrg* d, double* energies, qcm_trunc_result* trunc) {
    QCM_TRY
    if (!d || !energies) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_sweep: NULL argument");
    if (d->e->next_step != 0) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_sweep: a sweep is in progress (finish it with qcm_dmrg_run)");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    std::vector<double> E;
    std::vector<qcm::TruncResults> T;
    d->e->sweep(E, T);
    std::memcpy(energies, E.data(), E.size() * sizeof(double));
    if (trunc)
        for (std::size_t i = 0; i < T.size(); ++i)
            trunc[i] = qcm_trunc_result{T[i].bond_dimension, T[i].truncated_weight, T[i].truncated_fraction, T[i].smallest_ev};
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_group_sweep(qcm_dmrg* const* runs, int n, double* energies, qcm_trunc_result* trunc) {
    QCM_TRY
    if (!runs || n <= 0 || !energies) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_group_sweep: NULL argument");
    std::vector<qcm::DevDMRG*> e(n);
    for (int i = 0; i < n; ++i) {
        if (!runs[i]) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_group_sweep: NULL run");
        if (runs[i]->ctx != runs[0]->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_group_sweep: the runs use different contexts");
        for (int j = 0; j < i; ++j)
            if (runs[j] == runs[i]) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_group_sweep: a run appears twice");
        e[i] = runs[i]->e.get();
    }
    QCM_CUDA(cudaSetDevice(runs[0]->ctx->device));
    qcm::AllocStream scope(runs[0]->ctx->stream);
    std::vector<std::vector<double>> E;
    std::vector<std::vector<qcm::TruncResults>> T;
    qcm::dmrg_group_sweep(e, E, T);
    const std::size_t steps = E[0].size();
    for (int i = 0; i < n; ++i) {
        std::memcpy(energies + i * steps, E[i].data(), steps * sizeof(double));
        if (trunc)
            for (std::size_t k = 0; k < steps; ++k) {
                const qcm::TruncResults& t = T[i][k];
                trunc[i * steps + k] = qcm_trunc_result{t.bond_dimension, t.truncated_weight, t.truncated_fraction, t.smallest_ev};
            }
    }
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_get_stats(const qcm_dmrg* d, qcm_dmrg_stats* s) {
    if (!d || !s) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_get_stats: NULL argument");
    const qcm::DMRGStats& t = d->e->st;
    s->hpsi_count = t.hpsi_count;
    s->hpsi_flops = t.hpsi_flops;
    s->hpsi_count_fp64 = t.hpsi_count64;
    s->hpsi_flops_fp64 = t.hpsi_flops64;
    s->plan_s = t.plan_s;
    s->jd_s = t.jd_s;
    s->trunc_s = t.trunc_s;
    s->boundary_s = t.boundary_s;
    s->total_s = t.total_s;
    s->plans_built = t.plans_built;
    s->plans_reused = t.plans_reused;
    s->bsteps_built = t.bsteps_built;
    s->bsteps_reused = t.bsteps_reused;
    s->boundary_bytes_peak = t.boundary_bytes_peak;
    s->boundaries_offloaded = t.boundaries_offloaded;
    s->boundaries_fetched = t.boundaries_fetched;
    return QCM_OK;
}

int qcm_dmrg_set_coefficient_budget(qcm_dmrg* d, uint64_t max_bytes) {
    if (!d) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_set_coefficient_budget: NULL argument");
    if (max_bytes && d->e->p.precision != 0)
        return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_set_coefficient_budget: streamed coefficient blocks are for FP64 runs");
    d->e->coefficient_budget = max_bytes / sizeof(double);
    return QCM_OK;
}

int qcm_dmrg_set_apply_budget(qcm_dmrg* d, uint64_t max_bytes) {
    if (!d) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_set_apply_budget: NULL argument");
    if (max_bytes && d->e->p.precision != 0)
        return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_set_apply_budget: chunked applies are for FP64 runs");
    d->e->apply_budget = max_bytes / sizeof(double);
    return QCM_OK;
}

int qcm_dmrg_set_boundary_budget(qcm_dmrg* d, uint64_t bytes) {
    QCM_TRY
    if (!d) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_set_boundary_budget: NULL argument");
    QCM_CUDA(cudaSetDevice(d->ctx->device));
    qcm::AllocStream scope(d->ctx->stream);
    d->e->boundary_budget = bytes;
    d->e->st.boundary_bytes_peak = 0;  // the peak counts from here
    d->e->bnd_trim(d->e->next_step);
    QCM_CUDA(cudaStreamSynchronize(d->ctx->stream));
    return QCM_OK;
    QCM_CATCH
}

int qcm_dmrg_bond_dimensions(const qcm_dmrg* d, uint64_t* dims) {
    if (!d || !dims) return qcm::fail(QCM_ERR_ARG, "qcm_dmrg_bond_dimensions: NULL argument");
    const qcm::DevDMRG& e = *d->e;
    for (int i = 0; i + 1 < e.L; ++i) dims[i] = e.mps[i].right.sum_of_sizes();
    return QCM_OK;
}

void qcm_dmrg_free(qcm_dmrg* d) { delete d; }

}  // extern "C"
