// C-ABI: block-matrix truncation on the device (svd_truncate and heev_truncate of
// block_matrix_algorithms.h:185-240, 299-355).
#include <algorithm>
#include <memory>
#include <vector>

#include "../../include/qcm_b200.h"
#include "capi_types.hpp"
#include "capi_util.hpp"
#include "dmrg_dev.hpp"

namespace {

void to_result(const qcm::TruncResults& t, qcm_trunc_result* r) {
    if (!r) return;
    r->bond_dimension = t.bond_dimension;
    r->truncated_weight = t.truncated_weight;
    r->truncated_fraction = t.truncated_fraction;
    r->smallest_ev = t.smallest_ev;
}

// device block list (32-element aligned blocks) with the host blocks, concatenated column-major
qcm::DBlocks upload_blocks(qcm::Ctx& c, uint32_t n, const uint32_t* rows, const uint32_t* cols, const double* data) {
    qcm::DBlocks b;
    for (uint32_t k = 0; k < n; ++k) b.add(qcm::Charge(int(k), 0), qcm::Charge(int(k), 0), rows[k], cols[k]);
    b.allocate(c.s, true);
    uint64_t h = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const uint64_t e = uint64_t(rows[k]) * cols[k];
        if (e) QCM_CUDA(cudaMemcpyAsync(b.d.get() + b.off[k], data + h, e * sizeof(double), cudaMemcpyHostToDevice, c.s));
        h += e;
    }
    return b;
}

void download(qcm::Ctx& c, const double* d, double* h, uint64_t n) {
    if (n) QCM_CUDA(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, c.s));
}

}  // namespace

int qcm_truncate_svd(qcm_ctx* ctx, uint32_t n_blocks, const uint32_t* rows, const uint32_t* cols, const double* blocks,
                     uint64_t max_bond_dimension, double cutoff, uint32_t* keep, double* U, double* S, double* Vt,
                     qcm_trunc_result* result) {
    QCM_TRY
    if (!ctx || (n_blocks && (!rows || !cols || !blocks || !keep || !U || !S || !Vt)))
        return qcm::fail(QCM_ERR_ARG, "qcm_truncate_svd: NULL argument");
    if (n_blocks == 0) return qcm::fail(QCM_ERR_ARG, "qcm_truncate_svd: no blocks");
    QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx->stream);
    qcm::Ctx c;
    c.s = ctx->stream;
    c.device = ctx->device;
    qcm::DBlocks M = upload_blocks(c, n_blocks, rows, cols, blocks);  // the solver is made only if needed
    qcm::BlockSVD sv = qcm::svd_truncate(c, M, max_bond_dimension, cutoff);
    // U_k (rows x keep, ld rows), S_k (keep), Vt_k (keep x cols, ld keep) packed in block order
    std::vector<double> v;
    uint64_t pu = 0, ps = 0, pv = 0;
    for (uint32_t k = 0; k < n_blocks; ++k) {
        const uint32_t kp = sv.keep[k], m = rows[k], n = cols[k];
        keep[k] = kp;
        download(c, sv.U.get() + sv.uo[k], U + pu, uint64_t(m) * kp);
        std::copy(sv.vals[k].begin(), sv.vals[k].begin() + kp, S + ps);
        v.resize(uint64_t(n) * kp);
        download(c, sv.V.get() + sv.vo[k], v.data(), v.size());
        QCM_CUDA(cudaStreamSynchronize(c.s));
        for (uint32_t j = 0; j < kp; ++j)
            for (uint32_t i = 0; i < n; ++i) Vt[pv + j + uint64_t(i) * kp] = v[i + uint64_t(j) * n];
        pu += uint64_t(m) * kp; ps += kp; pv += uint64_t(kp) * n;
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
    to_result(sv.tr, result);
    return QCM_OK;
    QCM_CATCH
}

int qcm_truncate_heev(qcm_ctx* ctx, uint32_t n_blocks, const uint32_t* dims, const double* blocks, uint64_t max_bond_dimension,
                      double cutoff, uint32_t* keep, double* U, double* evals, qcm_trunc_result* result) {
    QCM_TRY
    if (!ctx || (n_blocks && (!dims || !blocks || !keep || !U || !evals)))
        return qcm::fail(QCM_ERR_ARG, "qcm_truncate_heev: NULL argument");
    if (n_blocks == 0) return qcm::fail(QCM_ERR_ARG, "qcm_truncate_heev: no blocks");
    QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx->stream);
    qcm::Ctx c;
    c.s = ctx->stream;
    c.device = ctx->device;
    qcm::DBlocks dm = upload_blocks(c, n_blocks, dims, dims, blocks);
    qcm::BlockHeev hv = qcm::heev_truncate(c, dm, max_bond_dimension, cutoff);
    // U_k = the kept eigenvectors in descending eigenvalue order (dim x keep, ld dim)
    std::vector<double> ev;
    uint64_t pu = 0, pe = 0;
    for (uint32_t k = 0; k < n_blocks; ++k) {
        const uint32_t kp = hv.keep[k], n = dims[k];
        keep[k] = kp;
        ev.resize(uint64_t(n) * n);
        download(c, dm.d.get() + dm.off[k], ev.data(), ev.size());
        QCM_CUDA(cudaStreamSynchronize(c.s));
        for (uint32_t j = 0; j < kp; ++j)
            std::copy(ev.begin() + uint64_t(n - 1 - j) * n, ev.begin() + uint64_t(n - j) * n, U + pu + uint64_t(j) * n);
        std::copy(hv.evals[k].begin(), hv.evals[k].begin() + kp, evals + pe);
        pu += uint64_t(n) * kp; pe += kp;
    }
    to_result(hv.tr, result);
    return QCM_OK;
    QCM_CATCH
}

extern "C" int qcm_qr_blocks(qcm_ctx* ctx, uint32_t n_blocks, const uint32_t* rows, const uint32_t* cols,
                             const double* blocks, int lq, double* Q, double* R) {
    QCM_TRY
    if (!ctx || !n_blocks || !rows || !cols || !blocks || !Q || !R) return qcm::fail(QCM_ERR_ARG, "qcm_qr_blocks: NULL argument");
    QCM_CUDA(cudaSetDevice(ctx->device));
    qcm::AllocStream scope(ctx->stream);
    qcm::Ctx c;
    c.s = ctx->stream;
    c.device = ctx->device;
    qcm::DBlocks M = upload_blocks(c, n_blocks, rows, cols, blocks);
    // outputs packed like the inputs: per block Q (m x k or k x n) then R / L, k = min(m, n)
    std::vector<uint64_t> qo(n_blocks), ro(n_blocks);
    uint64_t ql = 0, rl = 0, wl = 0;
    std::vector<qcm::QrJob> jobs;
    for (uint32_t k = 0; k < n_blocks; ++k) {
        const uint64_t m = rows[k], n = cols[k], kk = std::min(m, n);
        qo[k] = ql; ro[k] = rl;
        ql += kk * (lq ? n : m);
        rl += kk * (lq ? m : n);
        if (!m || !n) continue;
        jobs.push_back(qcm::QrJob{M.off[k], qo[k], ro[k], wl, uint32_t(m), uint32_t(n), uint32_t(lq != 0), 0});
        wl += (qcm::qr_scratch(uint32_t(m), uint32_t(n), lq != 0) + 31) / 32 * 32;
    }
    qcm::DBuf<double> dq(std::max<uint64_t>(ql, 1)), dr(std::max<uint64_t>(rl, 1)), dw(std::max<uint64_t>(wl, 1));
    qcm::batched_qr(jobs, M.d.get(), M.total, dq.get(), ql, dr.get(), rl, dw.get(), wl ? wl : 1, c.qjobs, c.s);
    download(c, dq.get(), Q, ql);
    download(c, dr.get(), R, rl);
    QCM_CUDA(cudaStreamSynchronize(c.s));
    return QCM_OK;
    QCM_CATCH
}
