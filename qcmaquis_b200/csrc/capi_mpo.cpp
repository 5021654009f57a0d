// C-ABI: MPO construction (input prep for the two-site H_eff path).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qcm_b200.h"
#include "capi_util.hpp"
#include "mpo.hpp"

struct qcm_mpo {
    qcm::MPO m;
    std::vector<char> unset;  // tensors qcm_mpo_create left for qcm_mpo_set_tensor
    std::shared_ptr<qcm::IntegralProvenance> prov;  // qcm_mpo_build_qc_tracked
};

namespace {

// an MPO handed in tensor by tensor is complete and its bonds agree on both sides
void check_complete(const qcm_mpo* p) {
    for (std::size_t i = 0; i < p->unset.size(); ++i)
        if (p->unset[i]) throw std::runtime_error("MPO tensor " + std::to_string(i) + " was never set (qcm_mpo_set_tensor)");
    // tensor i's right bond is the left bond of tensor i + 1 (i + 2 for two-site tensors)
    const auto& t = p->m.t;
    const std::size_t step = p->m.twosite ? 2 : 1;
    for (std::size_t i = 0; i + step < t.size(); ++i)
        if (t[i].cols != t[i + step].rows || t[i].herm_right != t[i + step].herm_left || t[i].phase_right != t[i + step].phase_left)
            throw std::runtime_error("MPO tensors " + std::to_string(i) + " and " + std::to_string(i + step) +
                                     " disagree on their shared bond (dimension or Hermitian pairs)");
}

void check_pairs(const int32_t* herm, const int32_t* phase, uint32_t n, const char* what) {
    if (!herm && !phase) return;
    if (!herm || !phase) throw std::runtime_error(std::string("qcm_mpo_set_tensor: ") + what + ": pairs and phases go together");
    for (uint32_t b = 0; b < n; ++b) {
        if (herm[b] < -1 || herm[b] >= int64_t(n)) throw std::runtime_error(std::string("qcm_mpo_set_tensor: ") + what + ": partner out of range");
        if (herm[b] >= 0 && herm[herm[b]] != int32_t(b)) throw std::runtime_error(std::string("qcm_mpo_set_tensor: ") + what + ": pairs are not symmetric");
        if (phase[b] != 1 && phase[b] != -1) throw std::runtime_error(std::string("qcm_mpo_set_tensor: ") + what + ": phase is not +-1");
    }
}

}  // namespace

extern "C" {

int qcm_mpo_build_qc(int L, const double* h, const double* V, double cutoff, qcm_mpo** out) {
    QCM_TRY
    if (!h || !V || !out || L < 2) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_build_qc: bad arguments");
    auto* p = new qcm_mpo;
    p->m = qcm::build_qc_mpo(L, h, V, cutoff);
    *out = p;
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_build_qc_tracked(int L, const double* h, const double* V, qcm_mpo** out) {
    QCM_TRY
    if (!h || !V || !out || L < 2) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_build_qc_tracked: bad arguments");
    auto p = std::make_unique<qcm_mpo>();
    p->prov = std::make_shared<qcm::IntegralProvenance>();
    p->m = qcm::build_qc_mpo(L, h, V, 0.0, p->prov.get());
    *out = p.release();
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_provenance(const qcm_mpo* m, int site, uint64_t* ptr, uint64_t* id, double* val, uint64_t cap, uint64_t* n) {
    QCM_TRY
    if (!m || !n) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_provenance: bad arguments");
    if (!m->prov) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_provenance: MPO built without provenance (qcm_mpo_build_qc_tracked)");
    if (site < 0 || std::size_t(site) >= m->prov->ptr.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_provenance: site out of range");
    const auto& pp = m->prov->ptr[std::size_t(site)];
    const uint64_t nr = pp.back();
    *n = nr;
    if (!ptr && !id && !val) return QCM_OK;
    if (!ptr || !id || !val || cap < nr) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_provenance: buffers too small");
    std::copy(pp.begin(), pp.end(), ptr);
    std::copy(m->prov->id[std::size_t(site)].begin(), m->prov->id[std::size_t(site)].end(), id);
    std::copy(m->prov->val[std::size_t(site)].begin(), m->prov->val[std::size_t(site)].end(), val);
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_make_twosite(const qcm_mpo* m, qcm_mpo** out) {
    QCM_TRY
    if (!m || !out) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_make_twosite: bad arguments");
    check_complete(m);
    if (m->m.twosite) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_make_twosite: input is already a two-site MPO");
    auto* p = new qcm_mpo;
    p->m = qcm::make_twosite_mpo(m->m);
    *out = p;
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_length(const qcm_mpo* m) { return m ? int(m->m.t.size()) : -1; }

int qcm_mpo_serialize(const qcm_mpo* m, void* buf, size_t cap, size_t* len) {
    QCM_TRY
    if (!m || !len) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_serialize: bad arguments");
    check_complete(m);
    std::vector<uint8_t> b = qcm::serialize_mpo(m->m);
    *len = b.size();
    if (buf) {
        if (cap < b.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_serialize: buffer too small");
        std::memcpy(buf, b.data(), b.size());
    }
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_deserialize(const void* buf, size_t len, qcm_mpo** out) {
    QCM_TRY
    if (!buf || !out) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_deserialize: bad arguments");
    auto* p = new qcm_mpo;
    p->m = qcm::deserialize_mpo(static_cast<const uint8_t*>(buf), len);
    *out = p;
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_tensor_terms(const qcm_mpo* m, int site, uint32_t* b1, uint32_t* b2, uint32_t* op, double* scale, uint64_t cap,
                         uint64_t* n) {
    QCM_TRY
    if (!m || !n) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_tensor_terms: bad arguments");
    if (site < 0 || std::size_t(site) >= m->m.t.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_tensor_terms: site out of range");
    const qcm::MPOTensor& t = m->m.t[std::size_t(site)];
    const std::size_t ne = t.scale.size();
    *n = ne;
    if (!b1 && !b2 && !op && !scale) return QCM_OK;
    if (cap < ne) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_tensor_terms: buffers too small");
    for (std::size_t e = 0; e < ne; ++e) {
        if (b1) b1[e] = t.b1[e];
        if (b2) b2[e] = t.b2[e];
        if (op) op[e] = t.op[e];
        if (scale) scale[e] = t.scale[e];
    }
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_set_scales(qcm_mpo* m, int site, const double* scale, uint64_t n) {
    QCM_TRY
    if (!m || !scale) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_scales: bad arguments");
    if (site < 0 || std::size_t(site) >= m->m.t.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_scales: site out of range");
    qcm::MPOTensor& t = m->m.t[std::size_t(site)];
    if (n != t.scale.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_scales: entry count mismatch");
    for (uint64_t e = 0; e < n; ++e)
        if (!std::isfinite(scale[e])) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_scales: non-finite scale");
    std::copy(scale, scale + n, t.scale.begin());
    t.finalize();  // drops the derived tables; plans built before keep theirs
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_create(int length, int twosite, qcm_mpo** out) {
    QCM_TRY
    if (!out || length < 1) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_create: bad arguments");
    auto* p = new qcm_mpo;
    p->m.twosite = twosite != 0;
    p->m.t.resize(std::size_t(length));
    p->unset.assign(std::size_t(length), 1);
    *out = p;
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_set_tensor(qcm_mpo* m, int site, const qcm_mpo_tensor_desc* d) {
    QCM_TRY
    if (!m || !d) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: bad arguments");
    if (site < 0 || std::size_t(site) >= m->m.t.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: site out of range");
    if (d->rows == 0 || d->cols == 0 || d->n_phys == 0 || !d->phys_charge || !d->phys_size)
        return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: empty dimensions or physical index");
    if (d->n_terms && (!d->b1 || !d->b2 || !d->op || !d->scale)) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: missing term arrays");
    if (d->n_ops && !d->op_ptr) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: missing operator pointers");
    qcm::MPOTensor T;
    T.rows = d->rows;
    T.cols = d->cols;
    for (uint32_t s = 0; s < d->n_phys; ++s) {
        if (d->phys_size[s] == 0) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: empty physical sector");
        qcm::Charge c(d->phys_charge[2 * s], d->phys_charge[2 * s + 1]);
        if (s && !(T.phys.d.back().first > c))
            return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: physical sectors not in strictly descending charge order");
        T.phys.d.push_back({c, d->phys_size[s]});
    }
    const uint64_t nst = T.phys.sum_of_sizes();
    auto ops = std::make_shared<std::vector<qcm::SparseOp>>(d->n_ops);
    for (uint32_t k = 0; k < d->n_ops; ++k) {
        const uint64_t a = d->op_ptr[k], b = d->op_ptr[k + 1];
        if (b < a || (b > a && (!d->op_in || !d->op_out || !d->op_val)))
            return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: operator pointers not increasing or arrays missing");
        for (uint64_t e = a; e < b; ++e) {
            if (d->op_in[e] >= nst || d->op_out[e] >= nst)
                return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: operator entry outside the physical basis");
            (*ops)[k].in.push_back(d->op_in[e]);
            (*ops)[k].out.push_back(d->op_out[e]);
            (*ops)[k].val.push_back(d->op_val[e]);
        }
    }
    T.ops = ops;
    // entries sorted by (b1, b2), the given order kept within a pair
    std::vector<uint64_t> ord(d->n_terms);
    for (uint64_t e = 0; e < d->n_terms; ++e) {
        if (d->b1[e] >= d->rows || d->b2[e] >= d->cols || d->op[e] >= d->n_ops)
            return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: term index out of range");
        if (!std::isfinite(d->scale[e])) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_set_tensor: non-finite scale");
        ord[e] = e;
    }
    std::stable_sort(ord.begin(), ord.end(), [&](uint64_t x, uint64_t y) {
        return d->b1[x] != d->b1[y] ? d->b1[x] < d->b1[y] : d->b2[x] < d->b2[y];
    });
    for (uint64_t e : ord) { T.b1.push_back(d->b1[e]); T.b2.push_back(d->b2[e]); T.op.push_back(d->op[e]); T.scale.push_back(d->scale[e]); }
    check_pairs(d->herm_left, d->phase_left, d->rows, "left bond");
    check_pairs(d->herm_right, d->phase_right, d->cols, "right bond");
    if (d->herm_left) { T.herm_left.assign(d->herm_left, d->herm_left + d->rows); T.phase_left.assign(d->phase_left, d->phase_left + d->rows); }
    if (d->herm_right) { T.herm_right.assign(d->herm_right, d->herm_right + d->cols); T.phase_right.assign(d->phase_right, d->phase_right + d->cols); }
    T.finalize();
    m->m.t[std::size_t(site)] = std::move(T);
    m->unset[std::size_t(site)] = 0;
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_tensor_info(const qcm_mpo* m, int site, uint32_t* rows, uint32_t* cols, uint32_t* n_ops, uint32_t* n_phys) {
    QCM_TRY
    if (!m) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_tensor_info: bad arguments");
    if (site < 0 || std::size_t(site) >= m->m.t.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_tensor_info: site out of range");
    const qcm::MPOTensor& t = m->m.t[std::size_t(site)];
    if (rows) *rows = t.rows;
    if (cols) *cols = t.cols;
    if (n_ops) *n_ops = t.ops ? uint32_t(t.ops->size()) : 0;
    if (n_phys) *n_phys = uint32_t(t.phys.size());
    return QCM_OK;
    QCM_CATCH
}

int qcm_mpo_tensor_hermitian(const qcm_mpo* m, int site, int32_t* herm_left, int32_t* phase_left, int32_t* herm_right,
                             int32_t* phase_right) {
    QCM_TRY
    if (!m) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_tensor_hermitian: bad arguments");
    if (site < 0 || std::size_t(site) >= m->m.t.size()) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_tensor_hermitian: site out of range");
    const qcm::MPOTensor& t = m->m.t[std::size_t(site)];
    if (herm_left) std::copy(t.herm_left.begin(), t.herm_left.end(), herm_left);
    if (phase_left) std::copy(t.phase_left.begin(), t.phase_left.end(), phase_left);
    if (herm_right) std::copy(t.herm_right.begin(), t.herm_right.end(), herm_right);
    if (phase_right) std::copy(t.phase_right.begin(), t.phase_right.end(), phase_right);
    return QCM_OK;
    QCM_CATCH
}

void qcm_mpo_free(qcm_mpo* m) { delete m; }

}  // extern "C"

namespace qcm {
const MPO& mpo_of(const qcm_mpo* m) {
    check_complete(m);
    return m->m;
}
}  // namespace qcm
