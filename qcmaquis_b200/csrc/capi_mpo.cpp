// C-ABI: MPO construction (input prep for the two-site H_eff path).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>

#include "../../include/qcm_b200.h"
#include "capi_util.hpp"
#include "mpo.hpp"

struct qcm_mpo {
    qcm::MPO m;
};

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

int qcm_mpo_make_twosite(const qcm_mpo* m, qcm_mpo** out) {
    QCM_TRY
    if (!m || !out) return qcm::fail(QCM_ERR_ARG, "qcm_mpo_make_twosite: bad arguments");
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

void qcm_mpo_free(qcm_mpo* m) { delete m; }

}  // extern "C"

namespace qcm {
const MPO& mpo_of(const qcm_mpo* m) { return m->m; }
}  // namespace qcm
