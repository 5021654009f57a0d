// Excited states on the device: the overlap boundaries between the current MPS and the ortho states
// (mps_detail::overlap_left_step / overlap_right_step, mp_tensors/mps.h:175-219) and the ortho vectors of
// a two-site step (contraction::site_ortho_boundaries, mp_tensors/contractions/special.hpp:38-62), as
// batched DMMA GEMMs over the charge blocks and the MPS reshapes.
#include <stdexcept>
#include <vector>

#include "dmrg_dev.hpp"

namespace qcm {

DBlocks unit_blocks(Ctx& c, const Index& i) {
    DBlocks b;
    for (std::size_t k = 0; k < i.size(); ++k) b.add(i[k].first, i[k].first, uint32_t(i[k].second), uint32_t(i[k].second));
    b.allocate(c.s, true);
    std::vector<double> h(b.total ? b.total : 1, 0.0);
    for (std::size_t k = 0; k < b.n(); ++k)
        for (uint32_t d = 0; d < b.rows[k]; ++d) h[b.off[k] + d + uint64_t(d) * b.rows[k]] = 1.0;
    QCM_CUDA(cudaMemcpyAsync(b.d.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
    return b;
}

DBlocks ortho_left_step(Ctx& c, const DMPS& bra_in, const DMPS& ket_in, const DBlocks& left) {
    const DMPS* bra = &bra_in;
    const DMPS* ket = &ket_in;
    DMPS bl, kr;
    if (bra->right_paired) { bl = left_paired_copy(c, *bra); bra = &bl; }
    if (!ket->right_paired) { kr = right_paired_copy(c, *ket); ket = &kr; }
    // t = left * ket, right-paired over (phys, bra left, ket right)
    DMPS t;
    t.phys = ket->phys; t.left = bra->left; t.right = ket->right; t.right_paired = true;
    t.b = layout_right_paired(t.phys, t.left, t.right);
    t.b.allocate(c.s, true);
    std::vector<GemmJob> jobs;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        const Charge q = t.b.lc[k];
        const std::size_t jl = left.find_l(q), jk = ket->b.find_l(q);
        if (jl == left.n() || jk == ket->b.n()) continue;
        if (left.rows[jl] != t.b.rows[k] || left.cols[jl] != ket->b.rows[jk] || ket->b.cols[jk] != t.b.cols[k])
            throw std::runtime_error("ortho left step: block shapes differ");
        GemmJob g{};
        g.a_off = left.off[jl]; g.lda = left.rows[jl];
        g.b_off = ket->b.off[jk]; g.ldb = ket->b.rows[jk];
        g.c_off = t.b.off[k]; g.ldc = t.b.rows[k];
        g.M = t.b.rows[k]; g.N = t.b.cols[k]; g.K = left.cols[jl]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    batched_gemm(jobs, left.d.get(), left.total, ket->b.d.get(), ket->b.total, t.b.d.get(), t.b.total, c.gjobs, c.gtiles, c.s);
    make_left_paired(c, t);  // reshape_right_to_left_new over the bra's left basis
    // out = bra^T t, per right charge
    DBlocks out;
    std::vector<std::pair<std::size_t, std::size_t>> pr;
    for (std::size_t k = 0; k < bra->b.n(); ++k) {
        const std::size_t jt = t.b.find_l(bra->b.rc[k]);
        if (jt == t.b.n()) continue;
        if (t.b.rows[jt] != bra->b.rows[k]) throw std::runtime_error("ortho left step: reshaped rows differ");
        out.add(bra->b.rc[k], bra->b.rc[k], bra->b.cols[k], t.b.cols[jt]);
        pr.push_back({k, jt});
    }
    out.allocate(c.s, true);
    jobs.clear();
    for (std::size_t o = 0; o < pr.size(); ++o) {
        const std::size_t k = pr[o].first, jt = pr[o].second;
        GemmJob g{};
        g.a_off = bra->b.off[k]; g.lda = bra->b.rows[k]; g.ta = 1;
        g.b_off = t.b.off[jt]; g.ldb = t.b.rows[jt];
        g.c_off = out.off[o]; g.ldc = out.rows[o];
        g.M = out.rows[o]; g.N = out.cols[o]; g.K = bra->b.rows[k]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    batched_gemm(jobs, bra->b.d.get(), bra->b.total, t.b.d.get(), t.b.total, out.d.get(), out.total, c.gjobs, c.gtiles, c.s);
    return out;
}

DBlocks ortho_right_step(Ctx& c, const DMPS& bra_in, const DMPS& ket_in, const DBlocks& right) {
    const DMPS* bra = &bra_in;
    const DMPS* ket = &ket_in;
    DMPS br, kl;
    if (!bra->right_paired) { br = right_paired_copy(c, *bra); bra = &br; }
    if (ket->right_paired) { kl = left_paired_copy(c, *ket); ket = &kl; }
    // t = ket * right^T, left-paired over (phys, ket left, bra right)
    DMPS t;
    t.phys = ket->phys; t.left = ket->left; t.right = bra->right; t.right_paired = false;
    t.b = layout_left_paired(t.phys, t.left, t.right);
    t.b.allocate(c.s, true);
    std::vector<GemmJob> jobs;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        const Charge q = t.b.rc[k];
        const std::size_t jk = ket->b.find_l(q), jr = right.find_l(q);
        if (jk == ket->b.n() || jr == right.n()) continue;
        if (ket->b.rows[jk] != t.b.rows[k] || ket->b.cols[jk] != right.cols[jr] || right.rows[jr] != t.b.cols[k])
            throw std::runtime_error("ortho right step: block shapes differ");
        GemmJob g{};
        g.a_off = ket->b.off[jk]; g.lda = ket->b.rows[jk];
        g.b_off = right.off[jr]; g.ldb = right.rows[jr]; g.tb = 1;
        g.c_off = t.b.off[k]; g.ldc = t.b.rows[k];
        g.M = t.b.rows[k]; g.N = t.b.cols[k]; g.K = ket->b.cols[jk]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    batched_gemm(jobs, ket->b.d.get(), ket->b.total, right.d.get(), right.total, t.b.d.get(), t.b.total, c.gjobs, c.gtiles, c.s);
    make_right_paired(c, t);  // reshape_left_to_right_new over the bra's right basis
    // out = bra t^T, per left charge
    DBlocks out;
    std::vector<std::pair<std::size_t, std::size_t>> pr;
    for (std::size_t k = 0; k < bra->b.n(); ++k) {
        const std::size_t jt = t.b.find_l(bra->b.lc[k]);
        if (jt == t.b.n()) continue;
        if (t.b.cols[jt] != bra->b.cols[k]) throw std::runtime_error("ortho right step: reshaped columns differ");
        out.add(bra->b.lc[k], bra->b.lc[k], bra->b.rows[k], t.b.rows[jt]);
        pr.push_back({k, jt});
    }
    out.allocate(c.s, true);
    jobs.clear();
    for (std::size_t o = 0; o < pr.size(); ++o) {
        const std::size_t k = pr[o].first, jt = pr[o].second;
        GemmJob g{};
        g.a_off = bra->b.off[k]; g.lda = bra->b.rows[k];
        g.b_off = t.b.off[jt]; g.ldb = t.b.rows[jt]; g.tb = 1;
        g.c_off = out.off[o]; g.ldc = out.rows[o];
        g.M = out.rows[o]; g.N = out.cols[o]; g.K = bra->b.cols[k]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    batched_gemm(jobs, bra->b.d.get(), bra->b.total, t.b.d.get(), t.b.total, out.d.get(), out.total, c.gjobs, c.gtiles, c.s);
    return out;
}

void ortho_vector(Ctx& c, const DMPS& twin, const DMPS& ot, const DBlocks& left, const DBlocks& right, double* v) {
    if (!twin.right_paired || !ot.right_paired) throw std::runtime_error("ortho vector: expects right-paired twins");
    if (twin.b.total) QCM_CUDA(cudaMemsetAsync(v, 0, twin.b.total * sizeof(double), c.s));
    // t = left * ortho twin per left charge
    DBlocks t;
    std::vector<std::size_t> tk(twin.b.n(), SIZE_MAX);
    std::vector<GemmJob> jobs;
    for (std::size_t k = 0; k < twin.b.n(); ++k) {
        const Charge q = twin.b.lc[k];
        const std::size_t jl = left.find_l(q), jo = ot.b.find_l(q);
        if (jl == left.n() || jo == ot.b.n()) continue;
        if (left.rows[jl] != twin.b.rows[k] || left.cols[jl] != ot.b.rows[jo])
            throw std::runtime_error("ortho vector: boundary and twin blocks differ");
        tk[k] = t.n();
        t.add(q, q, twin.b.rows[k], ot.b.cols[jo]);
        GemmJob g{};
        g.a_off = left.off[jl]; g.lda = left.rows[jl];
        g.b_off = ot.b.off[jo]; g.ldb = ot.b.rows[jo];
        g.c_off = t.off.back(); g.ldc = t.rows.back();
        g.M = t.rows.back(); g.N = t.cols.back(); g.K = left.cols[jl]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    t.allocate(c.s, false);
    batched_gemm(jobs, left.d.get(), left.total, ot.b.d.get(), ot.b.total, t.d.get(), t.total, c.gjobs, c.gtiles, c.s);
    // v(:, slice (phys state, right charge)) = t(:, the ortho twin's slice) * right^T
    ProductBasis cur_pb(twin.phys, twin.right, true), ort_pb(ot.phys, ot.right, true);
    jobs.clear();
    for (std::size_t k = 0; k < twin.b.n(); ++k) {
        if (tk[k] == SIZE_MAX) continue;
        const Charge q = twin.b.lc[k];
        const uint32_t ls = twin.b.rows[k];
        for (std::size_t s = 0; s < twin.phys.size(); ++s) {
            const Charge ph = twin.phys[s].first, rc = q + ph;
            if (!twin.right.has(rc) || !ot.right.has(rc)) continue;
            const std::size_t jr = right.find_l(rc);
            if (jr == right.n()) continue;
            const uint32_t rs_c = uint32_t(twin.right.size_of(rc)), rs_o = uint32_t(ot.right.size_of(rc));
            if (right.rows[jr] != rs_c || right.cols[jr] != rs_o) throw std::runtime_error("ortho vector: right boundary block differs");
            for (std::size_t ss = 0; ss < twin.phys[s].second; ++ss) {
                const uint64_t oc = ort_pb(ph, rc) + ss * rs_o, cc = cur_pb(ph, rc) + ss * rs_c;
                GemmJob g{};
                g.a_off = t.off[tk[k]] + oc * ls; g.lda = ls;
                g.b_off = right.off[jr]; g.ldb = rs_c; g.tb = 1;
                g.c_off = twin.b.off[k] + cc * ls; g.ldc = ls;
                g.M = ls; g.N = rs_c; g.K = rs_o; g.alpha = 1.0; g.beta = 0.0;
                jobs.push_back(g);
            }
        }
    }
    batched_gemm(jobs, t.d.get(), t.total, right.d.get(), right.total, v, twin.b.total, c.gjobs, c.gtiles, c.s);
}

}  // namespace qcm
