// ORACLE -- TEST INFRASTRUCTURE ONLY.  Contraction schedule and execution, restated
// from solver/tasks.cpp and mp_tensors/contractions/{create_schedule,boundary_ops}.
#include "engine.hpp"

#include <unordered_map>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

namespace {
// solver/tasks.cpp:49-62
void tr_tile_v(unsigned nrows, unsigned ncols, std::size_t cnt, const double* in, double* out) {
    for (std::size_t b = 0; b < cnt; ++b) {
        std::size_t off = b * nrows * ncols;
        for (unsigned i = 0; i < nrows; ++i)
            for (unsigned j = 0; j < ncols; ++j) out[off + std::size_t(ncols) * i + j] = in[off + std::size_t(nrows) * j + i];
    }
}
struct TiLookup {  // MPSBlock::get_ti (tasks.cpp:766-775): first (mps_offset, ci) match
    std::unordered_map<uint64_t, unsigned> m;
    void build(const std::vector<TJob>& ts) {
        m.clear();
        for (unsigned ti = 0; ti < ts.size(); ++ti) m.emplace((uint64_t(ts[ti].mps_offset) << 32) | ts[ti].ci, ti);
    }
    unsigned get(unsigned off, unsigned ci) const {
        auto it = m.find((uint64_t(off) << 32) | ci);
        return it == m.end() ? std::numeric_limits<unsigned>::max() : it->second;
    }
};
}  // namespace

Cohort::Cohort(const std::vector<std::size_t>& phys_i, unsigned l_block, unsigned r_block, unsigned l_size, unsigned r_size,
               unsigned ci_, unsigned ci_eff_, unsigned mpodim, bool left)
    : lb(l_block), rb(r_block), ls(l_size), rs(r_size), ci(ci_), ci_eff(ci_eff_), nSrows(mpodim),
      mpo_offsets(mpodim, 0), sfold(phys_i.size()) {
    unsigned ssum = 0;
    for (std::size_t s = 0; s < phys_i.size(); ++s) { sfold[s] = ssum; ssum += unsigned(phys_i[s]); }
    suv.resize(ssum);
    sblock = left ? rs : ls;
}

// tasks.cpp:506-526 (compute_mpo_offsets)
void Cohort::finalize() {
    std::vector<long> cpy = mpo_offsets;
    unsigned n_blocks = 0;
    for (auto& b : cpy) if (b) b = n_blocks++;
    nSrows = n_blocks;
    for (auto& x : suv)
        for (auto& b : x.b1) b = unsigned(cpy[b]);
    std::size_t block_size = std::size_t(ls) * rs;
    unsigned cnt = 0;
    for (auto& b : mpo_offsets) b = b ? long(block_size * cnt++) : -1;
}

std::size_t Cohort::n_flops() const {
    std::size_t r = 2ull * rs * ls * nSrows * stripe;
    for (auto& x : suv) r += 2ull * ls * x.ms * x.alpha.size();
    return r;
}

std::vector<double> Cohort::create_s(const TList& T) const {
    std::vector<double> ret(S_size(), 0.0);
    for (auto& x : suv) {
        if (x.alpha.empty()) continue;
        std::vector<double> buf(std::size_t(x.ms) * rs);
        unsigned seeker = 0;
        for (std::size_t b = 0; b < x.b2s.size(); ++b) {
            std::fill(buf.begin(), buf.end(), 0.0);
            for (unsigned ia = seeker; ia < seeker + x.b2s[b]; ++ia)
                daxpy(std::size_t(x.ms) * rs, x.alpha[ia], &T[x.tidx[2 * ia]][std::size_t(x.tidx[2 * ia + 1]) * rs], buf.data());
            unsigned bb = x.b1[b];
            for (unsigned c = 0; c < rs; ++c)
                std::copy(&buf[std::size_t(c) * x.ms], &buf[std::size_t(c) * x.ms] + x.ms,
                          ret.data() + std::size_t(stripe) * (std::size_t(bb) * rs + c) + x.offset);
            seeker += x.b2s[b];
        }
    }
    return ret;
}

std::vector<double> Cohort::create_s_r(const TList& T) const {
    std::vector<double> ret(S_size(), 0.0);
    for (auto& x : suv) {
        if (x.alpha.empty()) continue;
        std::vector<double> buf(std::size_t(ls) * x.ms);
        unsigned seeker = 0;
        for (std::size_t b = 0; b < x.b2s.size(); ++b) {
            std::fill(buf.begin(), buf.end(), 0.0);
            for (unsigned ia = seeker; ia < seeker + x.b2s[b]; ++ia)
                daxpy(std::size_t(x.ms) * ls, x.alpha[ia], &T[x.tidx[2 * ia]][std::size_t(x.tidx[2 * ia + 1]) * ls], buf.data());
            unsigned bb = x.b1[b];
            for (unsigned c = 0; c < x.ms; ++c)
                std::copy(&buf[std::size_t(c) * ls], &buf[std::size_t(c) * ls] + ls,
                          ret.data() + std::size_t(nSrows) * ls * (x.offset + c) + std::size_t(bb) * ls);
            seeker += x.b2s[b];
        }
    }
    return ret;
}

std::vector<double> Cohort::contract_buf(const std::vector<const double*>& left, const TList& T) const {
    std::vector<double> sloc = create_s_r(T);
    int M = int(rs), N = int(stripe), K = int(nSrows * ls);
    const double* luse = left[ci_eff];
    std::vector<double> lbuf;
    if (ci != ci_eff) {
        lbuf.resize(std::size_t(M) * K);
        tr_tile_v(ls, rs, nSrows, left[ci_eff], lbuf.data());
        luse = lbuf.data();
    }
    std::vector<double> buf(std::size_t(M) * N);
    dgemm('N', 'N', M, N, K, 1.0, luse, M, sloc.data(), K, 0.0, buf.data(), M);
    return buf;
}

void Cohort::contract(const std::vector<const double*>& left, const TList& T, double* out, std::mutex& mu) const {
    std::vector<double> sloc = create_s_r(T);
    int M = int(rs), N = int(stripe), K = int(nSrows * ls);
    const double* luse = left[ci_eff];
    std::vector<double> lbuf;
    if (ci != ci_eff) {
        lbuf.resize(std::size_t(M) * K);
        tr_tile_v(ls, rs, nSrows, left[ci_eff], lbuf.data());
        luse = lbuf.data();
    }
    std::vector<double> buf(std::size_t(M) * N);
    dgemm('N', 'N', M, N, K, 1.0, luse, M, sloc.data(), K, 0.0, buf.data(), M);
    std::lock_guard<std::mutex> lk(mu);
    daxpy(buf.size(), 1.0, buf.data(), out);
}

void Cohort::prop_l(const double* bra, const TList& T, double* new_left) const {
    std::vector<double> sloc = create_s(T);
    int M = int(ls), N = int(nSrows * rs);
    dgemm('T', 'N', M, N, int(stripe), 1.0, bra, int(stripe), sloc.data(), int(stripe), 0.0, new_left, M);
}

void Cohort::prop_r(const double* bra, const TList& T, double* new_right) const {
    std::vector<double> sloc = create_s_r(T);
    int M = int(nSrows * ls), N = int(rs);
    std::vector<double> buf(std::size_t(M) * N);
    dgemm('N', 'T', M, N, int(stripe), 1.0, sloc.data(), M, bra, int(rs), 0.0, buf.data(), M);
    for (unsigned b = 0; b < nSrows; ++b)
        for (unsigned col = 0; col < rs; ++col)
            std::copy(&buf[std::size_t(ls) * b + std::size_t(col) * M], &buf[std::size_t(ls) * b + std::size_t(col) * M] + ls,
                      new_right + (std::size_t(b) * rs + col) * ls);
}

void Cohort::lbtm(const TList& T, double* out, double alpha) const {
    std::vector<double> sloc = create_s(T);
    int M = int(stripe), K = M ? int(sloc.size() / M) : 0;
    std::vector<double> tmp(std::size_t(M) * M, 0.0);
    dgemm('N', 'T', M, M, K, alpha, sloc.data(), M, sloc.data(), M, 1.0, tmp.data(), M);
    daxpy(tmp.size(), 1.0, tmp.data(), out);
}

void Cohort::rbtm(const TList& T, double* out, double alpha) const {
    std::vector<double> sloc = create_s_r(T);
    int M = int(stripe), K = int(nSrows * ls);
    std::vector<double> tmp(std::size_t(M) * M, 0.0);
    dgemm('T', 'N', M, M, K, alpha, sloc.data(), K, sloc.data(), K, 1.0, tmp.data(), M);
    daxpy(tmp.size(), 1.0, tmp.data(), out);
}

unsigned MPSBlock::get_ti(unsigned mps_offset, unsigned ci_virt) const {
    for (unsigned ti = 0; ti < t_schedule.size(); ++ti)
        if (t_schedule[ti].mps_offset == mps_offset && t_schedule[ti].ci == ci_virt) return ti;
    return std::numeric_limits<unsigned>::max();
}

TList MPSBlock::create_T(const std::vector<const double*>& right, const std::vector<const double*>& mps) const {
    TList ret(t_schedule.size());
    for (unsigned ti = 0; ti < t_schedule.size(); ++ti) {
        const TJob& j = t_schedule[ti];
        int bls = int(right_rt->left_size(j.ci)), brs = int(right_rt->right_size(j.ci));
        int M = int((*lr_ket_sizes)[j.lb_ket]);
        int K = bls;
        unsigned nbk = unsigned(right_rt->n_blocks(j.ci_eff));
        const double* mpsdata = mps[j.lb_ket] + std::size_t(M) * j.mps_offset;
        ret[ti].assign(std::size_t(M) * nbk * brs, 0.0);
        for (unsigned b = 0; b < nbk; ++b) {
            std::size_t roff = std::size_t(b) * K * brs, ooff = std::size_t(b) * M * brs;
            if (j.ci != j.ci_eff)
                dgemm('N', 'T', M, brs, K, 1.0, mpsdata, M, right[j.ci_eff] + roff, brs, 0.0, ret[ti].data() + ooff, M);
            else
                dgemm('N', 'N', M, brs, K, 1.0, mpsdata, M, right[j.ci_eff] + roff, K, 0.0, ret[ti].data() + ooff, M);
        }
    }
    return ret;
}

TList MPSBlock::create_T_left(const std::vector<const double*>& left, const std::vector<const double*>& mps) const {
    TList ret(t_schedule.size());
    for (unsigned ti = 0; ti < t_schedule.size(); ++ti) {
        const TJob& j = t_schedule[ti];
        int M = int(left_rt->left_size(j.ci)), K = int(left_rt->right_size(j.ci));
        int N = int((*lr_ket_sizes)[rb_ket]);
        unsigned nbk = unsigned(left_rt->n_blocks(j.ci_eff));
        const double* mpsdata = mps[j.lb_ket] + std::size_t(K) * j.mps_offset;
        ret[ti].assign(std::size_t(M) * N * nbk, 0.0);
        for (unsigned b = 0; b < nbk; ++b) {
            std::size_t loff = std::size_t(b) * M * K, ooff = std::size_t(b) * M * N;
            if (j.ci != j.ci_eff)
                dgemm('T', 'N', M, N, K, 1.0, left[j.ci_eff] + loff, K, mpsdata, K, 0.0, ret[ti].data() + ooff, M);
            else
                dgemm('N', 'N', M, N, K, 1.0, left[j.ci_eff] + loff, M, mpsdata, K, 0.0, ret[ti].data() + ooff, M);
        }
    }
    return ret;
}

std::size_t MPSBlock::n_flops(const BoundaryIndex& right) const {
    std::size_t r = 0;
    for (auto& j : t_schedule) r += 2ull * (*lr_ket_sizes)[j.lb_ket] * right.cohort_size(j.ci_eff);
    for (auto& c : data) r += c.n_flops();
    return r;
}

// ---- schedule builders --------------------------------------------------------

namespace {

// create_schedule/op_iterate.hpp:38-70 (abelian: all four couplings equal the scale)
// term / dcoupling (H_eff schedules): the MPO entry of the alphas and their coupling without the
// entry's scale, recorded for the scale gradient
void op_iterate(const SiteOp& W, std::size_t w_block, double coupling, Cohort& cg, unsigned s, unsigned m2_size,
                const TiLookup& tl, unsigned mps_offset, unsigned ci, unsigned boundary_col,
                unsigned term = std::numeric_limits<unsigned>::max(), double dcoupling = 0.0) {
    const OpBlock& blk = W.blocks[w_block];
    for (std::size_t e = 0; e < blk.coeff.size(); ++e) {
        double scale = blk.coeff[e] * coupling;
        unsigned ti = tl.get(mps_offset + blk.ss1[e] * m2_size, ci);
        if (ti < std::numeric_limits<unsigned>::max()) {
            cg.push_back(s, blk.ss2[e], scale, ti, boundary_col);
            if (term != std::numeric_limits<unsigned>::max()) cg.push_term(s, blk.ss2[e], term, blk.coeff[e] * dcoupling);
        }
    }
}

// create_schedule/right_tasks.hpp:39-78
void rshtm_t_tasks(const BoundaryIndex& right, const Index& left_i, const Index& right_i, const Index& phys_i,
                   const ProductBasis& right_pb, unsigned lb_ket, MPSBlock& mpsb) {
    Q lc_ket = left_i[lb_ket].first;
    for (std::size_t s = 0; s < phys_i.size(); ++s) {
        Q phys_in = phys_i[s].first;
        Q rc_ket = lc_ket + phys_in;
        std::size_t rb_ket = right_i.position(rc_ket);
        if (rb_ket == right_i.size()) continue;
        unsigned rs_ket = unsigned(right_i[rb_ket].second);
        unsigned ket_offset = unsigned(right_pb(phys_in, rc_ket));
        for (std::size_t rb_bra = 0; rb_bra < right_i.size(); ++rb_bra) {
            unsigned ci = right.cohort_index(rc_ket, right_i[rb_bra].first);
            if (ci == right.n_cohorts()) continue;
            unsigned ci_eff = right.tr(ci) ? right.cohort_index(right_i[rb_bra].first, rc_ket) : ci;
            std::size_t sz = left_i[lb_ket].second * right_i[rb_bra].second * right.n_blocks(ci_eff);
            std::size_t sza = round_up(sz);
            mpsb.buf_size += phys_i[s].second * sza;
            for (unsigned ss = 0; ss < phys_i[s].second; ++ss)
                mpsb.t_schedule.push_back(TJob{ket_offset + ss * rs_ket, ci, ci_eff, lb_ket, sza});
        }
    }
}

// create_schedule/site_hamil_tasks.hpp:41-137
void shtm_tasks(const MPOTensor& mpo, const BoundaryIndex& left, const BoundaryIndex& right, const Index& left_i,
                const Index& right_i, const Index& phys_i, const ProductBasis& right_pb, unsigned lb_in, MPSBlock& mpsb) {
    std::vector<std::size_t> phys_s = phys_i.sizes();
    TiLookup tl;
    tl.build(mpsb.t_schedule);
    Q lc_in = left_i[lb_in].first;
    unsigned ls_in = unsigned(left_i[lb_in].second);
    for (unsigned lb_out = 0; lb_out < left_i.size(); ++lb_out) {
        Q lc_out = left_i[lb_out].first;
        unsigned ls_out = unsigned(left_i[lb_out].second);
        unsigned ci = left.cohort_index(lc_out, lc_in);
        if (ci == left.n_cohorts()) continue;
        unsigned ci_eff = left.tr(ci) ? left.cohort_index(lc_in, lc_out) : ci;
        Cohort cohort(phys_s, lb_in, lb_out, ls_in, ls_out, ci, ci_eff, unsigned(left.n_blocks(ci_eff)));
        for (unsigned s = 0; s < phys_i.size(); ++s) {
            Q phys_out = phys_i[s].first;
            Q rc_out = lc_out + phys_out;
            std::size_t rb_out = right_i.position(rc_out);
            if (rb_out == right_i.size()) continue;
            unsigned rs_out = unsigned(right_i[rb_out].second);
            unsigned out_offset = unsigned(right_pb(phys_out, rc_out));
            cohort.add_unit(s, unsigned(phys_i[s].second), rs_out, out_offset);
            for (unsigned b1 = 0; b1 < mpo.rows; ++b1) {
                if (!left.has_block(ci, b1)) continue;
                unsigned left_idx = unsigned(left.offset(ci, b1) / (long(ls_in) * ls_out));
                for (unsigned b2 : mpo.row_b2[b1]) {
                    const auto& ents = mpo.at.at({b1, b2});
                    for (unsigned e : ents) {
                        const SiteOp& W = mpo.ops[mpo.op[e]];
                        for (std::size_t wb = 0; wb < W.blocks.size(); ++wb) {
                            if (phys_out != mpo.phys[W.blocks[wb].out_sec].first) continue;
                            Q phys_in = mpo.phys[W.blocks[wb].in_sec].first;
                            Q rc_in = lc_in + phys_in;
                            unsigned ci_right = right.cohort_index(rc_in, rc_out);
                            if (!right.has_block(ci_right, b2)) continue;
                            std::size_t rb_in = right_i.position(rc_in);
                            if (rb_in == right_i.size()) continue;
                            unsigned rs_in = unsigned(right_i[rb_in].second);
                            unsigned in_offset = unsigned(right_pb(phys_in, rc_in));
                            long right_offset = right.offset(ci_right, b2);
                            double scale = right.conjugate_scale(ci_right, b2) * mpo.scale[e] * left.conjugate_scale(ci, b1);
                            double dscale = right.conjugate_scale(ci_right, b2) * left.conjugate_scale(ci, b1);
                            op_iterate(W, wb, scale, cohort, s, rs_in, tl, in_offset, ci_right, unsigned(right_offset / rs_in),
                                       e, dscale);
                        }
                    }
                }
                cohort.add_line(left_idx);
            }
        }
        if (cohort.n_tasks()) mpsb.data.push_back(std::move(cohort));
    }
}

// create_schedule/right_tasks.hpp:80-167
void rshtm_tasks(const MPOTensor& mpo, const BoundaryIndex& right, const Index& left_i, const Index& right_i,
                 const Index& phys_i, const ProductBasis& right_pb, unsigned lb_ket, MPSBlock& mpsb, bool skip) {
    std::vector<std::size_t> phys_s = phys_i.sizes();
    TiLookup tl;
    tl.build(mpsb.t_schedule);
    Q lc_ket = left_i[lb_ket].first;
    unsigned ls_ket = unsigned(left_i[lb_ket].second);
    for (unsigned lb_bra = 0; lb_bra < left_i.size(); ++lb_bra) {
        Q lc_bra = left_i[lb_bra].first;
        if (std::abs(particleNumber(lc_ket) - particleNumber(lc_bra)) > 2) continue;
        unsigned ls_bra = unsigned(left_i[lb_bra].second);
        Cohort cohort(phys_s, lb_ket, lb_bra, ls_ket, ls_bra, 0, 0, mpo.rows);
        for (unsigned s = 0; s < phys_i.size(); ++s) {
            Q phys_out = phys_i[s].first;
            Q rc_bra = lc_bra + phys_out;
            std::size_t rb_bra = right_i.position(rc_bra);
            if (rb_bra == right_i.size()) continue;
            unsigned rs_bra = unsigned(right_i[rb_bra].second);
            unsigned bra_offset = unsigned(right_pb(phys_out, rc_bra));
            cohort.add_unit(s, unsigned(phys_i[s].second), rs_bra, bra_offset);
            for (unsigned b1 = 0; b1 < mpo.rows; ++b1) {
                if (MPOTensor::skip(mpo.herm_left, b1, lc_ket, lc_bra) && skip) continue;
                for (unsigned b2 : mpo.row_b2[b1]) {
                    for (unsigned e : mpo.at.at({b1, b2})) {
                        const SiteOp& W = mpo.ops[mpo.op[e]];
                        for (std::size_t wb = 0; wb < W.blocks.size(); ++wb) {
                            if (phys_out != mpo.phys[W.blocks[wb].out_sec].first) continue;
                            Q phys_in = mpo.phys[W.blocks[wb].in_sec].first;
                            Q rc_ket = lc_ket + phys_in;
                            unsigned ci = right.cohort_index(rc_ket, rc_bra);
                            if (!right.has_block(ci, b2)) continue;
                            std::size_t rb_ket = right_i.position(rc_ket);
                            if (rb_ket == right_i.size()) continue;
                            unsigned rs_ket = unsigned(right_i[rb_ket].second);
                            unsigned ket_offset = unsigned(right_pb(phys_in, rc_ket));
                            long right_offset = right.offset(ci, b2);
                            double scale = right.conjugate_scale(ci, b2) * mpo.scale[e];
                            op_iterate(W, wb, scale, cohort, s, rs_ket, tl, ket_offset, ci, unsigned(right_offset / rs_ket));
                        }
                    }
                }
                cohort.add_line(b1);
            }
        }
        cohort.finalize();
        if (cohort.n_tasks()) mpsb.data.push_back(std::move(cohort));
    }
}

// create_schedule/left_tasks.hpp:38-74
void lshtm_t_tasks(const BoundaryIndex& left, const Index& left_i, const Index& right_i, const Index& phys_i,
                   const ProductBasis& right_pb, unsigned rb_ket, MPSBlock& mpsb) {
    Q rc_ket = right_i[rb_ket].first;
    unsigned rs_ket = unsigned(right_i[rb_ket].second);
    for (std::size_t s = 0; s < phys_i.size(); ++s) {
        Q phys_in = phys_i[s].first;
        Q lc_ket = rc_ket + (-phys_in);
        std::size_t lb_ket = left_i.position(lc_ket);
        if (lb_ket == left_i.size()) continue;
        unsigned ket_offset = unsigned(right_pb(phys_in, rc_ket));
        for (std::size_t lb_bra = 0; lb_bra < left_i.size(); ++lb_bra) {
            unsigned ci = left.cohort_index(left_i[lb_bra].first, lc_ket);
            if (ci == left.n_cohorts()) continue;
            unsigned ci_eff = left.tr(ci) ? left.cohort_index(lc_ket, left_i[lb_bra].first) : ci;
            std::size_t sz = left_i[lb_bra].second * rs_ket * left.n_blocks(ci_eff);
            std::size_t sza = round_up(sz);
            mpsb.buf_size += phys_i[s].second * sza;
            for (unsigned ss = 0; ss < phys_i[s].second; ++ss)
                mpsb.t_schedule.push_back(TJob{ket_offset + ss * rs_ket, ci, ci_eff, unsigned(lb_ket), sza});
        }
    }
}

// create_schedule/left_tasks.hpp:76-172
void lshtm_tasks(const MPOTensor& mpo, const MPSTensor& bra, const MPSTensor& ket, const BoundaryIndex& left,
                 const ProductBasis& bra_left_pb, const ProductBasis& ket_right_pb, unsigned rb_ket, MPSBlock& mpsb,
                 bool skip) {
    const Index& ket_left_i = ket.left;
    const Index& ket_right_i = ket.right;
    const Index& bra_left_i = bra.left;
    const Index& bra_right_i = bra.right;
    const Index& phys_i = ket.phys;
    std::vector<std::size_t> phys_s = phys_i.sizes();
    TiLookup tl;
    tl.build(mpsb.t_schedule);
    Q rc_ket = ket_right_i[rb_ket].first;
    unsigned rs_ket = unsigned(ket_right_i[rb_ket].second);
    for (unsigned rb_bra = 0; rb_bra < bra_right_i.size(); ++rb_bra) {
        Q rc_bra = bra_right_i[rb_bra].first;
        if (std::abs(particleNumber(rc_bra) - particleNumber(rc_ket)) > 2) continue;
        unsigned rs_bra = unsigned(bra_right_i[rb_bra].second);
        Cohort cohort(phys_s, rb_bra, rb_ket, rs_bra, rs_ket, 0, 0, mpo.cols, true);
        for (unsigned s = 0; s < phys_i.size(); ++s) {
            Q phys_out = phys_i[s].first;
            Q lc_bra = rc_bra + (-phys_out);
            std::size_t lb_bra = bra_left_i.position(lc_bra);
            if (lb_bra == bra_left_i.size()) continue;
            unsigned ls_bra = unsigned(bra_left_i[lb_bra].second);
            unsigned bra_offset = unsigned(bra_left_pb(phys_out, lc_bra));
            cohort.add_unit(s, unsigned(phys_i[s].second), ls_bra, bra_offset);
            for (unsigned b2 = 0; b2 < mpo.cols; ++b2) {
                if (MPOTensor::skip(mpo.herm_right, b2, rc_bra, rc_ket) && skip) continue;
                for (unsigned b1 : mpo.col_b1[b2]) {
                    for (unsigned e : mpo.at.at({b1, b2})) {
                        const SiteOp& W = mpo.ops[mpo.op[e]];
                        for (std::size_t wb = 0; wb < W.blocks.size(); ++wb) {
                            if (phys_out != mpo.phys[W.blocks[wb].out_sec].first) continue;
                            Q phys_in = mpo.phys[W.blocks[wb].in_sec].first;
                            Q lc_ket = rc_ket + (-phys_in);
                            std::size_t lb_ket = ket_left_i.position(lc_ket);
                            if (lb_ket == ket_left_i.size()) continue;
                            unsigned ci = left.cohort_index(lc_bra, lc_ket);
                            if (!left.has_block(ci, b1)) continue;
                            unsigned ls_ket = unsigned(ket_left_i[lb_ket].second);
                            unsigned ket_offset = unsigned(ket_right_pb(phys_in, rc_ket));
                            long left_offset = left.offset(ci, b1);
                            double scale = left.conjugate_scale(ci, b1) * mpo.scale[e];
                            op_iterate(W, wb, scale, cohort, s, rs_ket, tl, ket_offset, ci, unsigned(left_offset / ls_ket));
                        }
                    }
                }
                cohort.add_line(b2);
            }
        }
        cohort.finalize();
        if (cohort.n_tasks()) mpsb.data.push_back(std::move(cohort));
    }
}

std::vector<const double*> block_view(const MPSTensor& t, const Index& by, bool by_left) {
    std::vector<const double*> v(by.size(), nullptr);
    for (std::size_t i = 0; i < by.size(); ++i) {
        Q c = by[i].first;
        std::size_t k = t.data.find(c, c);
        (void)by_left;
        if (k < t.data.n_blocks()) v[i] = t.data.b[k].d.data();
    }
    return v;
}

std::vector<const double*> boundary_view(const Boundary& b) {
    std::vector<const double*> v(b.data.size());
    for (std::size_t i = 0; i < b.data.size(); ++i) v[i] = b.data[i].data();
    return v;
}

}  // namespace

std::unique_ptr<Schedule> create_contraction_schedule(MPSTensor& initial, const Boundary& left, const Boundary& right,
                                                      const MPOTensor& mpo) {
    initial.make_right_paired();
    const Index& phys_i = initial.phys;
    const Index& right_i = initial.right;
    const Index& left_i = initial.left;
    ProductBasis out_right_pb(phys_i, right_i, true);
    auto tasks = std::make_unique<Schedule>();
    tasks->lr_ket_sizes = left_i.sizes();
    tasks->blocks.resize(left_i.size());
    for (auto& b : initial.data.b) tasks->mps_block_sizes.push_back(b.r * b.c);
    for (unsigned mb = 0; mb < left_i.size(); ++mb) {
        MPSBlock& blk = tasks->blocks[mb];
        blk.lr_ket_sizes = &tasks->lr_ket_sizes;
        blk.left_rt = &left.index;
        blk.right_rt = &right.index;
        blk.rb_ket = mb;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int mb = 0; mb < int(left_i.size()); ++mb) {
        rshtm_t_tasks(right.index, left_i, right_i, phys_i, out_right_pb, unsigned(mb), tasks->blocks[mb]);
        shtm_tasks(mpo, left.index, right.index, left_i, right_i, phys_i, out_right_pb, unsigned(mb), tasks->blocks[mb]);
    }
    for (auto& b : tasks->blocks) tasks->total_flops += b.n_flops(right.index);
    return tasks;
}

void super_hamil_mv(const Schedule& sched, const Boundary& left, const Boundary& right,
                    const std::vector<const double*>& x, const std::vector<double*>& y) {
    // Cohort products are formed in parallel over ket blocks as in super_hamil_mv.hpp:121-132,
    // then added to each output block in a fixed (lb_in, cohort) order, so the result does
    // not depend on the thread count (the reference's mutex-ordered axpy does).
    std::vector<const double*> lv = boundary_view(left), rv = boundary_view(right);
    const std::size_t nb = sched.blocks.size();
    std::vector<std::vector<std::vector<double>>> part(nb);
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < int(nb); ++b) {
        const MPSBlock& blk = sched.blocks[b];
        if (blk.data.empty()) continue;
        TList T = blk.create_T(rv, x);
        part[b].resize(blk.data.size());
        for (std::size_t c = 0; c < blk.data.size(); ++c) part[b][c] = blk.data[c].contract_buf(lv, T);
    }
    std::vector<std::vector<std::pair<std::size_t, std::size_t>>> by_out(nb);
    for (std::size_t b = 0; b < nb; ++b)
        for (std::size_t c = 0; c < sched.blocks[b].data.size(); ++c) by_out[sched.blocks[b].data[c].rb].push_back({b, c});
#pragma omp parallel for schedule(dynamic, 1)
    for (int o = 0; o < int(nb); ++o)
        for (auto& bc : by_out[o]) {
            const std::vector<double>& buf = part[bc.first][bc.second];
            daxpy(buf.size(), 1.0, buf.data(), y[o]);
        }
}

void scale_gradient(const Schedule& sched, const Boundary& left, const Boundary& right, const std::vector<const double*>& x,
                    const std::vector<const double*>& ybar, std::size_t n_terms, std::vector<double>& grad) {
    std::vector<const double*> lv = boundary_view(left), rv = boundary_view(right);
    const std::size_t nb = sched.blocks.size();
    std::vector<std::vector<double>> part(nb);
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < int(nb); ++b) {
        const MPSBlock& blk = sched.blocks[b];
        if (blk.data.empty()) continue;
        part[b].assign(n_terms, 0.0);
        TList T = blk.create_T(rv, x);
        for (const Cohort& c : blk.data) {
            if (!ybar[c.rb]) continue;
            // Sbar (K x stripe) = L_eff^T ybar[lb_out], L_eff (ls_out x K) as contract uses it
            const int M = int(c.rs), N = int(c.stripe), K = int(c.nSrows * c.ls);
            const double* luse = lv[c.ci_eff];
            std::vector<double> lbuf;
            if (c.ci != c.ci_eff) {
                lbuf.resize(std::size_t(M) * K);
                tr_tile_v(c.ls, c.rs, c.nSrows, lv[c.ci_eff], lbuf.data());
                luse = lbuf.data();
            }
            std::vector<double> sbar(std::size_t(K) * N);
            dgemm('T', 'N', K, N, M, 1.0, luse, M, ybar[c.rb], M, 0.0, sbar.data(), K);
            // create_s_r's element map: S[K (offset + col) + bb ls + i] += alpha T[ti][(tidx1 + col) ls + i]
            for (const SUnit& u : c.suv) {
                if (u.alpha.empty()) continue;
                if (u.term.size() != u.alpha.size()) throw std::runtime_error("scale_gradient: schedule without term records");
                unsigned seeker = 0;
                for (std::size_t l = 0; l < u.b2s.size(); ++l) {
                    const std::size_t bb = u.b1[l];
                    for (unsigned ia = seeker; ia < seeker + u.b2s[l]; ++ia) {
                        const std::vector<double>& Tt = T[u.tidx[2 * ia]];
                        const std::size_t t1 = u.tidx[2 * ia + 1];
                        double abar = 0.0;
                        for (unsigned col = 0; col < u.ms; ++col) {
                            const double* sp = sbar.data() + std::size_t(K) * (u.offset + col) + bb * c.ls;
                            const double* tp = Tt.data() + (t1 + col) * c.ls;
                            for (unsigned i = 0; i < c.ls; ++i) abar += sp[i] * tp[i];
                        }
                        part[b][u.term[ia]] += abar * u.dalpha[ia];
                    }
                    seeker += u.b2s[l];
                }
            }
        }
    }
    grad.assign(n_terms, 0.0);
    for (std::size_t b = 0; b < nb; ++b)
        if (!part[b].empty())
            for (std::size_t e = 0; e < n_terms; ++e) grad[e] += part[b][e];
}

Boundary overlap_mpo_left_step(const MPSTensor& bra_in, const MPSTensor& ket_in, const Boundary& left, const MPOTensor& mpo,
                               bool symmetric) {
    MPSTensor bra = bra_in, ket = ket_in;
    ket.make_right_paired();
    bra.make_left_paired();
    const Index& physical_i = ket.phys;
    const Index& ket_right_i = ket.right;
    const Index& bra_right_i = bra.right;
    ProductBasis bra_right_pb(physical_i, bra.left);
    ProductBasis ket_right_pb(physical_i, ket_right_i, true);
    Schedule tasks;
    tasks.lr_ket_sizes = ket_right_i.sizes();
    tasks.blocks.resize(ket_right_i.size());
    for (unsigned rb = 0; rb < ket_right_i.size(); ++rb) {
        auto& blk = tasks.blocks[rb];
        blk.lr_ket_sizes = &tasks.lr_ket_sizes;
        blk.left_rt = blk.right_rt = &left.index;
        blk.rb_ket = rb;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int rb = 0; rb < int(ket_right_i.size()); ++rb) {
        lshtm_t_tasks(left.index, ket.left, ket_right_i, physical_i, ket_right_pb, unsigned(rb), tasks.blocks[rb]);
        lshtm_tasks(mpo, bra, ket, left.index, bra_right_pb, ket_right_pb, unsigned(rb), tasks.blocks[rb], symmetric);
    }
    Boundary ret;
    ret.index = BoundaryIndex(bra_right_i, ket_right_i);
    for (unsigned rb = 0; rb < ket_right_i.size(); ++rb)
        for (auto& e : tasks.blocks[rb].data) ret.index.add_cohort(e.lb, rb, e.mpo_offsets);
    if (symmetric) ret.index.complement_transpose(mpo.herm_right, mpo.phase_right, true);
    ret.allocate_all();
    std::vector<const double*> kv = block_view(ket, ket.left, true);
    std::vector<const double*> lv = boundary_view(left);
#pragma omp parallel for schedule(dynamic, 1)
    for (int rb = 0; rb < int(ket_right_i.size()); ++rb) {
        const MPSBlock& blk = tasks.blocks[rb];
        if (blk.data.empty()) continue;
        TList T = blk.create_T_left(lv, kv);
        for (const Cohort& c : blk.data) {
            unsigned ci = ret.index.cohort_index_pos(c.lb, unsigned(rb));
            Q rc_bra = bra_right_i[c.lb].first;
            std::size_t k = bra.data.find(rc_bra, rc_bra);
            c.prop_l(bra.data.b[k].d.data(), T, ret.data[ci].data());
        }
    }
    return ret;
}

Boundary overlap_mpo_right_step(const MPSTensor& bra_in, const MPSTensor& ket_in, const Boundary& right,
                                const MPOTensor& mpo, bool symmetric) {
    MPSTensor bra = bra_in, ket = ket_in;
    ket.make_right_paired();
    bra.make_right_paired();
    const Index& physical_i = bra.phys;
    const Index& bra_left_i = bra.left;
    const Index& bra_right_i = bra.right;
    const Index& ket_left_i = ket.left;
    ProductBasis bra_right_pb(physical_i, bra_right_i, true);
    Schedule tasks;
    tasks.lr_ket_sizes = ket_left_i.sizes();
    tasks.blocks.resize(ket_left_i.size());
    for (unsigned lb = 0; lb < ket_left_i.size(); ++lb) {
        auto& blk = tasks.blocks[lb];
        blk.lr_ket_sizes = &tasks.lr_ket_sizes;
        blk.left_rt = blk.right_rt = &right.index;
        blk.rb_ket = lb;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int lb = 0; lb < int(ket_left_i.size()); ++lb) {
        rshtm_t_tasks(right.index, bra_left_i, bra_right_i, physical_i, bra_right_pb, unsigned(lb), tasks.blocks[lb]);
        rshtm_tasks(mpo, right.index, bra_left_i, bra_right_i, physical_i, bra_right_pb, unsigned(lb), tasks.blocks[lb], symmetric);
    }
    Boundary ret;
    ret.index = BoundaryIndex(ket_left_i, bra_left_i);
    for (unsigned lb = 0; lb < ket_left_i.size(); ++lb)
        for (auto& e : tasks.blocks[lb].data) ret.index.add_cohort(lb, e.rb, e.mpo_offsets);
    ret.index.complement_transpose(mpo.herm_left, mpo.phase_left, false);
    ret.allocate_all();
    std::vector<const double*> kv = block_view(ket, ket.left, true);
    std::vector<const double*> rv = boundary_view(right);
#pragma omp parallel for schedule(dynamic, 1)
    for (int lb = 0; lb < int(ket_left_i.size()); ++lb) {
        const MPSBlock& blk = tasks.blocks[lb];
        if (blk.data.empty()) continue;
        TList T = blk.create_T(rv, kv);
        for (const Cohort& c : blk.data) {
            unsigned ci = ret.index.cohort_index_pos(unsigned(lb), c.rb);
            Q lc_bra = bra_left_i[c.rb].first;
            std::size_t k = bra.data.find(lc_bra, lc_bra);
            c.prop_r(bra.data.b[k].d.data(), T, ret.data[ci].data());
        }
    }
    return ret;
}

// move_boundary.hpp:37-89: schedule of the left step with bra = ket and no Hermitian
// skip, then lbtm of every cohort into the dm block of its bra right sector
void alpha_dm_direct(const MPSTensor& ket_in, const Boundary& left, const MPOTensor& mpo, BlockMatrix& dm, double alpha) {
    MPSTensor ket = ket_in;
    ket.make_right_paired();
    const Index& physical_i = ket.phys;
    const Index& left_i = ket.left;
    Index right_i = ket.right, out_left_i = physical_i * left_i;
    common_subset(out_left_i, right_i);
    ProductBasis left_pb(physical_i, left_i);
    ProductBasis right_pb(physical_i, right_i, true);
    MPSTensor view = ket;  // lshtm_tasks reads the indices from the tensors
    view.right = right_i;
    Schedule tasks;
    tasks.lr_ket_sizes = right_i.sizes();
    tasks.blocks.resize(right_i.size());
    for (unsigned rb = 0; rb < right_i.size(); ++rb) {
        auto& blk = tasks.blocks[rb];
        blk.lr_ket_sizes = &tasks.lr_ket_sizes;
        blk.left_rt = blk.right_rt = &left.index;
        blk.rb_ket = rb;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int rb = 0; rb < int(right_i.size()); ++rb) {
        lshtm_t_tasks(left.index, left_i, right_i, physical_i, right_pb, unsigned(rb), tasks.blocks[rb]);
        lshtm_tasks(mpo, view, view, left.index, left_pb, right_pb, unsigned(rb), tasks.blocks[rb], false);
    }
    std::vector<const double*> kv = block_view(ket, ket.left, true);
    std::vector<const double*> lv = boundary_view(left);
    // per-cohort products in parallel, added to dm in (rb_ket, cohort) order
    std::vector<std::vector<std::pair<std::size_t, std::vector<double>>>> part(right_i.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int rb = 0; rb < int(right_i.size()); ++rb) {
        const MPSBlock& blk = tasks.blocks[rb];
        if (blk.data.empty()) continue;
        TList T = blk.create_T_left(lv, kv);
        for (const Cohort& c : blk.data) {
            std::size_t k = dm.find(right_i[c.lb].first, right_i[c.lb].first);
            if (k == dm.n_blocks()) throw std::runtime_error("alpha_dm_direct: missing dm block");
            std::vector<double> acc(dm.b[k].d.size(), 0.0);
            c.lbtm(T, acc.data(), alpha);
            part[rb].push_back({k, std::move(acc)});
        }
    }
    for (auto& pr : part)
        for (auto& e : pr) daxpy(e.second.size(), 1.0, e.second.data(), dm.b[e.first].d.data());
}

// move_boundary.hpp:91-145
void alpha_dm_direct_right(const MPSTensor& ket_in, const Boundary& right, const MPOTensor& mpo, BlockMatrix& dm, double alpha) {
    MPSTensor ket = ket_in;
    ket.make_right_paired();
    const Index& physical_i = ket.phys;
    const Index& right_i = ket.right;
    const Index& left_i = ket.left;
    ProductBasis right_pb(physical_i, right_i, true);
    Schedule tasks;
    tasks.lr_ket_sizes = left_i.sizes();
    tasks.blocks.resize(left_i.size());
    for (unsigned lb = 0; lb < left_i.size(); ++lb) {
        auto& blk = tasks.blocks[lb];
        blk.lr_ket_sizes = &tasks.lr_ket_sizes;
        blk.left_rt = blk.right_rt = &right.index;
        blk.rb_ket = lb;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int lb = 0; lb < int(left_i.size()); ++lb) {
        rshtm_t_tasks(right.index, left_i, right_i, physical_i, right_pb, unsigned(lb), tasks.blocks[lb]);
        rshtm_tasks(mpo, right.index, left_i, right_i, physical_i, right_pb, unsigned(lb), tasks.blocks[lb], false);
    }
    std::vector<const double*> kv = block_view(ket, ket.left, true);
    std::vector<const double*> rv = boundary_view(right);
    std::vector<std::vector<std::pair<std::size_t, std::vector<double>>>> part(left_i.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int lb = 0; lb < int(left_i.size()); ++lb) {
        const MPSBlock& blk = tasks.blocks[lb];
        if (blk.data.empty()) continue;
        TList T = blk.create_T(rv, kv);
        for (const Cohort& c : blk.data) {
            std::size_t k = dm.find(left_i[c.rb].first, left_i[c.rb].first);
            if (k == dm.n_blocks()) throw std::runtime_error("alpha_dm_direct_right: missing dm block");
            std::vector<double> acc(dm.b[k].d.size(), 0.0);
            c.rbtm(T, acc.data(), alpha);
            part[lb].push_back({k, std::move(acc)});
        }
    }
    for (auto& pr : part)
        for (auto& e : pr) daxpy(e.second.size(), 1.0, e.second.data(), dm.b[e.first].d.data());
}

}  // namespace orc
