// Boundary propagation on the device (overlap_mpo_left/right_step,
// contractions/boundary_ops/move_boundary.hpp:147-404).
//
// Right step (rshtm_t_tasks / rshtm_tasks, right_tasks.hpp:39-167; prop_r, tasks.cpp:243-284):
//   T = ket_slab * R_old[ci_eff]          -> grouped T-GEMM (same kernel as H_eff)
//   S = sum alpha * T slices               -> unit S-GEMM (same kernel as H_eff)
//   R_new[b] = S_b * bra^T                 -> batched GEMM, one job per MPO row block
// Left step (lshtm_t_tasks / lshtm_tasks, left_tasks.hpp:38-172; create_T_left,
// create_s, prop_l, tasks.cpp:198-241, 425-454, 545-601):
//   T_b = L_old[ci_eff]_b(^T) * ket_slab   -> batched GEMM, one job per (T job, MPO block)
//   S (stripe x nS*rs_ket) = sum alpha * T slices  -> unit S-GEMM with the left layout
//   L_new = bra^T * S                      -> batched GEMM, one job per cohort
// Cohort offsets follow Cohort::finalize (tasks.cpp:506-526): MPO indices with
// coefficients get consecutive block positions in index order.
#include <algorithm>
#include <cstdlib>
#include <stdexcept>
#include <unordered_map>

#include "dmrg_dev.hpp"

namespace qcm {

namespace {
constexpr uint32_t NONE = 0xffffffffu;

void add_tiles(std::vector<TileD>* tiles, uint32_t item, uint32_t M, uint32_t N) {
    int sh = shape_for_rows(M);
    uint32_t bm = shape_bm(sh), bn = shape_bn(sh);
    for (uint32_t n0 = 0; n0 < N; n0 += bn)
        for (uint32_t m0 = 0; m0 < M; m0 += bm) tiles[sh].push_back(TileD{item, m0, n0, 0});
}
}  // namespace

void SBuild::add_unit(uint64_t s_off, uint64_t line_stride, uint32_t erows, uint32_t col_stride, uint32_t ne,
                      const std::vector<uint32_t>& lines, const std::vector<E>& ents) {
    if (ents.empty() || ne == 0) return;
    std::unordered_map<uint64_t, uint32_t> kid;
    std::vector<uint64_t> slices;
    std::vector<uint32_t> ek(ents.size());
    for (std::size_t i = 0; i < ents.size(); ++i) {
        auto ins = kid.emplace(ents[i].slice, uint32_t(slices.size()));
        if (ins.second) slices.push_back(ents[i].slice);
        ek[i] = ins.first->second;
    }
    UnitD u{};
    u.s_off = s_off; u.line_stride = line_stride; u.erows = erows; u.col_stride = col_stride; u.ne = ne;
    u.nl = uint32_t(lines.size()); u.line0 = uint32_t(line_b1.size());
    u.nk = uint32_t(slices.size()); u.slice0 = uint32_t(slice_off.size()); u.sptr0 = uint32_t(sptr.size());
    line_b1.insert(line_b1.end(), lines.begin(), lines.end());
    slice_off.insert(slice_off.end(), slices.begin(), slices.end());
    std::vector<uint32_t> cnt(u.nk + 1, 0);
    for (uint32_t k : ek) cnt[k + 1]++;
    for (uint32_t k = 0; k < u.nk; ++k) cnt[k + 1] += cnt[k];
    const uint32_t w0 = uint32_t(went.size());
    for (uint32_t k = 0; k <= u.nk; ++k) sptr.push_back(w0 + cnt[k]);
    went.resize(w0 + ents.size());
    std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
    for (std::size_t i = 0; i < ents.size(); ++i) went[w0 + fill[ek[i]]++] = WEntD{ents[i].line, ek[i], ents[i].a};
    int sh = shape_for_rows(u.nl);
    uint32_t bm = shape_bm(sh), bn = shape_bn(sh);
    for (uint32_t n0 = 0; n0 < u.ne; n0 += bn)
        for (uint32_t m0 = 0; m0 < u.nl; m0 += bm) utiles[sh].push_back(TileD{uint32_t(units.size()), m0, n0, 0});
    units.push_back(u);
}

void SBuild::validate(uint64_t t_len, uint64_t s_len) const {
    for (const UnitD& u : units) {
        if (!u.ne || !u.nl) continue;
        if (u.erows == 0 || u.ne % u.erows) throw std::runtime_error("S unit: element count is not a whole number of columns");
        uint32_t maxline = 0;
        for (uint32_t l = 0; l < u.nl; ++l) maxline = std::max(maxline, line_b1[u.line0 + l]);
        const uint64_t last = u.s_off + uint64_t(maxline) * u.line_stride + (u.erows - 1) + uint64_t(u.ne / u.erows - 1) * u.col_stride;
        if (last >= s_len) throw std::runtime_error("device work list out of bounds: S unit");
        for (uint32_t k = 0; k < u.nk; ++k)
            if (slice_off[u.slice0 + k] + u.ne > t_len) throw std::runtime_error("device work list out of bounds: T slice");
        for (uint32_t w = sptr[u.sptr0]; w < sptr[u.sptr0 + u.nk]; ++w)
            if (went[w].line >= u.nl || went[w].k >= u.nk) throw std::runtime_error("S unit: coefficient index out of range");
    }
}

void SBuild::upload(cudaStream_t s) {
    d_units.upload(units, s);
    for (int k = 0; k < N_SHAPES; ++k) d_utiles[k].upload(utiles[k], s);
    d_line_b1.upload(line_b1, s);
    d_sptr.upload(sptr, s);
    d_slice_off.upload(slice_off, s);
    d_went.upload(went, s);
}

void complement_transpose(BoundaryIndexH& x, const std::vector<int32_t>& herm, const std::vector<int32_t>& phase, bool forward) {
    // rebuild the (bra, ket) -> cohort map, add transposed partners, fill Hermitian blocks
    const uint32_t n0 = x.n_cohorts();
    auto lookup = [&](uint32_t a, uint32_t b) -> uint32_t {
        for (uint32_t ci = 0; ci < x.n_cohorts(); ++ci) if (x.cbra[ci] == a && x.cket[ci] == b) return ci;
        return NONE;
    };
    for (uint32_t ciA = 0; ciA < n0; ++ciA) {
        Charge lb = x.bra[x.cbra[ciA]].first, rb = x.ket[x.cket[ciA]].first;
        std::size_t pb = x.bra.position(rb), pk = x.ket.position(lb);
        if (pb >= x.bra.size() || pk >= x.ket.size()) continue;
        uint32_t ciB = lookup(uint32_t(pb), uint32_t(pk));
        if (ciB == NONE) {
            ciB = x.n_cohorts();
            x.cbra.push_back(uint32_t(pb)); x.cket.push_back(uint32_t(pk));
            x.lsz.push_back(uint32_t(x.bra[pb].second)); x.rsz.push_back(uint32_t(x.ket[pk].second));
            x.nb.push_back(0); x.tr.push_back(1);
            x.offsets.resize(x.offsets.size() + x.aux, -1);
            x.cscale.resize(x.cscale.size() + x.aux, 1.0);
        }
        for (uint32_t b = 0; b < x.aux; ++b) {
            // Hermitian::skip(b, ket charge, bra charge): l < r and b has a partner
            if (rb < lb && herm[b] >= 0) {
                x.offsets[std::size_t(ciB) * x.aux + b] = x.offsets[std::size_t(ciA) * x.aux + uint32_t(herm[b])];
                x.cscale[std::size_t(ciB) * x.aux + b] = double(phase[forward ? b : uint32_t(herm[b])]);
            }
        }
    }
}

namespace {

// T job extents: psi slab (a), boundary cohort (b: N/brs blocks of K x brs) and T output
void validate_tjobs(const std::vector<TJobD>& jobs, uint64_t a_len, uint64_t b_len, uint64_t t_len) {
    for (const TJobD& j : jobs) {
        check_extent(j.a_off, j.M, j.K, j.lda, a_len, "T-GEMM psi slab");
        if (j.N && j.K && j.b_off + uint64_t(j.N) * j.K > b_len) throw std::runtime_error("device work list out of bounds: T-GEMM boundary");
        if (j.brs == 0 || j.N % j.brs) throw std::runtime_error("T job: width is not a whole number of blocks");
        if (j.c_off + uint64_t(j.M) * j.N > t_len) throw std::runtime_error("device work list out of bounds: T output");
    }
}

std::unique_ptr<DevBoundary> finish_boundary(BoundaryIndexH& idx, cudaStream_t s) {
    auto B = std::make_unique<DevBoundary>();
    idx.finish();
    B->idx = std::move(idx);
    B->data.alloc(B->idx.total ? B->idx.total : 1);
    QCM_CUDA(cudaMemsetAsync(B->data.get(), 0, (B->idx.total ? B->idx.total : 1) * sizeof(double), s));
    return B;
}

}  // namespace

// ---------------------------------------------------------------------------
std::unique_ptr<DevBoundary> boundary_step_right(Ctx& c, const DevBoundary& Rold, const DMPS& ket, const MPOTensor& W,
                                                 bool symmetric) {
    if (!ket.right_paired) throw std::runtime_error("boundary_step_right: ket must be right-paired");
    const BoundaryIndexH& R = Rold.idx;
    const Index& phys = ket.phys;
    const Index& left = ket.left;
    const Index& right = ket.right;
    ProductBasis rpb(phys, right, true);
    StateMap sm(phys);
    const uint32_t nl = uint32_t(left.size()), nst = uint32_t(sm.nstates());
    // block offsets of the (right-paired) ket per left sector
    std::vector<uint64_t> koff(nl, 0);
    std::vector<uint32_t> kcols(nl, 0);
    std::vector<bool> kok(nl, false);
    for (uint32_t lb = 0; lb < nl; ++lb) {
        std::size_t k = ket.b.find_l(left[lb].first);
        if (k < ket.b.n()) { koff[lb] = ket.b.off[k]; kcols[lb] = ket.b.cols[k]; kok[lb] = true; }
    }
    std::vector<TJobD> tjobs;
    std::vector<TileD> ttiles[N_SHAPES];
    uint64_t t_len = 0;
    SBuild sb;
    uint64_t s_len = 0;
    std::vector<GemmJob> prop;
    BoundaryIndexH nidx;
    nidx.bra = left; nidx.ket = left; nidx.aux = W.rows;
    struct Pending { uint64_t s_off; uint32_t lb_ket, lb_bra, nS; std::vector<int64_t> offs; };
    std::vector<Pending> pend;
    for (uint32_t lb_ket = 0; lb_ket < nl; ++lb_ket) {
        if (!kok[lb_ket]) continue;
        const Charge lc_ket = left[lb_ket].first;
        const uint32_t ls_ket = uint32_t(left[lb_ket].second);
        // T jobs (rshtm_t_tasks): (mps offset, ci) -> job
        std::unordered_map<uint64_t, uint32_t> tmap;
        for (uint32_t s = 0; s < phys.size(); ++s) {
            Charge rc_ket = lc_ket + phys[s].first;
            std::size_t rbk = right.position(rc_ket);
            if (rbk == right.size()) continue;
            uint32_t rs_ket = uint32_t(right[rbk].second), koff_s = uint32_t(rpb(phys[s].first, rc_ket));
            for (std::size_t rbb = 0; rbb < right.size(); ++rbb) {
                uint32_t ci = R.cohort_index(rc_ket, right[rbb].first);
                if (ci == R.n_cohorts()) continue;
                uint32_t ce = R.tr[ci] ? R.cohort_index(right[rbb].first, rc_ket) : ci;
                for (uint32_t ss = 0; ss < phys[s].second; ++ss) {
                    uint32_t mo = koff_s + ss * rs_ket;
                    TJobD j{};
                    j.a_off = koff[lb_ket] + uint64_t(mo) * ls_ket;
                    j.b_off = Rold.idx.data_off[ce];
                    j.c_off = t_len;
                    j.M = ls_ket; j.K = rs_ket; j.brs = R.rsz[ci]; j.N = R.nb[ce] * j.brs; j.lda = ls_ket;
                    j.tr = ci != ce;
                    tmap.emplace((uint64_t(mo) << 32) | ci, uint32_t(tjobs.size()));
                    t_len += (uint64_t(j.M) * j.N + 31) / 32 * 32;
                    if (j.M && j.N) add_tiles(ttiles, uint32_t(tjobs.size()), j.M, j.N);
                    tjobs.push_back(j);
                }
            }
        }
        // cohorts (rshtm_tasks)
        for (uint32_t lb_bra = 0; lb_bra < nl; ++lb_bra) {
            const Charge lc_bra = left[lb_bra].first;
            if (std::abs(lc_ket.particles() - lc_bra.particles()) > 2) continue;
            if (!kok[lb_bra]) continue;
            const uint32_t ls_bra = uint32_t(left[lb_bra].second);
            struct U { uint32_t st, offset, ms; std::vector<std::pair<uint32_t, SBuild::E>> em; };
            std::vector<U> units;
            std::vector<int> unit_of(nst, -1);
            uint32_t stripe = 0;
            for (uint32_t st = 0; st < nst; ++st) {
                Charge rc_bra = lc_bra + phys[sm.sector[st]].first;
                std::size_t rbb = right.position(rc_bra);
                if (rbb == right.size()) continue;
                uint32_t rs = uint32_t(right[rbb].second);
                unit_of[st] = int(units.size());
                units.push_back(U{st, uint32_t(rpb(phys[sm.sector[st]].first, rc_bra)) + uint32_t(sm.sub[st]) * rs, rs, {}});
                stripe += rs;
            }
            std::vector<uint32_t> line_count(W.rows, 0);
            for (uint32_t b1 = 0; b1 < W.rows; ++b1) {
                if (symmetric && lc_ket < lc_bra && W.herm_left[b1] >= 0) continue;
                for (uint32_t e = W.row_ptr[b1]; e < W.row_ptr[b1 + 1]; ++e) {
                    const uint32_t b2 = W.b2[e];
                    const SparseOp& op = (*W.ops)[W.op[e]];
                    for (std::size_t k = 0; k < op.val.size(); ++k) {
                        int u = unit_of[op.out[k]];
                        if (u < 0) continue;
                        const uint32_t sti = op.in[k];
                        Charge rc_ket = lc_ket + phys[sm.sector[sti]].first;
                        Charge rc_bra = lc_bra + phys[sm.sector[units[u].st]].first;
                        uint32_t ci = R.cohort_index(rc_ket, rc_bra);
                        if (!R.has_block(ci, b2)) continue;
                        std::size_t rbk = right.position(rc_ket);
                        if (rbk == right.size()) continue;
                        uint32_t rs_ket = uint32_t(right[rbk].second);
                        uint32_t mo = uint32_t(rpb(phys[sm.sector[sti]].first, rc_ket)) + uint32_t(sm.sub[sti]) * rs_ket;
                        auto it = tmap.find((uint64_t(mo) << 32) | ci);
                        if (it == tmap.end()) continue;
                        uint32_t col = uint32_t(R.offset(ci, b2) / rs_ket);
                        double a = op.val[k] * R.conj_scale(ci, b2) * W.scale[e];
                        units[u].em.push_back({b1, SBuild::E{0, tjobs[it->second].c_off + uint64_t(col) * ls_ket, a}});
                        line_count[b1]++;
                    }
                }
            }
            // finalize: MPO rows with coefficients get consecutive positions
            std::vector<uint32_t> pos(W.rows, NONE);
            uint32_t nS = 0;
            for (uint32_t b1 = 0; b1 < W.rows; ++b1) if (line_count[b1]) pos[b1] = nS++;
            if (nS == 0) continue;
            const uint32_t K_c = nS * ls_ket;
            const uint64_t s_off = s_len;
            s_len += (uint64_t(K_c) * stripe + 31) / 32 * 32;
            for (U& u : units) {
                if (u.em.empty()) continue;
                std::vector<uint32_t> lines;
                std::vector<SBuild::E> ents;
                for (auto& pe : u.em) {
                    uint32_t p = pos[pe.first];
                    if (lines.empty() || lines.back() != p) lines.push_back(p);
                    SBuild::E e = pe.second;
                    e.line = uint32_t(lines.size() - 1);
                    ents.push_back(e);
                }
                sb.add_unit(s_off + uint64_t(u.offset) * K_c, ls_ket, ls_ket, K_c, ls_ket * u.ms, lines, ents);
            }
            Pending pd{s_off, lb_ket, lb_bra, nS, std::vector<int64_t>(W.rows, -1)};
            for (uint32_t b1 = 0; b1 < W.rows; ++b1)
                if (pos[b1] != NONE) pd.offs[b1] = int64_t(pos[b1]) * ls_ket * ls_bra;
            pend.push_back(std::move(pd));
        }
    }
    // new boundary index (BoundaryIndex(ket_left_i, bra_left_i), add_cohort(lb_ket, rb))
    for (auto& pd : pend) {
        nidx.cbra.push_back(pd.lb_ket); nidx.cket.push_back(pd.lb_bra);
        nidx.lsz.push_back(uint32_t(left[pd.lb_ket].second)); nidx.rsz.push_back(uint32_t(left[pd.lb_bra].second));
        nidx.nb.push_back(pd.nS); nidx.tr.push_back(0);
        nidx.offsets.insert(nidx.offsets.end(), pd.offs.begin(), pd.offs.end());
        nidx.cscale.insert(nidx.cscale.end(), W.rows, 1.0);
    }
    complement_transpose(nidx, W.herm_left, W.phase_left, false);
    auto Rn = finish_boundary(nidx, c.s);
    // execute
    Ctx::ensure(c.T, t_len ? t_len : 1);
    Ctx::ensure(c.S, s_len ? s_len : 1);
    validate_tjobs(tjobs, ket.b.total, Rold.idx.total, t_len);
    sb.validate(t_len, s_len);
    c.tjobs.upload(tjobs, c.s);
    for (int k = 0; k < N_SHAPES; ++k) c.ttiles[k].upload(ttiles[k], c.s);
    sb.upload(c.s);
    run_tgemm(c.tjobs.get(), c.ttiles, ttiles, ket.b.d.get(), Rold.data.get(), c.T.get(), c.s);
    if (s_len) QCM_CUDA(cudaMemsetAsync(c.S.get(), 0, s_len * sizeof(double), c.s));
    run_sgemm(sb.d_units.get(), sb.d_utiles, sb.utiles, sb.d_line_b1.get(), sb.d_slice_off.get(), sb.d_sptr.get(),
              sb.d_went.get(), c.T.get(), c.S.get(), c.s);
    // prop_r: new_R[b] (ls_ket x ls_bra) = S_b * bra^T
    for (std::size_t i = 0; i < pend.size(); ++i) {
        const Pending& pd = pend[i];
        const uint32_t ls = uint32_t(left[pd.lb_ket].second), lsb = uint32_t(left[pd.lb_bra].second);
        const uint32_t ci = Rn->idx.cohort_index(left[pd.lb_ket].first, left[pd.lb_bra].first);
        const uint32_t stripe = kcols[pd.lb_bra];
        for (uint32_t b = 0; b < pd.nS; ++b) {
            GemmJob g{};
            g.a_off = pd.s_off + uint64_t(b) * ls; g.lda = pd.nS * ls;
            g.b_off = koff[pd.lb_bra]; g.ldb = lsb; g.tb = 1;
            g.c_off = Rn->idx.data_off[ci] + uint64_t(b) * ls * lsb; g.ldc = ls;
            g.M = ls; g.N = lsb; g.K = stripe; g.alpha = 1.0; g.beta = 0.0;
            prop.push_back(g);
        }
    }
    // A = S scratch, B = ket data, C = new boundary: three different base pointers
    batched_gemm(prop, c.S.get(), s_len, ket.b.d.get(), ket.b.total, Rn->data.get(), Rn->idx.total, c.gjobs, c.gtiles, c.s);
    return Rn;
}

// ---------------------------------------------------------------------------
std::unique_ptr<DevBoundary> boundary_step_left(Ctx& c, const DevBoundary& Lold, const DMPS& ket, const DMPS& bra,
                                                const MPOTensor& W, bool symmetric) {
    if (!ket.right_paired || bra.right_paired) throw std::runtime_error("boundary_step_left: ket right-paired, bra left-paired");
    const BoundaryIndexH& L = Lold.idx;
    const Index& phys = ket.phys;
    const Index& left = ket.left;
    const Index& right = ket.right;
    ProductBasis kpb(phys, right, true);  // ket right-paired columns
    ProductBasis bpb(phys, left);         // bra left-paired rows
    StateMap sm(phys);
    const uint32_t nl = uint32_t(left.size()), nr = uint32_t(right.size()), nst = uint32_t(sm.nstates());
    std::vector<uint64_t> koff(nl, 0), boff(nr, 0);
    std::vector<bool> kok(nl, false), bok(nr, false);
    std::vector<uint32_t> brows(nr, 0);
    for (uint32_t lb = 0; lb < nl; ++lb) {
        std::size_t k = ket.b.find_l(left[lb].first);
        if (k < ket.b.n()) { koff[lb] = ket.b.off[k]; kok[lb] = true; }
    }
    for (uint32_t rb = 0; rb < nr; ++rb) {
        std::size_t k = bra.b.find_r(right[rb].first);
        if (k < bra.b.n()) { boff[rb] = bra.b.off[k]; brows[rb] = bra.b.rows[k]; bok[rb] = true; }
    }
    std::vector<GemmJob> tj_gemm, prop;
    uint64_t t_len = 0, s_len = 0;
    SBuild sb;
    BoundaryIndexH nidx;
    nidx.bra = right; nidx.ket = right; nidx.aux = W.cols;
    for (uint32_t rb_ket = 0; rb_ket < nr; ++rb_ket) {
        const Charge rc_ket = right[rb_ket].first;
        const uint32_t rs_ket = uint32_t(right[rb_ket].second);
        // T jobs (lshtm_t_tasks): T[ti] = nb blocks of ls_bra x rs_ket
        std::unordered_map<uint64_t, uint64_t> tmap;  // (mps offset, ci) -> T offset
        for (uint32_t s = 0; s < phys.size(); ++s) {
            Charge lc_ket = rc_ket + (-phys[s].first);
            std::size_t lbk = left.position(lc_ket);
            if (lbk == left.size() || !kok[lbk]) continue;
            const uint32_t ls_ket = uint32_t(left[lbk].second);
            const uint32_t ko = uint32_t(kpb(phys[s].first, rc_ket));
            for (uint32_t lb_bra = 0; lb_bra < nl; ++lb_bra) {
                uint32_t ci = L.cohort_index(left[lb_bra].first, lc_ket);
                if (ci == L.n_cohorts()) continue;
                uint32_t ce = L.tr[ci] ? L.cohort_index(lc_ket, left[lb_bra].first) : ci;
                const uint32_t ls_bra = uint32_t(left[lb_bra].second), nb = L.nb[ce];
                for (uint32_t ss = 0; ss < phys[s].second; ++ss) {
                    const uint32_t mo = ko + ss * rs_ket;
                    const uint64_t c_off = t_len;
                    tmap.emplace((uint64_t(mo) << 32) | ci, c_off);
                    t_len += (uint64_t(ls_bra) * rs_ket * nb + 31) / 32 * 32;
                    for (uint32_t b = 0; b < nb; ++b) {
                        GemmJob g{};
                        g.a_off = Lold.idx.data_off[ce] + uint64_t(b) * ls_bra * ls_ket;
                        g.ta = (ci != ce); g.lda = g.ta ? ls_ket : ls_bra;
                        g.b_off = koff[lbk] + uint64_t(mo) * ls_ket; g.ldb = ls_ket;
                        g.c_off = c_off + uint64_t(b) * ls_bra * rs_ket; g.ldc = ls_bra;
                        g.M = ls_bra; g.N = rs_ket; g.K = ls_ket; g.alpha = 1.0; g.beta = 0.0;
                        tj_gemm.push_back(g);
                    }
                }
            }
        }
        // cohorts (lshtm_tasks)
        for (uint32_t rb_bra = 0; rb_bra < nr; ++rb_bra) {
            const Charge rc_bra = right[rb_bra].first;
            if (std::abs(rc_bra.particles() - rc_ket.particles()) > 2 || !bok[rb_bra]) continue;
            const uint32_t rs_bra = uint32_t(right[rb_bra].second), stripe = brows[rb_bra];
            struct U { uint32_t st, offset, ms; Charge lc_bra; std::vector<std::pair<uint32_t, SBuild::E>> em; };
            std::vector<U> units;
            std::vector<int> unit_of(nst, -1);
            for (uint32_t st = 0; st < nst; ++st) {
                Charge lc_bra = rc_bra + (-phys[sm.sector[st]].first);
                std::size_t lbb = left.position(lc_bra);
                if (lbb == left.size()) continue;
                uint32_t ls_bra = uint32_t(left[lbb].second);
                unit_of[st] = int(units.size());
                units.push_back(U{st, uint32_t(bpb(phys[sm.sector[st]].first, lc_bra)) + uint32_t(sm.sub[st]) * ls_bra, ls_bra, lc_bra, {}});
            }
            std::vector<uint32_t> line_count(W.cols, 0);
            for (uint32_t b2 = 0; b2 < W.cols; ++b2) {
                if (symmetric && rc_bra < rc_ket && W.herm_right[b2] >= 0) continue;
                for (uint32_t q = W.col_ptr[b2]; q < W.col_ptr[b2 + 1]; ++q) {
                    const uint32_t e = W.col_ent[q], b1 = W.b1[e];
                    const SparseOp& op = (*W.ops)[W.op[e]];
                    for (std::size_t k = 0; k < op.val.size(); ++k) {
                        int u = unit_of[op.out[k]];
                        if (u < 0) continue;
                        const uint32_t sti = op.in[k];
                        Charge lc_ket = rc_ket + (-phys[sm.sector[sti]].first);
                        std::size_t lbk = left.position(lc_ket);
                        if (lbk == left.size() || !kok[lbk]) continue;
                        uint32_t ci = L.cohort_index(units[u].lc_bra, lc_ket);
                        if (!L.has_block(ci, b1)) continue;
                        const uint32_t ls_ket = uint32_t(left[lbk].second);
                        const uint32_t mo = uint32_t(kpb(phys[sm.sector[sti]].first, rc_ket)) + uint32_t(sm.sub[sti]) * rs_ket;
                        auto it = tmap.find((uint64_t(mo) << 32) | ci);
                        if (it == tmap.end()) continue;
                        const uint32_t col = uint32_t(L.offset(ci, b1) / ls_ket);
                        const double a = op.val[k] * L.conj_scale(ci, b1) * W.scale[e];
                        units[u].em.push_back({b2, SBuild::E{0, it->second + uint64_t(col) * rs_ket, a}});
                        line_count[b2]++;
                    }
                }
            }
            std::vector<uint32_t> pos(W.cols, NONE);
            uint32_t nS = 0;
            for (uint32_t b2 = 0; b2 < W.cols; ++b2) if (line_count[b2]) pos[b2] = nS++;
            if (nS == 0) continue;
            const uint64_t s_off = s_len;
            s_len += (uint64_t(stripe) * nS * rs_ket + 31) / 32 * 32;
            for (U& u : units) {
                if (u.em.empty()) continue;
                std::vector<uint32_t> lines;
                std::vector<SBuild::E> ents;
                for (auto& pe : u.em) {
                    uint32_t p = pos[pe.first];
                    if (lines.empty() || lines.back() != p) lines.push_back(p);
                    SBuild::E e = pe.second;
                    e.line = uint32_t(lines.size() - 1);
                    ents.push_back(e);
                }
                sb.add_unit(s_off + u.offset, uint64_t(rs_ket) * stripe, u.ms, stripe, u.ms * rs_ket, lines, ents);
            }
            // new cohort (rb_bra, rb_ket): nS blocks rs_bra x rs_ket
            nidx.cbra.push_back(rb_bra); nidx.cket.push_back(rb_ket);
            nidx.lsz.push_back(rs_bra); nidx.rsz.push_back(rs_ket);
            nidx.nb.push_back(nS); nidx.tr.push_back(0);
            for (uint32_t b2 = 0; b2 < W.cols; ++b2)
                nidx.offsets.push_back(pos[b2] == NONE ? -1 : int64_t(pos[b2]) * rs_bra * rs_ket);
            nidx.cscale.insert(nidx.cscale.end(), W.cols, 1.0);
            GemmJob g{};
            g.a_off = boff[rb_bra]; g.ta = 1; g.lda = stripe;
            g.b_off = s_off; g.ldb = stripe;
            g.c_off = uint64_t(nidx.n_cohorts() - 1);  // cohort index, resolved after the index is final
            g.M = rs_bra; g.N = nS * rs_ket; g.K = stripe; g.alpha = 1.0; g.beta = 0.0;
            prop.push_back(g);
        }
    }
    if (symmetric) complement_transpose(nidx, W.herm_right, W.phase_right, true);
    auto Ln = finish_boundary(nidx, c.s);
    for (auto& g : prop) { g.ldc = uint32_t(g.M); g.c_off = Ln->idx.data_off[g.c_off]; }
    Ctx::ensure(c.T, t_len ? t_len : 1);
    Ctx::ensure(c.S, s_len ? s_len : 1);
    batched_gemm(tj_gemm, Lold.data.get(), Lold.idx.total, ket.b.d.get(), ket.b.total, c.T.get(), t_len, c.gjobs, c.gtiles, c.s);
    sb.validate(t_len, s_len);
    sb.upload(c.s);
    if (s_len) QCM_CUDA(cudaMemsetAsync(c.S.get(), 0, s_len * sizeof(double), c.s));
    run_sgemm(sb.d_units.get(), sb.d_utiles, sb.utiles, sb.d_line_b1.get(), sb.d_slice_off.get(), sb.d_sptr.get(),
              sb.d_went.get(), c.T.get(), c.S.get(), c.s);
    batched_gemm(prop, bra.b.d.get(), bra.b.total, c.S.get(), s_len, Ln->data.get(), Ln->idx.total, c.gjobs, c.gtiles, c.s);
    return Ln;
}

}  // namespace qcm
