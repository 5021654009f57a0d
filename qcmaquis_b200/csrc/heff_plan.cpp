// Host-side construction of the flattened H_eff plan.
//
// Same bookkeeping as create_contraction_schedule
// (create_schedule/site_hamil_schedule.hpp:42-93): T jobs as in rshtm_t_tasks
// (right_tasks.hpp:39-78) and cohort coefficients as in shtm_tasks +
// op_iterate (site_hamil_tasks.hpp:41-137, op_iterate.hpp:38-70) --
//   alpha = op coefficient * MPO scale * R.conjugate_scale(ci_right, b2)
//           * L.conjugate_scale(ci, b1),
//   T slice = (ket offset + ss1 * rs_in, ci_right), column right_offset / rs_in,
//   S row block = position of b1 in the L cohort, column = unit offset.
// The result is laid out as device work lists.  Every lookup the inner loop
// needs (sector offsets, cohort indices, T jobs) is a flat table built once per
// plan, and the ket sectors are processed in parallel (OpenMP) and merged in
// sector order, so the plan does not depend on the thread count.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <stdexcept>

#include "heff.hpp"

namespace qcm {

void BoundaryIndexH::finish() {
    lbrb.assign(bra.size(), std::vector<uint32_t>(ket.size(), n_cohorts()));
    for (uint32_t ci = 0; ci < n_cohorts(); ++ci) {
        if (cbra[ci] >= bra.size() || cket[ci] >= ket.size()) throw std::runtime_error("boundary: cohort sector out of range");
        lbrb[cbra[ci]][cket[ci]] = ci;
    }
    data_off.resize(n_cohorts());
    total = 0;
    for (uint32_t ci = 0; ci < n_cohorts(); ++ci) {
        data_off[ci] = total;
        total += (cohort_size(ci) + 31) / 32 * 32;  // 256-byte aligned cohorts
    }
}

HeffPlan::~HeffPlan() {
    if (graph) cudaGraphExecDestroy(graph);
}

namespace {

constexpr uint32_t NONE = 0xffffffffu;
// K rows per split-K item of the L.S GEMM (measured at L=24 M=512: 512 -> 1.06 ms, 1024 -> 0.77 ms,
// 2048 -> 0.84 ms, 4096 -> 1.28 ms: more partial tiles to reduce below, fewer concurrent items above)
constexpr uint32_t KCHUNK = 1024;

void add_tiles(std::vector<TileD>* tiles, uint32_t item, uint32_t M, uint32_t N) {
    int sh = shape_for_rows(M);
    uint32_t bm = shape_bm(sh), bn = shape_bn(sh);
    for (uint32_t n0 = 0; n0 < N; n0 += bn)
        for (uint32_t m0 = 0; m0 < M; m0 += bm) tiles[sh].push_back(TileD{item, m0, n0, 0});
}

struct RSec { uint32_t rb, rs, off; };  // right sector of (left sector, phys sector), column offset

// Everything one ket sector (lb_in) contributes; offsets relative to the part.
struct Part {
    std::vector<TJobD> tjobs;
    std::vector<uint32_t> tjob_mps;  // mps column offset of each job (bookkeeping)
    uint64_t t_len = 0;
    std::vector<UnitD> units;
    std::vector<uint32_t> line_b1, sptr;
    std::vector<uint64_t> slice_off;
    std::vector<WEntD> went;
    uint64_t s_len = 0, w_len = 0;
    std::vector<std::pair<uint32_t, SegD>> segs;
    double flops_t = 0, flops_s = 0, flops_ls = 0, flops_sdense = 0;
    uint64_t g_elems = 0, g_reads = 0;
    std::vector<uint32_t> bk_int;
    std::vector<double> bk_alpha;
};

struct Em { uint32_t line, slice; double a; uint32_t mps, cir, col; };
struct U { uint32_t st, offset, ms, rb_out; std::vector<Em> em; std::vector<uint32_t> lines; };

}  // namespace

void add_unit_tiles(const UnitD& u, uint32_t item, const WEntD* ents, std::size_t n, std::vector<TileD>* utiles,
                    std::vector<uint16_t>& klist) {
    if (!u.nl || !u.ne || !u.nk || !n) return;
    constexpr uint32_t KS = 16;  // k-step of the S-GEMM (dm::BK), four DMMA k-groups of 4 slices
    const uint32_t nks = (u.nk + KS - 1) / KS;
    if (nks >= 4096) throw std::runtime_error("S unit: too many slices for the k-step list");
    // occupancy of (16 lines x 4 slices) coefficient groups as a 4-bit mask per (16 lines x 16 slices)
    // block; coarser line tiles OR rows together
    const uint32_t n16 = (u.nl + 15) / 16;
    std::vector<uint8_t> occ16(std::size_t(n16) * nks, 0);
    for (std::size_t i = 0; i < n; ++i)
        occ16[std::size_t(ents[i].line / 16) * nks + ents[i].k / KS] |= uint8_t(1u << ((ents[i].k % KS) / 4));
    auto occ_at = [&](uint32_t bm, std::vector<uint8_t>& occ) {
        const uint32_t f = bm / 16, nmt = (u.nl + bm - 1) / bm;
        occ.assign(std::size_t(nmt) * nks, 0);
        for (uint32_t r = 0; r < n16; ++r)
            for (uint32_t ks = 0; ks < nks; ++ks) occ[std::size_t(r / f) * nks + ks] |= occ16[std::size_t(r) * nks + ks];
    };
    auto groups = [](uint8_t m) { return (m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1); };
    // candidate shapes and a relative cost per tensor flop (the 16-row shape runs 2 x 4 fragments per warp)
    static const int cand[4] = {SHAPE_16, SHAPE_32, SHAPE_64, SHAPE_128};
    static const double eff[4] = {1.3, 1.0, 1.0, 1.05};
    int best = -1;
    double best_cost = 0;
    std::vector<uint8_t> occ, best_occ;
    for (int ci = 0; ci < 4; ++ci) {
        const uint32_t bm = shape_bm(cand[ci]), bn = shape_bn(cand[ci]);
        const uint32_t nnt = (u.ne + bn - 1) / bn;
        occ_at(bm, occ);
        std::size_t on = 0;
        for (uint8_t o : occ) on += groups(o);
        const double cost = eff[ci] * double(on) * bm * 4.0 * double(nnt) * bn;
        if (best < 0 || cost < best_cost) { best = ci; best_cost = cost; best_occ.swap(occ); }
    }
    const int sh = cand[best];
    const uint32_t bm = shape_bm(sh), bn = shape_bn(sh), nmt = (u.nl + bm - 1) / bm;
    for (uint32_t mt = 0; mt < nmt; ++mt) {
        const uint32_t off = uint32_t(klist.size());
        klist.push_back(0);
        uint16_t cnt = 0;
        for (uint32_t ks = 0; ks < nks; ++ks) {
            const uint8_t m = best_occ[std::size_t(mt) * nks + ks];
            if (m) { klist.push_back(uint16_t((ks << 4) | m)); ++cnt; }
        }
        klist[off] = cnt;
        if (!cnt) continue;
        for (uint32_t n0 = 0; n0 < u.ne; n0 += bn) utiles[sh].push_back(TileD{item, mt * bm, n0, off});
    }
}

std::unique_ptr<HeffPlan> build_heff_plan(const DevBoundary& Lb, const DevBoundary& Rb, const MPOTensor& W,
                                          const Index& phys, const Index& left, const Index& right, bool bookkeeping) {
    const BoundaryIndexH& L = Lb.idx;
    const BoundaryIndexH& R = Rb.idx;
    if (!(phys == W.phys)) throw std::runtime_error("heff plan: MPS physical index differs from the MPO's");
    if (W.rows != L.aux || W.cols != R.aux)
        throw std::runtime_error("heff plan: MPO bond dimensions do not match the boundaries");
    auto p = std::make_unique<HeffPlan>();
    p->phys = phys; p->left = left; p->right = right;
    p->L = &Lb; p->R = &Rb;
    ProductBasis rpb(phys, right, true);
    StateMap sm(phys);
    const uint32_t nl = uint32_t(left.size()), nr = uint32_t(right.size()), nps = uint32_t(phys.size());
    const uint32_t nst = uint32_t(sm.nstates());

    // vector layout: right-paired blocks in left-index order
    p->x_off.resize(nl);
    p->x_cols.resize(nl);
    for (uint32_t lb = 0; lb < nl; ++lb) {
        p->x_off[lb] = p->x_len;
        p->x_cols[lb] = uint32_t(rpb.size(left[lb].first));
        p->x_len += left[lb].second * p->x_cols[lb];
    }

    // ---- flat lookup tables ----
    std::vector<RSec> rsec(std::size_t(nl) * nps, RSec{NONE, 0, 0});
    for (uint32_t lb = 0; lb < nl; ++lb)
        for (uint32_t s = 0; s < nps; ++s) {
            Charge rc = left[lb].first + phys[s].first;
            std::size_t rb = right.position(rc);
            if (rb < nr) rsec[std::size_t(lb) * nps + s] = RSec{uint32_t(rb), uint32_t(right[rb].second), uint32_t(rpb(phys[s].first, rc))};
        }
    // R cohort of (ket right sector, bra right sector), and its storage partner
    std::vector<uint32_t> Rci(std::size_t(nr) * nr, NONE), Rcie(std::size_t(nr) * nr, NONE);
    for (uint32_t a = 0; a < nr; ++a)
        for (uint32_t b = 0; b < nr; ++b) {
            uint32_t ci = R.cohort_index(right[a].first, right[b].first);
            if (ci == R.n_cohorts()) continue;
            uint32_t ce = R.tr[ci] ? R.cohort_index(right[b].first, right[a].first) : ci;
            if (ce == R.n_cohorts()) throw std::runtime_error("heff plan: transposed cohort without partner");
            Rci[std::size_t(a) * nr + b] = ci;
            Rcie[std::size_t(a) * nr + b] = ce;
        }
    // op entries, CSR per operator: (input state, output state, value)
    const std::size_t nops = W.ops->size();
    std::vector<uint32_t> optr(nops + 1, 0), oin, oout;
    std::vector<double> oval;
    for (std::size_t o = 0; o < nops; ++o) {
        const SparseOp& s = (*W.ops)[o];
        optr[o] = uint32_t(oin.size());
        for (std::size_t e = 0; e < s.val.size(); ++e) { oin.push_back(s.in[e]); oout.push_back(s.out[e]); oval.push_back(s.val[e]); }
    }
    optr[nops] = uint32_t(oin.size());

    std::vector<Part> parts(nl);
    const bool tdbg = std::getenv("QCM_PLAN_TIMING") != nullptr;
    auto tnow = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    const double t_a = tnow();
#pragma omp parallel for schedule(dynamic, 1)
    for (int lbi = 0; lbi < int(nl); ++lbi) {
        const uint32_t lb_in = uint32_t(lbi);
        Part& P = parts[lb_in];
        const uint32_t ls_in = uint32_t(left[lb_in].second);
        // ---- T jobs: one per (input state, bra right sector) ----
        std::vector<uint32_t> tj(std::size_t(nst) * nr, NONE);
        for (uint32_t st = 0; st < nst; ++st) {
            const uint32_t s = uint32_t(sm.sector[st]), ss = uint32_t(sm.sub[st]);
            const RSec& ri = rsec[std::size_t(lb_in) * nps + s];
            if (ri.rb == NONE) continue;
            for (uint32_t rbb = 0; rbb < nr; ++rbb) {
                uint32_t ci = Rci[std::size_t(ri.rb) * nr + rbb];
                if (ci == NONE) continue;
                uint32_t ce = Rcie[std::size_t(ri.rb) * nr + rbb];
                TJobD j{};
                uint32_t mps_off = ri.off + ss * ri.rs;
                j.a_off = p->x_off[lb_in] + uint64_t(mps_off) * ls_in;
                j.b_off = R.data_off[ce];
                j.c_off = P.t_len;
                j.M = ls_in; j.K = ri.rs; j.brs = R.rsz[ci]; j.N = R.nb[ce] * j.brs; j.lda = ls_in;
                j.tr = (ci != ce) ? 1 : 0;
                P.flops_t += 2.0 * ls_in * double(R.cohort_size(ce));
                tj[std::size_t(st) * nr + rbb] = uint32_t(P.tjobs.size());
                P.t_len += (uint64_t(j.M) * j.N + 31) / 32 * 32;
                P.tjobs.push_back(j);
                P.tjob_mps.push_back(mps_off);
            }
        }
        // slice numbering: slot of (job, b2 position); cleared after each unit
        std::vector<uint32_t> job_pos0(P.tjobs.size() + 1, 0);
        for (std::size_t k = 0; k < P.tjobs.size(); ++k)
            job_pos0[k + 1] = job_pos0[k] + (P.tjobs[k].brs ? P.tjobs[k].N / P.tjobs[k].brs : 0);
        std::vector<uint32_t> slot(job_pos0.back() + 1, NONE);

        for (uint32_t lb_out = 0; lb_out < nl; ++lb_out) {
            uint32_t ci = L.cohort_index(left[lb_out].first, left[lb_in].first);
            if (ci == L.n_cohorts()) continue;
            uint32_t ce = L.tr[ci] ? L.cohort_index(left[lb_in].first, left[lb_out].first) : ci;
            if (ce == L.n_cohorts()) throw std::runtime_error("heff plan: transposed cohort without partner");
            const uint32_t ls_out = uint32_t(left[lb_out].second);
            const uint32_t nS = L.nb[ce];
            const uint32_t K_c = nS * ls_in;
            // units = output states whose right sector exists
            std::vector<U> units;
            uint32_t stripe = 0;
            for (uint32_t st = 0; st < nst; ++st) {
                const RSec& ro = rsec[std::size_t(lb_out) * nps + sm.sector[st]];
                if (ro.rb == NONE) continue;
                units.push_back(U{st, ro.off + uint32_t(sm.sub[st]) * ro.rs, ro.rs, ro.rb, {}, {}});
                stripe += ro.rs;
            }
            if (stripe != p->x_cols[lb_out]) throw std::runtime_error("heff plan: cohort stripe differs from the block width");
            // per (input state, unit): R cohort, T job and slice geometry
            std::vector<int> unit_of(nst, -1);
            for (std::size_t k = 0; k < units.size(); ++k) unit_of[units[k].st] = int(k);
            const std::size_t nu = units.size();
            std::vector<uint32_t> cir_t(std::size_t(nst) * nu, NONE), job_t(std::size_t(nst) * nu, NONE), rsin_t(nst, 0);
            for (uint32_t sti = 0; sti < nst; ++sti) {
                const RSec& ri = rsec[std::size_t(lb_in) * nps + sm.sector[sti]];
                if (ri.rb == NONE) continue;
                rsin_t[sti] = ri.rs;
                for (std::size_t k = 0; k < nu; ++k) {
                    cir_t[sti * nu + k] = Rci[std::size_t(ri.rb) * nr + units[k].rb_out];
                    job_t[sti * nu + k] = tj[std::size_t(sti) * nr + units[k].rb_out];
                }
            }
            const int64_t* Roff = R.offsets.data();
            const double* Rcs = R.cscale.data();
            const std::size_t Raux = R.aux;
            std::size_t n_alpha = 0;
            for (uint32_t b1 = 0; b1 < W.rows; ++b1) {
                if (!L.has_block(ci, b1)) continue;
                const uint32_t bpos = uint32_t(L.offset(ci, b1) / (int64_t(ls_in) * ls_out));
                const double lsc = L.conj_scale(ci, b1);
                for (uint32_t e = W.row_ptr[b1]; e < W.row_ptr[b1 + 1]; ++e) {
                    const uint32_t b2 = W.b2[e], op = W.op[e];
                    const double wsc = W.scale[e] * lsc;
                    for (uint32_t k = optr[op]; k < optr[op + 1]; ++k) {
                        const int u = unit_of[oout[k]];
                        if (u < 0) continue;
                        const uint32_t sti = oin[k];
                        const uint32_t cir = cir_t[sti * nu + u];
                        if (cir == NONE) continue;
                        const int64_t roff = Roff[cir * Raux + b2];
                        if (roff < 0) continue;
                        const uint32_t job = job_t[sti * nu + u];
                        if (job == NONE) continue;
                        U& un = units[u];
                        const uint32_t col = uint32_t(roff / rsin_t[sti]);
                        if (un.lines.empty() || un.lines.back() != bpos) un.lines.push_back(bpos);
                        un.em.push_back(Em{uint32_t(un.lines.size() - 1), job_pos0[job] + col / un.ms,
                                           oval[k] * Rcs[cir * Raux + b2] * wsc, P.tjob_mps[job], cir, col});
                        ++n_alpha;
                    }
                }
            }
            if (n_alpha == 0) continue;
            const uint64_t s_off = P.s_len;
            P.s_len += (uint64_t(K_c) * stripe + 31) / 32 * 32;
            for (U& u : units) {
                P.flops_s += 2.0 * ls_in * u.ms * double(u.em.size());
                if (u.em.empty()) continue;
                // number the unit's slices in first-use order
                std::vector<uint32_t> slices;
                for (Em& m : u.em) {
                    uint32_t& sl = slot[m.slice];
                    if (sl == NONE) { sl = uint32_t(slices.size()); slices.push_back(m.slice); }
                }
                UnitD ud{};
                ud.s_off = s_off + uint64_t(u.offset) * K_c;
                ud.line_stride = ls_in; ud.erows = ls_in; ud.col_stride = K_c; ud.ne = ls_in * u.ms;
                ud.nl = uint32_t(u.lines.size()); ud.line0 = uint32_t(P.line_b1.size());
                ud.nk = uint32_t(slices.size()); ud.slice0 = uint32_t(P.slice_off.size());
                ud.sptr0 = uint32_t(P.sptr.size());
                ud.w_off = P.w_len;
                P.w_len += uint64_t(ud.nl) * ud.nk;
                P.line_b1.insert(P.line_b1.end(), u.lines.begin(), u.lines.end());
                for (uint32_t gp : slices) {
                    // slot -> (job, b2 position) -> T offset of the slice
                    uint32_t job = uint32_t(std::upper_bound(job_pos0.begin(), job_pos0.end(), gp) - job_pos0.begin()) - 1;
                    uint32_t pos = gp - job_pos0[job];
                    P.slice_off.push_back(P.tjobs[job].c_off + uint64_t(pos) * u.ms * ls_in);
                }
                // entries sorted by slice, duplicates of (line, slice) summed
                std::vector<WEntD> ents;
                ents.reserve(u.em.size());
                for (Em& m : u.em) ents.push_back(WEntD{m.line, slot[m.slice], m.a});
                pack_unit_entries(std::move(ents), ud.nk, P.went, P.sptr);
                if (bookkeeping)
                    for (Em& m : u.em) {
                        uint32_t row[10] = {lb_in, lb_out, ci, ce, u.offset, u.ms, u.lines[m.line], m.mps, m.cir, m.col};
                        P.bk_int.insert(P.bk_int.end(), row, row + 10);
                        P.bk_alpha.push_back(m.a);
                    }
                for (uint32_t gp : slices) slot[gp] = NONE;
                P.units.push_back(ud);
                P.g_elems += uint64_t(ud.ne) * ud.nl;
                P.g_reads += uint64_t(ud.ne) * u.em.size();
                P.flops_sdense += 2.0 * ud.nl * ud.nk * double(ud.ne);
            }
            P.flops_ls += 2.0 * ls_out * ls_in * double(nS) * stripe;
            SegD sg{};
            sg.l_off = L.data_off[ce];
            sg.s_off = s_off;
            sg.ls_in = ls_in; sg.nS = nS; sg.tr = (ci != ce) ? 1 : 0;
            P.segs.push_back({lb_out, sg});
        }
    }

    const double t_b = tnow();
    // ---- merge the parts in ket-sector order: prefix offsets, one allocation, parallel copy ----
    struct Base { uint64_t t, s, w; uint32_t job, unit, line, slice, sptr, went; std::size_t bk; };
    std::vector<Base> base(nl + 1);
    base[0] = Base{0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = 0; i < nl; ++i) {
        const Part& P = parts[i];
        base[i + 1] = Base{base[i].t + P.t_len, base[i].s + P.s_len, base[i].w + P.w_len, base[i].job + uint32_t(P.tjobs.size()),
                           base[i].unit + uint32_t(P.units.size()), base[i].line + uint32_t(P.line_b1.size()),
                           base[i].slice + uint32_t(P.slice_off.size()), base[i].sptr + uint32_t(P.sptr.size()),
                           base[i].went + uint32_t(P.went.size()), base[i].bk + P.bk_alpha.size()};
    }
    const Base& tot = base[nl];
    p->tjobs.resize(tot.job);
    p->units.resize(tot.unit);
    p->line_b1.resize(tot.line);
    p->slice_off.resize(tot.slice);
    p->sptr.resize(tot.sptr);
    p->went.resize(tot.went);
    if (bookkeeping) { p->bk_int.resize(tot.bk * 10); p->bk_alpha.resize(tot.bk); }
#pragma omp parallel for schedule(dynamic, 1)
    for (int ii = 0; ii < int(nl); ++ii) {
        Part& P = parts[ii];
        const Base& B = base[ii];
        for (std::size_t k = 0; k < P.tjobs.size(); ++k) { TJobD j = P.tjobs[k]; j.c_off += B.t; p->tjobs[B.job + k] = j; }
        for (std::size_t k = 0; k < P.units.size(); ++k) {
            UnitD u = P.units[k];
            u.s_off += B.s; u.line0 += B.line; u.slice0 += B.slice; u.sptr0 += B.sptr; u.w_off += B.w;
            p->units[B.unit + k] = u;
        }
        std::copy(P.line_b1.begin(), P.line_b1.end(), p->line_b1.begin() + B.line);
        for (std::size_t k = 0; k < P.slice_off.size(); ++k) p->slice_off[B.slice + k] = P.slice_off[k] + B.t;
        for (std::size_t k = 0; k < P.sptr.size(); ++k) p->sptr[B.sptr + k] = P.sptr[k] + B.went;
        std::copy(P.went.begin(), P.went.end(), p->went.begin() + B.went);
        if (bookkeeping) {
            std::copy(P.bk_int.begin(), P.bk_int.end(), p->bk_int.begin() + B.bk * 10);
            std::copy(P.bk_alpha.begin(), P.bk_alpha.end(), p->bk_alpha.begin() + B.bk);
        }
        for (auto& sg : P.segs) sg.second.s_off += B.s;
        P.tjobs = {}; P.tjob_mps = {}; P.units = {}; P.line_b1 = {}; P.slice_off = {}; P.sptr = {}; P.went = {};
        P.bk_int = {}; P.bk_alpha = {};
    }
    p->t_len = tot.t;
    p->s_len = tot.s;
    p->w_len = tot.w;
    std::vector<std::vector<SegD>> per_out(nl);
    for (uint32_t i = 0; i < nl; ++i) {
        const Part& P = parts[i];
        for (auto& sg : P.segs) per_out[sg.first].push_back(sg.second);
        p->flops_t += P.flops_t; p->flops_s += P.flops_s; p->flops_ls += P.flops_ls; p->flops_sdense += P.flops_sdense;
        p->g_elems += P.g_elems; p->g_reads += P.g_reads;
    }
    for (uint32_t j = 0; j < p->tjobs.size(); ++j)
        if (p->tjobs[j].M && p->tjobs[j].N) add_tiles(p->ttiles, j, p->tjobs[j].M, p->tjobs[j].N);
    {
        // S-GEMM tiles and their non-empty k-steps, per unit in parallel, then concatenated in unit order
        const std::size_t nu = p->units.size();
        struct UT { std::vector<TileD> t[N_SHAPES]; std::vector<uint16_t> kl; };
        std::vector<UT> ut(nu);
#pragma omp parallel for schedule(dynamic, 16)
        for (long long kk = 0; kk < (long long)nu; ++kk) {
            const UnitD& u = p->units[kk];
            const uint32_t e0 = p->sptr[u.sptr0], e1 = p->sptr[u.sptr0 + u.nk];
            add_unit_tiles(u, uint32_t(kk), p->went.data() + e0, e1 - e0, ut[kk].t, ut[kk].kl);
        }
        for (std::size_t k = 0; k < nu; ++k) {
            const uint32_t kb = uint32_t(p->klist.size());
            for (int sh = 0; sh < N_SHAPES; ++sh)
                for (TileD t : ut[k].t[sh]) {
                    for (uint32_t i = 0; i < ut[k].kl[t.pad]; ++i) {
                        const uint16_t e = ut[k].kl[t.pad + 1 + i];
                        p->flops_sexec += 2.0 * 4.0 * (((e & 1) + ((e >> 1) & 1) + ((e >> 2) & 1) + ((e >> 3) & 1))) *
                                          shape_bm(sh) * shape_bn(sh);
                    }
                    t.pad += kb;
                    p->utiles[sh].push_back(t);
                }
            p->klist.insert(p->klist.end(), ut[k].kl.begin(), ut[k].kl.end());
        }
    }
    // output blocks, their segments (lb_in order) and split-K items
    for (uint32_t lb_out = 0; lb_out < nl; ++lb_out) {
        if (per_out[lb_out].empty()) continue;
        OutD o{};
        o.y_off = p->x_off[lb_out];
        o.M = uint32_t(left[lb_out].second);
        o.N = p->x_cols[lb_out];
        o.seg_start = uint32_t(p->segs.size());
        o.seg_count = uint32_t(per_out[lb_out].size());
        p->segs.insert(p->segs.end(), per_out[lb_out].begin(), per_out[lb_out].end());
        if (o.M && o.N) {
            int sh = shape_for_rows(o.M);
            uint32_t bm = shape_bm(sh), bn = shape_bn(sh);
            for (uint32_t n0 = 0; n0 < o.N; n0 += bn)
                for (uint32_t m0 = 0; m0 < o.M; m0 += bm) {
                    OTileD t{};
                    t.out = uint32_t(p->outs.size()); t.m0 = m0; t.n0 = n0;
                    t.part0 = uint32_t(p->kitems[sh].size());
                    for (uint32_t sg = o.seg_start; sg < o.seg_start + o.seg_count; ++sg) {
                        uint32_t Kc = p->segs[sg].nS * p->segs[sg].ls_in;
                        for (uint32_t k0 = 0; k0 < Kc; k0 += KCHUNK)
                            p->kitems[sh].push_back(KItemD{uint32_t(p->otiles[sh].size()), sg, k0, std::min(Kc, k0 + KCHUNK)});
                    }
                    t.nparts = uint32_t(p->kitems[sh].size()) - t.part0;
                    p->otiles[sh].push_back(t);
                }
        }
        p->outs.push_back(o);
    }
    if (tdbg) {
        std::fprintf(stderr, "plan: tables+parts %.3f s, merge %.3f s\n", t_b - t_a, tnow() - t_b);
        // S-build unit shapes: useful (nalpha), dense (nl*nk) and tile-padded work
        double w_alpha = 0, w_dense = 0, w_pad = 0;
        uint64_t hist_nl[8] = {0}, hist_nk[8] = {0};
        double fl_nl[8] = {0}, fl_nk[8] = {0};
        auto bin = [](uint32_t v) { int b = 0; while (b < 7 && v > (4u << b)) ++b; return b; };  // <=4,8,...,256,>256
        for (const UnitD& u : p->units) {
            const uint32_t na = p->sptr[u.sptr0 + u.nk] - p->sptr[u.sptr0];
            const int sh = shape_for_rows(u.nl);
            const double bm = shape_bm(sh), bn = shape_bn(sh);
            w_alpha += 2.0 * na * u.ne;
            w_dense += 2.0 * u.nl * double(u.nk) * u.ne;
            w_pad += 2.0 * std::ceil(u.nl / bm) * bm * std::ceil(u.nk / 16.0) * 16.0 * std::ceil(u.ne / bn) * bn;
            hist_nl[bin(u.nl)]++; hist_nk[bin(u.nk)]++;
            fl_nl[bin(u.nl)] += 2.0 * u.nl * double(u.nk) * u.ne;
            fl_nk[bin(u.nk)] += 2.0 * u.nl * double(u.nk) * u.ne;
        }
        std::fprintf(stderr, "plan: %zu units, %zu coefficients, %zu S tiles, S work alpha %.3e dense %.3e padded %.3e flop\n",
                     p->units.size(), p->went.size(), p->utiles[0].size() + p->utiles[1].size() + p->utiles[2].size() + p->utiles[3].size(),
                     w_alpha, w_dense, w_pad);
        // k-step occupancy of the coefficient tiles: work if all-zero (BM x 16) blocks were skipped
        for (int bmq : {16, 32, 64, 128}) {
            double w_skip = 0, w_full = 0;
            for (const UnitD& u : p->units) {
                const uint32_t nmt = (u.nl + bmq - 1) / bmq, nks = (u.nk + 15) / 16;
                std::vector<uint8_t> occ(std::size_t(nmt) * nks, 0);
                for (uint32_t w = p->sptr[u.sptr0]; w < p->sptr[u.sptr0 + u.nk]; ++w)
                    occ[std::size_t(p->went[w].line / bmq) * nks + p->went[w].k / 16] = 1;
                std::size_t on = 0;
                for (uint8_t o : occ) on += o;
                w_skip += 2.0 * on * bmq * 16.0 * u.ne;
                w_full += 2.0 * nmt * bmq * nks * 16.0 * u.ne;
            }
            std::fprintf(stderr, "  BM %3d: padded (lines, slices) work %.3e, nonzero-block work %.3e (%.2f)\n", bmq, w_full, w_skip,
                         w_skip / w_full);
        }
        for (int b = 0; b < 8; ++b)
            std::fprintf(stderr, "  bin <=%u: nl units %llu (dense flop %.2e) | nk units %llu (dense flop %.2e)\n", 4u << b,
                         (unsigned long long)hist_nl[b], fl_nl[b], (unsigned long long)hist_nk[b], fl_nk[b]);
    }
    uint64_t pl = 0;
    for (int sh = 0; sh < N_SHAPES; ++sh) pl = std::max<uint64_t>(pl, uint64_t(p->kitems[sh].size()) * shape_bm(sh) * shape_bn(sh));
    p->p_len = pl;
    p->flops = p->flops_t + p->flops_ls + p->flops_s;
    return p;
}

}  // namespace qcm
