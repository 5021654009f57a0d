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
// The result is laid out as device work lists instead of per-sector objects.
#include <algorithm>
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
void add_tiles(std::vector<TileD>* tiles, uint32_t item, uint32_t M, uint32_t N) {
    int sh = shape_for_rows(M);
    uint32_t bm = shape_bm(sh), bn = shape_bn(sh);
    for (uint32_t n0 = 0; n0 < N; n0 += bn)
        for (uint32_t m0 = 0; m0 < M; m0 += bm) tiles[sh].push_back(TileD{item, m0, n0, 0});
}
constexpr uint32_t KCHUNK = 512;  // K rows per split-K item of the L.S GEMM
}  // namespace

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

    // vector layout: right-paired blocks in left-index order
    p->x_off.resize(left.size());
    p->x_cols.resize(left.size());
    for (std::size_t lb = 0; lb < left.size(); ++lb) {
        p->x_off[lb] = p->x_len;
        p->x_cols[lb] = uint32_t(rpb.size(left[lb].first));
        p->x_len += left[lb].second * p->x_cols[lb];
    }

    // operators of the MPO tensor grouped per (op, output sector): (in state, out state, value)
    struct OE { uint32_t in, out; double v; };
    std::vector<std::vector<std::vector<OE>>> op_by_out(W.ops->size(), std::vector<std::vector<OE>>(phys.size()));
    for (std::size_t o = 0; o < W.ops->size(); ++o) {
        const SparseOp& s = (*W.ops)[o];
        for (std::size_t e = 0; e < s.val.size(); ++e)
            op_by_out[o][sm.sector[s.out[e]]].push_back(OE{s.in[e], s.out[e], s.val[e]});
    }

    std::vector<std::pair<uint32_t, SegD>> seg_tmp;
    for (uint32_t lb_in = 0; lb_in < left.size(); ++lb_in) {
        Charge lc_in = left[lb_in].first;
        uint32_t ls_in = uint32_t(left[lb_in].second);
        // ---- T jobs ----
        std::unordered_map<uint64_t, uint32_t> tmap;  // (mps col offset, ci_right) -> job
        for (uint32_t s = 0; s < phys.size(); ++s) {
            Charge rc_ket = lc_in + phys[s].first;
            std::size_t rbk = right.position(rc_ket);
            if (rbk == right.size()) continue;
            uint32_t rs_ket = uint32_t(right[rbk].second);
            uint32_t ket_off = uint32_t(rpb(phys[s].first, rc_ket));
            for (std::size_t rb_bra = 0; rb_bra < right.size(); ++rb_bra) {
                Charge rc_bra = right[rb_bra].first;
                uint32_t ci = R.cohort_index(rc_ket, rc_bra);
                if (ci == R.n_cohorts()) continue;
                uint32_t ci_eff = R.tr[ci] ? R.cohort_index(rc_bra, rc_ket) : ci;
                if (ci_eff == R.n_cohorts()) throw std::runtime_error("heff plan: transposed cohort without partner");
                for (uint32_t ss = 0; ss < phys[s].second; ++ss) {
                    uint32_t mps_off = ket_off + ss * rs_ket;
                    TJobD j{};
                    j.a_off = p->x_off[lb_in] + uint64_t(mps_off) * ls_in;
                    j.b_off = Rb.idx.data_off[ci_eff];
                    j.c_off = p->t_len;
                    j.M = ls_in; j.K = rs_ket; j.brs = R.rsz[ci]; j.N = R.nb[ci_eff] * j.brs; j.lda = ls_in;
                    j.tr = (ci != ci_eff) ? 1 : 0;
                    p->flops_t += 2.0 * ls_in * double(R.cohort_size(ci_eff));
                    if (tmap.emplace((uint64_t(mps_off) << 32) | ci, uint32_t(p->tjobs.size())).second) {
                        p->t_len += (uint64_t(j.M) * j.N + 31) / 32 * 32;
                        if (j.M && j.N) add_tiles(p->ttiles, uint32_t(p->tjobs.size()), j.M, j.N);
                        p->tjobs.push_back(j);
                    }
                }
            }
        }
        // ---- cohorts ----
        for (uint32_t lb_out = 0; lb_out < left.size(); ++lb_out) {
            Charge lc_out = left[lb_out].first;
            uint32_t ls_out = uint32_t(left[lb_out].second);
            uint32_t ci = L.cohort_index(lc_out, lc_in);
            if (ci == L.n_cohorts()) continue;
            uint32_t ci_eff = L.tr[ci] ? L.cohort_index(lc_in, lc_out) : ci;
            if (ci_eff == L.n_cohorts()) throw std::runtime_error("heff plan: transposed cohort without partner");
            uint32_t nS = L.nb[ci_eff];
            struct Unit { uint32_t offset, ms; std::vector<std::vector<std::pair<double, uint64_t>>> lines; std::vector<std::vector<uint32_t>> bk; };
            std::vector<Unit> units;
            std::vector<int> unit_of_state(sm.nstates(), -1);
            uint32_t stripe = 0;
            for (uint32_t s = 0; s < phys.size(); ++s) {
                Charge rc_out = lc_out + phys[s].first;
                std::size_t rbo = right.position(rc_out);
                if (rbo == right.size()) continue;
                uint32_t rs_out = uint32_t(right[rbo].second);
                uint32_t out_off = uint32_t(rpb(phys[s].first, rc_out));
                for (uint32_t ss2 = 0; ss2 < phys[s].second; ++ss2) {
                    unit_of_state[sm.first[s] + ss2] = int(units.size());
                    Unit u;
                    u.offset = out_off + ss2 * rs_out;
                    u.ms = rs_out;
                    u.lines.resize(nS);
                    if (bookkeeping) u.bk.resize(nS);
                    units.push_back(std::move(u));
                    stripe += rs_out;
                }
            }
            if (stripe != p->x_cols[lb_out]) throw std::runtime_error("heff plan: cohort stripe differs from the block width");
            std::size_t n_alpha = 0;
            for (uint32_t b1 = 0; b1 < W.rows; ++b1) {
                if (!L.has_block(ci, b1)) continue;
                uint32_t left_idx = uint32_t(L.offset(ci, b1) / (int64_t(ls_in) * ls_out));
                double lscale = L.conj_scale(ci, b1);
                for (uint32_t e = W.row_ptr[b1]; e < W.row_ptr[b1 + 1]; ++e) {
                    uint32_t b2 = W.b2[e];
                    const auto& by_out = op_by_out[W.op[e]];
                    for (uint32_t s = 0; s < phys.size(); ++s) {
                        Charge rc_out = lc_out + phys[s].first;
                        if (!right.has(rc_out)) continue;
                        for (const OE& oe : by_out[s]) {
                            Charge phys_in = phys[sm.sector[oe.in]].first;
                            Charge rc_in = lc_in + phys_in;
                            uint32_t ci_r = R.cohort_index(rc_in, rc_out);
                            if (!R.has_block(ci_r, b2)) continue;
                            std::size_t rbi = right.position(rc_in);
                            if (rbi == right.size()) continue;
                            uint32_t rs_in = uint32_t(right[rbi].second);
                            uint32_t in_off = uint32_t(rpb(phys_in, rc_in));
                            uint32_t mps_off = in_off + uint32_t(sm.sub[oe.in]) * rs_in;
                            auto it = tmap.find((uint64_t(mps_off) << 32) | ci_r);
                            if (it == tmap.end()) continue;
                            uint32_t col = uint32_t(R.offset(ci_r, b2) / rs_in);
                            double a = oe.v * R.conj_scale(ci_r, b2) * W.scale[e] * lscale;
                            const TJobD& tj = p->tjobs[it->second];
                            int u = unit_of_state[oe.out];
                            units[u].lines[left_idx].push_back({a, tj.c_off + uint64_t(col) * ls_in});
                            if (bookkeeping) {
                                auto& bk = units[u].bk[left_idx];
                                bk.push_back(mps_off); bk.push_back(ci_r); bk.push_back(col);
                            }
                            ++n_alpha;
                        }
                    }
                }
            }
            if (n_alpha == 0) continue;
            uint32_t K_c = nS * ls_in;
            uint64_t s_off = p->s_len;
            p->s_len += (uint64_t(K_c) * stripe + 31) / 32 * 32;
            for (auto& u : units) {
                // unit GEMM data: lines (b1 rows with coefficients), distinct T slices, entries by slice
                std::vector<uint32_t> lines;
                std::unordered_map<uint64_t, uint32_t> kidx;  // T offset -> slice index
                std::vector<uint64_t> slices;
                std::vector<std::vector<std::pair<uint32_t, double>>> by_slice;
                std::size_t nu = 0;
                for (uint32_t b = 0; b < nS; ++b) {
                    auto& ln = u.lines[b];
                    if (ln.empty()) continue;
                    uint32_t li = uint32_t(lines.size());
                    lines.push_back(b);
                    nu += ln.size();
                    for (std::size_t k = 0; k < ln.size(); ++k) {
                        auto ins = kidx.emplace(ln[k].second, uint32_t(slices.size()));
                        if (ins.second) { slices.push_back(ln[k].second); by_slice.emplace_back(); }
                        by_slice[ins.first->second].push_back({li, ln[k].first});
                        if (bookkeeping) {
                            const auto& bk = u.bk[b];
                            uint32_t row[10] = {lb_in, lb_out, ci, ci_eff, u.offset, u.ms, b, bk[3 * k], bk[3 * k + 1], bk[3 * k + 2]};
                            p->bk_int.insert(p->bk_int.end(), row, row + 10);
                            p->bk_alpha.push_back(ln[k].first);
                        }
                    }
                }
                p->flops_s += 2.0 * ls_in * u.ms * double(nu);
                if (lines.empty() || ls_in == 0 || u.ms == 0) continue;
                UnitD ud{};
                ud.s_off = s_off + uint64_t(u.offset) * K_c;
                ud.ldS = K_c; ud.ls = ls_in; ud.ne = ls_in * u.ms;
                ud.nl = uint32_t(lines.size()); ud.line0 = uint32_t(p->line_b1.size());
                ud.nk = uint32_t(slices.size()); ud.slice0 = uint32_t(p->slice_off.size());
                ud.sptr0 = uint32_t(p->sptr.size());
                p->line_b1.insert(p->line_b1.end(), lines.begin(), lines.end());
                p->slice_off.insert(p->slice_off.end(), slices.begin(), slices.end());
                for (uint32_t k = 0; k < ud.nk; ++k) {
                    p->sptr.push_back(uint32_t(p->went.size()));
                    for (auto& e : by_slice[k]) p->went.push_back(WEntD{e.first, k, e.second});
                }
                p->sptr.push_back(uint32_t(p->went.size()));
                int sh = shape_for_rows(ud.nl);
                uint32_t bm = shape_bm(sh), bn = shape_bn(sh);
                for (uint32_t n0 = 0; n0 < ud.ne; n0 += bn)
                    for (uint32_t m0 = 0; m0 < ud.nl; m0 += bm) p->utiles[sh].push_back(TileD{uint32_t(p->units.size()), m0, n0, 0});
                p->units.push_back(ud);
                p->g_elems += uint64_t(ls_in) * u.ms * ud.nl;
                p->g_reads += uint64_t(ls_in) * u.ms * nu;
                p->flops_sdense += 2.0 * ud.nl * ud.nk * double(ud.ne);
            }
            p->flops_ls += 2.0 * ls_out * ls_in * double(nS) * stripe;
            SegD sg{};
            sg.l_off = Lb.idx.data_off[ci_eff];
            sg.s_off = s_off;
            sg.ls_in = ls_in; sg.nS = nS; sg.tr = (ci != ci_eff) ? 1 : 0;
            seg_tmp.push_back({lb_out, sg});
        }
    }
    // group segments per output block; inside a block they stay in lb_in order
    {
        std::vector<std::vector<SegD>> per_out(left.size());
        for (std::size_t i = 0; i < seg_tmp.size(); ++i) per_out[seg_tmp[i].first].push_back(seg_tmp[i].second);
        for (uint32_t lb_out = 0; lb_out < left.size(); ++lb_out) {
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
    }
    uint64_t pl = 0;
    for (int sh = 0; sh < N_SHAPES; ++sh) pl = std::max<uint64_t>(pl, uint64_t(p->kitems[sh].size()) * shape_bm(sh) * shape_bn(sh));
    p->p_len = pl;
    p->flops = p->flops_t + p->flops_ls + p->flops_s;
    return p;
}

}  // namespace qcm
