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
#include <cstring>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>

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
// split-K chunk of the L.S GEMM (rows of K per work item): 512 gives about twice the CTAs of 1024 at the
// L=24, M=512 middle bond and took the L.S phase from 0.47 to 0.41 ms (with the per-element reduction of
// the partials); 256 was no faster
constexpr uint32_t KCHUNK = 512;

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
    CoefGen cg;  // part-local coefficient-generation units
    std::vector<uint32_t> line_b1;
    std::vector<uint64_t> slice_off;
    uint64_t s_len = 0, w_len = 0, n_alpha = 0;
    std::vector<std::pair<uint32_t, SegD>> segs;
    double flops_t = 0, flops_s = 0, flops_ls = 0, flops_sdense = 0;
    uint64_t g_elems = 0, g_reads = 0;
    std::vector<uint32_t> bk_int;
    std::vector<double> bk_alpha;
    std::vector<TileD> utiles[N_SHAPES];  // S-GEMM tiles, item = unit of this part, pad = klist offset
    std::vector<uint16_t> klist;
    double flops_sexec = 0;
};

// Output state of a cohort and its coefficient terms: (line, slice id in the part's T
// numbering), and with bookkeeping (mps column, R cohort, R column, alpha) per term.
struct U {
    uint32_t st, offset, ms, rb_out;
    uint64_t nterms = 0;
    std::vector<uint32_t> sl;   // slot -> slice id, first-use order
    std::vector<uint64_t> sig;  // per slot, nw words: the 16-line groups of its lines
    uint32_t nw = 0;
    std::vector<LKD> em;        // (line, slot) per term, with bookkeeping only
    std::vector<uint32_t> lines, rows, bk;  // lines: S row block of each line, rows: its MPO row b1
    std::vector<double> bk_a;
};

// (unit, input state) of a cohort: the R block positions of the input state's cohort (null: the
// unit has no T job for it) and the slice-id base of its T job
struct GRef {
    const int32_t* rp;
    uint32_t jbase;
};

}  // namespace

namespace {

constexpr uint32_t KS = 16;  // k-step of the S-GEMM (dm::BK), four DMMA k-groups of 4 slices

// S-GEMM tiling of a unit: the shape and the occupancy at its line tiles (one 4-bit mask of non-empty
// 4-slot groups per (line tile, k-step))
struct TileChoice {
    int sh = -1;
    double cost = 0;
    std::vector<uint8_t> occ;
};

// The cheapest shape for an occupancy occ16 (n16 x nks: 16-line groups x k-steps).  Coarser line
// tiles OR rows together; the cost is the tensor work of the occupied groups, weighted per shape
// (the 16-row shape runs 2 x 4 fragments per warp).
void choose_shape(const UnitD& u, const uint8_t* occ16, uint32_t nks, TileChoice& best, std::vector<uint8_t>& occ) {
    const uint32_t n16 = (u.nl + 15) / 16;
    auto groups = [](uint8_t m) { return (m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1); };
    static const int cand[4] = {SHAPE_16, SHAPE_32, SHAPE_64, SHAPE_128};
    static const double eff[4] = {1.3, 1.0, 1.0, 1.05};
    for (int ci = 0; ci < 4; ++ci) {
        const uint32_t bm = shape_bm(cand[ci]), bn = shape_bn(cand[ci]);
        const uint32_t f = bm / 16, nmt = (u.nl + bm - 1) / bm, nnt = (u.ne + bn - 1) / bn;
        occ.assign(std::size_t(nmt) * nks, 0);
        for (uint32_t r = 0; r < n16; ++r)
            for (uint32_t ks = 0; ks < nks; ++ks) occ[std::size_t(r / f) * nks + ks] |= occ16[std::size_t(r) * nks + ks];
        std::size_t on = 0;
        for (uint8_t o : occ) on += groups(o);
        const double cost = eff[ci] * double(on) * bm * 4.0 * double(nnt) * bn;
        if (best.sh < 0 || cost < best.cost) { best.sh = cand[ci]; best.cost = cost; best.occ.swap(occ); }
    }
}

void emit_tiles(const UnitD& u, uint32_t item, const TileChoice& c, std::vector<TileD>* utiles,
                std::vector<uint16_t>& klist) {
    const uint32_t nks = (u.nk + KS - 1) / KS;
    const int sh = c.sh;
    const uint32_t bm = shape_bm(sh), bn = shape_bn(sh), nmt = (u.nl + bm - 1) / bm;
    for (uint32_t mt = 0; mt < nmt; ++mt) {
        const uint32_t off = uint32_t(klist.size());
        klist.push_back(0);
        uint16_t cnt = 0;
        for (uint32_t ks = 0; ks < nks; ++ks) {
            const uint8_t m = c.occ[std::size_t(mt) * nks + ks];
            if (m) { klist.push_back(uint16_t((ks << 4) | m)); ++cnt; }
        }
        klist[off] = cnt;
        if (!cnt) continue;
        for (uint32_t n0 = 0; n0 < u.ne; n0 += bn) utiles[sh].push_back(TileD{item, mt * bm, n0, off});
    }
}

uint32_t checked_ksteps(const UnitD& u) {
    const uint32_t nks = (u.nk + KS - 1) / KS;
    if (nks >= 4096) throw std::runtime_error("S unit: too many slices for the k-step list");
    return nks;
}

// Slot order and tiling of an H_eff unit from its slot signatures: sig[slot * nw + w] bit r set where a
// line of 16-line group 64 w + r uses the slot.  For line tiles of 16, 64 and 128 lines the slots are
// sorted by the line tiles that use them (then by the 16-line groups; first-use order among equal
// sets), so that slots used by the same line tiles share 4-slot k-groups; the ordering and shape of
// least tensor work (over all four shapes) are kept.  order[new slot] = old slot.
void plan_unit_tiles(const UnitD& u, const uint64_t* sig, uint32_t nw, std::vector<uint32_t>& order, TileChoice& best) {
    const uint32_t nk = u.nk;
    order.resize(nk);
    for (uint32_t i = 0; i < nk; ++i) order[i] = i;
    if (!u.nl || !u.ne || !nk) return;
    const uint32_t nks = checked_ksteps(u), n16 = (u.nl + 15) / 16;
    std::vector<uint64_t> key;
    std::vector<uint32_t> ord(nk);
    std::vector<uint8_t> occ16, scratch;
    // line-tile coarseness of the ordering key: 16, 64 and 128 lines (32 won in 13 of 4,878 units at the
    // L=24, M=512 middle bond without changing the executed work; leaving it out saves 40 % of this step)
    for (uint32_t f : {1u, 4u, 8u}) {
        if (f > 1 && (n16 + f / 2 - 1) / (f / 2) <= 1) break;  // one coarse tile: the same order as before
        const uint32_t nc = (n16 + f - 1) / f, ncw = (nc + 63) / 64;
        auto by_sig = [&](uint32_t a, uint32_t b) {
            for (uint32_t w = nw; w-- > 0;) {
                const uint64_t x = sig[std::size_t(a) * nw + w], y = sig[std::size_t(b) * nw + w];
                if (x != y) return x < y;
            }
            return false;
        };
        for (uint32_t i = 0; i < nk; ++i) ord[i] = i;
        if (f == 1) {
            // 16-line tiles: the key is the signature itself
            std::stable_sort(ord.begin(), ord.end(), by_sig);
        } else {
            key.assign(std::size_t(nk) * ncw, 0);
            for (uint32_t sl = 0; sl < nk; ++sl)
                for (uint32_t w = 0; w < nw; ++w)
                    for (uint64_t bits = sig[std::size_t(sl) * nw + w]; bits; bits &= bits - 1) {
                        const uint32_t c = (64 * w + uint32_t(__builtin_ctzll(bits))) / f;
                        key[std::size_t(sl) * ncw + c / 64] |= 1ull << (c % 64);
                    }
            std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
                for (uint32_t w = ncw; w-- > 0;) {
                    const uint64_t x = key[std::size_t(a) * ncw + w], y = key[std::size_t(b) * ncw + w];
                    if (x != y) return x < y;
                }
                return by_sig(a, b);
            });
        }
        occ16.assign(std::size_t(n16) * nks, 0);
        for (uint32_t i = 0; i < nk; ++i) {
            const uint32_t sl = ord[i];
            const uint8_t bit = uint8_t(1u << ((i % KS) / 4));
            for (uint32_t w = 0; w < nw; ++w)
                for (uint64_t bits = sig[std::size_t(sl) * nw + w]; bits; bits &= bits - 1)
                    occ16[std::size_t(64 * w + uint32_t(__builtin_ctzll(bits))) * nks + i / KS] |= bit;
        }
        TileChoice c;
        choose_shape(u, occ16.data(), nks, c, scratch);
        if (best.sh < 0 || c.cost < best.cost) { best = std::move(c); order = ord; }
    }
}

}  // namespace

void add_unit_tiles(const UnitD& u, uint32_t item, const LKD* ents, std::size_t n, std::vector<TileD>* utiles,
                    std::vector<uint16_t>& klist) {
    if (!u.nl || !u.ne || !u.nk || !n) return;
    const uint32_t nks = checked_ksteps(u), n16 = (u.nl + 15) / 16;
    // occupancy of (16 lines x 4 slices) coefficient groups as a 4-bit mask per (16 lines x 16 slices) block
    std::vector<uint8_t> occ16(std::size_t(n16) * nks, 0), scratch;
    for (std::size_t i = 0; i < n; ++i)
        occ16[std::size_t(ents[i].line / 16) * nks + ents[i].k / KS] |= uint8_t(1u << ((ents[i].k % KS) / 4));
    TileChoice c;
    choose_shape(u, occ16.data(), nks, c, scratch);
    emit_tiles(u, item, c, utiles, klist);
}


uint64_t plan_structure_key(const BoundaryIndexH& L, const BoundaryIndexH& R, const Index& phys, const Index& left,
                            const Index& right) {
    KeyHash k;
    k.boundary(L);
    k.boundary(R);
    k.index(phys);
    k.index(left);
    k.index(right);
    return k.h;
}

uint64_t boundary_key(const DevBoundary& B) {
    if (!B.key) {
        KeyHash k;
        k.boundary(B.idx);
        B.key = k.h | 1;
    }
    return B.key;
}

uint64_t plan_structure_key(const DevBoundary& L, const DevBoundary& R, const Index& phys, const Index& left,
                            const Index& right) {
    KeyHash k;
    k.word(boundary_key(L));
    k.word(boundary_key(R));
    k.index(phys);
    k.index(left);
    k.index(right);
    return k.h;
}

std::shared_ptr<const MPOTables> build_mpo_tables(const MPOTensor& W) {
    auto t = std::make_shared<MPOTables>();
    t->nst = uint32_t(StateMap(W.phys).nstates());
    t->nops = W.ops ? W.ops->size() : 0;
    t->rows = W.rows; t->cols = W.cols;
    const uint32_t nst = t->nst;
    const std::size_t nops = t->nops, nent = W.b2.size();
    if (W.b1.size() != nent || W.op.size() != nent || W.scale.size() != nent) throw std::runtime_error("MPO tables: inconsistent MPO tensor");
    if (W.row_ptr.size() != std::size_t(W.rows) + 1 || W.row_ptr.back() != nent || W.col_ptr.size() != std::size_t(W.cols) + 1 ||
        W.col_ptr.back() != nent || W.col_ent.size() != nent)
        throw std::runtime_error("MPO tables: MPO tensor is not finalized");
    for (std::size_t i = 0; i < W.rows; ++i)
        if (W.row_ptr[i] > W.row_ptr[i + 1]) throw std::runtime_error("MPO tables: row pointers");
    for (std::size_t i = 0; i < W.cols; ++i)
        if (W.col_ptr[i] > W.col_ptr[i + 1]) throw std::runtime_error("MPO tables: column pointers");
    for (std::size_t e = 0; e < nent; ++e)
        if (W.b1[e] >= W.rows || W.b2[e] >= W.cols || W.op[e] >= nops || W.col_ent[e] >= nent)
            throw std::runtime_error("MPO tables: entry out of range");
    // operator terms
    t->optr.assign(nops + 1, 0);
    for (std::size_t o = 0; o < nops; ++o) {
        const SparseOp& op = (*W.ops)[o];
        if (op.in.size() != op.val.size() || op.out.size() != op.val.size()) throw std::runtime_error("MPO tables: operator arrays");
        t->optr[o] = uint32_t(t->oin.size());
        for (std::size_t e = 0; e < op.val.size(); ++e) {
            if (op.in[e] >= nst || op.out[e] >= nst) throw std::runtime_error("MPO tables: operator entry outside the physical basis");
            t->oin.push_back(op.in[e]); t->oout.push_back(op.out[e]); t->oval.push_back(op.val[e]);
        }
    }
    t->optr[nops] = uint32_t(t->oin.size());
    t->o_ptr.assign(nops * nst + 1, 0);
    for (std::size_t o = 0; o < nops; ++o)
        for (uint32_t k = t->optr[o]; k < t->optr[o + 1]; ++k) t->o_ptr[o * nst + t->oout[k] + 1]++;
    for (std::size_t i = 0; i < nops * nst; ++i) t->o_ptr[i + 1] += t->o_ptr[i];
    t->o_in.resize(t->oin.size());
    t->o_val.resize(t->oin.size());
    std::vector<uint32_t> fill(t->o_ptr.begin(), t->o_ptr.end() - 1);
    for (std::size_t o = 0; o < nops; ++o)
        for (uint32_t k = t->optr[o]; k < t->optr[o + 1]; ++k) {
            const uint32_t d = fill[o * nst + t->oout[k]]++;
            t->o_in[d] = t->oin[k];
            t->o_val[d] = t->oval[k];
        }
    t->o_one.assign(nops * nst, MPOTables::O_NONE);
    for (std::size_t i = 0; i < nops * nst; ++i) {
        const uint32_t n = t->o_ptr[i + 1] - t->o_ptr[i];
        if (n == 1) t->o_one[i] = t->o_in[t->o_ptr[i]];
        else if (n > 1) t->o_one[i] = MPOTables::O_MANY;
    }
    t->row_qb.resize(nent);
    for (std::size_t e = 0; e < nent; ++e) t->row_qb[e] = (uint64_t(W.op[e]) * nst << 32) | W.b2[e];
    // entries by row and by column
    t->row_ptr = W.row_ptr;
    t->row_other = W.b2; t->row_op = W.op; t->row_scale = W.scale;
    t->col_ptr = W.col_ptr;
    t->col_other.resize(nent); t->col_op.resize(nent); t->col_scale.resize(nent);
    for (std::size_t q = 0; q < nent; ++q) {
        const uint32_t e = W.col_ent[q];
        t->col_other[q] = W.b1[e]; t->col_op[q] = W.op[e]; t->col_scale[q] = W.scale[e];
    }
    return t;
}

std::shared_ptr<const MPOTables> MPOTensor::tables() const {
    static std::mutex m;
    std::lock_guard<std::mutex> g(m);
    if (!tables_) tables_ = build_mpo_tables(*this);
    return tables_;
}

void CoefGen::set_mpo(const MPOTensor& W, bool row) {
    mt = W.tables();
    nst = mt->nst;
    by_row = row;
}

void CoefGen::set_boundary(const BoundaryIndexH& B) {
    b_aux = B.aux;
    b_cs = &B.cscale;
    b_pos.resize(B.offsets.size());
    for (uint32_t c = 0; c < B.n_cohorts(); ++c) {
        const int64_t bs = std::max<int64_t>(1, int64_t(B.lsz[c]) * B.rsz[c]);
        for (uint32_t b = 0; b < B.aux; ++b) {
            const int64_t o = B.offsets[std::size_t(c) * B.aux + b];
            b_pos[std::size_t(c) * B.aux + b] = o < 0 ? -1 : int32_t(o / bs);
        }
    }
}

void CoefGen::append_units(const CoefGen& x, uint32_t line_base, uint32_t map_base, uint64_t w_base) {
    for (WGenUnitD g : x.units) {
        g.w_off += w_base; g.line0 += line_base; g.map0 += map_base;
        units.push_back(g);
    }
    gin.insert(gin.end(), x.gin.begin(), x.gin.end());
    line_major.insert(line_major.end(), x.line_major.begin(), x.line_major.end());
    line_scale.insert(line_scale.end(), x.line_scale.begin(), x.line_scale.end());
    smap_id.insert(smap_id.end(), x.smap_id.begin(), x.smap_id.end());
    smap_slot.insert(smap_slot.end(), x.smap_slot.begin(), x.smap_slot.end());
}

void CoefGen::add_unit(uint64_t w_off, uint32_t wld, uint32_t st_out, const uint32_t* majors, const double* scales, uint32_t nl,
                       const std::vector<uint32_t>& slices, const WGenInD* in_row) {
    WGenUnitD g{};
    g.w_off = w_off; g.wld = wld; g.st_out = st_out;
    g.line0 = uint32_t(line_major.size()); g.nl = nl;
    g.map0 = uint32_t(smap_id.size()); g.nk = uint32_t(slices.size());
    line_major.insert(line_major.end(), majors, majors + nl);
    line_scale.insert(line_scale.end(), scales, scales + nl);
    const std::size_t m0 = smap_id.size();
    for (uint32_t i = 0; i < g.nk; ++i) { smap_id.push_back(slices[i]); smap_slot.push_back(i); }
    // (slice id, slot) pairs sorted by id
    std::vector<std::pair<uint32_t, uint32_t>> pr(g.nk);
    for (uint32_t i = 0; i < g.nk; ++i) pr[i] = {slices[i], i};
    std::sort(pr.begin(), pr.end());
    for (uint32_t i = 0; i < g.nk; ++i) { smap_id[m0 + i] = pr[i].first; smap_slot[m0 + i] = pr[i].second; }
    gin.insert(gin.end(), in_row, in_row + nst);
    units.push_back(g);
}

std::unique_ptr<HeffPlan> build_heff_plan(const DevBoundary& Lb, const DevBoundary& Rb, const MPOTensor& W,
                                          const Index& phys, const Index& left, const Index& right, bool bookkeeping) {
    const BoundaryIndexH& L = Lb.idx;
    const BoundaryIndexH& R = Rb.idx;
    if (!(phys == W.phys)) throw std::runtime_error("heff plan: MPS physical index differs from the MPO's");
    if (W.rows != L.aux || W.cols != R.aux)
        throw std::runtime_error("heff plan: MPO bond dimensions do not match the boundaries");
    const double t_0 = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
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
    // operator terms, CSR per operator: (input state, output state, value)
    const std::shared_ptr<const MPOTables> mt = W.tables();
    if (mt->nst != nst) throw std::runtime_error("heff plan: MPO physical basis differs");
    const std::vector<uint32_t>& optr = mt->optr;
    const std::vector<uint32_t>& oin = mt->oin;
    const std::vector<uint32_t>& oout = mt->oout;
    // the same grouped by (operator, output state), in their order within the operator
    const std::vector<uint32_t>& og_ptr = mt->o_ptr;
    const std::vector<uint32_t>& og_in = mt->o_in;
    const uint32_t* o_one = mt->o_one.data();
    const uint64_t* row_qb = mt->row_qb.data();
    const std::vector<double>& og_val = mt->o_val;
    // coefficient generation: lines iterate MPO rows b1, slices come from R cohorts
    p->cg.set_mpo(W, true);
    p->cg.set_boundary(R);

    std::vector<Part> parts(nl);
    // ket sectors in decreasing estimated work (the L blocks of their cohorts), so that dynamic
    // scheduling starts the largest parts first and no large part is left for the end
    std::vector<uint32_t> part_order(nl);
    {
        std::vector<uint64_t> est(nl, 0);
        for (uint32_t a = 0; a < nl; ++a) {
            part_order[a] = a;
            for (uint32_t b = 0; b < nl; ++b) {
                const uint32_t ci = L.cohort_index(left[b].first, left[a].first);
                if (ci == L.n_cohorts()) continue;
                const uint32_t ce = L.tr[ci] ? L.cohort_index(left[a].first, left[b].first) : ci;
                if (ce < L.n_cohorts()) est[a] += L.nb[ce];
            }
        }
        std::stable_sort(part_order.begin(), part_order.end(), [&](uint32_t x, uint32_t y) { return est[x] > est[y]; });
    }
    const bool tdbg = std::getenv("QCM_PLAN_TIMING") != nullptr;
    std::vector<double> part_s(tdbg ? nl : 0);
    double sum_terms = 0, sum_tiles = 0;  // QCM_PLAN_TIMING: thread time in the term enumeration / tile planning
    auto tnow = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    const double t_a = tnow();
    std::string err;
#pragma omp parallel
    {
    // per-thread scratch, reused across cohorts
    std::vector<U> units;
    std::vector<uint32_t> slices;
    std::vector<double> lscale;
    std::vector<uint32_t> corder, crank, ctmp;
    std::vector<GRef> gref;
    std::vector<std::pair<uint32_t, uint32_t>> lrows;
#pragma omp for schedule(dynamic, 1)
    for (int oi = 0; oi < int(nl); ++oi) try {
        const uint32_t lb_in = part_order[std::size_t(oi)];
        Part& P = parts[lb_in];
        const double tp0 = tdbg ? tnow() : 0.0;
        P.cg.nst = nst;
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
                j.sst = slice_stride(j.brs, j.M);
                P.flops_t += 2.0 * ls_in * double(R.cohort_size(ce));
                tj[std::size_t(st) * nr + rbb] = uint32_t(P.tjobs.size());
                P.t_len += (uint64_t(R.nb[ce]) * j.sst + 31) / 32 * 32;
                P.tjobs.push_back(j);
                P.tjob_mps.push_back(mps_off);
            }
        }
        // slice ids: (job, b2 position) -> job_pos0[job] + position; slot of an id within the
        // current unit, cleared after each unit
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
            std::size_t nu = 0;
            uint32_t stripe = 0;
            for (uint32_t st = 0; st < nst; ++st) {
                const RSec& ro = rsec[std::size_t(lb_out) * nps + sm.sector[st]];
                if (ro.rb == NONE) continue;
                if (nu == units.size()) units.emplace_back();
                U& x = units[nu++];
                x.st = st; x.offset = ro.off + uint32_t(sm.sub[st]) * ro.rs; x.ms = ro.rs; x.rb_out = ro.rb;
                x.em.clear(); x.lines.clear(); x.rows.clear(); x.bk.clear(); x.bk_a.clear();
                x.nterms = 0; x.sl.clear(); x.sig.clear();
                stripe += ro.rs;
            }
            if (stripe != p->x_cols[lb_out]) throw std::runtime_error("heff plan: cohort stripe differs from the block width");
            // per (input state, unit): R cohort and slice-id base of its T job
            std::vector<WGenInD> gin(nu * nst, WGenInD{WGEN_NONE, WGEN_NONE});  // [unit][input state]
            std::vector<uint32_t> rsin_t(nst, 0);
            for (uint32_t sti = 0; sti < nst; ++sti) {
                const RSec& ri = rsec[std::size_t(lb_in) * nps + sm.sector[sti]];
                if (ri.rb == NONE) continue;
                rsin_t[sti] = ri.rs;
                for (std::size_t k = 0; k < nu; ++k) {
                    const uint32_t cir = Rci[std::size_t(ri.rb) * nr + units[k].rb_out];
                    const uint32_t job = tj[std::size_t(sti) * nr + units[k].rb_out];
                    if (cir != NONE && job != NONE) gin[k * nst + sti] = WGenInD{cir, job_pos0[job]};
                }
            }
            // L blocks of the cohort: MPO row b1 and its S row block
            lrows.clear();
            for (uint32_t b1 = 0; b1 < W.rows; ++b1)
                if (L.has_block(ci, b1)) lrows.push_back({b1, uint32_t(L.offset(ci, b1) / (int64_t(ls_in) * ls_out))});
            // lines in decreasing MPO row length (the rows with most terms first; stable): lines of similar
            // density share S-GEMM line tiles, so the tiles of sparse lines occupy few slot groups
            // (executed tensor work at the L=24, M=512 middle bond: -18 %)
            std::stable_sort(lrows.begin(), lrows.end(), [&](const std::pair<uint32_t, uint32_t>& a,
                                                             const std::pair<uint32_t, uint32_t>& b) {
                return W.row_ptr[a.first + 1] - W.row_ptr[a.first] > W.row_ptr[b.first + 1] - W.row_ptr[b.first];
            });
            const uint32_t nw16 = (uint32_t(lrows.size()) + 1023) / 1024;  // signature words: 64 groups of 16 lines
            // per (unit, input state): the R block positions of the input state's cohort and the
            // slice-id base of its T job (rp = null: no T job)
            const int32_t* Rpos = p->cg.b_pos.data();
            const std::size_t Raux = R.aux;
            gref.assign(nu * nst, GRef{nullptr, 0});
            for (std::size_t i = 0; i < nu * nst; ++i)
                if (gin[i].c != WGEN_NONE) gref[i] = GRef{Rpos + std::size_t(gin[i].c) * Raux, gin[i].jbase};
            // each unit's terms in (b1, MPO entry, operator term) order: slots numbered at first use, the
            // 16-line groups of every slot's lines recorded, lines appended once they have a term
            std::size_t n_alpha = 0;
            const double tt0 = tdbg ? tnow() : 0.0;
            for (std::size_t ui = 0; ui < nu; ++ui) {
                U& un = units[ui];
                un.nw = nw16;
                const GRef* gu = gref.data() + ui * nst;
                for (const auto& lr : lrows) {
                    const uint32_t b1 = lr.first, line = uint32_t(un.lines.size());
                    const uint64_t before = un.nterms;
                    const uint32_t gw = (line >> 4) >> 6;
                    const uint64_t gbit = 1ull << ((line >> 4) & 63);
                    // one term: input state sti of the entry's operator (term k), MPO column b2
                    auto term = [&](uint32_t sti, uint32_t k, uint32_t b2, uint32_t e) {
                        const GRef g = gu[sti];
                        if (!g.rp) return;
                        const int32_t pos = g.rp[b2];
                        if (pos < 0) return;
                        const uint32_t id = g.jbase + uint32_t(pos);
                        uint32_t& sl = slot[id];
                        if (sl == NONE) {
                            sl = uint32_t(un.sl.size());
                            un.sl.push_back(id);
                            un.sig.resize(un.sig.size() + nw16, 0);
                        }
                        un.sig[std::size_t(sl) * nw16 + gw] |= gbit;
                        ++un.nterms;
                        if (bookkeeping) {
                            un.em.push_back(LKD{line, sl});
                            const uint32_t c = gin[ui * nst + sti].c;
                            const uint32_t col = uint32_t(R.offset(c, b2) / rsin_t[sti]);
                            const uint32_t job = tj[std::size_t(sti) * nr + un.rb_out];
                            const uint32_t row[3] = {P.tjob_mps[job], c, col};
                            un.bk.insert(un.bk.end(), row, row + 3);
                            un.bk_a.push_back(og_val[k] * R.conj_scale(c, b2) * (W.scale[e] * L.conj_scale(ci, b1)));
                        }
                    };
                    for (uint32_t e = W.row_ptr[b1]; e < W.row_ptr[b1 + 1]; ++e) {
                        const uint64_t x = row_qb[e];
                        const uint32_t b2 = uint32_t(x), q = uint32_t(x >> 32) + un.st;
                        const uint32_t one = o_one[q];
                        if (one < MPOTables::O_NONE) term(one, og_ptr[q], b2, e);
                        else if (one == MPOTables::O_MANY)
                            for (uint32_t k = og_ptr[q]; k < og_ptr[q + 1]; ++k) term(og_in[k], k, b2, e);
                    }
                    if (un.nterms != before) { un.lines.push_back(lr.second); un.rows.push_back(b1); }
                }
                for (uint32_t id : un.sl) slot[id] = NONE;
                n_alpha += un.nterms;
            }
            if (tdbg) {
#pragma omp atomic
                sum_terms += tnow() - tt0;
            }
            if (n_alpha == 0) continue;
            P.n_alpha += n_alpha;
            const uint64_t s_off = P.s_len;
            P.s_len += (uint64_t(K_c) * stripe + 31) / 32 * 32;
            for (std::size_t ui = 0; ui < nu; ++ui) {
                U& u = units[ui];
                P.flops_s += 2.0 * ls_in * u.ms * double(u.nterms);
                if (!u.nterms) continue;
                slices.assign(u.sl.begin(), u.sl.end());
                // slot order and S-GEMM tiling from the slot signatures
                UnitD ud{};
                ud.nl = uint32_t(u.lines.size()); ud.nk = uint32_t(slices.size()); ud.ne = ls_in * u.ms;
                TileChoice tch;
                const double tt1 = tdbg ? tnow() : 0.0;
                plan_unit_tiles(ud, u.sig.data(), u.nw, corder, tch);
                if (tdbg) {
#pragma omp atomic
                    sum_tiles += tnow() - tt1;
                }
                ctmp.assign(slices.begin(), slices.end());
                for (std::size_t i = 0; i < slices.size(); ++i) slices[i] = ctmp[corder[i]];
                if (bookkeeping) {
                    crank.resize(slices.size());
                    for (uint32_t i = 0; i < uint32_t(slices.size()); ++i) crank[corder[i]] = i;
                    for (LKD& m : u.em) m.k = crank[m.k];
                }
                ud.s_off = s_off + uint64_t(u.offset) * K_c;
                ud.line_stride = ls_in; ud.erows = ls_in; ud.col_stride = K_c; ud.ne = ls_in * u.ms;
                ud.nl = uint32_t(u.lines.size()); ud.line0 = uint32_t(P.line_b1.size());
                ud.nk = uint32_t(slices.size()); ud.slice0 = uint32_t(P.slice_off.size());
                ud.w_off = P.w_len;
                ud.wld = coef_ld(ud.nl);
                P.w_len += uint64_t(ud.wld) * ud.nk;
                for (uint32_t gp : slices) {
                    // slice id -> (job, b2 position) -> T offset of the slice
                    uint32_t job = uint32_t(std::upper_bound(job_pos0.begin(), job_pos0.end(), gp) - job_pos0.begin()) - 1;
                    uint32_t pos = gp - job_pos0[job];
                    P.slice_off.push_back(P.tjobs[job].c_off + uint64_t(pos) * P.tjobs[job].sst);
                }
                // coefficient generation: lines with their L conj scales, slot -> slice id
                lscale.resize(ud.nl);
                for (uint32_t l = 0; l < ud.nl; ++l) lscale[l] = L.conj_scale(ci, u.rows[l]);
                P.cg.add_unit(ud.w_off, ud.wld, u.st, u.rows.data(), lscale.data(), ud.nl, slices, &gin[ui * nst]);
                if (bookkeeping)
                    for (std::size_t i = 0; i < u.em.size(); ++i) {
                        uint32_t row[10] = {lb_in, lb_out, ci, ce, u.offset, u.ms, u.lines[u.em[i].line],
                                            u.bk[3 * i], u.bk[3 * i + 1], u.bk[3 * i + 2]};
                        P.bk_int.insert(P.bk_int.end(), row, row + 10);
                        P.bk_alpha.push_back(u.bk_a[i]);
                    }
                P.line_b1.insert(P.line_b1.end(), u.lines.begin(), u.lines.end());
                // S-GEMM tiles of the unit and the tensor work they execute
                std::size_t tb[N_SHAPES];
                for (int sh = 0; sh < N_SHAPES; ++sh) tb[sh] = P.utiles[sh].size();
                emit_tiles(ud, uint32_t(P.units.size()), tch, P.utiles, P.klist);
                for (int sh = 0; sh < N_SHAPES; ++sh)
                    for (std::size_t t = tb[sh]; t < P.utiles[sh].size(); ++t) {
                        const uint32_t o = P.utiles[sh][t].pad;
                        uint32_t g = 0;
                        for (uint32_t i = 0; i < P.klist[o]; ++i) g += __builtin_popcount(P.klist[o + 1 + i] & 15u);
                        P.flops_sexec += 2.0 * 4.0 * g * shape_bm(sh) * shape_bn(sh);
                    }
                P.units.push_back(ud);
                P.g_elems += uint64_t(ud.ne) * ud.nl;
                P.g_reads += uint64_t(ud.ne) * u.nterms;
                P.flops_sdense += 2.0 * ud.nl * ud.nk * double(ud.ne);  // padding lines not counted
            }
            P.flops_ls += 2.0 * ls_out * ls_in * double(nS) * stripe;
            SegD sg{};
            sg.l_off = L.data_off[ce];
            sg.s_off = s_off;
            sg.ls_in = ls_in; sg.nS = nS; sg.tr = (ci != ce) ? 1 : 0;
            P.segs.push_back({lb_out, sg});
        }
        if (tdbg) part_s[lb_in] = tnow() - tp0;
    } catch (const std::exception& e) {
#pragma omp critical
        err = e.what();
    }
    }
    if (!err.empty()) throw std::runtime_error(err);

    const double t_b = tnow();
    // ---- merge the parts in ket-sector order: prefix offsets, one allocation, parallel copy ----
    struct Base { uint64_t t, s, w, na; uint32_t job, unit, line, slice, smap, kl; std::size_t bk; std::size_t tile[N_SHAPES]; };
    std::vector<Base> base(nl + 1);
    base[0] = Base{};
    for (uint32_t i = 0; i < nl; ++i) {
        const Part& P = parts[i];
        const Base& b = base[i];
        Base& n = base[i + 1];
        n = Base{b.t + P.t_len, b.s + P.s_len, b.w + P.w_len, b.na + P.n_alpha, b.job + uint32_t(P.tjobs.size()),
                 b.unit + uint32_t(P.units.size()), b.line + uint32_t(P.line_b1.size()),
                 b.slice + uint32_t(P.slice_off.size()), b.smap + uint32_t(P.cg.smap_id.size()),
                 b.kl + uint32_t(P.klist.size()), b.bk + P.bk_alpha.size(), {}};
        for (int sh = 0; sh < N_SHAPES; ++sh) n.tile[sh] = b.tile[sh] + P.utiles[sh].size();
        p->flops_sexec += P.flops_sexec;
    }
    const Base& tot = base[nl];
    p->part_job.resize(nl + 1); p->part_unit.resize(nl + 1);
    p->part_t.resize(nl + 1); p->part_s.resize(nl + 1); p->part_w.resize(nl + 1);
    for (uint32_t i = 0; i <= nl; ++i) {
        p->part_job[i] = base[i].job; p->part_unit[i] = base[i].unit;
        p->part_t[i] = base[i].t; p->part_s[i] = base[i].s; p->part_w[i] = base[i].w;
    }
    p->tjobs.resize(tot.job);
    p->units.resize(tot.unit);
    CoefGen& cg = p->cg;
    cg.units.resize(tot.unit);
    cg.gin.resize(std::size_t(tot.unit) * nst);
    cg.line_major.resize(tot.line);
    cg.line_scale.resize(tot.line);
    cg.smap_id.resize(tot.smap);
    cg.smap_slot.resize(tot.smap);
    p->line_b1.resize(tot.line);
    p->slice_off.resize(tot.slice);
    p->klist.resize(tot.kl);
    p->n_alpha = tot.na;
    for (int sh = 0; sh < N_SHAPES; ++sh) p->utiles[sh].resize(tot.tile[sh]);
    if (bookkeeping) { p->bk_int.resize(tot.bk * 10); p->bk_alpha.resize(tot.bk); }
#pragma omp parallel for schedule(dynamic, 1)
    for (int ii = 0; ii < int(nl); ++ii) {
        Part& P = parts[ii];
        const Base& B = base[ii];
        for (std::size_t k = 0; k < P.tjobs.size(); ++k) { TJobD j = P.tjobs[k]; j.c_off += B.t; p->tjobs[B.job + k] = j; }
        for (std::size_t k = 0; k < P.units.size(); ++k) {
            UnitD u = P.units[k];
            u.s_off += B.s; u.line0 += B.line; u.slice0 += B.slice; u.w_off += B.w;
            p->units[B.unit + k] = u;
            WGenUnitD g = P.cg.units[k];
            g.w_off += B.w; g.line0 += B.line; g.map0 += B.smap;
            cg.units[B.unit + k] = g;
        }
        std::copy(P.cg.gin.begin(), P.cg.gin.end(), cg.gin.begin() + std::size_t(B.unit) * nst);
        std::copy(P.cg.line_major.begin(), P.cg.line_major.end(), cg.line_major.begin() + B.line);
        std::copy(P.cg.line_scale.begin(), P.cg.line_scale.end(), cg.line_scale.begin() + B.line);
        std::copy(P.line_b1.begin(), P.line_b1.end(), p->line_b1.begin() + B.line);
        for (std::size_t k = 0; k < P.slice_off.size(); ++k) p->slice_off[B.slice + k] = P.slice_off[k] + B.t;
        std::copy(P.cg.smap_id.begin(), P.cg.smap_id.end(), cg.smap_id.begin() + B.smap);
        std::copy(P.cg.smap_slot.begin(), P.cg.smap_slot.end(), cg.smap_slot.begin() + B.smap);
        if (bookkeeping) {
            std::copy(P.bk_int.begin(), P.bk_int.end(), p->bk_int.begin() + B.bk * 10);
            std::copy(P.bk_alpha.begin(), P.bk_alpha.end(), p->bk_alpha.begin() + B.bk);
        }
        std::copy(P.klist.begin(), P.klist.end(), p->klist.begin() + B.kl);
        for (int sh = 0; sh < N_SHAPES; ++sh)
            for (std::size_t k = 0; k < P.utiles[sh].size(); ++k) {
                TileD t = P.utiles[sh][k];
                t.item += B.unit; t.pad += B.kl;
                p->utiles[sh][B.tile[sh] + k] = t;
            }
        for (auto& sg : P.segs) sg.second.s_off += B.s;
        for (int sh = 0; sh < N_SHAPES; ++sh) P.utiles[sh] = {};
        P.klist = {};
        P.tjobs = {}; P.tjob_mps = {}; P.units = {}; P.cg = CoefGen(); P.line_b1 = {}; P.slice_off = {};
        P.bk_int = {}; P.bk_alpha = {};
    }
    p->t_len = tot.t;
    p->s_len = tot.s;
    p->w_len = tot.w;
    cg.w_len = tot.w;
    std::vector<std::vector<SegD>> per_out(nl);
    for (uint32_t i = 0; i < nl; ++i) {
        const Part& P = parts[i];
        for (auto& sg : P.segs) per_out[sg.first].push_back(sg.second);
        p->flops_t += P.flops_t; p->flops_s += P.flops_s; p->flops_ls += P.flops_ls; p->flops_sdense += P.flops_sdense;
        p->g_elems += P.g_elems; p->g_reads += P.g_reads;
    }
    for (uint32_t j = 0; j < p->tjobs.size(); ++j)
        if (p->tjobs[j].M && p->tjobs[j].N) add_tiles(p->ttiles, j, p->tjobs[j].M, p->tjobs[j].N);
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
                            p->kitems[sh].push_back(KItemD{uint32_t(p->otiles[sh].size()), sg, k0, std::min(Kc, k0 + KCHUNK),
                                                           uint32_t(p->kitems[sh].size())});
                    }
                    t.nparts = uint32_t(p->kitems[sh].size()) - t.part0;
                    p->otiles[sh].push_back(t);
                }
        }
        p->outs.push_back(o);
    }
    if (tdbg) {
        double psum = 0, pmax = 0;
        for (double t : part_s) { psum += t; pmax = std::max(pmax, t); }
        std::fprintf(stderr, "plan: tables %.4f s, parts %.4f s (sum %.4f s: terms %.4f, tiles %.4f; largest %.4f s), merge %.4f s; "
                     "%zu units, %llu coefficient terms, %zu S tiles, %.3e dense coefficients\n", t_a - t_0, t_b - t_a, psum,
                     sum_terms, sum_tiles, pmax, tnow() - t_b,
                     p->units.size(), (unsigned long long)p->n_alpha,
                     p->utiles[0].size() + p->utiles[1].size() + p->utiles[2].size() + p->utiles[3].size(), double(p->w_len));
    }
    uint64_t pl = 0;
    for (int sh = 0; sh < N_SHAPES; ++sh) pl = std::max<uint64_t>(pl, uint64_t(p->kitems[sh].size()) * shape_bm(sh) * shape_bn(sh));
    p->p_len = pl;
    p->flops = p->flops_t + p->flops_ls + p->flops_s;
    return p;
}

}  // namespace qcm
