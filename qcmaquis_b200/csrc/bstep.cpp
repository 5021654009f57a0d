// Boundary propagation on the device (overlap_mpo_left/right_step,
// contractions/boundary_ops/move_boundary.hpp:147-404).
//
// Right step (rshtm_t_tasks / rshtm_tasks, right_tasks.hpp:39-167; prop_r, tasks.cpp:243-284):
//   T = ket_slab * R_old[ci_eff]          -> grouped T-GEMM (same kernel as H_eff)
//   S = sum alpha * T slices               -> unit S-GEMM (same kernel as H_eff)
//   R_new[b] = S_b * bra^T                 -> batched GEMM, one row-blocked job per cohort
// Left step (lshtm_t_tasks / lshtm_tasks, left_tasks.hpp:38-172; create_T_left,
// create_s, prop_l, tasks.cpp:198-241, 425-454, 545-601):
//   T_b = L_old[ci_eff]_b(^T) * ket_slab   -> batched GEMM, one row-blocked job per T job
//   S (stripe x nS*rs_ket) = sum alpha * T slices  -> unit S-GEMM with the left layout
//   L_new = bra^T * S                      -> batched GEMM, one job per cohort
// Cohort offsets follow Cohort::finalize (tasks.cpp:506-526): MPO indices with
// coefficients get consecutive block positions in index order.
//
// The schedule is built per ket sector in parallel (OpenMP) from flat lookup
// tables and merged in sector order, so the result does not depend on the
// thread count.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <unordered_map>

#include "dmrg_dev.hpp"

namespace qcm {

namespace {
constexpr uint32_t NONE = 0xffffffffu;

// QCM_STEP_TIMING=1 prints host schedule time and device time of every boundary step
double step_now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
void step_report(const char* side, double t0, double tp, double t1, cudaStream_t s) {
    static const bool on = std::getenv("QCM_STEP_TIMING") != nullptr;
    if (!on) return;
    QCM_CUDA(cudaStreamSynchronize(s));
    std::fprintf(stderr, "[bstep %s] schedule %.4f s (parts %.4f, merge %.4f), device %.4f s\n", side, t1 - t0, tp - t0,
                 t1 - tp, step_now() - t1);
}

void add_tiles(std::vector<TileD>* tiles, uint32_t item, uint32_t M, uint32_t N) {
    int sh = shape_for_rows(M);
    uint32_t bm = shape_bm(sh), bn = shape_bn(sh);
    for (uint32_t n0 = 0; n0 < N; n0 += bn)
        for (uint32_t m0 = 0; m0 < M; m0 += bm) tiles[sh].push_back(TileD{item, m0, n0, 0});
}

// sparse operator entries of an MPO tensor, CSR per operator (the tensor's cached tables)
struct OpCSR {
    std::shared_ptr<const MPOTables> t;
    const std::vector<uint32_t>& ptr;
    const std::vector<uint32_t>& in;
    const std::vector<uint32_t>& out;
    explicit OpCSR(const MPOTensor& W) : t(W.tables()), ptr(t->optr), in(t->oin), out(t->oout) {}
};

// cohort of (sector a, sector b) by positions, and its storage partner
void cohort_tables(const BoundaryIndexH& B, const Index& ia, const Index& ib, std::vector<uint32_t>& ci_t,
                   std::vector<uint32_t>& ce_t) {
    const std::size_t na = ia.size(), nb = ib.size();
    ci_t.assign(na * nb, NONE);
    ce_t.assign(na * nb, NONE);
    for (std::size_t a = 0; a < na; ++a)
        for (std::size_t b = 0; b < nb; ++b) {
            uint32_t ci = B.cohort_index(ia[a].first, ib[b].first);
            if (ci == B.n_cohorts()) continue;
            uint32_t ce = B.tr[ci] ? B.cohort_index(ib[b].first, ia[a].first) : ci;
            if (ce == B.n_cohorts()) throw std::runtime_error("boundary step: transposed cohort without partner");
            ci_t[a * nb + b] = ci;
            ce_t[a * nb + b] = ce;
        }
}

// One ket sector's share of a boundary step; all offsets relative to the part.
struct BPart {
    std::vector<TJobD> tjobs;      // right step: grouped T-GEMM jobs
    std::vector<GemmJob> tgemm;    // left step: T_b jobs (batched GEMM)
    uint64_t t_len = 0;
    SBuild sb;
    uint64_t s_len = 0;
    struct Coh { uint32_t bra, ket, nS; uint64_t s_off; std::vector<int64_t> offs; };
    std::vector<Coh> coh;
};

// MPO entries bucketed by the charge difference D of the (bra, ket) sector pair they can
// contribute to.  In a symmetric boundary every block (cohort, b) has the same cohort charge
// difference q(b), and a TwoU1 operator changes the charge by a fixed amount, so an entry
// (line m, other index x, operator o) contributes only when D = sign * q(x) + dq(o), with
// (sign, the operator's change) fixed by the step direction.  Entries whose key is not
// defined (an index seen with two differences, an operator with mixed changes) go to every
// bucket; entries whose other index has no block in the boundary contribute nothing and are
// dropped.  Within a bucket the entries keep the line order of the MPO tensor.
struct EntryBuckets {
    std::vector<Charge> keys;
    std::vector<std::vector<uint32_t>> ptr, ent;  // per bucket: CSR over lines -> entry index
    int wild = -1;                                // bucket of the keyless entries alone
    int find(Charge d) const {
        for (std::size_t i = 0; i < keys.size(); ++i)
            if (keys[i] == d) return int(i);
        return wild;
    }
};

// by_row: lines = rows b1 (entry order of row_ptr), other index b2, key = -q(b2) - dq;
// otherwise lines = columns b2 (col_ptr / col_ent order), other index b1, key = q(b1) + dq.
EntryBuckets bucket_entries(const MPOTensor& W, const BoundaryIndexH& B, const Index& phys, bool by_row) {
    StateMap sm(phys);
    const uint32_t nst = uint32_t(sm.nstates());
    // q(b): cohort charge difference (bra - ket) of the blocks at MPO index b
    std::vector<Charge> qb(B.aux);
    std::vector<uint8_t> qstate(B.aux, 0);  // 0 = no block, 1 = defined, 2 = inconsistent
    for (uint32_t c = 0; c < B.n_cohorts(); ++c) {
        const Charge d = B.bra[B.cbra[c]].first - B.ket[B.cket[c]].first;
        for (uint32_t b = 0; b < B.aux; ++b) {
            if (B.offsets[std::size_t(c) * B.aux + b] < 0) continue;
            if (qstate[b] == 0) { qb[b] = d; qstate[b] = 1; }
            else if (qstate[b] == 1 && !(qb[b] == d)) qstate[b] = 2;
        }
    }
    // dq(o) = q(out) - q(in) of every term of operator o
    const std::size_t nops = W.ops->size();
    std::vector<Charge> dq(nops);
    std::vector<uint8_t> dstate(nops, 0);
    for (std::size_t o = 0; o < nops; ++o) {
        const SparseOp& op = (*W.ops)[o];
        for (std::size_t e = 0; e < op.val.size(); ++e) {
            if (op.in[e] >= nst || op.out[e] >= nst) { dstate[o] = 2; break; }
            const Charge d = phys[sm.sector[op.out[e]]].first - phys[sm.sector[op.in[e]]].first;
            if (dstate[o] == 0) { dq[o] = d; dstate[o] = 1; }
            else if (!(dq[o] == d)) { dstate[o] = 2; break; }
        }
    }
    const uint32_t nlines = by_row ? W.rows : W.cols;
    const std::vector<uint32_t>& lptr = by_row ? W.row_ptr : W.col_ptr;
    EntryBuckets eb;
    // key of each entry (in line order): bucket index, -2 = keyless, -1 = dropped
    std::vector<int> kb(W.b1.size(), -1);
    for (uint32_t m = 0; m < nlines; ++m)
        for (uint32_t q = lptr[m]; q < lptr[m + 1]; ++q) {
            const uint32_t e = by_row ? q : W.col_ent[q];
            const uint32_t x = by_row ? W.b2[e] : W.b1[e], o = W.op[e];
            if (x >= B.aux || qstate[x] == 0) continue;  // no block: the entry contributes nothing
            if (qstate[x] == 2 || dstate[o] != 1) { kb[q] = -2; continue; }
            const Charge key = by_row ? -qb[x] - dq[o] : qb[x] + dq[o];
            std::size_t i = 0;
            while (i < eb.keys.size() && !(eb.keys[i] == key)) ++i;
            if (i == eb.keys.size()) eb.keys.push_back(key);
            kb[q] = int(i);
        }
    const std::size_t nk = eb.keys.size();
    eb.wild = int(nk);
    eb.ptr.assign(nk + 1, std::vector<uint32_t>(nlines + 1, 0));
    eb.ent.assign(nk + 1, {});
    for (uint32_t m = 0; m < nlines; ++m) {
        for (std::size_t i = 0; i <= nk; ++i) eb.ptr[i][m] = uint32_t(eb.ent[i].size());
        for (uint32_t q = lptr[m]; q < lptr[m + 1]; ++q) {
            const uint32_t e = by_row ? q : W.col_ent[q];
            if (kb[q] == -1) continue;
            if (kb[q] == -2) {
                for (std::size_t i = 0; i <= nk; ++i) eb.ent[i].push_back(e);
            } else {
                eb.ent[std::size_t(kb[q])].push_back(e);
            }
        }
    }
    for (std::size_t i = 0; i <= nk; ++i) eb.ptr[i][nlines] = uint32_t(eb.ent[i].size());
    return eb;
}

// One cohort's terms of one unit: lines = distinct MPO line indices in visiting order (they
// ascend), terms = (local line, slice id)
struct UnitTerms {
    std::vector<uint32_t> majors, rows;
    std::vector<LKD> em;
    void clear() { majors.clear(); rows.clear(); em.clear(); }
    void add(uint32_t major, uint32_t id) {
        if (majors.empty() || majors.back() != major) majors.push_back(major);
        em.push_back(LKD{uint32_t(majors.size() - 1), id});
    }
};

// Units of one cohort -> SBuild; S row block of a line = pos[its MPO index] (finalize positions)
void emit_units(BPart& P, const std::vector<uint32_t>& pos, uint64_t s_off, const std::vector<uint64_t>& unit_off,
                uint64_t line_stride, const std::vector<uint32_t>& erows, uint32_t col_stride, const std::vector<uint32_t>& ne,
                const std::vector<uint32_t>& ust, std::vector<UnitTerms>& ut, const std::vector<WGenInD>& gin, uint32_t nst,
                std::vector<uint32_t>& slot, const JobSlices& js) {
    for (std::size_t u = 0; u < ust.size(); ++u) {
        UnitTerms& x = ut[u];
        if (x.em.empty()) continue;
        x.rows.resize(x.majors.size());
        for (std::size_t l = 0; l < x.majors.size(); ++l) x.rows[l] = pos[x.majors[l]];
        P.sb.add_unit(s_off + unit_off[u], line_stride, erows[u], col_stride, ne[u], ust[u], x.rows, x.majors, x.em, slot, js,
                      &gin[u * nst]);
    }
}

// Concatenates the parts' S-build lists in part order (offsets relative to each part), with
// the parts' T / S buffer bases; the copies run in parallel over parts.
template <class Part>
void merge_sbuilds(std::vector<Part>& parts, SBuild& dst, const std::vector<uint64_t>& t_base,
                   const std::vector<uint64_t>& s_base) {
    const std::size_t np = parts.size();
    const uint32_t nst = dst.cg.nst;
    struct B { std::size_t unit, line, slice, smap, kl; uint64_t w; std::size_t tile[N_SHAPES]; };
    std::vector<B> base(np + 1);
    base[0] = B{};
    for (std::size_t i = 0; i < np; ++i) {
        const SBuild& x = parts[i].sb;
        B b = base[i];
        b.unit += x.units.size(); b.line += x.line_b1.size(); b.slice += x.slice_off.size(); b.smap += x.cg.smap_id.size();
        b.kl += x.klist.size(); b.w += x.w_len;
        for (int k = 0; k < N_SHAPES; ++k) b.tile[k] += x.utiles[k].size();
        base[i + 1] = b;
    }
    const B& tot = base[np];
    dst.units.resize(tot.unit); dst.line_b1.resize(tot.line); dst.slice_off.resize(tot.slice);
    dst.klist.resize(tot.kl); dst.w_len = tot.w;
    CoefGen& cg = dst.cg;
    cg.units.resize(tot.unit); cg.gin.resize(tot.unit * nst); cg.line_major.resize(tot.line); cg.line_scale.resize(tot.line);
    cg.smap_id.resize(tot.smap); cg.smap_slot.resize(tot.smap); cg.w_len = tot.w;
    for (int k = 0; k < N_SHAPES; ++k) dst.utiles[k].resize(tot.tile[k]);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long ii = 0; ii < (long long)np; ++ii) {
        SBuild& x = parts[ii].sb;
        const B& b = base[ii];
        for (std::size_t k = 0; k < x.units.size(); ++k) {
            UnitD u = x.units[k];
            u.s_off += s_base[ii]; u.line0 += uint32_t(b.line); u.slice0 += uint32_t(b.slice); u.w_off += b.w;
            dst.units[b.unit + k] = u;
            WGenUnitD g = x.cg.units[k];
            g.w_off += b.w; g.line0 += uint32_t(b.line); g.map0 += uint32_t(b.smap);
            cg.units[b.unit + k] = g;
        }
        std::copy(x.cg.gin.begin(), x.cg.gin.end(), cg.gin.begin() + b.unit * nst);
        std::copy(x.cg.line_major.begin(), x.cg.line_major.end(), cg.line_major.begin() + b.line);
        std::copy(x.cg.line_scale.begin(), x.cg.line_scale.end(), cg.line_scale.begin() + b.line);
        std::copy(x.cg.smap_id.begin(), x.cg.smap_id.end(), cg.smap_id.begin() + b.smap);
        std::copy(x.cg.smap_slot.begin(), x.cg.smap_slot.end(), cg.smap_slot.begin() + b.smap);
        std::copy(x.line_b1.begin(), x.line_b1.end(), dst.line_b1.begin() + b.line);
        for (std::size_t k = 0; k < x.slice_off.size(); ++k) dst.slice_off[b.slice + k] = x.slice_off[k] + t_base[ii];
        std::copy(x.klist.begin(), x.klist.end(), dst.klist.begin() + b.kl);
        for (int sh = 0; sh < N_SHAPES; ++sh)
            for (std::size_t k = 0; k < x.utiles[sh].size(); ++k) {
                TileD t = x.utiles[sh][k];
                t.item += uint32_t(b.unit); t.pad += uint32_t(b.kl);
                dst.utiles[sh][b.tile[sh] + k] = t;
            }
        x = SBuild();
    }
}

}  // namespace

uint64_t JobSlices::offset(uint32_t id) const {
    const std::size_t j = std::size_t(std::upper_bound(pos0.begin(), pos0.end(), id) - pos0.begin());
    if (j == 0 || j >= pos0.size()) throw std::runtime_error("S unit: slice id outside the T jobs");
    return c_off[j - 1] + uint64_t(id - pos0[j - 1]) * bsize[j - 1];
}

void SBuild::add_unit(uint64_t s_off, uint64_t line_stride, uint32_t erows, uint32_t col_stride, uint32_t ne, uint32_t st_out,
                      const std::vector<uint32_t>& rows, const std::vector<uint32_t>& majors, std::vector<LKD>& ents,
                      std::vector<uint32_t>& slot, const JobSlices& js, const WGenInD* in_row) {
    if (ents.empty() || ne == 0) return;
    // slices numbered in first-use order
    std::vector<uint32_t> slices;
    for (LKD& e : ents) {
        uint32_t& sl = slot[e.k];
        if (sl == NONE) { sl = uint32_t(slices.size()); slices.push_back(e.k); }
        e.k = sl;
    }
    for (uint32_t id : slices) slot[id] = NONE;
    UnitD u{};
    u.s_off = s_off; u.line_stride = line_stride; u.erows = erows; u.col_stride = col_stride; u.ne = ne;
    u.nl = uint32_t(rows.size()); u.line0 = uint32_t(line_b1.size());
    u.nk = uint32_t(slices.size()); u.slice0 = uint32_t(slice_off.size());
    u.w_off = w_len;
    u.wld = coef_ld(u.nl);
    w_len += uint64_t(u.wld) * u.nk;
    line_b1.insert(line_b1.end(), rows.begin(), rows.end());
    for (uint32_t id : slices) slice_off.push_back(js.offset(id));
    const std::vector<double> ones(u.nl, 1.0);
    cg.add_unit(u.w_off, u.wld, st_out, majors.data(), ones.data(), u.nl, slices, in_row);
    add_unit_tiles(u, uint32_t(units.size()), ents.data(), ents.size(), utiles, klist);
    units.push_back(u);
}

void SBuild::validate(uint64_t t_len, uint64_t s_len) const {
    if (cg.units.size() != units.size() || cg.w_len != w_len) throw std::runtime_error("S build: coefficient tables differ from the units");
    for (std::size_t i = 0; i < units.size(); ++i) {
        const UnitD& u = units[i];
        if (!u.ne || !u.nl) continue;
        const WGenUnitD& g = cg.units[i];
        if (g.w_off != u.w_off || g.wld != u.wld || g.nl != u.nl || g.nk != u.nk || g.line0 != u.line0)
            throw std::runtime_error("S build: coefficient unit differs from its S unit");
        if (u.wld < u.nl || u.wld % 4 || u.w_off % 4 || u.w_off + uint64_t(u.wld) * u.nk > w_len)
            throw std::runtime_error("device work list out of bounds: coefficient block");
        if (u.erows == 0 || u.ne % u.erows) throw std::runtime_error("S unit: element count is not a whole number of columns");
        uint32_t maxline = 0;
        for (uint32_t l = 0; l < u.nl; ++l) maxline = std::max(maxline, line_b1[u.line0 + l]);
        const uint64_t last = u.s_off + uint64_t(maxline) * u.line_stride + (u.erows - 1) + uint64_t(u.ne / u.erows - 1) * u.col_stride;
        if (last >= s_len) throw std::runtime_error("device work list out of bounds: S unit");
        for (uint32_t k = 0; k < u.nk; ++k)
            if (slice_off[u.slice0 + k] + u.ne > t_len) throw std::runtime_error("device work list out of bounds: T slice");
    }
    for (int sh = 0; sh < N_SHAPES; ++sh)
        for (const TileD& t : utiles[sh]) {
            if (t.item >= units.size() || std::size_t(t.pad) >= klist.size() || std::size_t(t.pad) + 1 + klist[t.pad] > klist.size())
                throw std::runtime_error("S tile outside its work lists");
            const UnitD& u = units[t.item];
            for (uint32_t i = 0; i < klist[t.pad]; ++i)
                if (uint32_t(klist[t.pad + 1 + i] >> 4) * 16 >= u.nk) throw std::runtime_error("S tile: k-step out of range");
        }
}

void SBuild::upload(cudaStream_t s) {
    d_units.upload(units, s);
    for (int k = 0; k < N_SHAPES; ++k) d_utiles[k].upload(utiles[k], s);
    d_line_b1.upload(line_b1, s);
    d_slice_off.upload(slice_off, s);
    d_klist.upload(klist, s);
    cg.upload(s);
}

void complement_transpose(BoundaryIndexH& x, const std::vector<int32_t>& herm, const std::vector<int32_t>& phase, bool forward) {
    // add transposed partners of every cohort and fill Hermitian blocks (boundary.h:150-179)
    const uint32_t n0 = x.n_cohorts();
    std::unordered_map<uint64_t, uint32_t> where;
    for (uint32_t ci = 0; ci < n0; ++ci) where[(uint64_t(x.cbra[ci]) << 32) | x.cket[ci]] = ci;
    for (uint32_t ciA = 0; ciA < n0; ++ciA) {
        Charge lb = x.bra[x.cbra[ciA]].first, rb = x.ket[x.cket[ciA]].first;
        std::size_t pb = x.bra.position(rb), pk = x.ket.position(lb);
        if (pb >= x.bra.size() || pk >= x.ket.size()) continue;
        auto it = where.find((uint64_t(pb) << 32) | pk);
        uint32_t ciB;
        if (it == where.end()) {
            ciB = x.n_cohorts();
            where[(uint64_t(pb) << 32) | pk] = ciB;
            x.cbra.push_back(uint32_t(pb)); x.cket.push_back(uint32_t(pk));
            x.lsz.push_back(uint32_t(x.bra[pb].second)); x.rsz.push_back(uint32_t(x.ket[pk].second));
            x.nb.push_back(0); x.tr.push_back(1);
            x.offsets.resize(x.offsets.size() + x.aux, -1);
            x.cscale.resize(x.cscale.size() + x.aux, 1.0);
        } else {
            ciB = it->second;
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
        if (j.sst < j.brs * j.M || j.sst % 4 || j.c_off % 4 || j.c_off + uint64_t(j.N / j.brs) * j.sst > t_len)
            throw std::runtime_error("device work list out of bounds: T output");
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

// a new boundary of a finished index (copied), zeroed
std::unique_ptr<DevBoundary> alloc_boundary(const BoundaryIndexH& idx, cudaStream_t s) {
    auto B = std::make_unique<DevBoundary>();
    B->idx = idx;
    B->data.alloc(B->idx.total ? B->idx.total : 1);
    QCM_CUDA(cudaMemsetAsync(B->data.get(), 0, (B->idx.total ? B->idx.total : 1) * sizeof(double), s));
    return B;
}

template <class T> uint64_t dbytes(const DBuf<T>& b) { return uint64_t(b.size()) * sizeof(T); }

void hash_blocks(KeyHash& k, const DBlocks& b) {
    k.word(b.n());
    k.word(b.total);
    for (std::size_t i = 0; i < b.n(); ++i) {
        k.word(uint64_t(uint32_t(b.lc[i].a)) | (uint64_t(uint32_t(b.lc[i].b)) << 32));
        k.word(uint64_t(uint32_t(b.rc[i].a)) | (uint64_t(uint32_t(b.rc[i].b)) << 32));
        k.word(uint64_t(b.rows[i]) | (uint64_t(b.cols[i]) << 32));
        k.word(b.off[i]);
    }
}

// structure of a boundary step: side, old boundary, site tensors (indices and block layouts), MPO tensor
uint64_t step_key(int side, const DevBoundary& B, const DMPS& ket, const DMPS* bra, const MPOTensor& W, bool symmetric) {
    KeyHash k;
    k.word(uint64_t(side));
    k.word(boundary_key(B));
    k.index(ket.phys);
    k.index(ket.left);
    k.index(ket.right);
    hash_blocks(k, ket.b);
    if (bra) {
        k.index(bra->left);
        k.index(bra->right);
        hash_blocks(k, bra->b);
    }
    k.word(uint64_t(reinterpret_cast<uintptr_t>(&W)));
    k.word(W.b1.size());
    k.word(symmetric ? 1 : 0);
    return k.h;
}

}  // namespace

// One boundary step's schedule, built once and run again while the structure stays the same.
struct BStepPlan {
    std::vector<GemmJob> tj_gemm;  // left step: T_b jobs (A = old boundary, B = ket)
    std::vector<TJobD> tjobs;      // right step: T-GEMM jobs and tiles (A = ket, B = old boundary)
    std::vector<TileD> ttiles[N_SHAPES];
    DBuf<TJobD> d_tjobs;
    DBuf<TileD> d_ttiles[N_SHAPES];
    SBuild sb;                     // units and coefficient tables, on the device
    BoundaryIndexH nidx;           // the new boundary's index (finished)
    std::vector<GemmJob> prop;     // new boundary from S and the bra / ket
    uint64_t t_len = 0, s_len = 0;
    uint64_t device_bytes() const {
        uint64_t b = dbytes(d_tjobs) + dbytes(sb.d_units) + dbytes(sb.d_klist) + dbytes(sb.d_line_b1) + dbytes(sb.d_slice_off);
        for (int k = 0; k < N_SHAPES; ++k) b += dbytes(d_ttiles[k]) + dbytes(sb.d_utiles[k]);
        const CoefGen& g = sb.cg;
        b += dbytes(g.d_units) + dbytes(g.d_gin) + dbytes(g.d_line_major) + dbytes(g.d_smap_id) + dbytes(g.d_smap_slot) +
             dbytes(g.d_m_ptr) + dbytes(g.d_m_other) + dbytes(g.d_m_op) + dbytes(g.d_o_ptr) + dbytes(g.d_o_in) +
             dbytes(g.d_line_scale) + dbytes(g.d_m_scale) + dbytes(g.d_o_val) + dbytes(g.d_b_cs) + dbytes(g.d_b_pos);
        return b;
    }
};

namespace {

// T, S and the projections of a left step's schedule
std::unique_ptr<DevBoundary> run_left(Ctx& c, BStepPlan& P, const DevBoundary& Lold, const DMPS& ket, const DMPS& bra) {
    auto Ln = alloc_boundary(P.nidx, c.s);
    Ctx::ensure(c.T, P.t_len ? P.t_len : 1);
    Ctx::ensure(c.S, P.s_len ? P.s_len : 1);
    batched_gemm(P.tj_gemm, Lold.data.get(), Lold.idx.total, ket.b.d.get(), ket.b.total, c.T.get(), P.t_len, c.gjobs, c.gtiles,
                 c.s);
    if (P.s_len) QCM_CUDA(cudaMemsetAsync(c.S.get(), 0, P.s_len * sizeof(double), c.s));
    Ctx::ensure(c.W, P.sb.w_len ? P.sb.w_len : 1);
    P.sb.cg.generate(c.W.get(), c.s);
    run_sgemm(P.sb.d_units.get(), P.sb.d_utiles, P.sb.utiles, P.sb.d_line_b1.get(), P.sb.d_slice_off.get(), P.sb.d_klist.get(),
              c.W.get(), c.T.get(), c.S.get(), c.s);
    batched_gemm(P.prop, bra.b.d.get(), bra.b.total, c.S.get(), P.s_len, Ln->data.get(), Ln->idx.total, c.gjobs, c.gtiles, c.s);
    return Ln;
}

// the same for a right step
std::unique_ptr<DevBoundary> run_right(Ctx& c, BStepPlan& P, const DevBoundary& Rold, const DMPS& ket) {
    auto Rn = alloc_boundary(P.nidx, c.s);
    Ctx::ensure(c.T, P.t_len ? P.t_len : 1);
    Ctx::ensure(c.S, P.s_len ? P.s_len : 1);
    run_tgemm(P.d_tjobs.get(), P.d_ttiles, P.ttiles, ket.b.d.get(), Rold.data.get(), c.T.get(), c.s);
    if (P.s_len) QCM_CUDA(cudaMemsetAsync(c.S.get(), 0, P.s_len * sizeof(double), c.s));
    Ctx::ensure(c.W, P.sb.w_len ? P.sb.w_len : 1);
    P.sb.cg.generate(c.W.get(), c.s);
    run_sgemm(P.sb.d_units.get(), P.sb.d_utiles, P.sb.utiles, P.sb.d_line_b1.get(), P.sb.d_slice_off.get(), P.sb.d_klist.get(),
              c.W.get(), c.T.get(), c.S.get(), c.s);
    // A = S scratch, B = ket data, C = new boundary: three different base pointers
    batched_gemm(P.prop, c.S.get(), P.s_len, ket.b.d.get(), ket.b.total, Rn->data.get(), Rn->idx.total, c.gjobs, c.gtiles, c.s);
    return Rn;
}

}  // namespace

namespace {
// GEMM jobs that add into shared target blocks, run in rounds (round r = the r-th job of every
// target) so that each block is summed in job order
void run_accumulating(const std::vector<GemmJob>& jobs, const std::vector<std::size_t>& target, const double* A, uint64_t a_len,
                      const double* B, uint64_t b_len, double* C, uint64_t c_len, Ctx& c) {
    std::unordered_map<std::size_t, std::size_t> seen;
    std::vector<std::vector<GemmJob>> rounds;
    for (std::size_t i = 0; i < jobs.size(); ++i) {
        const std::size_t r = seen[target[i]]++;
        if (rounds.size() <= r) rounds.resize(r + 1);
        rounds[r].push_back(jobs[i]);
    }
    for (auto& r : rounds) batched_gemm(r, A, a_len, B, b_len, C, c_len, c.gjobs, c.gtiles, c.s);
}
}  // namespace

// ---------------------------------------------------------------------------
static std::unique_ptr<DevBoundary> step_right(Ctx& c, const DevBoundary& Rold, const DMPS& ket, const MPOTensor& W,
                                               bool symmetric, DensityNoise* dn, BStepCache* cache) {
    if (!ket.right_paired) throw std::runtime_error("boundary_step_right: ket must be right-paired");
    const double tb0 = step_now();
    uint64_t key = 0;
    if (cache && !dn) {
        key = step_key(1, Rold, ket, nullptr, W, symmetric);
        if (cache->plan && cache->key == key) {
            auto Rn = run_right(c, *cache->plan, Rold, ket);
            cache->hit = true;
            step_report("right (cached)", tb0, tb0, tb0, c.s);
            return Rn;
        }
        cache->plan.reset();
        cache->bytes = 0;
        cache->hit = false;
    }
    const BoundaryIndexH& R = Rold.idx;
    const Index& phys = ket.phys;
    const Index& left = ket.left;
    const Index& right = ket.right;
    if (W.cols != R.aux) throw std::runtime_error("boundary_step_right: MPO column dimension differs from the boundary");
    ProductBasis rpb(phys, right, true);
    StateMap sm(phys);
    const uint32_t nl = uint32_t(left.size()), nr = uint32_t(right.size()), nps = uint32_t(phys.size());
    const uint32_t nst = uint32_t(sm.nstates());
    // block offsets of the (right-paired) ket per left sector
    std::vector<uint64_t> koff(nl, 0);
    std::vector<uint32_t> kcols(nl, 0);
    std::vector<uint8_t> kok(nl, 0);
    for (uint32_t lb = 0; lb < nl; ++lb) {
        std::size_t k = ket.b.find_l(left[lb].first);
        if (k < ket.b.n()) { koff[lb] = ket.b.off[k]; kcols[lb] = ket.b.cols[k]; kok[lb] = 1; }
    }
    // right sector, its size and column offset for (left sector, phys sector)
    struct RSec { uint32_t rb, rs, off; };
    std::vector<RSec> rsec(std::size_t(nl) * nps, RSec{NONE, 0, 0});
    for (uint32_t lb = 0; lb < nl; ++lb)
        for (uint32_t s = 0; s < nps; ++s) {
            const Charge rc = left[lb].first + phys[s].first;
            const std::size_t rb = right.position(rc);
            if (rb < nr) rsec[std::size_t(lb) * nps + s] = RSec{uint32_t(rb), uint32_t(right[rb].second), uint32_t(rpb(phys[s].first, rc))};
        }
    std::vector<uint32_t> Rci, Rce;
    cohort_tables(R, right, right, Rci, Rce);
    const OpCSR oc(W);

    // coefficient generation: lines iterate MPO rows b1, slices come from R_old cohorts
    SBuild sb;
    sb.cg.set_mpo(W, true);
    if (sb.cg.nst != nst) throw std::runtime_error("boundary_step_right: MPO physical basis differs from the MPS");
    sb.cg.set_boundary(R);
    const int32_t* Rpos = sb.cg.b_pos.data();
    const std::size_t Raux = R.aux;
    const EntryBuckets eb = bucket_entries(W, R, phys, true);

    std::vector<BPart> parts(nl);
    std::string err;
#pragma omp parallel
    {
    std::vector<UnitTerms> ut;
#pragma omp for schedule(dynamic, 1)
    for (int lbi = 0; lbi < int(nl); ++lbi) try {
        const uint32_t lb_ket = uint32_t(lbi);
        if (!kok[lb_ket]) continue;
        BPart& P = parts[lb_ket];
        P.sb.cg.nst = nst;
        const Charge lc_ket = left[lb_ket].first;
        const uint32_t ls_ket = uint32_t(left[lb_ket].second);
        // T jobs (rshtm_t_tasks): one per (input state, bra right sector); slice ids per R block
        std::vector<uint32_t> tj(std::size_t(nst) * nr, NONE);
        JobSlices js;
        std::vector<uint32_t> tj_first, tj_count;
        for (uint32_t st = 0; st < nst; ++st) {
            const RSec& ri = rsec[std::size_t(lb_ket) * nps + sm.sector[st]];
            if (ri.rb == NONE) continue;
            for (uint32_t rbb = 0; rbb < nr; ++rbb) {
                const uint32_t ci = Rci[std::size_t(ri.rb) * nr + rbb];
                if (ci == NONE) continue;
                const uint32_t ce = Rce[std::size_t(ri.rb) * nr + rbb];
                TJobD j{};
                j.a_off = koff[lb_ket] + uint64_t(ri.off + uint32_t(sm.sub[st]) * ri.rs) * ls_ket;
                j.b_off = R.data_off[ce];
                j.c_off = P.t_len;
                j.M = ls_ket; j.K = ri.rs; j.brs = R.rsz[ci]; j.N = R.nb[ce] * j.brs; j.lda = ls_ket;
                j.tr = ci != ce;
                j.sst = slice_stride(j.brs, j.M);
                tj[std::size_t(st) * nr + rbb] = uint32_t(P.tjobs.size());
                tj_first.push_back(js.add(j.c_off, j.sst, R.nb[ce]));
                tj_count.push_back(R.nb[ce]);
                P.t_len += (uint64_t(R.nb[ce]) * j.sst + 31) / 32 * 32;
                P.tjobs.push_back(j);
            }
        }
        std::vector<uint32_t> slot(js.pos0.back() + 1, NONE);
        // cohorts (rshtm_tasks)
        std::vector<int> unit_of(nst, -1);
        std::vector<uint32_t> line_count(W.rows, 0), pos(W.rows, NONE);
        for (uint32_t lb_bra = 0; lb_bra < nl; ++lb_bra) {
            const Charge lc_bra = left[lb_bra].first;
            if (std::abs(lc_ket.particles() - lc_bra.particles()) > 2 || !kok[lb_bra]) continue;
            const uint32_t ls_bra = uint32_t(left[lb_bra].second);
            // units: output states whose right sector exists
            std::vector<uint32_t> ust, urbb, uer, une;
            std::vector<uint64_t> uoff;
            std::fill(unit_of.begin(), unit_of.end(), -1);
            for (uint32_t st = 0; st < nst; ++st) {
                const RSec& ro = rsec[std::size_t(lb_bra) * nps + sm.sector[st]];
                if (ro.rb == NONE) continue;
                unit_of[st] = int(ust.size());
                ust.push_back(st); urbb.push_back(ro.rb);
                uoff.push_back(uint64_t(ro.off + uint32_t(sm.sub[st]) * ro.rs));
                uer.push_back(ls_ket); une.push_back(ls_ket * ro.rs);
            }
            const std::size_t nu = ust.size();
            if (ut.size() < nu) ut.resize(nu);
            for (std::size_t u = 0; u < nu; ++u) ut[u].clear();
            // (R cohort, first slice id) of each (unit, input state) and its number of blocks
            std::vector<WGenInD> gin(nu * nst, WGenInD{WGEN_NONE, WGEN_NONE});
            std::vector<uint32_t> gcnt(nu * nst, 0);
            for (uint32_t sti = 0; sti < nst; ++sti) {
                const RSec& ri = rsec[std::size_t(lb_ket) * nps + sm.sector[sti]];
                if (ri.rb == NONE) continue;
                for (std::size_t u = 0; u < nu; ++u) {
                    const uint32_t ci = Rci[std::size_t(ri.rb) * nr + urbb[u]];
                    const uint32_t job = tj[std::size_t(sti) * nr + urbb[u]];
                    if (ci == NONE || job == NONE) continue;
                    gin[u * nst + sti] = WGenInD{ci, tj_first[job]};
                    gcnt[u * nst + sti] = tj_count[job];
                }
            }
            std::fill(line_count.begin(), line_count.end(), 0);
            const int bk = eb.find(lc_bra - lc_ket);
            const std::vector<uint32_t>& bptr = eb.ptr[bk];
            const std::vector<uint32_t>& bent = eb.ent[bk];
            for (uint32_t b1 = 0; b1 < W.rows; ++b1) {
                if (bptr[b1] == bptr[b1 + 1]) continue;
                if (symmetric && lc_ket < lc_bra && W.herm_left[b1] >= 0) continue;
                for (uint32_t qi = bptr[b1]; qi < bptr[b1 + 1]; ++qi) {
                    const uint32_t e = bent[qi], b2 = W.b2[e], o = W.op[e];
                    for (uint32_t k = oc.ptr[o]; k < oc.ptr[o + 1]; ++k) {
                        const int u = unit_of[oc.out[k]];
                        if (u < 0) continue;
                        const std::size_t gi = std::size_t(u) * nst + oc.in[k];
                        const WGenInD g = gin[gi];
                        if (g.c == WGEN_NONE) continue;
                        const int32_t bp = Rpos[g.c * Raux + b2];
                        if (bp < 0) continue;
                        if (uint32_t(bp) >= gcnt[gi]) throw std::runtime_error("boundary_step_right: R block position outside its T job");
                        ut[u].add(b1, g.jbase + uint32_t(bp));
                        line_count[b1]++;
                    }
                }
            }
            // finalize: MPO rows with coefficients get consecutive positions
            uint32_t nS = 0;
            for (uint32_t b1 = 0; b1 < W.rows; ++b1) pos[b1] = line_count[b1] ? nS++ : NONE;
            if (nS == 0) continue;
            const uint32_t K_c = nS * ls_ket;
            const uint64_t s_off = P.s_len;
            P.s_len += (uint64_t(K_c) * kcols[lb_bra] + 31) / 32 * 32;
            for (auto& x : uoff) x *= K_c;
            emit_units(P, pos, s_off, uoff, ls_ket, uer, K_c, une, ust, ut, gin, nst, slot, js);
            BPart::Coh ch{lb_ket, lb_bra, nS, s_off, std::vector<int64_t>(W.rows, -1)};
            for (uint32_t b1 = 0; b1 < W.rows; ++b1)
                if (pos[b1] != NONE) ch.offs[b1] = int64_t(pos[b1]) * ls_ket * ls_bra;
            P.coh.push_back(std::move(ch));
        }
    } catch (const std::exception& e) {
#pragma omp critical
        err = e.what();
    }
    }
    if (!err.empty()) throw std::runtime_error(err);

    const double tbp = step_now();
    // merge in ket-sector order; new index (BoundaryIndex(ket_left_i, bra_left_i))
    std::vector<TJobD> tjobs;
    std::vector<TileD> ttiles[N_SHAPES];
    uint64_t t_len = 0, s_len = 0;
    BoundaryIndexH nidx;
    nidx.bra = left; nidx.ket = left; nidx.aux = W.rows;
    struct Pend { uint32_t ci_new; uint32_t lb_ket, lb_bra, nS; uint64_t s_off; };
    std::vector<Pend> pend;
    std::vector<uint64_t> tb(nl), sbase(nl);
    {
        uint64_t t = 0, sx = 0;
        for (uint32_t lb = 0; lb < nl; ++lb) { tb[lb] = t; sbase[lb] = sx; t += parts[lb].t_len; sx += parts[lb].s_len; }
    }
    merge_sbuilds(parts, sb, tb, sbase);
    for (uint32_t lb = 0; lb < nl; ++lb) {
        BPart& P = parts[lb];
        for (TJobD j : P.tjobs) {
            j.c_off += t_len;
            if (j.M && j.N) add_tiles(ttiles, uint32_t(tjobs.size()), j.M, j.N);
            tjobs.push_back(j);
        }
        for (auto& ch : P.coh) {
            pend.push_back(Pend{nidx.n_cohorts(), ch.bra, ch.ket, ch.nS, ch.s_off + s_len});
            nidx.cbra.push_back(ch.bra); nidx.cket.push_back(ch.ket);
            nidx.lsz.push_back(uint32_t(left[ch.bra].second)); nidx.rsz.push_back(uint32_t(left[ch.ket].second));
            nidx.nb.push_back(ch.nS); nidx.tr.push_back(0);
            nidx.offsets.insert(nidx.offsets.end(), ch.offs.begin(), ch.offs.end());
            nidx.cscale.insert(nidx.cscale.end(), W.rows, 1.0);
        }
        t_len += P.t_len;
        s_len += P.s_len;
        P = BPart();
    }
    if (!dn) {
        auto P = std::make_shared<BStepPlan>();
        if (symmetric) complement_transpose(nidx, W.herm_left, W.phase_left, false);
        nidx.finish();
        // prop_r: new_R[b] (ls_ket x ls_bra) = S_b * bra^T for all b of a cohort in one job
        // (rows b-major in S; C row blocks = the cohort's MPO-index blocks)
        for (const Pend& pd : pend) {
            const uint32_t ls = uint32_t(left[pd.lb_ket].second), lsb = uint32_t(left[pd.lb_bra].second);
            GemmJob g{};
            g.a_off = pd.s_off; g.lda = pd.nS * ls;
            g.b_off = koff[pd.lb_bra]; g.ldb = lsb; g.tb = 1;
            g.c_off = nidx.data_off[pd.ci_new]; g.ldc = ls; g.crb = ls; g.c_bs = uint64_t(ls) * lsb;
            g.M = pd.nS * ls; g.N = lsb; g.K = kcols[pd.lb_bra]; g.alpha = 1.0; g.beta = 0.0;
            P->prop.push_back(g);
        }
        validate_tjobs(tjobs, ket.b.total, Rold.idx.total, t_len);
        sb.validate(t_len, s_len);
        P->tjobs = std::move(tjobs);
        for (int k = 0; k < N_SHAPES; ++k) P->ttiles[k] = std::move(ttiles[k]);
        P->d_tjobs.upload(P->tjobs, c.s);
        for (int k = 0; k < N_SHAPES; ++k) P->d_ttiles[k].upload(P->ttiles[k], c.s);
        P->sb = std::move(sb);
        P->sb.upload(c.s);
        P->sb.cg.b_cs = nullptr;  // uploaded; the old boundary's scales are not read again
        P->nidx = std::move(nidx);
        P->t_len = t_len;
        P->s_len = s_len;
        const double tb1 = step_now();
        auto Rn = run_right(c, *P, Rold, ket);
        if (cache) {
            cache->key = key;
            cache->bytes = P->device_bytes();
            cache->plan = std::move(P);
        }
        step_report("right", tb0, tbp, tb1, c.s);
        return Rn;
    }
    const double tb1 = step_now();
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
    Ctx::ensure(c.W, sb.w_len ? sb.w_len : 1);
    sb.cg.generate(c.W.get(), c.s);
    run_sgemm(sb.d_units.get(), sb.d_utiles, sb.utiles, sb.d_line_b1.get(), sb.d_slice_off.get(), sb.d_klist.get(), c.W.get(),
              c.T.get(), c.S.get(), c.s);
    {
        // rbtm (tasks.cpp:364-380): dm[lb_bra] += alpha S^T S, S = (nS*ls_ket) x stripe
        std::vector<GemmJob> acc;
        std::vector<std::size_t> tgt;
        for (const Pend& pd : pend) {
            const std::size_t k = dn->dm->find_l(left[pd.lb_bra].first);
            if (k == dn->dm->n()) throw std::runtime_error("rbtm: missing density-matrix block");
            const uint32_t K = pd.nS * uint32_t(left[pd.lb_ket].second), st = kcols[pd.lb_bra];
            if (dn->dm->rows[k] != st || dn->dm->cols[k] != st) throw std::runtime_error("rbtm: density-matrix block shape");
            GemmJob g{};
            g.a_off = pd.s_off; g.ta = 1; g.lda = K;
            g.b_off = pd.s_off; g.ldb = K;
            g.c_off = dn->dm->off[k]; g.ldc = st;
            g.M = st; g.N = st; g.K = K; g.alpha = dn->alpha; g.beta = 1.0;
            acc.push_back(g);
            tgt.push_back(k);
        }
        run_accumulating(acc, tgt, c.S.get(), s_len, c.S.get(), s_len, dn->dm->d.get(), dn->dm->total, c);
    }
    step_report("right (noise)", tb0, tbp, tb1, c.s);
    return nullptr;
}

std::unique_ptr<DevBoundary> boundary_step_right(Ctx& c, const DevBoundary& Rold, const DMPS& ket, const MPOTensor& W,
                                                 bool symmetric, BStepCache* cache) {
    return step_right(c, Rold, ket, W, symmetric, nullptr, cache);
}

void rbtm_accumulate(Ctx& c, const DevBoundary& R, const DMPS& ket_rp, const MPOTensor& W, DBlocks& dm, double alpha) {
    DensityNoise dn{&dm, alpha};
    step_right(c, R, ket_rp, W, false, &dn, nullptr);
}

// ---------------------------------------------------------------------------
static std::unique_ptr<DevBoundary> step_left(Ctx& c, const DevBoundary& Lold, const DMPS& ket, const DMPS& bra,
                                              const MPOTensor& W, bool symmetric, DensityNoise* dn, BStepCache* cache) {
    if (!ket.right_paired || bra.right_paired) throw std::runtime_error("boundary_step_left: ket right-paired, bra left-paired");
    const double tb0 = step_now();
    uint64_t key = 0;
    if (cache && !dn) {
        key = step_key(0, Lold, ket, &bra, W, symmetric);
        if (cache->plan && cache->key == key) {
            auto Ln = run_left(c, *cache->plan, Lold, ket, bra);
            cache->hit = true;
            step_report("left (cached)", tb0, tb0, tb0, c.s);
            return Ln;
        }
        cache->plan.reset();
        cache->bytes = 0;
        cache->hit = false;
    }
    const BoundaryIndexH& L = Lold.idx;
    const Index& phys = ket.phys;
    const Index& left = ket.left;
    const Index& right = ket.right;
    if (W.rows != L.aux) throw std::runtime_error("boundary_step_left: MPO row dimension differs from the boundary");
    ProductBasis kpb(phys, right, true);  // ket right-paired columns
    ProductBasis bpb(phys, left);         // bra left-paired rows
    StateMap sm(phys);
    const uint32_t nl = uint32_t(left.size()), nr = uint32_t(right.size()), nps = uint32_t(phys.size());
    const uint32_t nst = uint32_t(sm.nstates());
    std::vector<uint64_t> koff(nl, 0), boff(nr, 0);
    std::vector<uint8_t> kok(nl, 0), bok(nr, 0);
    std::vector<uint32_t> brows(nr, 0);
    for (uint32_t lb = 0; lb < nl; ++lb) {
        std::size_t k = ket.b.find_l(left[lb].first);
        if (k < ket.b.n()) { koff[lb] = ket.b.off[k]; kok[lb] = 1; }
    }
    for (uint32_t rb = 0; rb < nr; ++rb) {
        std::size_t k = bra.b.find_r(right[rb].first);
        if (k < bra.b.n()) { boff[rb] = bra.b.off[k]; brows[rb] = bra.b.rows[k]; bok[rb] = 1; }
    }
    // left sector, its size, ket column offset (right-paired) and bra row offset (left-paired)
    // of (right sector, phys sector)
    struct LSec { uint32_t lb, ls, koff, boff; };
    std::vector<LSec> lsec(std::size_t(nr) * nps, LSec{NONE, 0, 0, 0});
    for (uint32_t rb = 0; rb < nr; ++rb)
        for (uint32_t s = 0; s < nps; ++s) {
            const Charge lc = right[rb].first - phys[s].first;
            const std::size_t lb = left.position(lc);
            if (lb < nl)
                lsec[std::size_t(rb) * nps + s] = LSec{uint32_t(lb), uint32_t(left[lb].second),
                                                       uint32_t(kpb(phys[s].first, right[rb].first)), uint32_t(bpb(phys[s].first, lc))};
        }
    std::vector<uint32_t> Lci, Lce;
    cohort_tables(L, left, left, Lci, Lce);
    const OpCSR oc(W);

    // coefficient generation: lines iterate MPO columns b2, slices come from L_old cohorts
    SBuild sb;
    sb.cg.set_mpo(W, false);
    if (sb.cg.nst != nst) throw std::runtime_error("boundary_step_left: MPO physical basis differs from the MPS");
    sb.cg.set_boundary(L);
    const int32_t* Lpos = sb.cg.b_pos.data();
    const std::size_t Laux = L.aux;
    const EntryBuckets eb = bucket_entries(W, L, phys, false);

    std::vector<BPart> parts(nr);
    std::string err;
#pragma omp parallel
    {
    std::vector<UnitTerms> ut;
#pragma omp for schedule(dynamic, 1)
    for (int rbi = 0; rbi < int(nr); ++rbi) try {
        const uint32_t rb_ket = uint32_t(rbi);
        BPart& P = parts[rb_ket];
        P.sb.cg.nst = nst;
        const Charge rc_ket = right[rb_ket].first;
        const uint32_t rs_ket = uint32_t(right[rb_ket].second);
        // T jobs (lshtm_t_tasks): per (input state, bra left sector), nb GEMMs of ls_bra x rs_ket;
        // slice ids per L block
        std::vector<uint32_t> tj(std::size_t(nst) * nl, NONE);
        JobSlices js;
        std::vector<uint32_t> tj_first, tj_count;
        for (uint32_t st = 0; st < nst; ++st) {
            const LSec& li = lsec[std::size_t(rb_ket) * nps + sm.sector[st]];
            if (li.lb == NONE || !kok[li.lb]) continue;
            const uint32_t ls_ket = li.ls, mo = li.koff + uint32_t(sm.sub[st]) * rs_ket;
            for (uint32_t lb_bra = 0; lb_bra < nl; ++lb_bra) {
                const uint32_t ci = Lci[std::size_t(lb_bra) * nl + li.lb];
                if (ci == NONE) continue;
                const uint32_t ce = Lce[std::size_t(lb_bra) * nl + li.lb];
                const uint32_t ls_bra = uint32_t(left[lb_bra].second), nb = L.nb[ce];
                const uint64_t c_off = P.t_len;
                tj[std::size_t(st) * nl + lb_bra] = uint32_t(tj_first.size());
                const uint32_t bs = slice_stride(rs_ket, ls_bra);  // each T_b block 16-byte aligned
                tj_first.push_back(js.add(c_off, bs, nb));
                tj_count.push_back(nb);
                P.t_len += (uint64_t(bs) * nb + 31) / 32 * 32;
                if (nb == 0) continue;
                // all nb blocks of the cohort in one job: A and C row blocks = MPO-index blocks
                GemmJob g{};
                g.a_off = L.data_off[ce]; g.arb = ls_bra; g.a_bs = uint64_t(ls_bra) * ls_ket;
                g.ta = (ci != ce); g.lda = g.ta ? ls_ket : ls_bra;
                g.b_off = koff[li.lb] + uint64_t(mo) * ls_ket; g.ldb = ls_ket;
                g.c_off = c_off; g.crb = ls_bra; g.c_bs = bs; g.ldc = ls_bra;
                g.M = nb * ls_bra; g.N = rs_ket; g.K = ls_ket; g.alpha = 1.0; g.beta = 0.0;
                P.tgemm.push_back(g);
            }
        }
        std::vector<uint32_t> slot(js.pos0.back() + 1, NONE);
        // cohorts (lshtm_tasks)
        std::vector<int> unit_of(nst, -1);
        std::vector<uint32_t> line_count(W.cols, 0), pos(W.cols, NONE);
        for (uint32_t rb_bra = 0; rb_bra < nr; ++rb_bra) {
            const Charge rc_bra = right[rb_bra].first;
            if (std::abs(rc_bra.particles() - rc_ket.particles()) > 2 || !bok[rb_bra]) continue;
            const uint32_t rs_bra = uint32_t(right[rb_bra].second), stripe = brows[rb_bra];
            std::vector<uint32_t> ust, ulb, uer, une;
            std::vector<uint64_t> uoff;
            std::fill(unit_of.begin(), unit_of.end(), -1);
            for (uint32_t st = 0; st < nst; ++st) {
                const LSec& lo = lsec[std::size_t(rb_bra) * nps + sm.sector[st]];
                if (lo.lb == NONE) continue;
                unit_of[st] = int(ust.size());
                ust.push_back(st); ulb.push_back(lo.lb);
                uoff.push_back(uint64_t(lo.boff + uint32_t(sm.sub[st]) * lo.ls));
                uer.push_back(lo.ls); une.push_back(lo.ls * rs_ket);
            }
            const std::size_t nu = ust.size();
            if (ut.size() < nu) ut.resize(nu);
            for (std::size_t u = 0; u < nu; ++u) ut[u].clear();
            // (L cohort, first slice id) of each (unit, input state) and its number of blocks
            std::vector<WGenInD> gin(nu * nst, WGenInD{WGEN_NONE, WGEN_NONE});
            std::vector<uint32_t> gcnt(nu * nst, 0);
            for (uint32_t sti = 0; sti < nst; ++sti) {
                const LSec& li = lsec[std::size_t(rb_ket) * nps + sm.sector[sti]];
                if (li.lb == NONE || !kok[li.lb]) continue;
                for (std::size_t u = 0; u < nu; ++u) {
                    const uint32_t ci = Lci[std::size_t(ulb[u]) * nl + li.lb];
                    const uint32_t job = tj[std::size_t(sti) * nl + ulb[u]];
                    if (ci == NONE || job == NONE) continue;
                    gin[u * nst + sti] = WGenInD{ci, tj_first[job]};
                    gcnt[u * nst + sti] = tj_count[job];
                }
            }
            std::fill(line_count.begin(), line_count.end(), 0);
            const int bk = eb.find(rc_bra - rc_ket);
            const std::vector<uint32_t>& bptr = eb.ptr[bk];
            const std::vector<uint32_t>& bent = eb.ent[bk];
            for (uint32_t b2 = 0; b2 < W.cols; ++b2) {
                if (bptr[b2] == bptr[b2 + 1]) continue;
                if (symmetric && rc_bra < rc_ket && W.herm_right[b2] >= 0) continue;
                for (uint32_t qi = bptr[b2]; qi < bptr[b2 + 1]; ++qi) {
                    const uint32_t e = bent[qi], b1 = W.b1[e], o = W.op[e];
                    for (uint32_t k = oc.ptr[o]; k < oc.ptr[o + 1]; ++k) {
                        const int u = unit_of[oc.out[k]];
                        if (u < 0) continue;
                        const std::size_t gi = std::size_t(u) * nst + oc.in[k];
                        const WGenInD g = gin[gi];
                        if (g.c == WGEN_NONE) continue;
                        const int32_t bp = Lpos[g.c * Laux + b1];
                        if (bp < 0) continue;
                        if (uint32_t(bp) >= gcnt[gi]) throw std::runtime_error("boundary_step_left: L block position outside its T job");
                        ut[u].add(b2, g.jbase + uint32_t(bp));
                        line_count[b2]++;
                    }
                }
            }
            uint32_t nS = 0;
            for (uint32_t b2 = 0; b2 < W.cols; ++b2) pos[b2] = line_count[b2] ? nS++ : NONE;
            if (nS == 0) continue;
            const uint64_t s_off = P.s_len;
            P.s_len += (uint64_t(stripe) * nS * rs_ket + 31) / 32 * 32;
            emit_units(P, pos, s_off, uoff, uint64_t(rs_ket) * stripe, uer, stripe, une, ust, ut, gin, nst, slot, js);
            BPart::Coh ch{rb_bra, rb_ket, nS, s_off, std::vector<int64_t>(W.cols, -1)};
            for (uint32_t b2 = 0; b2 < W.cols; ++b2)
                if (pos[b2] != NONE) ch.offs[b2] = int64_t(pos[b2]) * rs_bra * rs_ket;
            P.coh.push_back(std::move(ch));
        }
    } catch (const std::exception& e) {
#pragma omp critical
        err = e.what();
    }
    }
    if (!err.empty()) throw std::runtime_error(err);

    const double tbp = step_now();
    // merge in ket-sector order; new index (BoundaryIndex(bra_right_i, ket_right_i))
    std::vector<GemmJob> tj_gemm;
    uint64_t t_len = 0, s_len = 0;
    BoundaryIndexH nidx;
    nidx.bra = right; nidx.ket = right; nidx.aux = W.cols;
    struct Pend { uint32_t ci_new, rb_bra, nS; uint64_t s_off; uint32_t rs_ket; };
    std::vector<Pend> pend;
    std::vector<uint64_t> tb(nr), sbase(nr);
    {
        uint64_t t = 0, sx = 0;
        for (uint32_t rb = 0; rb < nr; ++rb) { tb[rb] = t; sbase[rb] = sx; t += parts[rb].t_len; sx += parts[rb].s_len; }
    }
    merge_sbuilds(parts, sb, tb, sbase);
    for (uint32_t rb = 0; rb < nr; ++rb) {
        BPart& P = parts[rb];
        for (GemmJob g : P.tgemm) { g.c_off += t_len; tj_gemm.push_back(g); }
        for (auto& ch : P.coh) {
            pend.push_back(Pend{nidx.n_cohorts(), ch.bra, ch.nS, ch.s_off + s_len, uint32_t(right[ch.ket].second)});
            nidx.cbra.push_back(ch.bra); nidx.cket.push_back(ch.ket);
            nidx.lsz.push_back(uint32_t(right[ch.bra].second)); nidx.rsz.push_back(uint32_t(right[ch.ket].second));
            nidx.nb.push_back(ch.nS); nidx.tr.push_back(0);
            nidx.offsets.insert(nidx.offsets.end(), ch.offs.begin(), ch.offs.end());
            nidx.cscale.insert(nidx.cscale.end(), W.cols, 1.0);
        }
        t_len += P.t_len;
        s_len += P.s_len;
        P = BPart();
    }
    if (!dn) {
        auto P = std::make_shared<BStepPlan>();
        if (symmetric) complement_transpose(nidx, W.herm_right, W.phase_right, true);
        nidx.finish();
        // prop_l: L_new (rs_bra x nS*rs_ket) = bra^T * S
        for (const Pend& pd : pend) {
            GemmJob g{};
            g.a_off = boff[pd.rb_bra]; g.ta = 1; g.lda = brows[pd.rb_bra];
            g.b_off = pd.s_off; g.ldb = brows[pd.rb_bra];
            g.c_off = nidx.data_off[pd.ci_new]; g.ldc = uint32_t(right[pd.rb_bra].second);
            g.M = uint32_t(right[pd.rb_bra].second); g.N = pd.nS * pd.rs_ket; g.K = brows[pd.rb_bra];
            g.alpha = 1.0; g.beta = 0.0;
            P->prop.push_back(g);
        }
        sb.validate(t_len, s_len);
        P->tj_gemm = std::move(tj_gemm);
        P->sb = std::move(sb);
        P->sb.upload(c.s);
        P->sb.cg.b_cs = nullptr;  // uploaded; the old boundary's scales are not read again
        P->nidx = std::move(nidx);
        P->t_len = t_len;
        P->s_len = s_len;
        const double tb1 = step_now();
        auto Ln = run_left(c, *P, Lold, ket, bra);
        if (cache) {
            cache->key = key;
            cache->bytes = P->device_bytes();
            cache->plan = std::move(P);
        }
        step_report("left", tb0, tbp, tb1, c.s);
        return Ln;
    }
    const double tb1 = step_now();
    Ctx::ensure(c.T, t_len ? t_len : 1);
    Ctx::ensure(c.S, s_len ? s_len : 1);
    batched_gemm(tj_gemm, Lold.data.get(), Lold.idx.total, ket.b.d.get(), ket.b.total, c.T.get(), t_len, c.gjobs, c.gtiles, c.s);
    sb.validate(t_len, s_len);
    sb.upload(c.s);
    if (s_len) QCM_CUDA(cudaMemsetAsync(c.S.get(), 0, s_len * sizeof(double), c.s));
    Ctx::ensure(c.W, sb.w_len ? sb.w_len : 1);
    sb.cg.generate(c.W.get(), c.s);
    run_sgemm(sb.d_units.get(), sb.d_utiles, sb.utiles, sb.d_line_b1.get(), sb.d_slice_off.get(), sb.d_klist.get(), c.W.get(),
              c.T.get(), c.S.get(), c.s);
    {
        // lbtm (tasks.cpp:346-362): dm[rb_bra] += alpha S S^T, S = stripe x (nS*rs_ket)
        std::vector<GemmJob> acc;
        std::vector<std::size_t> tgt;
        for (const Pend& pd : pend) {
            const std::size_t k = dn->dm->find_r(right[pd.rb_bra].first);
            if (k == dn->dm->n()) throw std::runtime_error("lbtm: missing density-matrix block");
            const uint32_t st = brows[pd.rb_bra], K = pd.nS * pd.rs_ket;
            if (dn->dm->rows[k] != st || dn->dm->cols[k] != st) throw std::runtime_error("lbtm: density-matrix block shape");
            GemmJob g{};
            g.a_off = pd.s_off; g.lda = st;
            g.b_off = pd.s_off; g.tb = 1; g.ldb = st;
            g.c_off = dn->dm->off[k]; g.ldc = st;
            g.M = st; g.N = st; g.K = K; g.alpha = dn->alpha; g.beta = 1.0;
            acc.push_back(g);
            tgt.push_back(k);
        }
        run_accumulating(acc, tgt, c.S.get(), s_len, c.S.get(), s_len, dn->dm->d.get(), dn->dm->total, c);
    }
    step_report("left (noise)", tb0, tbp, tb1, c.s);
    return nullptr;
}

std::unique_ptr<DevBoundary> boundary_step_left(Ctx& c, const DevBoundary& Lold, const DMPS& ket, const DMPS& bra,
                                                const MPOTensor& W, bool symmetric, BStepCache* cache) {
    return step_left(c, Lold, ket, bra, W, symmetric, nullptr, cache);
}

void lbtm_accumulate(Ctx& c, const DevBoundary& L, const DMPS& ket_rp, const DMPS& bra_lp, const MPOTensor& W, DBlocks& dm,
                     double alpha) {
    DensityNoise dn{&dm, alpha};
    step_left(c, L, ket_rp, bra_lp, W, false, &dn, nullptr);
}

}  // namespace qcm
