// ORACLE -- TEST INFRASTRUCTURE ONLY.  extern "C" entry points used by tests/, smoke()
// and bench.py (cpu_baseline / --impl reference) through ctypes.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

#include "dmrg.hpp"
#include "mpo.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

namespace {
thread_local std::string g_err;
int fail(const std::string& m) { g_err = m; return -1; }
void* dup_blob(const std::vector<uint8_t>& b, std::size_t* len) {
    void* p = std::malloc(b.size() ? b.size() : 1);
    std::memcpy(p, b.data(), b.size());
    *len = b.size();
    return p;
}
struct W {
    std::vector<uint8_t> b;
    template <class T> void put(T v) { const uint8_t* p = reinterpret_cast<const uint8_t*>(&v); b.insert(b.end(), p, p + sizeof(T)); }
};
}  // namespace

struct orc_dmrg { DMRG* d; };

namespace {
// block k of the host list gets charges (n - 1 - k, 0), so BlockMatrix keeps the input order
BlockMatrix host_blocks(uint32_t n, const uint32_t* rows, const uint32_t* cols, const double* data) {
    BlockMatrix M;
    uint64_t h = 0;
    for (uint32_t k = 0; k < n; ++k) {
        Mat m(rows[k], cols[k]);
        std::copy(data + h, data + h + m.d.size(), m.d.begin());
        h += m.d.size();
        M.lc.push_back(Q(int(n - 1 - k), 0));
        M.rc.push_back(Q(int(n - 1 - k), 0));
        M.b.push_back(std::move(m));
    }
    return M;
}
void put_result(const TruncationResults& t, double* res) {
    res[0] = double(t.bond_dimension); res[1] = t.truncated_weight; res[2] = t.truncated_fraction; res[3] = t.smallest_ev;
}
}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_init(const char* blas_path, int nthreads) {
    std::string err;
    if (!blas_init(blas_path, err)) return fail("blas_init: " + err);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_free(void* p) { std::free(p); }

// The QC MPO of integrals h (L x L) and V (L^4), built by the package's builder (input preparation),
// as a "QMPO" blob; free with orc_free.
int orc_mpo_build_qc(int L, const double* h, const double* V, double cutoff, void** out, size_t* len) {
    try {
        if (L < 2 || !h || !V || !out || !len) return fail("orc_mpo_build_qc: bad arguments");
        *out = dup_blob(qcm::serialize_mpo(qcm::build_qc_mpo(L, h, V, cutoff)), len);
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// The two-site site problem ("QSPB") at (site1, site1 + 1) of the MPS given as n_sites "QMPS" blobs,
// with boundaries built from that MPS (no optimisation); free with orc_free.
int orc_site_problem(const void* mpo_blob, size_t mn, int n_sites, const void* const* blobs, const size_t* lens, int site1,
                     void** out, size_t* len) {
    try {
        bool ts = false;
        auto mpo = load_mpo_blob(static_cast<const uint8_t*>(mpo_blob), mn, ts);
        if (ts) return fail("orc_site_problem: expected a single-site MPO");
        if (n_sites != int(mpo.size()) || !blobs || !lens || !out || !len) return fail("orc_site_problem: bad arguments");
        std::vector<MPSTensor> mps;
        for (int i = 0; i < n_sites; ++i) mps.push_back(load_mps_tensor(static_cast<const uint8_t*>(blobs[i]), lens[i]));
        *out = dup_blob(site_problem_from_mps(mpo, mps, site1), len);
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

int orc_dmrg_create(const void* blob, size_t n, int nup, int ndown, size_t Mmax, size_t init_bd, double cutoff, double tol,
                    int maxiter, double ecore, orc_dmrg** out) {
    try {
        bool ts = false;
        auto mpo = load_mpo_blob(static_cast<const uint8_t*>(blob), n, ts);
        if (ts) return fail("orc_dmrg_create: expected a single-site MPO");
        DMRGParams p;
        p.Mmax = Mmax; p.init_bond_dimension = init_bd; p.cutoff = cutoff; p.jcd_tol = tol; p.jcd_maxiter = maxiter; p.ecore = ecore;
        *out = new orc_dmrg{new DMRG(std::move(mpo), nup, ndown, p)};
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

void orc_dmrg_free(orc_dmrg* h) { if (h) { delete h->d; delete h; } }

int orc_dmrg_set_mmax(orc_dmrg* h, size_t Mmax) { h->d->p.Mmax = Mmax; return 0; }

// twosite_truncation = heev with alpha_initial / alpha_main / alpha_final over ngrowsweeps / nmainsweeps
int orc_dmrg_set_heev(orc_dmrg* h, int heev, double a_init, double a_main, double a_final, int ngrow, int nmain) {
    DMRGParams& p = h->d->p;
    p.heev = heev != 0; p.alpha_initial = a_init; p.alpha_main = a_main; p.alpha_final = a_final;
    p.ngrowsweeps = ngrow; p.nmainsweeps = nmain;
    return 0;
}

// excited states: n_states ortho states of L site tensors each ("QMPS" blobs, state-major), kept
// orthogonal to every solution; call at the start of a sweep
int orc_dmrg_set_ortho(orc_dmrg* h, int n_states, const void* const* blobs, const size_t* lens) {
    try {
        DMRG& d = *h->d;
        if (n_states < 0 || (n_states > 0 && (!blobs || !lens))) return fail("orc_dmrg_set_ortho: bad arguments");
        std::vector<std::vector<MPSTensor>> st(static_cast<std::size_t>(n_states));
        for (int o = 0; o < n_states; ++o)
            for (int i = 0; i < d.L; ++i) {
                const std::size_t k = std::size_t(o) * d.L + i;
                st[o].push_back(load_mps_tensor(static_cast<const uint8_t*>(blobs[k]), lens[k]));
            }
        d.set_ortho(std::move(st));
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// ietl_jcd_gmres of the sweep's solves
// optimization = singlesite (1) or twosite (0); a sweep then has 2L (or 2L - 2) steps
int orc_dmrg_set_single_site(orc_dmrg* h, int on) {
    h->d->p.single_site = on != 0;
    return 0;
}

int orc_dmrg_steps_per_sweep(orc_dmrg* h) { return h->d->steps_per_sweep(); }

int orc_dmrg_set_gmres(orc_dmrg* h, int gmres) {
    if (gmres < 0) return fail("orc_dmrg_set_gmres: gmres < 0");
    h->d->p.jcd_gmres = gmres;
    return 0;
}

// energies/tw/tf/bond: arrays of steps_per_sweep.  If stop_step >= 0, the frozen site problem of
// that step is returned in *snap (free with orc_free) and the sweep stops there.
int orc_dmrg_sweep(orc_dmrg* h, int sweep, double* energies, double* tw, double* tf, uint64_t* bond, int stop_step,
                   void** snap, size_t* snap_len) {
    try {
        std::vector<double> E;
        std::vector<TruncationResults> T;
        std::vector<uint8_t> sb;
        h->d->sweep(sweep, E, T, stop_step, &sb);
        if (stop_step >= 0 && snap) { *snap = dup_blob(sb, snap_len); return 0; }
        for (std::size_t i = 0; i < E.size(); ++i) {
            if (energies) energies[i] = E[i];
            if (tw) tw[i] = T[i].truncated_weight;
            if (tf) tf[i] = T[i].truncated_fraction;
            if (bond) bond[i] = T[i].bond_dimension;
        }
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// Boundary step case from the current state (call after a sweep stopped at a step of the
// left-to-right half): side 0 = overlap_mpo_left_step(mps[site], left_[site]),
// side 1 = overlap_mpo_right_step(mps[site], right_[site + 1]); free with orc_free.
int orc_dmrg_boundary_export(orc_dmrg* h, int side, int site, void** out, size_t* len) {
    try {
        DMRG& d = *h->d;
        if (site < 0 || site >= d.L) return fail("orc_dmrg_boundary_export: site out of range");
        auto same = [](const Index& a, const Index& b) {
            if (a.size() != b.size()) return false;
            for (std::size_t i = 0; i < a.size(); ++i)
                if (!(a[i].first == b[i].first) || a[i].second != b[i].second) return false;
            return true;
        };
        if (side == 0) {
            const Boundary& in = d.left_[site];
            if (!same(in.index.bra, d.mps[site].left)) return fail("orc_dmrg_boundary_export: left boundary does not match the site");
            Boundary res = overlap_mpo_left_step(d.mps[site], d.mps[site], in, d.mpo[site], true);
            *out = dup_blob(save_boundary_step(0, site, d.mps[site], in, res), len);
        } else {
            const Boundary& in = d.right_[site + 1];
            if (!same(in.index.bra, d.mps[site].right)) return fail("orc_dmrg_boundary_export: right boundary does not match the site");
            Boundary res = overlap_mpo_right_step(d.mps[site], d.mps[site], in, d.mpo[site], true);
            *out = dup_blob(save_boundary_step(1, site, d.mps[site], in, res), len);
        }
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// Current site tensor `site` ("QMPS" v1, right-paired); free with orc_free.
int orc_dmrg_mps_export(orc_dmrg* h, int site, void** out, size_t* len) {
    try {
        DMRG& d = *h->d;
        if (site < 0 || site >= d.L) return fail("orc_dmrg_mps_export: site out of range");
        *out = dup_blob(save_mps_tensor(d.mps[site]), len);
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// [hpsi_count, hpsi_time, hpsi_flops, jd_time, schedule_time, trunc_time, boundary_time]
int orc_dmrg_stats(orc_dmrg* h, double* out) {
    DMRG& d = *h->d;
    out[0] = double(d.hpsi_count); out[1] = d.hpsi_time; out[2] = double(d.hpsi_flops);
    out[3] = d.jd_time; out[4] = d.schedule_time; out[5] = d.trunc_time; out[6] = d.boundary_time;
    return 0;
}

// H_eff x for a frozen site problem; x, y are the twin blocks concatenated in block order.
int orc_heff_apply(const void* snap, size_t n, const void* mpo_blob, size_t mn, int site1, const double* x, double* y,
                   size_t len, int repeat, double* flops, double* seconds) {
    try {
        bool ts = false;
        auto mpo = load_mpo_blob(static_cast<const uint8_t*>(mpo_blob), mn, ts);
        MPOTensor W = ts ? mpo[site1] : make_twosite_mpo(mpo[site1], mpo[site1 + 1]);
        MPSTensor twin;
        Boundary Lb, Rb;
        load_site_problem(static_cast<const uint8_t*>(snap), n, twin, Lb, Rb);
        auto sched = create_contraction_schedule(twin, Lb, Rb, W);
        std::vector<const double*> xv(twin.left.size(), nullptr);
        std::vector<double*> yv(twin.left.size(), nullptr);
        std::size_t off = 0;
        for (std::size_t k = 0; k < twin.data.n_blocks(); ++k) {
            std::size_t lb = twin.left.position(twin.data.lc[k]);
            xv[lb] = x + off;
            yv[lb] = y + off;
            off += twin.data.b[k].d.size();
        }
        if (off != len) return fail("orc_heff_apply: vector length mismatch");
        auto t0 = std::chrono::steady_clock::now();
        for (int r = 0; r < std::max(1, repeat); ++r) {
            std::fill(y, y + len, 0.0);
            super_hamil_mv(*sched, Lb, Rb, xv, yv);
        }
        auto t1 = std::chrono::steady_clock::now();
        if (flops) *flops = double(sched->total_flops);
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count() / std::max(1, repeat);
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// Jacobi-Davidson on a frozen site problem (solve_ietl_jcd, ietl_jacobi_davidson.h:35-76): start
// vector x0, n_ortho ortho vectors of len doubles each (contiguous), GMRES(gmres) corrections.
int orc_jd_solve(const void* snap, size_t n, const void* mpo_blob, size_t mn, int site1, const double* x0, size_t len,
                 const double* ortho, int n_ortho, int gmres, double tol, int maxiter, double* out, double* eval,
                 int* iters, int* applies) {
    try {
        bool ts = false;
        auto mpo = load_mpo_blob(static_cast<const uint8_t*>(mpo_blob), mn, ts);
        MPOTensor W = ts ? mpo[site1] : make_twosite_mpo(mpo[site1], mpo[site1 + 1]);
        MPSTensor twin;
        Boundary Lb, Rb;
        load_site_problem(static_cast<const uint8_t*>(snap), n, twin, Lb, Rb);
        auto sched = create_contraction_schedule(twin, Lb, Rb, W);
        std::vector<std::size_t> off(twin.left.size(), SIZE_MAX);
        std::size_t tot = 0;
        for (std::size_t k = 0; k < twin.data.n_blocks(); ++k) {
            off[twin.left.position(twin.data.lc[k])] = tot;
            tot += twin.data.b[k].d.size();
        }
        if (tot != len) return fail("orc_jd_solve: vector length mismatch");
        if (maxiter < 1 || gmres < 0 || n_ortho < 0) return fail("orc_jd_solve: bad iteration counts");
        auto mult = [&](const std::vector<double>& x, std::vector<double>& y) {
            std::vector<const double*> xv(twin.left.size(), nullptr);
            std::vector<double*> yv(twin.left.size(), nullptr);
            for (std::size_t lb = 0; lb < off.size(); ++lb)
                if (off[lb] != SIZE_MAX) { xv[lb] = x.data() + off[lb]; yv[lb] = y.data() + off[lb]; }
            std::fill(y.begin(), y.end(), 0.0);
            super_hamil_mv(*sched, Lb, Rb, xv, yv);
        };
        std::vector<std::vector<double>> O;
        O.resize(std::size_t(n_ortho));
        for (int i = 0; i < n_ortho; ++i) O[i].assign(ortho + std::size_t(i) * len, ortho + std::size_t(i + 1) * len);
        std::vector<double> x(x0, x0 + len), xo;
        int it = 0;
        *eval = jacobi_davidson(mult, x, tol, maxiter, xo, it, gmres, O, applies);
        std::copy(xo.begin(), xo.end(), out);
        if (iters) *iters = it;
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// Adjoint of H_eff x on a frozen site problem (the differentiation form): psi_bar = H ybar (H_eff is
// symmetric) and grad[e] = d (ybar . H x) / d scale_e for the n_terms entries of the site's two-site
// MPO tensor, in the tensor's entry order.
int orc_heff_adjoint(const void* snap, size_t n, const void* mpo_blob, size_t mn, int site1, const double* x,
                     const double* ybar, size_t len, double* psi_bar, double* grad, size_t n_terms) {
    try {
        bool ts = false;
        auto mpo = load_mpo_blob(static_cast<const uint8_t*>(mpo_blob), mn, ts);
        MPOTensor W = ts ? mpo[site1] : make_twosite_mpo(mpo[site1], mpo[site1 + 1]);
        if (n_terms != W.scale.size()) return fail("orc_heff_adjoint: term count mismatch");
        MPSTensor twin;
        Boundary Lb, Rb;
        load_site_problem(static_cast<const uint8_t*>(snap), n, twin, Lb, Rb);
        auto sched = create_contraction_schedule(twin, Lb, Rb, W);
        std::vector<const double*> xv(twin.left.size(), nullptr), yb(twin.left.size(), nullptr);
        std::vector<double*> pv(twin.left.size(), nullptr);
        std::size_t off = 0;
        for (std::size_t k = 0; k < twin.data.n_blocks(); ++k) {
            std::size_t lb = twin.left.position(twin.data.lc[k]);
            xv[lb] = x + off;
            yb[lb] = ybar + off;
            pv[lb] = psi_bar + off;
            off += twin.data.b[k].d.size();
        }
        if (off != len) return fail("orc_heff_adjoint: vector length mismatch");
        std::fill(psi_bar, psi_bar + len, 0.0);
        super_hamil_mv(*sched, Lb, Rb, yb, pv);
        std::vector<double> g;
        scale_gradient(*sched, Lb, Rb, xv, yb, n_terms, g);
        std::copy(g.begin(), g.end(), grad);
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// Flat export of the schedule (bookkeeping parity).  Layout ("QSCH" v1):
// u32 nblocks; per block: u32 ntj, ntj x (u32 mps_offset, ci, ci_eff, lb_ket);
//   u32 ncoh; per cohort: u32 lb, rb, ls, rs, ci, ci_eff, nSrows, stripe, nunits;
//   per unit: u32 offset, ms, nlines, nalpha; nlines x (u32 b1, u32 count); nalpha x (f64 alpha, u32 ti, u32 col)
int orc_schedule_export(const void* snap, size_t n, const void* mpo_blob, size_t mn, int site1, void** out, size_t* len,
                        double* flops) {
    try {
        bool ts = false;
        auto mpo = load_mpo_blob(static_cast<const uint8_t*>(mpo_blob), mn, ts);
        MPOTensor Wt = ts ? mpo[site1] : make_twosite_mpo(mpo[site1], mpo[site1 + 1]);
        MPSTensor twin;
        Boundary Lb, Rb;
        load_site_problem(static_cast<const uint8_t*>(snap), n, twin, Lb, Rb);
        auto s = create_contraction_schedule(twin, Lb, Rb, Wt);
        W w;
        w.put<uint32_t>(0x48435351u);
        w.put<uint32_t>(uint32_t(s->blocks.size()));
        for (auto& b : s->blocks) {
            w.put<uint32_t>(uint32_t(b.t_schedule.size()));
            for (auto& j : b.t_schedule) { w.put(j.mps_offset); w.put(j.ci); w.put(j.ci_eff); w.put(j.lb_ket); }
            w.put<uint32_t>(uint32_t(b.data.size()));
            for (auto& c : b.data) {
                w.put(c.lb); w.put(c.rb); w.put(c.ls); w.put(c.rs); w.put(c.ci); w.put(c.ci_eff); w.put(c.nSrows); w.put(c.stripe);
                w.put<uint32_t>(uint32_t(c.suv.size()));
                for (auto& u : c.suv) {
                    w.put(u.offset); w.put(u.ms); w.put<uint32_t>(uint32_t(u.b1.size())); w.put<uint32_t>(uint32_t(u.alpha.size()));
                    for (std::size_t l = 0; l < u.b1.size(); ++l) { w.put(u.b1[l]); w.put(u.b2s[l]); }
                    for (std::size_t a = 0; a < u.alpha.size(); ++a) { w.put(u.alpha[a]); w.put(u.tidx[2 * a]); w.put(u.tidx[2 * a + 1]); }
                }
            }
        }
        if (flops) *flops = double(s->total_flops);
        *out = dup_blob(w.b, len);
        return 0;
    } catch (const std::exception& e) { return fail(e.what()); }
}

// svd_truncate on host blocks (column-major, concatenated): per block k keep[k], U_k (rows x
// keep), S_k (keep), Vt_k (keep x cols) packed in block order; res = (bond dimension,
// truncated weight, truncated fraction, smallest ev)
int orc_truncate_svd(uint32_t n, const uint32_t* rows, const uint32_t* cols, const double* blocks, uint64_t Mmax, double cutoff,
                     uint32_t* keep, double* U, double* S, double* Vt, double* res) {
    try {
        BlockMatrix M = host_blocks(n, rows, cols, blocks);
        BlockMatrix Ub, Vb;
        std::vector<std::vector<double>> Sv;
        const TruncationResults tr = svd_truncate(M, Ub, Vb, Sv, cutoff, Mmax);
        uint64_t pu = 0, ps = 0, pv = 0;
        std::size_t si = 0;
        for (uint32_t k = 0; k < n; ++k) {
            const Q q(int(n - 1 - k), 0);
            const std::size_t i = Ub.find(q, q);
            if (i == Ub.n_blocks()) { keep[k] = 0; continue; }
            const Mat& u = Ub.b[i];
            const Mat& v = Vb.b[Vb.find(q, q)];
            keep[k] = uint32_t(u.c);
            std::copy(u.d.begin(), u.d.end(), U + pu);
            std::copy(Sv[si].begin(), Sv[si].end(), S + ps);
            std::copy(v.d.begin(), v.d.end(), Vt + pv);
            pu += u.d.size(); ps += Sv[si].size(); pv += v.d.size();
            ++si;
        }
        put_result(tr, res);
        return 0;
    } catch (const std::exception& e) {
        return fail(e.what());
    }
}

// heev_truncate on host symmetric blocks: per block keep[k], U_k (dim x keep, descending) and
// the kept eigenvalues (descending), packed in block order
int orc_truncate_heev(uint32_t n, const uint32_t* dims, const double* blocks, uint64_t Mmax, double cutoff, uint32_t* keep,
                      double* U, double* evals, double* res) {
    try {
        BlockMatrix dm = host_blocks(n, dims, dims, blocks);
        BlockMatrix Ub;
        const TruncationResults tr = heev_truncate(dm, Ub, cutoff, Mmax);
        uint64_t pu = 0, pe = 0;
        for (uint32_t k = 0; k < n; ++k) {
            const Q q(int(n - 1 - k), 0);
            const std::size_t i = Ub.find(q, q);
            if (i == Ub.n_blocks()) { keep[k] = 0; continue; }
            const Mat& u = Ub.b[i];
            keep[k] = uint32_t(u.c);
            std::copy(u.d.begin(), u.d.end(), U + pu);
            Mat ev;
            std::vector<double> w;
            heev_desc(dm.b[k], ev, w);
            std::copy(w.begin(), w.begin() + long(u.c), evals + pe);
            pu += u.d.size(); pe += u.c;
        }
        put_result(tr, res);
        return 0;
    } catch (const std::exception& e) {
        return fail(e.what());
    }
}

}  // extern "C"
