// MPS tensors, two-site tensors and their factorizations on the device.
//
// Reshapes (mp_tensors/reshapes.h, mpstensor.hpp:211-240) are sub-block copies
// between the left-paired ((phys x left) x right) and right-paired
// (left x (phys x right)) forms; the two-site tensor (twositetensor.hpp:29-199,
// ts_reshape.h) is the block product of a left-paired and a right-paired site
// tensor, re-blocked over the fused physical index.  Truncation follows
// svd_truncate / estimate_truncation (block_matrix_algorithms.h:136-240) with
// the per-block SVDs on the device and the global cut on the host.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <stdexcept>
#include <string>

#include "dmrg_dev.hpp"

namespace qcm {

namespace {
double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

namespace {

std::size_t find_block(const DBlocks& b, Charge c) {
    for (std::size_t k = 0; k < b.n(); ++k) if (b.lc[k] == c) return k;
    return b.n();
}

DMPS reshaped_left(Ctx& c, const DMPS& t) {
    DMPS o;
    o.phys = t.phys; o.left = t.left; o.right = t.right; o.right_paired = false;
    o.b = layout_left_paired(t.phys, t.left, t.right);
    o.b.allocate(c.s, true);
    ProductBasis out_left(t.phys, t.left), in_right(t.phys, t.right, true);
    std::vector<CopyJob> jobs;
    for (std::size_t k = 0; k < o.b.n(); ++k) {
        const Charge rc = o.b.rc[k];
        const uint32_t rdim = o.b.cols[k];
        for (std::size_t s = 0; s < t.phys.size(); ++s) {
            const Charge p = t.phys[s].first, lc = rc - p;
            const std::size_t lb = t.left.position(lc);
            if (lb == t.left.size()) continue;
            const std::size_t ks = find_block(t.b, lc);
            if (ks == t.b.n()) continue;
            const uint32_t ldim = uint32_t(t.left[lb].second);
            if (t.b.rows[ks] != ldim) throw std::runtime_error("reshape: block rows differ from the left index");
            const uint64_t ol = out_left(p, lc), ir = in_right(p, rc);
            for (uint32_t ss = 0; ss < t.phys[s].second; ++ss)
                jobs.push_back(CopyJob{t.b.off[ks] + (ir + uint64_t(ss) * rdim) * ldim, o.b.off[k] + ol + uint64_t(ss) * ldim,
                                       ldim, rdim, ldim, o.b.rows[k], 0, 0});
        }
    }
    batched_copy(jobs, t.b.d.get(), t.b.total, o.b.d.get(), o.b.total, c.cjobs, c.s);
    return o;
}

DMPS reshaped_right(Ctx& c, const DMPS& t) {
    DMPS o;
    o.phys = t.phys; o.left = t.left; o.right = t.right; o.right_paired = true;
    o.b = layout_right_paired(t.phys, t.left, t.right);
    o.b.allocate(c.s, true);
    ProductBasis in_left(t.phys, t.left), out_right(t.phys, t.right, true);
    std::vector<CopyJob> jobs;
    for (std::size_t k = 0; k < o.b.n(); ++k) {
        const Charge lc = o.b.lc[k];
        const uint32_t ldim = o.b.rows[k];
        for (std::size_t s = 0; s < t.phys.size(); ++s) {
            const Charge p = t.phys[s].first, rc = lc + p;
            const std::size_t rb = t.right.position(rc);
            if (rb == t.right.size()) continue;
            const std::size_t ks = find_block(t.b, rc);
            if (ks == t.b.n()) continue;
            const uint32_t rdim = uint32_t(t.right[rb].second);
            if (t.b.cols[ks] != rdim) throw std::runtime_error("reshape: block columns differ from the right index");
            const uint64_t il = in_left(p, lc), orr = out_right(p, rc);
            for (uint32_t ss = 0; ss < t.phys[s].second; ++ss)
                jobs.push_back(CopyJob{t.b.off[ks] + il + uint64_t(ss) * ldim, o.b.off[k] + (orr + uint64_t(ss) * rdim) * ldim,
                                       ldim, rdim, t.b.rows[ks], ldim, 0, 0});
        }
    }
    batched_copy(jobs, t.b.d.get(), t.b.total, o.b.d.get(), o.b.total, c.cjobs, c.s);
    return o;
}

// estimate_truncation (block_matrix_algorithms.h:136-183) on per-block values in descending order
TruncResults estimate_cut(const std::vector<std::vector<double>>& vals, uint64_t Mmax, double cutoff,
                          std::vector<uint32_t>& keep) {
    std::vector<double> all;
    for (auto& v : vals) all.insert(all.end(), v.begin(), v.end());
    std::sort(all.begin(), all.end(), std::greater<double>());
    TruncResults tr;
    if (all.empty() || all[0] == 0.0) throw std::runtime_error("truncation: two-site tensor is zero");
    double evalscut = cutoff * all[0];
    if (all.size() > Mmax) evalscut = std::max(evalscut, all[Mmax]);
    tr.smallest_ev = evalscut / all[0];
    double tf = 0, tw = 0, sum = 0, sum2 = 0;
    for (double x : all) {
        sum += x; sum2 += x * x;
        if (x < evalscut) { tf += x; tw += x * x; }
    }
    tr.truncated_fraction = tf / sum;
    tr.truncated_weight = tw / sum2;
    keep.assign(vals.size(), 0);
    for (std::size_t k = 0; k < vals.size(); ++k) {
        uint32_t n = 0;
        while (n < vals[k].size() && !(vals[k][n] < evalscut)) ++n;
        keep[k] = n;
        tr.bond_dimension += n;
    }
    return tr;
}

Index sorted_basis(const std::vector<std::pair<Charge, std::size_t>>& v) {
    Index r;
    r.d = v;
    r.sort();
    return r;
}

}  // namespace

DBlocks layout_right_paired(const Index& phys, const Index& left, const Index& right, bool packed) {
    ProductBasis pb(phys, right, true);
    DBlocks b;
    for (std::size_t lb = 0; lb < left.size(); ++lb) {
        const Charge c = left[lb].first;
        const std::size_t n = pb.size(c);
        if (n == 0 || left[lb].second == 0) continue;
        b.add(c, c, uint32_t(left[lb].second), uint32_t(n), packed);
    }
    return b;
}

DBlocks layout_left_paired(const Index& phys, const Index& left, const Index& right) {
    ProductBasis pb(phys, left);
    DBlocks b;
    for (std::size_t rb = 0; rb < right.size(); ++rb) {
        const Charge c = right[rb].first;
        const std::size_t n = pb.size(c);
        if (n == 0 || right[rb].second == 0) continue;
        b.add(c, c, uint32_t(n), uint32_t(right[rb].second));
    }
    return b;
}

void make_left_paired(Ctx& c, DMPS& t) {
    if (!t.right_paired) return;
    t = reshaped_left(c, t);
}

void make_right_paired(Ctx& c, DMPS& t) {
    if (t.right_paired) return;
    t = reshaped_right(c, t);
}

DMPS right_paired_copy(Ctx& c, const DMPS& t) {
    if (!t.right_paired) return reshaped_right(c, t);
    DMPS o;
    o.phys = t.phys; o.left = t.left; o.right = t.right; o.right_paired = true;
    o.b.lc = t.b.lc; o.b.rc = t.b.rc; o.b.rows = t.b.rows; o.b.cols = t.b.cols; o.b.off = t.b.off; o.b.total = t.b.total;
    o.b.allocate(c.s, false);
    QCM_CUDA(cudaMemcpyAsync(o.b.d.get(), t.b.d.get(), std::max<uint64_t>(t.b.total, 1) * sizeof(double),
                             cudaMemcpyDeviceToDevice, c.s));
    return o;
}

DMPS left_paired_copy(Ctx& c, const DMPS& t) {
    if (t.right_paired) return reshaped_left(c, t);
    DMPS o;
    o.phys = t.phys; o.left = t.left; o.right = t.right; o.right_paired = false;
    o.b.lc = t.b.lc; o.b.rc = t.b.rc; o.b.rows = t.b.rows; o.b.cols = t.b.cols; o.b.off = t.b.off; o.b.total = t.b.total;
    o.b.allocate(c.s, false);
    QCM_CUDA(cudaMemcpyAsync(o.b.d.get(), t.b.d.get(), std::max<uint64_t>(t.b.total, 1) * sizeof(double),
                             cudaMemcpyDeviceToDevice, c.s));
    return o;
}

double norm2(Ctx& c, const DBlocks& b) {
    if (!b.total) return 0.0;
    Ctx::ensure(c.scal, 64 + DOT_PARTS);
    dev_dots(b.d.get(), 0, 1, b.d.get(), b.total, c.scal.get(), c.scal.get() + 64, c.s);
    double r = 0;
    QCM_CUDA(cudaMemcpyAsync(&r, c.scal.get(), sizeof(double), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
    return r;
}

void scale(Ctx& c, DBlocks& b, double f) {
    if (b.total) dev_axpby(f, b.d.get(), 0.0, b.d.get(), b.total, c.s);
}

DBlocks normalize_left(Ctx& c, DMPS& t) {
    make_left_paired(c, t);
    DBlocks Q, R;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        const uint32_t m = t.b.rows[k], n = t.b.cols[k], kk = std::min(m, n);
        Q.add(t.b.lc[k], t.b.rc[k], m, kk);
        R.add(t.b.rc[k], t.b.rc[k], kk, n);
    }
    Q.allocate(c.s, true);
    R.allocate(c.s, true);
    // every block's thin QR in one launch (qr, alps/matrix/algorithms.hpp:260-291)
    std::vector<QrJob> jobs;
    uint64_t wl = 0;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        if (!t.b.rows[k] || !t.b.cols[k]) continue;
        jobs.push_back(QrJob{t.b.off[k], Q.off[k], R.off[k], wl, t.b.rows[k], t.b.cols[k], 0, 0});
        wl += (qr_scratch(t.b.rows[k], t.b.cols[k], false) + 31) / 32 * 32;
    }
    Ctx::ensure(c.qrw, std::max<uint64_t>(wl, 1));
    batched_qr(jobs, t.b.d.get(), t.b.total, Q.d.get(), Q.total, R.d.get(), R.total, c.qrw.get(), c.qrw.size(), c.qjobs, c.s);
    t.b = std::move(Q);
    t.right = t.b.right_basis();
    return R;
}

DBlocks normalize_right(Ctx& c, DMPS& t) {
    make_right_paired(c, t);
    DBlocks Lm, Q;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        const uint32_t m = t.b.rows[k], n = t.b.cols[k], kk = std::min(m, n);
        Lm.add(t.b.lc[k], t.b.lc[k], m, kk);
        Q.add(t.b.lc[k], t.b.rc[k], kk, n);
    }
    Lm.allocate(c.s, true);
    Q.allocate(c.s, true);
    // every block's thin LQ in one launch (lq, alps/matrix/algorithms.hpp:293-325)
    std::vector<QrJob> jobs;
    uint64_t wl = 0;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        if (!t.b.rows[k] || !t.b.cols[k]) continue;
        jobs.push_back(QrJob{t.b.off[k], Q.off[k], Lm.off[k], wl, t.b.rows[k], t.b.cols[k], 1, 0});
        wl += (qr_scratch(t.b.rows[k], t.b.cols[k], true) + 31) / 32 * 32;
    }
    Ctx::ensure(c.qrw, std::max<uint64_t>(wl, 1));
    batched_qr(jobs, t.b.d.get(), t.b.total, Q.d.get(), Q.total, Lm.d.get(), Lm.total, c.qrw.get(), c.qrw.size(), c.qjobs, c.s);
    t.b = std::move(Q);
    t.left = t.b.left_basis();
    return Lm;
}

void multiply_from_left(Ctx& c, DMPS& t, const DBlocks& N) {
    make_right_paired(c, t);
    DBlocks o;
    std::vector<GemmJob> jobs;
    for (std::size_t j = 0; j < N.n(); ++j) {
        const std::size_t ks = find_block(t.b, N.rc[j]);
        if (ks == t.b.n()) continue;
        if (t.b.rows[ks] != N.cols[j]) throw std::runtime_error("multiply_from_left: inner dimensions differ");
        o.add(N.lc[j], t.b.rc[ks], N.rows[j], t.b.cols[ks]);
        GemmJob g{};
        g.a_off = N.off[j]; g.lda = N.rows[j];
        g.b_off = t.b.off[ks]; g.ldb = t.b.rows[ks];
        g.c_off = o.off.back(); g.ldc = N.rows[j];
        g.M = N.rows[j]; g.N = t.b.cols[ks]; g.K = N.cols[j]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    o.allocate(c.s, true);
    batched_gemm(jobs, N.d.get(), N.total, t.b.d.get(), t.b.total, o.d.get(), o.total, c.gjobs, c.gtiles, c.s);
    t.b = std::move(o);
    t.left = t.b.left_basis();
}

void multiply_from_right(Ctx& c, DMPS& t, const DBlocks& N) {
    make_left_paired(c, t);
    DBlocks o;
    std::vector<GemmJob> jobs;
    for (std::size_t k = 0; k < t.b.n(); ++k) {
        const std::size_t j = find_block(N, t.b.rc[k]);
        if (j == N.n()) continue;
        if (N.rows[j] != t.b.cols[k]) throw std::runtime_error("multiply_from_right: inner dimensions differ");
        o.add(t.b.lc[k], N.rc[j], t.b.rows[k], N.cols[j]);
        GemmJob g{};
        g.a_off = t.b.off[k]; g.lda = t.b.rows[k];
        g.b_off = N.off[j]; g.ldb = N.rows[j];
        g.c_off = o.off.back(); g.ldc = t.b.rows[k];
        g.M = t.b.rows[k]; g.N = N.cols[j]; g.K = t.b.cols[k]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    o.allocate(c.s, true);
    batched_gemm(jobs, t.b.d.get(), t.b.total, N.d.get(), N.total, o.d.get(), o.total, c.gjobs, c.gtiles, c.s);
    t.b = std::move(o);
    t.right = t.b.right_basis();
}

// ---------------------------------------------------------------------------
// two-site tensor
void DTwoSite::build(Ctx& c, const DMPS& a, const DMPS& b) {
    if (a.right_paired || !b.right_paired) throw std::runtime_error("two-site tensor: expects left-paired a, right-paired b");
    phys1 = a.phys; phys2 = b.phys; phys = index_product(phys1, phys2); left = a.left; right = b.right;
    ProductBasis in_left(phys1, left), in_right(phys2, right, true), out_right(phys, right, true), ppb(phys1, phys2);
    // both-paired layout: every middle charge with rows and columns (ts_reshape.h creates the
    // blocks the product leaves out when reshaping back)
    both = DBlocks();
    prod.clear();
    std::vector<GemmJob> jobs;
    Index mids = index_product(phys1, left);
    for (std::size_t i = 0; i < mids.size(); ++i) {
        const Charge m = mids[i].first;
        const std::size_t rows = in_left.size(m), cols = in_right.size(m);
        if (!rows || !cols) continue;
        both.add(m, m, uint32_t(rows), uint32_t(cols));
        const std::size_t ka = find_block(a.b, m), kb = find_block(b.b, m);
        const bool pr = ka < a.b.n() && kb < b.b.n();
        prod.push_back(pr ? 1 : 0);
        if (!pr) continue;
        if (a.b.rows[ka] != rows || b.b.cols[kb] != cols || a.b.cols[ka] != b.b.rows[kb])
            throw std::runtime_error("two-site tensor: block shapes differ from the product bases");
        GemmJob g{};
        g.a_off = a.b.off[ka]; g.lda = a.b.rows[ka];
        g.b_off = b.b.off[kb]; g.ldb = b.b.rows[kb];
        g.c_off = both.off.back(); g.ldc = uint32_t(rows);
        g.M = uint32_t(rows); g.N = uint32_t(cols); g.K = a.b.cols[ka]; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    both.allocate(c.s, true);
    batched_gemm(jobs, a.b.d.get(), a.b.total, b.b.d.get(), b.b.total, both.d.get(), both.total, c.gjobs, c.gtiles, c.s);

    // twin (make_mps): right-paired blocks for the left charges the product blocks reach
    std::vector<uint8_t> need(left.size(), 0);
    for (std::size_t k = 0; k < both.n(); ++k) {
        if (!prod[k]) continue;
        for (std::size_t s1 = 0; s1 < phys1.size(); ++s1) {
            const std::size_t l = left.position(both.lc[k] - phys1[s1].first);
            if (l == left.size()) continue;
            for (std::size_t s2 = 0; s2 < phys2.size(); ++s2)
                if (right.has(both.lc[k] + phys2[s2].first)) need[l] = 1;
        }
    }
    twin = DMPS();
    twin.phys = phys; twin.right = right; twin.right_paired = true;
    for (std::size_t l = 0; l < left.size(); ++l)
        if (need[l] && out_right.size(left[l].first)) twin.left.d.push_back(left[l]);
    twin.b = layout_right_paired(phys, twin.left, right, true);
    twin.b.allocate(c.s, true);
    std::vector<CopyJob> cj;
    for (std::size_t k = 0; k < both.n(); ++k) {
        if (!prod[k]) continue;
        const Charge m = both.lc[k];
        for (std::size_t s1 = 0; s1 < phys1.size(); ++s1) {
            const Charge p1 = phys1[s1].first, lc = m - p1;
            const std::size_t l = left.position(lc);
            if (l == left.size()) continue;
            const std::size_t kt = find_block(twin.b, lc);
            for (std::size_t s2 = 0; s2 < phys2.size(); ++s2) {
                const Charge p2 = phys2[s2].first, rc = m + p2;
                const std::size_t r = right.position(rc);
                if (r == right.size()) continue;
                const uint32_t ldim = uint32_t(left[l].second), rdim = uint32_t(right[r].second);
                const uint32_t sd1 = uint32_t(phys1[s1].second), sd2 = uint32_t(phys2[s2].second);
                const uint64_t ilo = in_left(p1, lc), iro = in_right(p2, rc), oro = out_right(p1 + p2, rc), opo = ppb(p1, p2);
                for (uint32_t ss1 = 0; ss1 < sd1; ++ss1)
                    for (uint32_t ss2 = 0; ss2 < sd2; ++ss2) {
                        const uint64_t so = opo + uint64_t(ss1) * sd2 + ss2;
                        cj.push_back(CopyJob{both.off[k] + ilo + uint64_t(ss1) * ldim + (iro + uint64_t(ss2) * rdim) * both.rows[k],
                                             twin.b.off[kt] + (oro + so * rdim) * ldim, ldim, rdim, both.rows[k], ldim, 0, 0});
                    }
            }
        }
    }
    batched_copy(cj, both.d.get(), both.total, twin.b.d.get(), twin.b.total, c.cjobs, c.s);
}

void DTwoSite::twin_to_both(Ctx& c) {
    ProductBasis in_left(phys1, left), in_right(phys2, right, true), out_right(phys, right, true), ppb(phys1, phys2);
    if (both.total) QCM_CUDA(cudaMemsetAsync(both.d.get(), 0, both.total * sizeof(double), c.s));
    std::vector<CopyJob> cj;
    for (std::size_t kt = 0; kt < twin.b.n(); ++kt) {
        const Charge lc = twin.b.lc[kt];
        const std::size_t l = left.position(lc);
        for (std::size_t s1 = 0; s1 < phys1.size(); ++s1)
            for (std::size_t s2 = 0; s2 < phys2.size(); ++s2) {
                const Charge p1 = phys1[s1].first, p2 = phys2[s2].first, rc = lc + p1 + p2;
                const std::size_t r = right.position(rc);
                if (r == right.size()) continue;
                const std::size_t k = find_block(both, lc + p1);
                if (k == both.n()) throw std::runtime_error("two-site tensor: missing both-paired block");
                const uint32_t ldim = uint32_t(left[l].second), rdim = uint32_t(right[r].second);
                const uint32_t sd1 = uint32_t(phys1[s1].second), sd2 = uint32_t(phys2[s2].second);
                const uint64_t ilo = in_left(p1, lc), iro = in_right(p2, rc), oro = out_right(p1 + p2, rc), opo = ppb(p1, p2);
                for (uint32_t ss1 = 0; ss1 < sd1; ++ss1)
                    for (uint32_t ss2 = 0; ss2 < sd2; ++ss2) {
                        const uint64_t so = opo + uint64_t(ss1) * sd2 + ss2;
                        cj.push_back(CopyJob{twin.b.off[kt] + (oro + so * rdim) * ldim,
                                             both.off[k] + ilo + uint64_t(ss1) * ldim + (iro + uint64_t(ss2) * rdim) * both.rows[k],
                                             ldim, rdim, ldim, both.rows[k], 0, 0});
                    }
            }
    }
    batched_copy(cj, twin.b.d.get(), twin.b.total, both.d.get(), both.total, c.cjobs, c.s);
}

namespace {

uint64_t round32(uint64_t n) { return (n + 31) / 32 * 32; }

// Thin SVDs of the blocks of `both` into r.U, r.S, r.V (the BlockSVD layout), by the preconditioned
// one-sided Jacobi method (Drmac and Veselic, SIAM J. Matrix Anal. Appl. 29, 2008): F = A (rows >= cols)
// or A^T, a Householder QR with column pivoting F P = Q R, the one-sided Jacobi SVD of X = R^T
// (k x k, k = min(rows, cols)), X = Ux S Vx^T; then F = (Q Vx) S (P Ux)^T.  The pivoted R's rows are
// graded, so the Jacobi sweeps converge in a few sweeps over k-long columns.  F's left factor is one
// GEMM per block, its right factor the rows of Ux scattered by the permutation.  Zero singular values
// leave zero columns in the scattered factor (V for rows >= cols, U otherwise).
void preconditioned_svd(Ctx& c, const DBlocks& both, BlockSVD& r, int* zero_count, int* sweeps) {
    const std::size_t nb = both.n();
    std::vector<QrJob> qj;
    std::vector<SvdJob> sj;
    std::vector<GemmJob> gu, gv;
    std::vector<PermJob> pu, pv;
    uint64_t ql = 0, xl = 0, pl = 0, wq = 0, wj = 0;
    for (std::size_t k = 0; k < nb; ++k) {
        const uint32_t kk = r.kk[k], m = both.rows[k], n = both.cols[k];
        if (!kk) continue;
        const bool tall = m >= n;
        const uint64_t qo = ql, xo = xl, po = pl;
        ql += round32(uint64_t(m) * n);  // Q: m x k (QR of A) or k x n (LQ of A)
        xl += round32(uint64_t(kk) * kk);  // X, Ux and Vx at the same offsets of three buffers
        pl += kk;
        qj.push_back(QrJob{both.off[k], qo, xo, wq, m, n, tall ? 0u : 1u, QR_PIVOT | (tall ? QR_RT : 0u), po});
        wq += qr_scratch(m, n, !tall);
        sj.push_back(SvdJob{xo, xo, r.so[k], xo, wj, kk, kk, uint32_t(k), 0});
        wj += jacobi_svd_scratch(kk, kk);
        GemmJob g{};
        g.alpha = 1.0; g.beta = 0.0;
        g.b_off = xo; g.ldb = kk; g.tb = 0; g.N = kk; g.K = kk;
        if (tall) {
            // U (m x k) = Q (m x k) Vx; V = P Ux
            g.a_off = qo; g.lda = m; g.ta = 0; g.c_off = r.uo[k]; g.ldc = m; g.M = m;
            gu.push_back(g);
            pv.push_back(PermJob{xo, r.vo[k], po, kk, n});
        } else {
            // V (n x k) = (Q (k x n))^T Vx; U = P Ux
            g.a_off = qo; g.lda = kk; g.ta = 1; g.c_off = r.vo[k]; g.ldc = n; g.M = n;
            gv.push_back(g);
            pu.push_back(PermJob{xo, r.uo[k], po, kk, m});
        }
    }
    if (qj.empty()) return;
    DBuf<double> Qb(ql), Xb(xl), Uxb(xl), Vxb(xl), Wq(wq), Wjb(wj);
    DBuf<uint32_t> Pb(pl);
    // QCM_SVD_STATS=1: the time of each part
    cudaEvent_t ev[4] = {};
    if (sweeps)
        for (auto& e : ev) QCM_CUDA(cudaEventCreate(&e));
    if (sweeps) QCM_CUDA(cudaEventRecord(ev[0], c.s));
    batched_qr(qj, both.d.get(), both.total, Qb.get(), ql, Xb.get(), xl, Wq.get(), wq, c.qjobs, c.s, Pb.get(), pl);
    if (sweeps) QCM_CUDA(cudaEventRecord(ev[1], c.s));
    batched_jacobi_svd(sj, Xb.get(), xl, Uxb.get(), xl, r.S.get(), r.s_len, Vxb.get(), xl, Wjb.get(), wj, zero_count, c.sjobs,
                       c.s, sweeps);
    if (sweeps) QCM_CUDA(cudaEventRecord(ev[2], c.s));
    if (!gu.empty()) batched_gemm(gu, Qb.get(), ql, Vxb.get(), xl, r.U.get(), r.u_len, c.gjobs, c.gtiles, c.s);
    if (!gv.empty()) batched_gemm(gv, Qb.get(), ql, Vxb.get(), xl, r.V.get(), r.v_len, c.gjobs, c.gtiles, c.s);
    batched_permute_rows(pv, Uxb.get(), xl, r.V.get(), r.v_len, Pb.get(), pl, c.pjobs, c.s);
    batched_permute_rows(pu, Uxb.get(), xl, r.U.get(), r.u_len, Pb.get(), pl, c.pjobs, c.s);
    if (sweeps) {
        QCM_CUDA(cudaEventRecord(ev[3], c.s));
        QCM_CUDA(cudaEventSynchronize(ev[3]));
        float t[3];
        for (int i = 0; i < 3; ++i) QCM_CUDA(cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]));
        std::fprintf(stderr, "[svd parts] qr %.3f ms, jacobi %.3f ms, assembly %.3f ms\n", t[0], t[1], t[2]);
        for (auto& e : ev) cudaEventDestroy(e);
    }
}

}  // namespace

BlockSVD svd_truncate(Ctx& c, const DBlocks& both, uint64_t Mmax, double cutoff) {
    BlockSVD r = svd_truncate_groups(c, both, {0, both.n()}, {Mmax}, {cutoff});
    r.tr = r.gtr[0];
    return r;
}

BlockSVD svd_truncate_groups(Ctx& c, const DBlocks& both, const std::vector<std::size_t>& g0,
                             const std::vector<uint64_t>& Mmax, const std::vector<double>& cutoff) {
    const std::size_t nb = both.n(), ng = Mmax.size();
    if (g0.size() != ng + 1 || cutoff.size() != ng || g0.front() != 0 || g0.back() != nb)
        throw std::runtime_error("svd_truncate_groups: group ranges do not cover the blocks");
    // the cut of group g over its blocks' singular values: keep[k] for its blocks
    auto cut = [&](std::size_t g, const std::vector<std::vector<double>>& vals, std::vector<uint32_t>& keep) {
        std::vector<std::vector<double>> gv(vals.begin() + long(g0[g]), vals.begin() + long(g0[g + 1]));
        std::vector<uint32_t> gk;
        const TruncResults t = estimate_cut(gv, Mmax[g], cutoff[g], gk);
        std::copy(gk.begin(), gk.end(), keep.begin() + long(g0[g]));
        return t;
    };
    BlockSVD r;
    r.uo.resize(nb); r.so.resize(nb); r.vo.resize(nb); r.kk.resize(nb);
    uint64_t ul = 0, sl = 0, vl = 0;
    for (std::size_t k = 0; k < nb; ++k) {
        r.kk[k] = std::min(both.rows[k], both.cols[k]);
        r.uo[k] = ul; ul += (uint64_t(both.rows[k]) * r.kk[k] + 31) / 32 * 32;
        r.so[k] = sl; sl += r.kk[k];
        r.vo[k] = vl; vl += (uint64_t(both.cols[k]) * r.kk[k] + 31) / 32 * 32;
    }
    r.u_len = std::max<uint64_t>(ul, 1); r.s_len = std::max<uint64_t>(sl, 1); r.v_len = std::max<uint64_t>(vl, 1);
    r.U.alloc(r.u_len); r.S.alloc(r.s_len); r.V.alloc(r.v_len);
    // all blocks at once: pivoted QR, one-sided Jacobi on R^T, assembly (preconditioned_svd)
    DBuf<int> zc(std::max<std::size_t>(nb, 1));
    // QCM_SVD_STATS=1 prints the kernel time and the Jacobi sweeps of every batch
    static const bool stats = std::getenv("QCM_SVD_STATS") != nullptr;
    DBuf<int> swp;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        swp.alloc(std::max<std::size_t>(nb, 1));
        QCM_CUDA(cudaMemsetAsync(swp.get(), 0, std::max<std::size_t>(nb, 1) * sizeof(int), c.s));
        QCM_CUDA(cudaEventCreate(&e0));
        QCM_CUDA(cudaEventCreate(&e1));
        QCM_CUDA(cudaEventRecord(e0, c.s));
    }
    preconditioned_svd(c, both, r, zc.get(), stats ? swp.get() : nullptr);
    if (stats) {
        QCM_CUDA(cudaEventRecord(e1, c.s));
        QCM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        QCM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        std::vector<int> hsw(nb, 0);
        if (nb) QCM_CUDA(cudaMemcpyAsync(hsw.data(), swp.get(), nb * sizeof(int), cudaMemcpyDeviceToHost, c.s));
        QCM_CUDA(cudaStreamSynchronize(c.s));
        uint32_t mr = 0, mc = 0;
        std::size_t kbig = 0;
        int modes[3] = {0, 0, 0};  // work matrix and rotations in shared memory / work matrix only / neither
        for (std::size_t k = 0; k < nb; ++k) {
            mr = std::max(mr, both.rows[k]);
            mc = std::max(mc, both.cols[k]);
            // the Jacobi runs on the k x k factor R^T
            const uint64_t cc = std::min(both.rows[k], both.cols[k]), cpd = (cc + (cc & 1)) * cc;
            if (uint64_t(both.rows[k]) * both.cols[k] > uint64_t(both.rows[kbig]) * both.cols[kbig]) kbig = k;
            modes[2 * cpd <= jacobi_svd_smem_doubles() ? 0 : (cpd <= jacobi_svd_smem_doubles() ? 1 : 2)]++;
        }
        std::fprintf(stderr, "[svd] %zu blocks (max %u x %u): %.3f ms, Jacobi sweeps max %d; largest %u x %u: %d sweeps; modes %d/%d/%d\n",
                     nb, mr, mc, ms, hsw.empty() ? 0 : *std::max_element(hsw.begin(), hsw.end()), both.rows[kbig],
                     both.cols[kbig], nb ? hsw[kbig] : 0, modes[0], modes[1], modes[2]);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    std::vector<double> hs(sl);
    std::vector<int> hz(nb, 0);
    if (sl) QCM_CUDA(cudaMemcpyAsync(hs.data(), r.S.get(), sl * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    if (nb) QCM_CUDA(cudaMemcpyAsync(hz.data(), zc.get(), nb * sizeof(int), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
    r.vals.assign(nb, {});
    for (std::size_t k = 0; k < nb; ++k) r.vals[k].assign(hs.begin() + r.so[k], hs.begin() + r.so[k] + r.kk[k]);
    {
        // a kept singular value of exactly zero needs an orthonormal completion of its singular
        // vectors: such blocks are recomputed by cuSOLVER's gesvdj
        std::vector<uint32_t> keep0(nb, 0);
        for (std::size_t g = 0; g < ng; ++g) cut(g, r.vals, keep0);
        std::vector<std::size_t> redo;
        for (std::size_t k = 0; k < nb; ++k)
            if (hz[k] && keep0[k] + uint32_t(hz[k]) > r.kk[k]) redo.push_back(k);
        if (!redo.empty()) {
            if (!c.sv) c.sv = std::make_unique<Solver>();
            int* info = c.sv->reserve_info(uint32_t(redo.size()), c.s);
            c.sv->fork(c.s);
            for (std::size_t i = 0; i < redo.size(); ++i) {
                const std::size_t k = redo[i];
                svd_thin_lane(*c.sv, 0, both.d.get() + both.off[k], int(both.rows[k]), int(both.cols[k]), r.U.get() + r.uo[k],
                              r.S.get() + r.so[k], r.V.get() + r.vo[k], info + i);
            }
            c.sv->join(c.s);
            c.sv->check(c.s);
            for (std::size_t k : redo)
                QCM_CUDA(cudaMemcpyAsync(hs.data() + r.so[k], r.S.get() + r.so[k], r.kk[k] * sizeof(double), cudaMemcpyDeviceToHost,
                                         c.s));
            QCM_CUDA(cudaStreamSynchronize(c.s));
            for (std::size_t k : redo) r.vals[k].assign(hs.begin() + r.so[k], hs.begin() + r.so[k] + r.kk[k]);
        }
    }
    r.keep.assign(nb, 0);
    r.gtr.resize(ng);
    for (std::size_t g = 0; g < ng; ++g) r.gtr[g] = cut(g, r.vals, r.keep);
    return r;
}

TruncResults DTwoSite::split(Ctx& c, bool l2r, uint64_t Mmax, double cutoff, DMPS& m1, DMPS& m2) {
    BlockSVD sv = svd_truncate(c, both, Mmax, cutoff);
    return split_from(c, l2r, sv, 0, 0, m1, m2);
}

TruncResults DTwoSite::split_from(Ctx& c, bool l2r, const BlockSVD& sv, std::size_t b0, std::size_t g, DMPS& m1, DMPS& m2) {
    const std::size_t nb = both.n();
    if (b0 + nb > sv.keep.size() || g >= sv.gtr.size()) throw std::runtime_error("split: blocks outside the decomposition");
    const std::vector<uint32_t> keep(sv.keep.begin() + long(b0), sv.keep.begin() + long(b0 + nb));
    const TruncResults tr = sv.gtr[g];
    const std::vector<uint64_t> uo(sv.uo.begin() + long(b0), sv.uo.begin() + long(b0 + nb));
    const std::vector<uint64_t> so(sv.so.begin() + long(b0), sv.so.begin() + long(b0 + nb));
    const std::vector<uint64_t> vo(sv.vo.begin() + long(b0), sv.vo.begin() + long(b0 + nb));
    const DBuf<double>& U = sv.U;
    const DBuf<double>& S = sv.S;
    const DBuf<double>& V = sv.V;
    const uint64_t ul = sv.u_len, vl = sv.v_len;
    // U[:, :keep] and V^T[:keep, :], with S multiplied into V^T (l2r) or U (r2l)
    m1 = DMPS(); m2 = DMPS();
    m1.phys = phys1; m1.left = left; m1.right_paired = false;
    m2.phys = phys2; m2.right = right; m2.right_paired = true;
    std::vector<std::pair<Charge, std::size_t>> mid;
    for (std::size_t k = 0; k < nb; ++k) {
        if (!keep[k]) continue;
        mid.push_back({both.lc[k], keep[k]});
        m1.b.add(both.lc[k], both.lc[k], both.rows[k], keep[k]);
        m2.b.add(both.lc[k], both.lc[k], keep[k], both.cols[k]);
    }
    m1.right = sorted_basis(mid);
    m2.left = m1.right;
    m1.b.allocate(c.s, true);
    m2.b.allocate(c.s, true);
    std::vector<CopyJob> ju, jv;
    std::size_t i = 0;
    for (std::size_t k = 0; k < nb; ++k) {
        if (!keep[k]) continue;
        ju.push_back(CopyJob{uo[k], m1.b.off[i], both.rows[k], keep[k], both.rows[k], both.rows[k], 0, 0});
        jv.push_back(CopyJob{vo[k], m2.b.off[i], both.cols[k], keep[k], both.cols[k], keep[k], 1, 0});
        ++i;
    }
    batched_copy(ju, U.get(), ul, m1.b.d.get(), m1.b.total, c.cjobs, c.s);
    batched_copy(jv, V.get(), vl, m2.b.d.get(), m2.b.total, c.cjobs, c.s);
    i = 0;
    for (std::size_t k = 0; k < nb; ++k) {
        if (!keep[k]) continue;
        if (l2r) dev_scale_rows(m2.b.d.get() + m2.b.off[i], keep[k], both.cols[k], keep[k], S.get() + so[k], c.s);
        else dev_scale_cols(m1.b.d.get() + m1.b.off[i], both.rows[k], keep[k], both.rows[k], S.get() + so[k], c.s);
        ++i;
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));  // the decomposition's buffers may be released on return
    return tr;
}

BlockHeev heev_truncate(Ctx& c, DBlocks& dm, uint64_t Mmax, double cutoff) {
    const std::size_t nb = dm.n();
    for (std::size_t k = 0; k < nb; ++k)
        if (dm.rows[k] != dm.cols[k]) throw std::runtime_error("heev_truncate: density-matrix block is not square");
    if (!c.sv) c.sv = std::make_unique<Solver>();
    // heev per block (lanes, one host thread each), eigenvalues ascending on the device
    std::vector<uint64_t> wo(nb);
    uint64_t wl = 0;
    for (std::size_t k = 0; k < nb; ++k) { wo[k] = wl; wl += dm.rows[k]; }
    DBuf<double> Wv(std::max<uint64_t>(wl, 1));
    int* info = c.sv->reserve_info(uint32_t(nb), c.s);
    std::vector<std::size_t> order(nb);
    for (std::size_t k = 0; k < nb; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](std::size_t x, std::size_t y) { return dm.rows[x] > dm.rows[y]; });
    double t_heev = 0.0;
    static const bool stats = std::getenv("QCM_SVD_STATS") != nullptr;
    if (stats) {
        QCM_CUDA(cudaStreamSynchronize(c.s));
        t_heev = now_ms();
    }
    c.sv->fork(c.s);
    std::string err;
#pragma omp parallel for num_threads(Solver::LANES) schedule(static, 1)
    for (int lane = 0; lane < Solver::LANES; ++lane) {
        try {
            QCM_CUDA(cudaSetDevice(c.device));
            for (std::size_t i = std::size_t(lane); i < nb; i += Solver::LANES) {
                const std::size_t k = order[i];
                syevd_lane(*c.sv, lane, dm.d.get() + dm.off[k], int(dm.rows[k]), Wv.get() + wo[k], info + k);
            }
        } catch (const std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if (!err.empty()) throw std::runtime_error(err);
    c.sv->join(c.s);
    c.sv->check(c.s);
    if (stats) {
        QCM_CUDA(cudaStreamSynchronize(c.s));
        uint32_t mn = 0;
        uint64_t n3 = 0;
        for (std::size_t k = 0; k < nb; ++k) { mn = std::max(mn, dm.rows[k]); n3 += uint64_t(dm.rows[k]) * dm.rows[k] * dm.rows[k]; }
        std::fprintf(stderr, "[heev] %zu blocks (max %u, sum n^3 %.3g): %.3f ms\n", nb, mn, double(n3), now_ms() - t_heev);
    }
    std::vector<double> hw(wl);
    if (wl) QCM_CUDA(cudaMemcpyAsync(hw.data(), Wv.get(), wl * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
    // descending order; the cut is on sqrt of the positive eigenvalues (others kept as they are)
    std::vector<std::vector<double>> vals(nb);
    for (std::size_t k = 0; k < nb; ++k) {
        vals[k].resize(dm.rows[k]);
        for (uint32_t i = 0; i < dm.rows[k]; ++i) {
            const double x = hw[wo[k] + dm.rows[k] - 1 - i];
            vals[k][i] = x > 0.0 ? std::sqrt(x) : x;
        }
    }
    BlockHeev r;
    r.tr = estimate_cut(vals, Mmax, cutoff, r.keep);
    r.tr.truncated_weight = r.tr.truncated_fraction;  // heev_truncate reports the fraction in both fields
    r.evals.assign(nb, {});
    for (std::size_t k = 0; k < nb; ++k)
        for (uint32_t i = 0; i < dm.rows[k]; ++i) r.evals[k].push_back(hw[wo[k] + dm.rows[k] - 1 - i]);
    return r;
}

// ---------------------------------------------------------------------------
// predict_split_l2r / _r2l (contractions/boundary_ops/prediction.hpp:152-236) with
// heev_truncate (block_matrix_algorithms.h:299-355)
TruncResults DTwoSite::predict_split(Ctx& c, bool l2r, uint64_t Mmax, double cutoff, double alpha, const DevBoundary& B,
                                     const MPOTensor& W, DMPS& m1, DMPS& m2) {
    if (alpha == 0.0) return split(c, l2r, Mmax, cutoff, m1, m2);
    const std::size_t nb = both.n();
    // reduced density matrix: both both^T (l2r, rows x rows) or both^T both (r2l, cols x cols)
    DBlocks dm;
    std::vector<GemmJob> jobs;
    for (std::size_t k = 0; k < nb; ++k) {
        const uint32_t m = both.rows[k], n = both.cols[k], d = l2r ? m : n;
        dm.add(both.lc[k], both.lc[k], d, d);
        GemmJob g{};
        g.a_off = both.off[k]; g.lda = m; g.b_off = both.off[k]; g.ldb = m;
        if (l2r) { g.tb = 1; g.M = m; g.N = m; g.K = n; }
        else { g.ta = 1; g.M = n; g.N = n; g.K = m; }
        g.c_off = dm.off.back(); g.ldc = d; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    dm.allocate(c.s, true);
    batched_gemm(jobs, both.d.get(), both.total, both.d.get(), both.total, dm.d.get(), dm.total, c.gjobs, c.gtiles, c.s);
    // noise term on the both-paired data seen as a site tensor of the boundary step
    {
        DMPS tmp;
        std::vector<std::pair<Charge, std::size_t>> fused;
        for (std::size_t k = 0; k < nb; ++k) fused.push_back({both.lc[k], l2r ? both.cols[k] : both.rows[k]});
        if (l2r) { tmp.phys = phys1; tmp.left = left; tmp.right = sorted_basis(fused); tmp.right_paired = false; }
        else { tmp.phys = phys2; tmp.left = sorted_basis(fused); tmp.right = right; tmp.right_paired = true; }
        tmp.b.lc = both.lc; tmp.b.rc = both.rc; tmp.b.rows = both.rows; tmp.b.cols = both.cols; tmp.b.off = both.off;
        tmp.b.total = both.total;
        tmp.b.allocate(c.s, false);
        QCM_CUDA(cudaMemcpyAsync(tmp.b.d.get(), both.d.get(), std::max<uint64_t>(both.total, 1) * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c.s));
        if (l2r) {
            DMPS ket = right_paired_copy(c, tmp);
            lbtm_accumulate(c, B, ket, tmp, W, dm, alpha);
        } else {
            rbtm_accumulate(c, B, tmp, W, dm, alpha);
        }
    }
    BlockHeev hv = heev_truncate(c, dm, Mmax, cutoff);
    const std::vector<uint32_t>& keep = hv.keep;
    const TruncResults tr = hv.tr;
    // U = kept eigenvectors, descending (columns n-1, n-2, ...)
    m1 = DMPS(); m2 = DMPS();
    m1.phys = phys1; m1.left = left; m1.right_paired = false;
    m2.phys = phys2; m2.right = right; m2.right_paired = true;
    std::vector<std::pair<Charge, std::size_t>> mid;
    for (std::size_t k = 0; k < nb; ++k) {
        if (!keep[k]) continue;
        mid.push_back({both.lc[k], keep[k]});
        m1.b.add(both.lc[k], both.lc[k], both.rows[k], keep[k]);
        m2.b.add(both.lc[k], both.lc[k], keep[k], both.cols[k]);
    }
    m1.right = sorted_basis(mid);
    m2.left = m1.right;
    m1.b.allocate(c.s, true);
    m2.b.allocate(c.s, true);
    std::vector<CopyJob> cj;
    std::vector<GemmJob> gj;
    std::size_t i = 0;
    for (std::size_t k = 0; k < nb; ++k) {
        if (!keep[k]) continue;
        const uint32_t n = dm.rows[k], kp = keep[k], rows = both.rows[k], cols = both.cols[k];
        const uint64_t src = dm.off[k] + uint64_t(n - kp) * n;  // last kp eigenvectors, read in reverse
        GemmJob g{};
        if (l2r) {
            // site 1 = U (rows x kp); site 2 = U^T both (kp x cols)
            cj.push_back(CopyJob{src, m1.b.off[i], n, kp, n, rows, 0, 1});
            g.a_off = m1.b.off[i]; g.ta = 1; g.lda = rows;
            g.b_off = both.off[k]; g.ldb = rows;
            g.c_off = m2.b.off[i]; g.ldc = kp;
            g.M = kp; g.N = cols; g.K = rows;
        } else {
            // site 2 = U^T (kp x cols); site 1 = both U = both (site 2)^T (rows x kp)
            cj.push_back(CopyJob{src, m2.b.off[i], n, kp, n, kp, 1, 1});
            g.a_off = both.off[k]; g.lda = rows;
            g.b_off = m2.b.off[i]; g.tb = 1; g.ldb = kp;
            g.c_off = m1.b.off[i]; g.ldc = rows;
            g.M = rows; g.N = kp; g.K = cols;
        }
        g.alpha = 1.0; g.beta = 0.0;
        gj.push_back(g);
        ++i;
    }
    if (l2r) {
        batched_copy(cj, dm.d.get(), dm.total, m1.b.d.get(), m1.b.total, c.cjobs, c.s);
        batched_gemm(gj, m1.b.d.get(), m1.b.total, both.d.get(), both.total, m2.b.d.get(), m2.b.total, c.gjobs, c.gtiles, c.s);
    } else {
        batched_copy(cj, dm.d.get(), dm.total, m2.b.d.get(), m2.b.total, c.cjobs, c.s);
        batched_gemm(gj, both.d.get(), both.total, m2.b.d.get(), m2.b.total, m1.b.d.get(), m1.b.total, c.gjobs, c.gtiles, c.s);
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
    return tr;
}

}  // namespace qcm

namespace qcm {

// ---------------------------------------------------------------------------
// single-site growth (contractions/engine.hpp:85-123, boundary_ops/prediction.hpp:41-148)
TruncResults grow_l2r(Ctx& c, DMPS& a, DMPS& b, const DevBoundary& L, const MPOTensor& W, double alpha, uint64_t Mmax,
                      double cutoff) {
    make_left_paired(c, a);
    const std::size_t nb = a.b.n();
    // alpha_dm: a a^T per right sector, plus alpha times the noise of the left boundary step
    DBlocks dm;
    std::vector<GemmJob> jobs;
    for (std::size_t k = 0; k < nb; ++k) {
        const uint32_t m = a.b.rows[k], n = a.b.cols[k];
        dm.add(a.b.rc[k], a.b.rc[k], m, m);
        GemmJob g{};
        g.a_off = a.b.off[k]; g.lda = m; g.b_off = a.b.off[k]; g.ldb = m; g.tb = 1;
        g.M = m; g.N = m; g.K = n; g.c_off = dm.off.back(); g.ldc = m; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    dm.allocate(c.s, true);
    batched_gemm(jobs, a.b.d.get(), a.b.total, a.b.d.get(), a.b.total, dm.d.get(), dm.total, c.gjobs, c.gtiles, c.s);
    {
        DMPS ket = right_paired_copy(c, a);
        lbtm_accumulate(c, L, ket, a, W, dm, alpha);
    }
    BlockHeev hv = heev_truncate(c, dm, Mmax, cutoff);
    // new a = U (kept eigenvectors, descending); t = U^T a_old (kept x old right sector)
    DMPS u;
    u.phys = a.phys; u.left = a.left; u.right_paired = false;
    DBlocks t;
    std::vector<std::pair<Charge, std::size_t>> kept;
    std::vector<CopyJob> cj;
    std::vector<GemmJob> gj;
    for (std::size_t k = 0; k < nb; ++k) {
        const uint32_t kp = hv.keep[k];
        if (!kp) continue;
        const uint32_t n = dm.rows[k], cols = a.b.cols[k];
        kept.push_back({a.b.rc[k], kp});
        u.b.add(a.b.rc[k], a.b.rc[k], n, kp);
        t.add(a.b.rc[k], a.b.rc[k], kp, cols);
        cj.push_back(CopyJob{dm.off[k] + uint64_t(n - kp) * n, u.b.off.back(), n, kp, n, n, 0, 1});
        GemmJob g{};
        g.a_off = u.b.off.back(); g.ta = 1; g.lda = n;
        g.b_off = a.b.off[k]; g.ldb = n;
        g.c_off = t.off.back(); g.ldc = kp;
        g.M = kp; g.N = cols; g.K = n; g.alpha = 1.0; g.beta = 0.0;
        gj.push_back(g);
    }
    u.right = sorted_basis(kept);
    u.b.allocate(c.s, true);
    t.allocate(c.s, true);
    batched_copy(cj, dm.d.get(), dm.total, u.b.d.get(), u.b.total, c.cjobs, c.s);
    batched_gemm(gj, u.b.d.get(), u.b.total, a.b.d.get(), a.b.total, t.d.get(), t.total, c.gjobs, c.gtiles, c.s);
    multiply_from_left(c, b, t);
    a = std::move(u);
    QCM_CUDA(cudaStreamSynchronize(c.s));
    return hv.tr;
}

TruncResults grow_r2l(Ctx& c, DMPS& a, DMPS& b, const DevBoundary& R, const MPOTensor& W, double alpha, uint64_t Mmax,
                      double cutoff) {
    make_right_paired(c, a);
    const std::size_t nb = a.b.n();
    // alpha_dm_right: a^T a per left sector, plus alpha times the noise of the right boundary step
    DBlocks dm;
    std::vector<GemmJob> jobs;
    for (std::size_t k = 0; k < nb; ++k) {
        const uint32_t m = a.b.rows[k], n = a.b.cols[k];
        dm.add(a.b.lc[k], a.b.lc[k], n, n);
        GemmJob g{};
        g.a_off = a.b.off[k]; g.lda = m; g.b_off = a.b.off[k]; g.ldb = m; g.ta = 1;
        g.M = n; g.N = n; g.K = m; g.c_off = dm.off.back(); g.ldc = n; g.alpha = 1.0; g.beta = 0.0;
        jobs.push_back(g);
    }
    dm.allocate(c.s, true);
    batched_gemm(jobs, a.b.d.get(), a.b.total, a.b.d.get(), a.b.total, dm.d.get(), dm.total, c.gjobs, c.gtiles, c.s);
    rbtm_accumulate(c, R, a, W, dm, alpha);
    BlockHeev hv = heev_truncate(c, dm, Mmax, cutoff);
    // new a = U^T (right-paired, kept x phys.right); t = a_old U (old left sector x kept)
    DMPS u;
    u.phys = a.phys; u.right = a.right; u.right_paired = true;
    DBlocks t;
    std::vector<std::pair<Charge, std::size_t>> kept;
    std::vector<CopyJob> cj;
    std::vector<GemmJob> gj;
    for (std::size_t k = 0; k < nb; ++k) {
        const uint32_t kp = hv.keep[k];
        if (!kp) continue;
        const uint32_t n = dm.rows[k], rows = a.b.rows[k];
        kept.push_back({a.b.lc[k], kp});
        u.b.add(a.b.lc[k], a.b.lc[k], kp, n);
        t.add(a.b.lc[k], a.b.lc[k], rows, kp);
        cj.push_back(CopyJob{dm.off[k] + uint64_t(n - kp) * n, u.b.off.back(), n, kp, n, kp, 1, 1});
        GemmJob g{};
        g.a_off = a.b.off[k]; g.lda = rows;
        g.b_off = u.b.off.back(); g.tb = 1; g.ldb = kp;
        g.c_off = t.off.back(); g.ldc = rows;
        g.M = rows; g.N = kp; g.K = n; g.alpha = 1.0; g.beta = 0.0;
        gj.push_back(g);
    }
    u.left = sorted_basis(kept);
    u.b.allocate(c.s, true);
    t.allocate(c.s, true);
    batched_copy(cj, dm.d.get(), dm.total, u.b.d.get(), u.b.total, c.cjobs, c.s);
    batched_gemm(gj, a.b.d.get(), a.b.total, u.b.d.get(), u.b.total, t.d.get(), t.total, c.gjobs, c.gtiles, c.s);
    multiply_from_right(c, b, t);
    a = std::move(u);
    QCM_CUDA(cudaStreamSynchronize(c.s));
    return hv.tr;
}

}  // namespace qcm
