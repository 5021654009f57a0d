// ORACLE -- TEST INFRASTRUCTURE ONLY.  Two-site tensors, truncation, JD and the sweep,
// restated from mp_tensors/{twositetensor.hpp,ts_ops.hpp,mpstensor.hpp,mps.hpp,
// mps_initializers.h,mps_sectors.h}, block_matrix/block_matrix_algorithms.h,
// ietl/jacobi.h and optimize/{ts_optimize.hpp,optimize.h}.
#include "dmrg.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace orc {

namespace {
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
Mat matmul(const Mat& A, const Mat& B) {
    Mat C(A.r, B.c);
    dgemm('N', 'N', int(A.r), int(B.c), int(A.c), 1.0, A.d.data(), int(std::max<std::size_t>(A.r, 1)), B.d.data(),
          int(std::max<std::size_t>(B.r, 1)), 0.0, C.d.data(), int(std::max<std::size_t>(C.r, 1)));
    return C;
}
// block_matrix gemm (block_matrix_algorithms.h:64-90) for charge-diagonal operands
Mat matmul_tn(const Mat& A, const Mat& B) {  // A^T B
    Mat C(A.c, B.c);
    if (A.r && A.c && B.c)
        dgemm('T', 'N', int(A.c), int(B.c), int(A.r), 1.0, A.d.data(), int(A.r), B.d.data(), int(B.r), 0.0, C.d.data(), int(A.c));
    return C;
}
Mat matmul_nt(const Mat& A, const Mat& B) {  // A B^T
    Mat C(A.r, B.r);
    if (A.r && B.r && A.c)
        dgemm('N', 'T', int(A.r), int(B.r), int(A.c), 1.0, A.d.data(), int(A.r), B.d.data(), int(B.r), 0.0, C.d.data(), int(A.r));
    return C;
}

BlockMatrix bm_gemm(const BlockMatrix& A, const BlockMatrix& B) {
    BlockMatrix C;
    for (std::size_t k = 0; k < A.n_blocks(); ++k) {
        std::size_t j = B.find_left(A.rc[k]);
        if (j == B.n_blocks()) continue;
        C.insert(A.lc[k], B.rc[j], matmul(A.b[k], B.b[j]));
    }
    return C;
}
}  // namespace

// ---------------------------------------------------------------------------
// two-site MPO (ts_ops.hpp:97-168).  An entry with several operators takes all of
// them (the reference's single-summand branch reads operator 0 only; its MPOs
// carry one operator per entry).
MPOTensor make_twosite_mpo(const MPOTensor& W1, const MPOTensor& W2) {
    MPOTensor T;
    T.rows = W1.rows;
    T.cols = W2.cols;
    T.phys = W1.phys * W2.phys;
    T.herm_left = W1.herm_left; T.phase_left = W1.phase_left;
    T.herm_right = W2.herm_right; T.phase_right = W2.phase_right;
    ProductBasis pb(W1.phys, W2.phys);
    // sub-index of (s1, ss1) x (s2, ss2) inside the fused sector: pb + ss1*d2 + ss2 (alps_detail.hpp op_kron)
    auto sector_sub = [&](std::size_t s1, unsigned ss1, std::size_t s2, unsigned ss2, std::size_t& sec, unsigned& sub) {
        Q c = W1.phys[s1].first + W2.phys[s2].first;
        sec = T.phys.position(c);
        sub = unsigned(pb(W1.phys[s1].first, W2.phys[s2].first) + ss1 * W2.phys[s2].second + ss2);
    };
    auto kron_into = [&](const SiteOp& a, const SiteOp& b, double f, std::map<std::tuple<std::size_t, std::size_t, unsigned, unsigned>, double>& acc) {
        for (auto& ba : a.blocks)
            for (auto& bb : b.blocks)
                for (std::size_t i = 0; i < ba.coeff.size(); ++i)
                    for (std::size_t j = 0; j < bb.coeff.size(); ++j) {
                        std::size_t si, so;
                        unsigned ui, uo;
                        sector_sub(ba.in_sec, ba.ss1[i], bb.in_sec, bb.ss1[j], si, ui);
                        sector_sub(ba.out_sec, ba.ss2[i], bb.out_sec, bb.ss2[j], so, uo);
                        acc[{si, so, ui, uo}] += f * ba.coeff[i] * bb.coeff[j];
                    }
    };
    for (unsigned b1 = 0; b1 < W1.rows; ++b1) {
        std::map<unsigned, std::vector<unsigned>> summands;  // b3 -> b2 list
        for (unsigned b2 : W1.row_b2[b1])
            for (unsigned b3 : W2.row_b2[b2]) summands[b3].push_back(b2);
        for (auto& kv : summands) {
            unsigned b3 = kv.first;
            std::map<std::tuple<std::size_t, std::size_t, unsigned, unsigned>, double> acc;
            double scale = 1.0;
            const auto& e1s = W1.at.at({b1, kv.second[0]});
            const auto& e2s = W2.at.at({kv.second[0], b3});
            if (kv.second.size() == 1 && e1s.size() == 1 && e2s.size() == 1) {
                kron_into(W1.ops[W1.op[e1s[0]]], W2.ops[W2.op[e2s[0]]], 1.0, acc);
                scale = W1.scale[e1s[0]] * W2.scale[e2s[0]];
            } else {
                for (unsigned b2 : kv.second)
                    for (unsigned e1 : W1.at.at({b1, b2}))
                        for (unsigned e2 : W2.at.at({b2, b3}))
                            kron_into(W1.ops[W1.op[e1]], W2.ops[W2.op[e2]], W1.scale[e1] * W2.scale[e2], acc);
            }
            SiteOp op;
            for (auto& a : acc) {
                if (a.second == 0.0) continue;
                std::size_t si = std::get<0>(a.first), so = std::get<1>(a.first);
                std::size_t bi = 0;
                while (bi < op.blocks.size() && !(op.blocks[bi].in_sec == si && op.blocks[bi].out_sec == so)) ++bi;
                if (bi == op.blocks.size()) op.blocks.push_back(OpBlock{si, so, {}, {}, {}});
                op.blocks[bi].ss1.push_back(std::get<2>(a.first));
                op.blocks[bi].ss2.push_back(std::get<3>(a.first));
                op.blocks[bi].coeff.push_back(a.second);
            }
            if (op.blocks.empty()) continue;
            unsigned e = unsigned(T.b1.size());
            T.b1.push_back(b1); T.b2.push_back(b3); T.op.push_back(unsigned(T.ops.size())); T.scale.push_back(scale);
            T.ops.push_back(std::move(op));
            T.at[{b1, b3}].push_back(e);
        }
    }
    T.row_b2.resize(T.rows);
    T.col_b1.resize(T.cols);
    for (auto& kv : T.at) { T.row_b2[kv.first.first].push_back(kv.first.second); T.col_b1[kv.first.second].push_back(kv.first.first); }
    for (auto& v : T.row_b2) std::sort(v.begin(), v.end());
    for (auto& v : T.col_b1) std::sort(v.begin(), v.end());
    return T;
}

// ---------------------------------------------------------------------------
// two-site tensor (twositetensor.hpp:29-199, ts_reshape.h)
TwoSite::TwoSite(MPSTensor a, MPSTensor b) {
    phys1 = a.phys; phys2 = b.phys; phys = phys1 * phys2; left = a.left; right = b.right;
    a.make_left_paired();
    b.make_right_paired();
    both = bm_gemm(a.data, b.data);
}

MPSTensor TwoSite::make_mps() const {
    ProductBasis in_left(phys1, left), in_right(phys2, right, true), out_right(phys, right, true), ppb(phys1, phys2);
    MPSTensor t;
    t.phys = phys; t.left = left; t.right = right; t.pairing = RightPaired;
    for (std::size_t k = 0; k < both.n_blocks(); ++k) {
        Q c = both.lc[k];
        const Mat& in = both.b[k];
        for (std::size_t s1 = 0; s1 < phys1.size(); ++s1) {
            Q p1 = phys1[s1].first;
            std::size_t l = left.position(c + (-p1));
            if (l == left.size()) continue;
            for (std::size_t s2 = 0; s2 < phys2.size(); ++s2) {
                Q p2 = phys2[s2].first;
                std::size_t r = right.position(c + p2);
                if (r == right.size()) continue;
                Q lc = left[l].first, rc = right[r].first, sc = p1 + p2;
                std::size_t ob = t.data.find(lc, lc);
                if (ob == t.data.n_blocks()) ob = t.data.insert(lc, lc, Mat(left[l].second, out_right.size(lc)));
                Mat& out = t.data.b[ob];
                std::size_t ldim = left[l].second, rdim = right[r].second, sd1 = phys1[s1].second, sd2 = phys2[s2].second;
                std::size_t ilo = in_left(p1, lc), iro = in_right(p2, rc), oro = out_right(sc, rc), opo = ppb(p1, p2);
                for (std::size_t ss1 = 0; ss1 < sd1; ++ss1)
                    for (std::size_t ss2 = 0; ss2 < sd2; ++ss2) {
                        std::size_t so = opo + ss1 * sd2 + ss2;
                        for (std::size_t rr = 0; rr < rdim; ++rr)
                            for (std::size_t ll = 0; ll < ldim; ++ll)
                                out(ll, oro + so * rdim + rr) = in(ilo + ss1 * ldim + ll, iro + ss2 * rdim + rr);
                    }
            }
        }
    }
    return t;
}

void TwoSite::set_from_mps(const MPSTensor& tw) {
    ProductBasis in_left(phys1, left), in_right(phys2, right, true), out_right(phys, right, true), ppb(phys1, phys2);
    for (auto& m : both.b) std::fill(m.d.begin(), m.d.end(), 0.0);
    for (std::size_t k = 0; k < tw.data.n_blocks(); ++k) {
        Q lc = tw.data.lc[k];
        std::size_t l = left.position(lc);
        const Mat& src = tw.data.b[k];
        for (std::size_t s1 = 0; s1 < phys1.size(); ++s1)
            for (std::size_t s2 = 0; s2 < phys2.size(); ++s2) {
                Q p1 = phys1[s1].first, p2 = phys2[s2].first;
                Q rc = lc + p1 + p2;
                std::size_t r = right.position(rc);
                if (r == right.size()) continue;
                Q c = lc + p1;
                std::size_t bb = both.find(c, c);
                if (bb == both.n_blocks())  // ts_reshape.h: the both-paired block is created when missing
                    bb = both.insert(c, c, Mat(in_left.size(c), in_right.size(c)));
                Mat& dst = both.b[bb];
                std::size_t ldim = left[l].second, rdim = right[r].second, sd1 = phys1[s1].second, sd2 = phys2[s2].second;
                std::size_t ilo = in_left(p1, lc), iro = in_right(p2, rc), oro = out_right(p1 + p2, rc), opo = ppb(p1, p2);
                for (std::size_t ss1 = 0; ss1 < sd1; ++ss1)
                    for (std::size_t ss2 = 0; ss2 < sd2; ++ss2) {
                        std::size_t so = opo + ss1 * sd2 + ss2;
                        for (std::size_t rr = 0; rr < rdim; ++rr)
                            for (std::size_t ll = 0; ll < ldim; ++ll)
                                dst(ilo + ss1 * ldim + ll, iro + ss2 * rdim + rr) = src(ll, oro + so * rdim + rr);
                    }
            }
    }
}

TruncationResults estimate_truncation(const std::vector<std::vector<double>>& vals, std::size_t Mmax, double cutoff,
                                      std::vector<std::size_t>& keeps) {
    std::vector<double> all;
    for (auto& s : vals) all.insert(all.end(), s.begin(), s.end());
    std::sort(all.begin(), all.end());
    std::reverse(all.begin(), all.end());
    TruncationResults tr;
    double evalscut = cutoff * all[0];
    if (all.size() > Mmax) evalscut = std::max(evalscut, all[Mmax]);
    tr.smallest_ev = evalscut / all[0];
    double tf = 0, tw = 0, sum = 0, sum2 = 0;
    auto it = std::find_if(all.begin(), all.end(), [&](double x) { return x < evalscut; });
    for (; it != all.end(); ++it) { tf += *it; tw += (*it) * (*it); }
    for (double x : all) { sum += x; sum2 += x * x; }
    tr.truncated_fraction = tf / sum;
    tr.truncated_weight = tw / sum2;
    keeps.assign(vals.size(), 0);
    for (std::size_t k = 0; k < vals.size(); ++k)
        keeps[k] = std::size_t(std::find_if(vals[k].begin(), vals[k].end(), [&](double x) { return x < evalscut; }) - vals[k].begin());
    return tr;
}

TruncationResults heev_truncate(const BlockMatrix& dm, BlockMatrix& U, double cutoff, std::size_t Mmax) {
    const std::size_t nb = dm.n_blocks();
    std::vector<Mat> ev(nb);
    std::vector<std::vector<double>> w(nb), wsq(nb);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < int(nb); ++k) heev_desc(dm.b[k], ev[k], w[k]);
    for (std::size_t k = 0; k < nb; ++k) {
        wsq[k] = w[k];
        for (double& x : wsq[k]) if (x > 0.0) x = std::sqrt(x);
    }
    std::vector<std::size_t> keeps;
    TruncationResults tr = estimate_truncation(wsq, Mmax, cutoff, keeps);
    U = BlockMatrix();
    for (std::size_t k = 0; k < nb; ++k) {
        if (keeps[k] == 0) continue;
        Mat u(ev[k].r, keeps[k]);
        for (std::size_t j = 0; j < keeps[k]; ++j)
            for (std::size_t i = 0; i < ev[k].r; ++i) u(i, j) = ev[k](i, j);
        U.insert(dm.lc[k], dm.rc[k], std::move(u));
        tr.bond_dimension += keeps[k];
    }
    tr.truncated_weight = tr.truncated_fraction;  // heev_truncate reports the fraction in both fields
    return tr;
}

TruncationResults svd_truncate(const BlockMatrix& M, BlockMatrix& U, BlockMatrix& V, std::vector<std::vector<double>>& S,
                               double cutoff, std::size_t Mmax) {
    std::size_t nb = M.n_blocks();
    U = BlockMatrix(); V = BlockMatrix();
    std::vector<Mat> Ub(nb), Vb(nb);
    S.assign(nb, {});
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < int(nb); ++k) dgesvd_thin(M.b[k], Ub[k], S[k], Vb[k]);
    std::vector<std::size_t> keeps;
    TruncationResults tr = estimate_truncation(S, Mmax, cutoff, keeps);
    for (std::size_t k = 0; k < nb; ++k) {
        const std::size_t keep = keeps[k];
        if (keep == 0) { S[k].clear(); continue; }
        Mat u(Ub[k].r, keep), v(keep, Vb[k].c);
        for (std::size_t j = 0; j < keep; ++j)
            for (std::size_t i = 0; i < Ub[k].r; ++i) u(i, j) = Ub[k](i, j);
        for (std::size_t j = 0; j < Vb[k].c; ++j)
            for (std::size_t i = 0; i < keep; ++i) v(i, j) = Vb[k](i, j);
        S[k].resize(keep);
        U.insert(M.lc[k], M.rc[k], std::move(u));
        V.insert(M.lc[k], M.rc[k], std::move(v));
        tr.bond_dimension += keep;
    }
    std::vector<std::vector<double>> Sk;
    for (std::size_t k = 0; k < nb; ++k) if (!S[k].empty()) Sk.push_back(S[k]);
    S = Sk;
    return tr;
}

void TwoSite::split_l2r(std::size_t Mmax, double cutoff, MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const {
    BlockMatrix U, V;
    std::vector<std::vector<double>> S;
    tr = svd_truncate(both, U, V, S, cutoff, Mmax);
    m1 = MPSTensor();
    m1.phys = phys1; m1.left = left; m1.right = U.right_basis(); m1.pairing = LeftPaired; m1.data = U;
    for (std::size_t k = 0; k < V.n_blocks(); ++k)
        for (std::size_t j = 0; j < V.b[k].c; ++j)
            for (std::size_t i = 0; i < V.b[k].r; ++i) V.b[k](i, j) *= S[k][i];
    m2 = MPSTensor();
    m2.phys = phys2; m2.left = V.left_basis(); m2.right = right; m2.pairing = RightPaired; m2.data = V;
}

void TwoSite::split_r2l(std::size_t Mmax, double cutoff, MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const {
    BlockMatrix U, V;
    std::vector<std::vector<double>> S;
    tr = svd_truncate(both, U, V, S, cutoff, Mmax);
    m2 = MPSTensor();
    m2.phys = phys2; m2.left = V.left_basis(); m2.right = right; m2.pairing = RightPaired; m2.data = V;
    for (std::size_t k = 0; k < U.n_blocks(); ++k)
        for (std::size_t j = 0; j < U.b[k].c; ++j)
            for (std::size_t i = 0; i < U.b[k].r; ++i) U.b[k](i, j) *= S[k][j];
    m1 = MPSTensor();
    m1.phys = phys1; m1.left = left; m1.right = U.right_basis(); m1.pairing = LeftPaired; m1.data = U;
}

void TwoSite::predict_split_l2r(std::size_t Mmax, double cutoff, double alpha, const Boundary& lb, const MPOTensor& mpo,
                                MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const {
    if (alpha == 0.0) { split_l2r(Mmax, cutoff, m1, m2, tr); return; }
    // the both-paired data as a left-paired tensor over (phys1, left) x (adjoin(phys2) * right)
    MPSTensor tmp;
    tmp.phys = phys1; tmp.left = left; tmp.right = adjoin(phys2) * right; tmp.pairing = LeftPaired; tmp.data = both;
    BlockMatrix dm;
    for (std::size_t k = 0; k < both.n_blocks(); ++k) {
        const Mat& b = both.b[k];
        Mat d(b.r, b.r);
        dgemm('N', 'T', int(b.r), int(b.r), int(b.c), 1.0, b.d.data(), int(std::max<std::size_t>(b.r, 1)), b.d.data(),
              int(std::max<std::size_t>(b.r, 1)), 0.0, d.d.data(), int(std::max<std::size_t>(b.r, 1)));
        dm.insert(both.lc[k], both.lc[k], std::move(d));
    }
    alpha_dm_direct(tmp, lb, mpo, dm, alpha);
    BlockMatrix U;
    tr = heev_truncate(dm, U, cutoff, Mmax);
    m1 = MPSTensor();
    m1.phys = phys1; m1.left = left; m1.right = U.right_basis(); m1.pairing = LeftPaired; m1.data = U;
    BlockMatrix V;  // U^T both
    for (std::size_t k = 0; k < U.n_blocks(); ++k) {
        const std::size_t j = both.find(U.lc[k], U.lc[k]);
        const Mat& u = U.b[k];
        const Mat& b = both.b[j];
        Mat v(u.c, b.c);
        dgemm('T', 'N', int(u.c), int(b.c), int(u.r), 1.0, u.d.data(), int(u.r), b.d.data(), int(b.r), 0.0, v.d.data(), int(u.c));
        V.insert(U.lc[k], U.lc[k], std::move(v));
    }
    m2 = MPSTensor();
    m2.phys = phys2; m2.left = V.left_basis(); m2.right = right; m2.pairing = RightPaired; m2.data = V;
}

void TwoSite::predict_split_r2l(std::size_t Mmax, double cutoff, double alpha, const Boundary& rb, const MPOTensor& mpo,
                                MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const {
    if (alpha == 0.0) { split_r2l(Mmax, cutoff, m1, m2, tr); return; }
    // the both-paired data as a right-paired tensor over (phys1 * left) x (phys2, right)
    MPSTensor tmp;
    tmp.phys = phys2; tmp.left = phys1 * left; tmp.right = right; tmp.pairing = RightPaired; tmp.data = both;
    BlockMatrix dm;
    for (std::size_t k = 0; k < both.n_blocks(); ++k) {
        const Mat& b = both.b[k];
        Mat d(b.c, b.c);
        dgemm('T', 'N', int(b.c), int(b.c), int(b.r), 1.0, b.d.data(), int(std::max<std::size_t>(b.r, 1)), b.d.data(),
              int(std::max<std::size_t>(b.r, 1)), 0.0, d.d.data(), int(std::max<std::size_t>(b.c, 1)));
        dm.insert(both.lc[k], both.lc[k], std::move(d));
    }
    alpha_dm_direct_right(tmp, rb, mpo, dm, alpha);
    BlockMatrix U;
    tr = heev_truncate(dm, U, cutoff, Mmax);
    BlockMatrix Ut, V;  // U^T (right-paired site 2) and both U (left-paired site 1)
    for (std::size_t k = 0; k < U.n_blocks(); ++k) {
        const Mat& u = U.b[k];
        Mat t(u.c, u.r);
        for (std::size_t j = 0; j < u.c; ++j)
            for (std::size_t i = 0; i < u.r; ++i) t(j, i) = u(i, j);
        Ut.insert(U.lc[k], U.lc[k], std::move(t));
        const std::size_t jb = both.find(U.lc[k], U.lc[k]);
        const Mat& b = both.b[jb];
        Mat v(b.r, u.c);
        dgemm('N', 'N', int(b.r), int(u.c), int(b.c), 1.0, b.d.data(), int(b.r), u.d.data(), int(u.r), 0.0, v.d.data(), int(b.r));
        V.insert(U.lc[k], U.lc[k], std::move(v));
    }
    m2 = MPSTensor();
    m2.phys = phys2; m2.left = Ut.left_basis(); m2.right = right; m2.pairing = RightPaired; m2.data = Ut;
    m1 = MPSTensor();
    m1.phys = phys1; m1.left = left; m1.right = V.right_basis(); m1.pairing = LeftPaired; m1.data = V;
}

TruncationResults grow_l2r(MPSTensor& a, MPSTensor& b, const Boundary& left, const MPOTensor& mpo, double alpha,
                           double cutoff, std::size_t Mmax) {
    a.make_left_paired();
    // alpha_dm (prediction.hpp:41-55): a a^T per right sector, then the noise term
    BlockMatrix dm;
    for (std::size_t k = 0; k < a.data.n_blocks(); ++k) dm.insert(a.data.lc[k], a.data.rc[k], matmul_nt(a.data.b[k], a.data.b[k]));
    alpha_dm_direct(a, left, mpo, dm, alpha);
    BlockMatrix U;
    TruncationResults tr = heev_truncate(dm, U, cutoff, Mmax);
    BlockMatrix t;  // U^T a: kept states x old right sector
    for (std::size_t k = 0; k < U.n_blocks(); ++k) {
        const std::size_t j = a.data.find(U.lc[k], U.rc[k]);
        t.insert(U.rc[k], a.data.rc[j], matmul_tn(U.b[k], a.data.b[j]));
    }
    multiply_from_left(b, t);
    a.data = U;
    a.right = U.right_basis();
    return tr;
}

TruncationResults grow_r2l(MPSTensor& a, MPSTensor& b, const Boundary& right, const MPOTensor& mpo, double alpha,
                           double cutoff, std::size_t Mmax) {
    a.make_right_paired();
    // alpha_dm_right (prediction.hpp:57-71): a^T a per left sector, then the noise term
    BlockMatrix dm;
    for (std::size_t k = 0; k < a.data.n_blocks(); ++k) dm.insert(a.data.lc[k], a.data.rc[k], matmul_tn(a.data.b[k], a.data.b[k]));
    alpha_dm_direct_right(a, right, mpo, dm, alpha);
    BlockMatrix U;
    TruncationResults tr = heev_truncate(dm, U, cutoff, Mmax);
    BlockMatrix t, Ut;  // a U: old left sector x kept states; U^T the new right-paired site tensor
    for (std::size_t k = 0; k < U.n_blocks(); ++k) {
        const std::size_t j = a.data.find(U.lc[k], U.rc[k]);
        t.insert(a.data.lc[j], U.rc[k], matmul(a.data.b[j], U.b[k]));
        const Mat& u = U.b[k];
        Mat ut(u.c, u.r);
        for (std::size_t c = 0; c < u.c; ++c)
            for (std::size_t r = 0; r < u.r; ++r) ut(c, r) = u(r, c);
        Ut.insert(U.rc[k], U.lc[k], std::move(ut));
    }
    multiply_from_right(b, t);
    a.data = Ut;
    a.left = Ut.left_basis();
    return tr;
}

BlockMatrix normalize_left(MPSTensor& t) {
    t.make_left_paired();
    BlockMatrix Qm, R;
    for (std::size_t k = 0; k < t.data.n_blocks(); ++k) {
        Mat q, r;
        qr(t.data.b[k], q, r);
        Qm.insert(t.data.lc[k], t.data.rc[k], std::move(q));
        R.insert(t.data.rc[k], t.data.rc[k], std::move(r));
    }
    t.data = Qm;
    t.right = Qm.right_basis();
    return R;
}

BlockMatrix normalize_right(MPSTensor& t) {
    t.make_right_paired();
    BlockMatrix Lm, Qm;
    for (std::size_t k = 0; k < t.data.n_blocks(); ++k) {
        Mat l, q;
        lq(t.data.b[k], l, q);
        Lm.insert(t.data.lc[k], t.data.lc[k], std::move(l));
        Qm.insert(t.data.lc[k], t.data.rc[k], std::move(q));
    }
    t.data = Qm;
    t.left = Qm.left_basis();
    return Lm;
}

void multiply_from_left(MPSTensor& t, const BlockMatrix& N) {
    t.make_right_paired();
    t.data = bm_gemm(N, t.data);
    t.left = t.data.left_basis();
}

void multiply_from_right(MPSTensor& t, const BlockMatrix& N) {
    t.make_left_paired();
    t.data = bm_gemm(t.data, N);
    t.right = t.data.right_basis();
}

// ---------------------------------------------------------------------------
// Jacobi-Davidson for the lowest eigenpair: solve_ietl_jcd (dmrg/solver/ietl_jacobi_davidson.h:35-76)
// -> jacobi_davidson::calculate_eigenvalue (ietl/jacobi.h:386-474), the correction equation by
// jcd_gmres_solver (ietl/jacobi.h:126-164) through ietl_gmres (ietl/gmres.h:78-146) on the operator
// (I - uu*)(A - theta)(I - uu*) (jcd_solver_operator, ietl/jacobi.h:249-268), and the projection
// against the ortho vectors (DavidsonVS::project, dmrg/solver/ietl_interface_dv.h:94-99).
namespace {
using Vec = std::vector<double>;
double vdot(const Vec& a, const Vec& b) {
    double s = 0;
    for (std::size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}
void vaxpy(double a, const Vec& x, Vec& y) {
    for (std::size_t i = 0; i < y.size(); ++i) y[i] += a * x[i];
}

// GeneratePlaneRotation / ApplyPlaneRotation (ietl/gmres.h:40-66)
void gen_rot(double dx, double dy, double& cs, double& sn) {
    if (dy == 0.0) { cs = 1; sn = 0; }
    else if (std::fabs(dy) > std::fabs(dx)) { double t = dx / dy; sn = 1.0 / std::sqrt(1.0 + t * t); cs = t * sn; }
    else { double t = dy / dx; cs = 1.0 / std::sqrt(1.0 + t * t); sn = t * cs; }
}
void apply_rot(double& dx, double& dy, double cs, double sn) {
    const double r0 = cs * dx + sn * dy, r1 = -sn * dx + cs * dy;
    dx = r0; dy = r1;
}

// ietl_gmres::operator() (ietl/gmres.h:92-146).  On a break at inner step i the update uses the
// first i directions only (Update(H, s, i), :66-75 and :140), as the reference does.
Vec gmres(const std::function<void(const Vec&, Vec&)>& A, const Vec& b, const Vec& x0, double abs_tol, int max_iter) {
    const std::size_t m = std::size_t(max_iter);
    Vec s(m + 1, 0.0), cs(m + 1, 0.0), sn(m + 1, 0.0);
    std::vector<Vec> v(m + 1);
    A(x0, v[0]);
    Vec r = b;
    vaxpy(-1.0, v[0], r);
    s[0] = std::sqrt(vdot(r, r));
    if (std::fabs(s[0]) < abs_tol) return x0;
    v[0] = r;
    for (double& e : v[0]) e /= s[0];
    std::vector<double> H((m + 1) * (m + 1), 0.0);
    auto h = [&](std::size_t i, std::size_t j) -> double& { return H[i + j * (m + 1)]; };
    std::size_t i = 0;
    Vec w;
    for (; i + 1 < m; ++i) {
        A(v[i], w);
        for (std::size_t k = 0; k <= i; ++k) {
            h(k, i) = vdot(w, v[k]);
            vaxpy(-h(k, i), v[k], w);
        }
        h(i + 1, i) = std::sqrt(vdot(w, w));
        v[i + 1] = w;
        for (double& e : v[i + 1]) e /= h(i + 1, i);
        for (std::size_t k = 0; k < i; ++k) apply_rot(h(k, i), h(k + 1, i), cs[k], sn[k]);
        gen_rot(h(i, i), h(i + 1, i), cs[i], sn[i]);
        apply_rot(h(i, i), h(i + 1, i), cs[i], sn[i]);
        apply_rot(s[i], s[i + 1], cs[i], sn[i]);
        if (std::fabs(s[i + 1]) < abs_tol) break;
    }
    Vec y(s.begin(), s.begin() + i);
    for (std::ptrdiff_t a = std::ptrdiff_t(i) - 1; a >= 0; --a) {
        y[a] /= h(a, a);
        for (std::ptrdiff_t c = a - 1; c >= 0; --c) y[c] -= h(c, a) * y[a];
    }
    Vec out = x0;
    for (std::size_t k = 0; k < i; ++k) vaxpy(y[k], v[k], out);
    return out;
}
}  // namespace

double jacobi_davidson(const std::function<void(const std::vector<double>&, std::vector<double>&)>& mult,
                       const std::vector<double>& x0, double tol, int maxiter, std::vector<double>& out, int& iters,
                       int gmres_iter, const std::vector<std::vector<double>>& ortho_in, int* applies) {
    const std::size_t n = x0.size();
    int napply = 0;
    auto A = [&](const Vec& x, Vec& y) { y.assign(n, 0.0); mult(x, y); ++napply; };
    // ortho vectors: at most n - 1, Gram-Schmidt among themselves (ietl_jacobi_davidson.h:41-48)
    std::vector<Vec> O(ortho_in.begin(), ortho_in.begin() + std::min(ortho_in.size(), n ? n - 1 : 0));
    for (std::size_t a = 1; a < O.size(); ++a)
        for (std::size_t b = 0; b < a; ++b) vaxpy(-vdot(O[b], O[a]) / vdot(O[b], O[b]), O[b], O[a]);
    auto project = [&](Vec& t) { for (const Vec& o : O) vaxpy(-vdot(o, t) / vdot(o, o), o, t); };
    auto nrm = [&](const Vec& a) { return std::sqrt(vdot(a, a)); };
    std::vector<Vec> V(maxiter), VA(maxiter);
    std::vector<double> M(std::size_t(maxiter) * maxiter, 0.0);
    V[0] = x0;
    project(V[0]);
    int it = 0;
    double theta = 0;
    std::vector<double> s;
    Vec u(n), uA(n);
    while (true) {
        Vec& t = V[it];
        double tau = nrm(t);
        for (int i = 1; i <= it; ++i) vaxpy(-vdot(V[i - 1], t), V[i - 1], t);
        if (nrm(t) < 0.25 * tau)
            for (int i = 1; i <= it; ++i) vaxpy(-vdot(V[i - 1], t), V[i - 1], t);
        project(t);
        double tn = nrm(t);
        for (auto& x : t) x /= tn;
        A(t, VA[it]);
        for (int i = 1; i <= it + 1; ++i) M[(i - 1) + std::size_t(it) * maxiter] = vdot(V[i - 1], VA[it]);
        dsyevx_lowest(M.data(), maxiter, it + 1, tol, theta, s);
        for (std::size_t k = 0; k < n; ++k) { u[k] = V[0][k] * s[0]; uA[k] = VA[0][k] * s[0]; }
        for (int j = 1; j <= it; ++j)
            for (std::size_t k = 0; k < n; ++k) { u[k] += V[j][k] * s[j]; uA[k] += VA[j][k] * s[j]; }
        project(uA);
        Vec& r = uA;
        vaxpy(-theta, u, r);
        ++it;
        double rn = nrm(r);
        if (rn <= tol * std::fabs(theta) || rn < tol || it >= maxiter) {
            out = u;
            iters = it;
            if (applies) *applies = napply;
            return theta;
        }
        // jcd_gmres_solver::operator() (ietl/jacobi.h:141-157): start t0 = -r + (r.u)/(u.u) u, then
        // GMRES(max_iter = ietl_jcd_gmres) on -r with abs_tol 2^-(it+1)
        const double dru = vdot(r, u), duu = vdot(u, u);
        Vec t0(n);
        for (std::size_t k = 0; k < n; ++k) t0[k] = -r[k] + dru / duu * u[k];
        if (gmres_iter > 0) {
            const double th = theta;
            auto op = [&](const Vec& x, Vec& y) {
                Vec t2 = x;
                vaxpy(-vdot(u, x), u, t2);
                A(t2, y);
                vaxpy(-th, t2, y);
                vaxpy(-vdot(u, y), u, y);
            };
            Vec inh(n);
            for (std::size_t k = 0; k < n; ++k) inh[k] = -r[k];
            V[it] = gmres(op, inh, t0, 1.0 / std::pow(2.0, double(it + 1)), gmres_iter);
        } else {
            V[it] = std::move(t0);
        }
    }
}

// ---------------------------------------------------------------------------
// MPS initialisation: allowed_sectors (mps_sectors.h:52-140) + const_mps_init
// (mps_initializers.h:84-100) + MPS::normalize_left (mps.hpp:129-136)
namespace {
std::vector<Index> allowed_sectors(int L, const Index& phys, Q right_end, std::size_t Mmax) {
    Index physc = phys;
    physc.sort();
    Q maxc = physc.v.front().first, minc = physc.v.back().first;
    if (minc > maxc) std::swap(maxc, minc);
    Q maxt, mint;
    for (int i = 0; i < L; ++i) { maxt = maxt + maxc; mint = mint + minc; }
    std::vector<Index> la(L + 1), ra(L + 1), allowed(L + 1);
    la[0].insert(Q(0, 0), 1);
    ra[L].insert(right_end, 1);
    Q cmaxi = maxt, cmini = mint;
    for (int i = 1; i <= L; ++i) {
        la[i] = phys * la[i - 1];
        cmaxi = cmaxi + (-maxc);
        cmini = cmini + (-minc);
        Index keep;
        for (auto& e : la[i].v) {
            if ((e.first + cmaxi) < right_end) continue;
            if ((e.first + cmini) > right_end) continue;
            keep.v.push_back({e.first, std::min(Mmax, e.second)});
        }
        la[i] = keep;
    }
    cmaxi = maxt; cmini = mint;
    for (int i = L - 1; i >= 0; --i) {
        ra[i] = adjoin(phys) * ra[i + 1];
        cmaxi = cmaxi + (-maxc);
        cmini = cmini + (-minc);
        Index keep;
        for (auto& e : ra[i].v) {
            if ((e.first + (-cmaxi)) > Q(0, 0)) continue;
            if ((e.first + (-cmini)) < Q(0, 0)) continue;
            keep.v.push_back({e.first, std::min(Mmax, e.second)});
        }
        ra[i] = keep;
    }
    for (int i = 0; i <= L; ++i) {
        Index a = la[i], b = ra[i];
        common_subset(a, b);
        for (auto& e : a.v) e.second = std::min(Mmax, std::min(la[i].size_of_block(e.first), ra[i].size_of_block(e.first)));
        allowed[i] = a;
    }
    return allowed;
}

// MPSTensor(sd, ld, rd, fillrand=false, val) (mpstensor.hpp:40-71)
MPSTensor const_tensor(const Index& sd, const Index& ld, const Index& rd, double val) {
    MPSTensor t;
    t.phys = sd;
    Index lb = sd * ld, rb = rd;
    common_subset(lb, rb);
    t.right = rb;
    Index possible = adjoin(sd) * t.right, ltemp = ld;
    common_subset(ltemp, possible);
    t.left = ltemp;
    lb.sort(); rb.sort(); t.left.sort(); t.right.sort();
    t.pairing = LeftPaired;
    for (std::size_t k = 0; k < lb.size(); ++k) t.data.insert(lb[k].first, rb[k].first, Mat(lb[k].second, rb[k].second, val));
    return t;
}
}  // namespace

DMRG::DMRG(std::vector<MPOTensor> mpo_single, int nup, int ndown, const DMRGParams& prm) : mpo(std::move(mpo_single)), p(prm) {
    L = int(mpo.size());
    for (int i = 0; i + 1 < L; ++i) ts_mpo.push_back(make_twosite_mpo(mpo[i], mpo[i + 1]));
    Index phys = mpo[0].phys;
    std::vector<Index> allowed = allowed_sectors(L, phys, Q(nup, ndown), p.init_bond_dimension);
    mps.resize(L);
    for (int i = 0; i < L; ++i) {
        mps[i] = const_tensor(phys, allowed[i], allowed[i + 1], 1.0);
        mps[i].scale(1.0 / mps[i].norm());
    }
    // MPS::normalize_left: canonize(L-1) then normalise the last site
    for (int i = 0; i < L - 1; ++i) {
        BlockMatrix t = normalize_left(mps[i]);
        multiply_from_left(mps[i + 1], t);
        mps[i + 1].scale(1.0 / mps[i + 1].norm());
    }
    normalize_left(mps[L - 1]);
    // optimizer_base: mps.canonize(0)
    for (int i = L - 1; i > 0; --i) {
        BlockMatrix t = normalize_right(mps[i]);
        multiply_from_right(mps[i - 1], t);
        mps[i - 1].scale(1.0 / mps[i - 1].norm());
    }
    // init_left_right (optimize.h:158-195)
    left_.resize(L + 1);
    right_.resize(L + 1);
    left_[0] = trivial_boundary(mps[0].left, mpo[0].rows);
    right_[L] = trivial_boundary(mps[L - 1].right, mpo[L - 1].cols);
    for (int i = L - 1; i >= 0; --i) right_[i] = overlap_mpo_right_step(mps[i], mps[i], right_[i + 1], mpo[i], true);
}

// ---------------------------------------------------------------------------
// Excited states.  overlap_left_step (mp_tensors/mps.h:178-197): t = left * ket (right-paired), reshaped
// to left-paired over the bra's left basis, then bra^T t.
BlockMatrix ortho_left_step(const MPSTensor& bra_in, const MPSTensor& ket_in, const BlockMatrix& left) {
    MPSTensor bra = bra_in, ket = ket_in;
    bra.make_left_paired();
    ket.make_right_paired();
    MPSTensor t;
    t.phys = ket.phys; t.left = bra.left; t.right = ket.right; t.pairing = RightPaired;
    t.data = bm_gemm(left, ket.data);
    t.make_left_paired();
    BlockMatrix out;
    for (std::size_t k = 0; k < bra.data.n_blocks(); ++k) {
        const std::size_t j = t.data.find(bra.data.rc[k], bra.data.rc[k]);
        if (j == t.data.n_blocks()) continue;
        out.insert(bra.data.rc[k], bra.data.rc[k], matmul_tn(bra.data.b[k], t.data.b[j]));
    }
    return out;
}

// overlap_right_step (mp_tensors/mps.h:200-219): t = ket (left-paired) * right^T, reshaped to right-paired
// over the bra's right basis, then bra t^T.
BlockMatrix ortho_right_step(const MPSTensor& bra_in, const MPSTensor& ket_in, const BlockMatrix& right) {
    MPSTensor bra = bra_in, ket = ket_in;
    bra.make_right_paired();
    ket.make_left_paired();
    MPSTensor t;
    t.phys = ket.phys; t.left = ket.left; t.right = bra.right; t.pairing = LeftPaired;
    for (std::size_t k = 0; k < ket.data.n_blocks(); ++k) {
        const std::size_t j = right.find(ket.data.rc[k], ket.data.rc[k]);
        if (j == right.n_blocks()) continue;
        t.data.insert(ket.data.rc[k], ket.data.rc[k], matmul_nt(ket.data.b[k], right.b[j]));
    }
    t.make_right_paired();
    BlockMatrix out;
    for (std::size_t k = 0; k < bra.data.n_blocks(); ++k) {
        const std::size_t j = t.data.find(bra.data.lc[k], bra.data.lc[k]);
        if (j == t.data.n_blocks()) continue;
        out.insert(bra.data.lc[k], bra.data.lc[k], matmul_nt(bra.data.b[k], t.data.b[j]));
    }
    return out;
}

// site_ortho_boundaries (contractions/special.hpp:38-62): left * ortho twin, then each (phys state,
// right sector) column slice times right^T, placed in the current twin's right-paired layout; blocks and
// slices the ortho product does not reach stay zero
std::vector<double> ortho_vector(const MPSTensor& twin, const MPSTensor& ortho_in, const BlockMatrix& left,
                                 const BlockMatrix& right) {
    MPSTensor ot = ortho_in;
    ot.make_right_paired();
    ProductBasis cur_pb(twin.phys, twin.right, true), ort_pb(ot.phys, ot.right, true);
    std::vector<double> v;
    for (std::size_t k = 0; k < twin.data.n_blocks(); ++k) {
        const Q lc = twin.data.lc[k];
        Mat blk(twin.data.b[k].r, twin.data.b[k].c);
        const std::size_t jl = left.find(lc, lc), jo = ot.data.find(lc, lc);
        if (jl < left.n_blocks() && jo < ot.data.n_blocks()) {
            const Mat t = matmul(left.b[jl], ot.data.b[jo]);
            for (std::size_t s = 0; s < twin.phys.size(); ++s) {
                const Q ph = twin.phys[s].first, rc = lc + ph;
                if (!twin.right.has(rc) || !ot.right.has(rc)) continue;
                const std::size_t jr = right.find(rc, rc);
                if (jr == right.n_blocks()) continue;
                const std::size_t rs_c = twin.right.size_of_block(rc), rs_o = ot.right.size_of_block(rc);
                for (std::size_t ss = 0; ss < twin.phys[s].second; ++ss) {
                    const std::size_t oc = ort_pb(ph, rc) + ss * rs_o, cc = cur_pb(ph, rc) + ss * rs_c;
                    Mat slice(t.r, rs_o);
                    for (std::size_t j = 0; j < rs_o; ++j)
                        for (std::size_t i = 0; i < t.r; ++i) slice(i, j) = t(i, oc + j);
                    const Mat pr = matmul_nt(slice, right.b[jr]);
                    for (std::size_t j = 0; j < rs_c; ++j)
                        for (std::size_t i = 0; i < pr.r; ++i) blk(i, cc + j) = pr(i, j);
                }
            }
        }
        v.insert(v.end(), blk.d.begin(), blk.d.end());
    }
    return v;
}

namespace {
// left_boundary_bm / right_boundary_bm (mp_tensors/mps.hpp:241-264): unit blocks of the end index
BlockMatrix unit_boundary(const Index& i) {
    BlockMatrix b;
    for (std::size_t k = 0; k < i.size(); ++k) {
        Mat m(i[k].second, i[k].second);
        for (std::size_t d = 0; d < i[k].second; ++d) m(d, d) = 1.0;
        b.insert(i[k].first, i[k].first, std::move(m));
    }
    return b;
}
}  // namespace

void DMRG::set_ortho(std::vector<std::vector<MPSTensor>> states) {
    for (auto& st : states)
        if (int(st.size()) != L) throw std::runtime_error("set_ortho: an ortho state with the wrong length");
    ortho_mps = std::move(states);
    const std::size_t n = ortho_mps.size();
    ortho_left_.assign(n, std::vector<BlockMatrix>(L + 1));
    ortho_right_.assign(n, std::vector<BlockMatrix>(L + 1));
    for (std::size_t o = 0; o < n; ++o) {
        ortho_left_[o][0] = unit_boundary(mps[0].left);
        ortho_right_[o][L] = unit_boundary(mps[L - 1].right);
        for (int i = L - 1; i >= 0; --i) ortho_right_[o][i] = ortho_right_step(mps[i], ortho_mps[o][i], ortho_right_[o][i + 1]);
    }
}

void DMRG::sweep_single(int sweep_no, std::vector<double>& energies, std::vector<TruncationResults>& trunc) {
    energies.clear();
    trunc.clear();
    for (int _site = 0; _site < 2 * L; ++_site) {
        const int lr = _site < L ? 1 : -1;
        const int site = _site < L ? _site : 2 * L - 1 - _site;  // to_site (ss_optimize.hpp:57-62)
        MPSTensor& x = mps[site];
        x.make_right_paired();
        // solve_site_problem with the single-site MPO (ss_optimize.hpp:120)
        double t0 = now_s();
        auto sched = create_contraction_schedule(x, left_[site], right_[site + 1], mpo[site]);
        double t1 = now_s();
        schedule_time += t1 - t0;
        std::vector<std::size_t> off;
        std::size_t tot = 0;
        for (auto& b : x.data.b) { off.push_back(tot); tot += b.d.size(); }
        std::vector<double> x0(tot);
        for (std::size_t k = 0; k < x.data.n_blocks(); ++k) std::copy(x.data.b[k].d.begin(), x.data.b[k].d.end(), x0.begin() + off[k]);
        auto mult = [&](const std::vector<double>& in, std::vector<double>& out) {
            double h0 = now_s();
            std::vector<const double*> xv(x.left.size(), nullptr);
            std::vector<double*> yv(x.left.size(), nullptr);
            std::fill(out.begin(), out.end(), 0.0);
            for (std::size_t lb = 0; lb < x.left.size(); ++lb) {
                std::size_t k = x.data.find(x.left[lb].first, x.left[lb].first);
                if (k == x.data.n_blocks()) continue;
                xv[lb] = in.data() + off[k];
                yv[lb] = out.data() + off[k];
            }
            super_hamil_mv(*sched, left_[site], right_[site + 1], xv, yv);
            hpsi_time += now_s() - h0;
            hpsi_count++;
            hpsi_flops += sched->total_flops;
        };
        // ortho vectors (ss_optimize.hpp:104-109)
        std::vector<std::vector<double>> ortho_vecs;
        for (std::size_t o = 0; o < ortho_mps.size(); ++o) {
            MPSTensor ot = ortho_mps[o][site];
            ot.make_right_paired();
            ortho_vecs.push_back(ortho_vector(x, ot, ortho_left_[o][site], ortho_right_[o][site + 1]));
        }
        std::vector<double> xo;
        int iters = 0;
        double E = jacobi_davidson(mult, x0, p.jcd_tol, p.jcd_maxiter, xo, iters, p.jcd_gmres, ortho_vecs);
        jd_time += now_s() - t1;
        for (std::size_t k = 0; k < x.data.n_blocks(); ++k)
            std::copy(xo.begin() + off[k], xo.begin() + off[k] + x.data.b[k].d.size(), x.data.b[k].d.begin());
        energies.push_back(E + p.ecore);
        // alpha, cutoff and Mmax of this sweep (ss_optimize.hpp:143-155)
        const double alpha = sweep_no < p.ngrowsweeps ? p.alpha_initial
                             : (sweep_no < p.ngrowsweeps + p.nmainsweeps ? p.alpha_main : p.alpha_final);
        TruncationResults tr;
        double t2 = now_s();
        if (lr == 1) {
            // ss_optimize.hpp:158-173
            if (site < L - 1) tr = grow_l2r(x, mps[site + 1], left_[site], mpo[site], alpha, p.cutoff, p.Mmax);
            else normalize_left(x);
            double t3 = now_s();
            trunc_time += t3 - t2;
            left_[site + 1] = overlap_mpo_left_step(x, x, left_[site], mpo[site], true);
            for (std::size_t o = 0; o < ortho_mps.size(); ++o)
                ortho_left_[o][site + 1] = ortho_left_step(x, ortho_mps[o][site], ortho_left_[o][site]);
            boundary_time += now_s() - t3;
        } else {
            // ss_optimize.hpp:174-186
            if (site > 0) tr = grow_r2l(x, mps[site - 1], right_[site + 1], mpo[site], alpha, p.cutoff, p.Mmax);
            else normalize_right(x);
            double t3 = now_s();
            trunc_time += t3 - t2;
            right_[site] = overlap_mpo_right_step(x, x, right_[site + 1], mpo[site], true);
            for (std::size_t o = 0; o < ortho_mps.size(); ++o)
                ortho_right_[o][site] = ortho_right_step(x, ortho_mps[o][site], ortho_right_[o][site + 1]);
            boundary_time += now_s() - t3;
        }
        trunc.push_back(tr);
    }
}

void DMRG::sweep(int sweep_no, std::vector<double>& energies, std::vector<TruncationResults>& trunc, int stop_step,
                 std::vector<uint8_t>* snap) {
    if (p.single_site) {
        if (stop_step >= 0) throw std::runtime_error("DMRG: site-problem snapshots of two-site sweeps only");
        sweep_single(sweep_no, energies, trunc);
        return;
    }
    energies.clear();
    trunc.clear();
    for (int _site = 0; _site < 2 * L - 2; ++_site) {
        int lr, site1, site2;
        int site = (_site < L - 1) ? _site : 2 * L - 2 - _site;
        if (_site < L - 1) { lr = 1; site1 = site; site2 = site + 1; }
        else { lr = -1; site1 = site - 1; site2 = site; }
        TwoSite tst(mps[site1], mps[site2]);
        MPSTensor twin = tst.make_mps();
        if (stop_step == _site && snap) {
            *snap = save_site_problem(twin, left_[site1], right_[site2 + 1]);
            return;
        }
        // solve_site_problem (solver_interface.hpp:30-77)
        double t0 = now_s();
        auto sched = create_contraction_schedule(twin, left_[site1], right_[site2 + 1], ts_mpo[site1]);
        double t1 = now_s();
        schedule_time += t1 - t0;
        std::vector<std::size_t> off;
        std::size_t tot = 0;
        for (auto& b : twin.data.b) { off.push_back(tot); tot += b.d.size(); }
        std::vector<double> x0(tot);
        for (std::size_t k = 0; k < twin.data.n_blocks(); ++k) std::copy(twin.data.b[k].d.begin(), twin.data.b[k].d.end(), x0.begin() + off[k]);
        auto mult = [&](const std::vector<double>& x, std::vector<double>& y) {
            double h0 = now_s();
            std::vector<const double*> xv(twin.left.size(), nullptr);
            std::vector<double*> yv(twin.left.size(), nullptr);
            std::fill(y.begin(), y.end(), 0.0);
            for (std::size_t lb = 0; lb < twin.left.size(); ++lb) {
                std::size_t k = twin.data.find(twin.left[lb].first, twin.left[lb].first);
                if (k == twin.data.n_blocks()) continue;
                xv[lb] = x.data() + off[k];
                yv[lb] = y.data() + off[k];
            }
            super_hamil_mv(*sched, left_[site1], right_[site2 + 1], xv, yv);
            hpsi_time += now_s() - h0;
            hpsi_count++;
            hpsi_flops += sched->total_flops;
        };
        // ortho vectors of this step (ts_optimize.hpp:217-223)
        std::vector<std::vector<double>> ortho_vecs;
        for (std::size_t o = 0; o < ortho_mps.size(); ++o) {
            TwoSite ts_o(ortho_mps[o][site1], ortho_mps[o][site2]);
            ortho_vecs.push_back(ortho_vector(twin, ts_o.make_mps(), ortho_left_[o][site1], ortho_right_[o][site2 + 1]));
        }
        std::vector<double> xo;
        int iters = 0;
        double E = jacobi_davidson(mult, x0, p.jcd_tol, p.jcd_maxiter, xo, iters, p.jcd_gmres, ortho_vecs);
        jd_time += now_s() - t1;
        for (std::size_t k = 0; k < twin.data.n_blocks(); ++k)
            std::copy(xo.begin() + off[k], xo.begin() + off[k] + twin.data.b[k].d.size(), twin.data.b[k].d.begin());
        tst.set_from_mps(twin);
        static const bool dbg = std::getenv("ORC_DEBUG") != nullptr;
        if (dbg) {
            double nt = 0; for (auto& b : twin.data.b) for (double v : b.d) nt += v * v;
            std::fprintf(stderr, "step %d: |twin|^2=%.12f |both|^2=%.12f\n", _site, nt, tst.both.norm2());
        }
        energies.push_back(E + p.ecore);
        TruncationResults tr;
        double t2 = now_s();
        // alpha of this sweep (ts_optimize.hpp:275-282)
        const double alpha = sweep_no < p.ngrowsweeps ? p.alpha_initial
                             : (sweep_no < p.ngrowsweeps + p.nmainsweeps ? p.alpha_main : p.alpha_final);
        if (lr == 1) {
            if (p.heev) tst.predict_split_l2r(p.Mmax, p.cutoff, alpha, left_[site1], mpo[site1], mps[site1], mps[site2], tr);
            else tst.split_l2r(p.Mmax, p.cutoff, mps[site1], mps[site2], tr);
            if (dbg) std::fprintf(stderr, "   split: |U|^2=%.12f |SV|^2=%.12f tw=%.3e\n", mps[site1].data.norm2(), mps[site2].data.norm2(), tr.truncated_weight);
            BlockMatrix t = normalize_left(mps[site2]);
            if (dbg) std::fprintf(stderr, "   qr: |Q|^2=%.12f |R|^2=%.12f\n", mps[site2].data.norm2(), t.norm2());
            if (site2 < L - 1) multiply_from_left(mps[site2 + 1], t);
            if (dbg && site2 < L - 1) std::fprintf(stderr, "   next: |RB|^2=%.12f\n", mps[site2 + 1].data.norm2());
            double t3 = now_s();
            trunc_time += t3 - t2;
            left_[site2] = overlap_mpo_left_step(mps[site1], mps[site1], left_[site1], mpo[site1], true);
            for (std::size_t o = 0; o < ortho_mps.size(); ++o)
                ortho_left_[o][site2] = ortho_left_step(mps[site1], ortho_mps[o][site1], ortho_left_[o][site1]);
            boundary_time += now_s() - t3;
        } else {
            if (p.heev) tst.predict_split_r2l(p.Mmax, p.cutoff, alpha, right_[site2 + 1], mpo[site2], mps[site1], mps[site2], tr);
            else tst.split_r2l(p.Mmax, p.cutoff, mps[site1], mps[site2], tr);
            BlockMatrix t = normalize_right(mps[site1]);
            if (site1 > 0) multiply_from_right(mps[site1 - 1], t);
            double t3 = now_s();
            trunc_time += t3 - t2;
            right_[site2] = overlap_mpo_right_step(mps[site2], mps[site2], right_[site2 + 1], mpo[site2], true);
            for (std::size_t o = 0; o < ortho_mps.size(); ++o)
                ortho_right_[o][site2] = ortho_right_step(mps[site2], ortho_mps[o][site2], ortho_right_[o][site2 + 1]);
            boundary_time += now_s() - t3;
        }
        trunc.push_back(tr);
    }
}

// ---------------------------------------------------------------------------
// "QSPB" v1 site-problem blob
namespace {
struct W {
    std::vector<uint8_t> b;
    template <class T> void put(T v) { const uint8_t* p = reinterpret_cast<const uint8_t*>(&v); b.insert(b.end(), p, p + sizeof(T)); }
    void idx(const Index& i) { put<uint32_t>(uint32_t(i.size())); for (auto& e : i.v) { put<int32_t>(e.first.n[0]); put<int32_t>(e.first.n[1]); put<uint32_t>(uint32_t(e.second)); } }
    void bnd(const Boundary& B) {
        const BoundaryIndex& x = B.index;
        idx(x.bra); idx(x.ket);
        uint32_t aux = x.n_cohorts() ? uint32_t(x.offsets[0].size()) : 0;
        put<uint32_t>(x.n_cohorts()); put<uint32_t>(aux);
        for (unsigned ci = 0; ci < x.n_cohorts(); ++ci) {
            uint32_t lb = 0, rb = 0;
            for (std::size_t i = 0; i < x.lbrb.size(); ++i)
                for (std::size_t j = 0; j < x.lbrb[i].size(); ++j) if (x.lbrb[i][j] == ci) { lb = uint32_t(i); rb = uint32_t(j); }
            put<uint32_t>(lb); put<uint32_t>(rb); put<uint8_t>(uint8_t(x.tr_[ci]));
            put<uint32_t>(uint32_t(x.lsz[ci])); put<uint32_t>(uint32_t(x.rsz[ci])); put<uint32_t>(x.nb[ci]);
            for (uint32_t b = 0; b < aux; ++b) put<int64_t>(x.offsets[ci][b]);
            for (uint32_t b = 0; b < aux; ++b) put<double>(x.cscale[ci][b]);
            put<uint64_t>(B.data[ci].size());
            for (double v : B.data[ci]) put<double>(v);
        }
    }
};
struct R {
    const uint8_t* p; std::size_t n, k = 0;
    template <class T> T get() { if (k + sizeof(T) > n) throw std::runtime_error("site problem blob truncated"); T v; std::memcpy(&v, p + k, sizeof(T)); k += sizeof(T); return v; }
    Index idx() { Index i; uint32_t m = get<uint32_t>(); for (uint32_t s = 0; s < m; ++s) { int a = get<int32_t>(), b = get<int32_t>(); uint32_t z = get<uint32_t>(); i.v.push_back({Q(a, b), z}); } return i; }
    Boundary bnd() {
        Boundary B;
        Index bra = idx(), ket = idx();
        B.index = BoundaryIndex(bra, ket);
        uint32_t nc = get<uint32_t>(), aux = get<uint32_t>();
        B.data.resize(nc);
        for (uint32_t ci = 0; ci < nc; ++ci) {
            uint32_t lb = get<uint32_t>(), rb = get<uint32_t>();
            uint8_t tr = get<uint8_t>();
            uint32_t ls = get<uint32_t>(), rs = get<uint32_t>(), nb = get<uint32_t>();
            std::vector<long> off(aux);
            std::vector<double> cs(aux);
            for (auto& o : off) o = long(get<int64_t>());
            for (auto& c : cs) c = get<double>();
            B.index.lbrb[lb][rb] = ci;
            B.index.offsets.push_back(off); B.index.cscale.push_back(cs);
            B.index.trans.push_back(std::vector<char>(aux, 0)); B.index.tr_.push_back(char(tr));
            B.index.lsz.push_back(ls); B.index.rsz.push_back(rs); B.index.nb.push_back(nb);
            uint64_t nd = get<uint64_t>();
            B.data[ci].resize(nd);
            for (auto& v : B.data[ci]) v = get<double>();
        }
        return B;
    }
};
}  // namespace

std::vector<uint8_t> save_site_problem(const MPSTensor& twin0, const Boundary& L, const Boundary& Rb) {
    MPSTensor twin = twin0;
    twin.make_right_paired();
    W w;
    w.put<uint32_t>(0x42505351u);  // "QSPB"
    w.put<uint32_t>(1);
    w.idx(twin.phys); w.idx(twin.left); w.idx(twin.right);
    w.put<uint32_t>(uint32_t(twin.data.n_blocks()));
    for (std::size_t k = 0; k < twin.data.n_blocks(); ++k) {
        w.put<int32_t>(twin.data.lc[k].n[0]); w.put<int32_t>(twin.data.lc[k].n[1]);
        w.put<uint32_t>(uint32_t(twin.data.b[k].r)); w.put<uint32_t>(uint32_t(twin.data.b[k].c));
        for (double v : twin.data.b[k].d) w.put<double>(v);
    }
    w.bnd(L);
    w.bnd(Rb);
    return w.b;
}

std::vector<uint8_t> site_problem_from_mps(const std::vector<MPOTensor>& mpo, const std::vector<MPSTensor>& mps, int site1) {
    const int L = int(mps.size());
    if (int(mpo.size()) != L || site1 < 0 || site1 + 1 >= L) throw std::runtime_error("site problem: bad site or lengths");
    Boundary left = trivial_boundary(mps[0].left, mpo[0].rows);
    for (int i = 0; i < site1; ++i) left = overlap_mpo_left_step(mps[i], mps[i], left, mpo[i], true);
    Boundary right = trivial_boundary(mps[L - 1].right, mpo[L - 1].cols);
    for (int i = L - 1; i > site1 + 1; --i) right = overlap_mpo_right_step(mps[i], mps[i], right, mpo[i], true);
    TwoSite tst(mps[site1], mps[site1 + 1]);
    return save_site_problem(tst.make_mps(), left, right);
}

std::vector<uint8_t> save_mps_tensor(const MPSTensor& m0) {
    MPSTensor m = m0;
    m.make_right_paired();
    W w;
    w.put<uint32_t>(0x53504D51u);  // "QMPS"
    w.put<uint32_t>(1);
    w.idx(m.phys); w.idx(m.left); w.idx(m.right);
    w.put<uint32_t>(uint32_t(m.data.n_blocks()));
    for (std::size_t k = 0; k < m.data.n_blocks(); ++k) {
        w.put<int32_t>(m.data.lc[k].n[0]); w.put<int32_t>(m.data.lc[k].n[1]);
        w.put<uint32_t>(uint32_t(m.data.b[k].r)); w.put<uint32_t>(uint32_t(m.data.b[k].c));
        for (double v : m.data.b[k].d) w.put<double>(v);
    }
    return w.b;
}

MPSTensor load_mps_tensor(const uint8_t* p, std::size_t n) {
    R r{p, n};
    if (r.get<uint32_t>() != 0x53504D51u || r.get<uint32_t>() != 1) throw std::runtime_error("bad MPS tensor blob");
    MPSTensor m;
    m.phys = r.idx(); m.left = r.idx(); m.right = r.idx();
    m.pairing = RightPaired;
    const uint32_t nb = r.get<uint32_t>();
    for (uint32_t k = 0; k < nb; ++k) {
        int a = r.get<int32_t>(), b = r.get<int32_t>();
        uint32_t rows = r.get<uint32_t>(), cols = r.get<uint32_t>();
        Mat x(rows, cols);
        for (auto& v : x.d) v = r.get<double>();
        m.data.insert(Q(a, b), Q(a, b), std::move(x));
    }
    return m;
}

std::vector<uint8_t> save_boundary_step(int side, int site, const MPSTensor& m0, const Boundary& in, const Boundary& out) {
    MPSTensor m = m0;
    m.make_right_paired();
    W w;
    w.put<uint32_t>(0x50534251u);  // "QBSP"
    w.put<uint32_t>(1);
    w.put<uint32_t>(uint32_t(side));
    w.put<uint32_t>(uint32_t(site));
    w.idx(m.phys); w.idx(m.left); w.idx(m.right);
    w.put<uint32_t>(uint32_t(m.data.n_blocks()));
    for (std::size_t k = 0; k < m.data.n_blocks(); ++k) {
        w.put<int32_t>(m.data.lc[k].n[0]); w.put<int32_t>(m.data.lc[k].n[1]);
        w.put<uint32_t>(uint32_t(m.data.b[k].r)); w.put<uint32_t>(uint32_t(m.data.b[k].c));
        for (double v : m.data.b[k].d) w.put<double>(v);
    }
    w.bnd(in);
    w.bnd(out);
    return w.b;
}

void load_site_problem(const uint8_t* p, std::size_t n, MPSTensor& twin, Boundary& Lb, Boundary& Rb) {
    R r{p, n};
    if (r.get<uint32_t>() != 0x42505351u || r.get<uint32_t>() != 1) throw std::runtime_error("bad site problem blob");
    twin = MPSTensor();
    twin.phys = r.idx(); twin.left = r.idx(); twin.right = r.idx();
    twin.pairing = RightPaired;
    uint32_t nb = r.get<uint32_t>();
    for (uint32_t k = 0; k < nb; ++k) {
        int a = r.get<int32_t>(), b = r.get<int32_t>();
        uint32_t rows = r.get<uint32_t>(), cols = r.get<uint32_t>();
        Mat m(rows, cols);
        for (auto& v : m.d) v = r.get<double>();
        twin.data.insert(Q(a, b), Q(a, b), std::move(m));
    }
    Lb = r.bnd();
    Rb = r.bnd();
}

}  // namespace orc
