// ORACLE -- TEST INFRASTRUCTURE ONLY.  Core containers of the CPU restatement.
#include "core.hpp"

#include <dlfcn.h>

#include <cstring>
#include <mutex>

namespace orc {

// indexing_stable.hpp:434-451
Index operator*(const Index& a, const Index& b) {
    Index r;
    for (auto& x : a.v)
        for (auto& y : b.v) {
            Q c = x.first + y.first;
            std::size_t p = r.position(c);
            if (p < r.size()) r[p].second += x.second * y.second;
            else r.insert(c, x.second * y.second);
        }
    r.sort();
    return r;
}

Index adjoin(const Index& a) {
    Index r;
    for (auto& x : a.v) r.insert(-x.first, x.second);
    return r;
}

void common_subset(Index& a, Index& b) {
    Index na, nb;
    for (auto& x : a.v) if (b.has(x.first)) na.v.push_back(x);
    for (auto& x : b.v) if (na.has(x.first)) nb.v.push_back(x);
    a = na;
    b = nb;
}

ProductBasis::ProductBasis(const Index& a, const Index& b, bool neg_first) {
    for (auto& x : a.v)
        for (auto& y : b.v) {
            Q pc = neg_first ? (-x.first + y.first) : (x.first + y.first);
            std::size_t& t = sz[{pc.n[0], pc.n[1]}];
            kv[{{x.first.n[0], x.first.n[1]}, {y.first.n[0], y.first.n[1]}}] = t;
            t += x.second * y.second;
        }
}

std::size_t ProductBasis::operator()(Q a, Q b) const {
    auto it = kv.find({{a.n[0], a.n[1]}, {b.n[0], b.n[1]}});
    if (it == kv.end()) throw std::runtime_error("oracle ProductBasis: missing pair");
    return it->second;
}

std::size_t BlockMatrix::insert(Q l, Q r, Mat m) {
    std::size_t k = 0;
    while (k < b.size() && (lc[k] > l || (lc[k] == l && rc[k] > r))) ++k;
    lc.insert(lc.begin() + k, l);
    rc.insert(rc.begin() + k, r);
    b.insert(b.begin() + k, std::move(m));
    return k;
}

Index BlockMatrix::left_basis() const {
    Index r;
    for (std::size_t k = 0; k < b.size(); ++k) r.v.push_back({lc[k], b[k].r});
    return r;
}
Index BlockMatrix::right_basis() const {
    Index r;
    for (std::size_t k = 0; k < b.size(); ++k) r.v.push_back({rc[k], b[k].c});
    return r;
}

// reshapes.h:197-... (reshape_left_to_right_new): left-paired (phys*left) x right
// -> right-paired left x (phys*right), column offset ProductBasis(phys, right, -p + r)
void MPSTensor::make_right_paired() {
    if (pairing == RightPaired) return;
    ProductBasis in_left(phys, left);
    ProductBasis out_right(phys, right, true);
    BlockMatrix out;
    for (std::size_t lb = 0; lb < left.size(); ++lb) {
        Q lc = left[lb].first;
        std::size_t ldim = left[lb].second;
        std::size_t ncol = 0;
        for (std::size_t s = 0; s < phys.size(); ++s) {
            Q rc = lc + phys[s].first;
            if (right.has(rc)) ncol = std::max(ncol, out_right(phys[s].first, rc) + phys[s].second * right.size_of_block(rc));
        }
        if (ncol == 0) continue;
        Mat m(ldim, ncol);
        for (std::size_t s = 0; s < phys.size(); ++s) {
            Q p = phys[s].first;
            Q rc = lc + p;
            std::size_t rb = right.position(rc);
            if (rb == right.size()) continue;
            std::size_t k = data.find(rc, rc);
            if (k == data.n_blocks()) continue;
            std::size_t rdim = right[rb].second, sdim = phys[s].second;
            std::size_t il = in_left(p, lc), orr = out_right(p, rc);
            const Mat& src = data.b[k];
            for (std::size_t ss = 0; ss < sdim; ++ss)
                for (std::size_t rr = 0; rr < rdim; ++rr)
                    for (std::size_t ll = 0; ll < ldim; ++ll)
                        m(ll, orr + ss * rdim + rr) = src(il + ss * ldim + ll, rr);
        }
        out.insert(lc, lc, std::move(m));
    }
    data = std::move(out);
    pairing = RightPaired;
}

// reshapes.h:309-... (reshape_right_to_left_new)
void MPSTensor::make_left_paired() {
    if (pairing == LeftPaired) return;
    ProductBasis out_left(phys, left);
    ProductBasis in_right(phys, right, true);
    BlockMatrix out;
    for (std::size_t rb = 0; rb < right.size(); ++rb) {
        Q rc = right[rb].first;
        std::size_t rdim = right[rb].second;
        std::size_t nrow = 0;
        for (std::size_t s = 0; s < phys.size(); ++s) {
            Q lc = rc + (-phys[s].first);
            if (left.has(lc)) nrow = std::max(nrow, out_left(phys[s].first, lc) + phys[s].second * left.size_of_block(lc));
        }
        if (nrow == 0) continue;
        Mat m(nrow, rdim);
        for (std::size_t s = 0; s < phys.size(); ++s) {
            Q p = phys[s].first;
            Q lc = rc + (-p);
            std::size_t lb = left.position(lc);
            if (lb == left.size()) continue;
            std::size_t k = data.find(lc, lc);
            if (k == data.n_blocks()) continue;
            std::size_t ldim = left[lb].second, sdim = phys[s].second;
            std::size_t ol = out_left(p, lc), ir = in_right(p, rc);
            const Mat& src = data.b[k];
            for (std::size_t ss = 0; ss < sdim; ++ss)
                for (std::size_t rr = 0; rr < rdim; ++rr)
                    for (std::size_t ll = 0; ll < ldim; ++ll)
                        m(ol + ss * ldim + ll, rr) = src(ll, ir + ss * rdim + rr);
        }
        out.insert(rc, rc, std::move(m));
    }
    data = std::move(out);
    pairing = LeftPaired;
}

// ---- MPO blob ("QMPO" v1, written by the product's input prep) --------------
namespace {
struct Rd {
    const uint8_t* p; std::size_t n, k = 0;
    template <class T> T get() {
        if (k + sizeof(T) > n) throw std::runtime_error("oracle: MPO blob truncated");
        T v; std::memcpy(&v, p + k, sizeof(T)); k += sizeof(T); return v;
    }
};
}  // namespace

std::vector<MPOTensor> load_mpo_blob(const uint8_t* p, std::size_t n, bool& twosite) {
    Rd r{p, n};
    if (r.get<uint32_t>() != 0x4F504D51u || r.get<uint32_t>() != 1) throw std::runtime_error("oracle: bad MPO blob");
    uint32_t nt = r.get<uint32_t>();
    twosite = r.get<uint32_t>() != 0;
    std::vector<MPOTensor> out(nt);
    for (auto& T : out) {
        uint32_t ns = r.get<uint32_t>();
        for (uint32_t s = 0; s < ns; ++s) {
            int a = r.get<int32_t>(), b = r.get<int32_t>();
            uint32_t sz = r.get<uint32_t>();
            T.phys.v.push_back({Q(a, b), sz});
        }
        T.rows = r.get<uint32_t>(); T.cols = r.get<uint32_t>();
        uint64_t nnz = r.get<uint64_t>();
        for (uint64_t e = 0; e < nnz; ++e) {
            T.b1.push_back(r.get<uint32_t>()); T.b2.push_back(r.get<uint32_t>());
            T.op.push_back(r.get<uint32_t>()); T.scale.push_back(r.get<double>());
        }
        T.herm_left.resize(T.rows); T.phase_left.resize(T.rows);
        T.herm_right.resize(T.cols); T.phase_right.resize(T.cols);
        for (uint32_t i = 0; i < T.rows; ++i) { T.herm_left[i] = r.get<int32_t>(); T.phase_left[i] = r.get<int32_t>(); }
        for (uint32_t i = 0; i < T.cols; ++i) { T.herm_right[i] = r.get<int32_t>(); T.phase_right[i] = r.get<int32_t>(); }
        // state -> (sector, sub)
        std::vector<std::size_t> sec, sub;
        for (std::size_t s = 0; s < T.phys.size(); ++s)
            for (std::size_t j = 0; j < T.phys[s].second; ++j) { sec.push_back(s); sub.push_back(j); }
        uint32_t no = r.get<uint32_t>();
        T.ops.resize(no);
        for (auto& o : T.ops) {
            uint32_t k = r.get<uint32_t>();
            for (uint32_t i = 0; i < k; ++i) {
                uint32_t in = r.get<uint32_t>(), ou = r.get<uint32_t>();
                double v = r.get<double>();
                std::size_t bi = 0;
                while (bi < o.blocks.size() && !(o.blocks[bi].in_sec == sec[in] && o.blocks[bi].out_sec == sec[ou])) ++bi;
                if (bi == o.blocks.size()) o.blocks.push_back(OpBlock{sec[in], sec[ou], {}, {}, {}});
                o.blocks[bi].ss1.push_back(unsigned(sub[in]));
                o.blocks[bi].ss2.push_back(unsigned(sub[ou]));
                o.blocks[bi].coeff.push_back(v);
            }
        }
        T.row_b2.resize(T.rows);
        T.col_b1.resize(T.cols);
        for (std::size_t e = 0; e < T.b1.size(); ++e) {
            auto& lst = T.at[{T.b1[e], T.b2[e]}];
            if (lst.empty()) { T.row_b2[T.b1[e]].push_back(T.b2[e]); T.col_b1[T.b2[e]].push_back(T.b1[e]); }
            lst.push_back(unsigned(e));
        }
        for (auto& v : T.row_b2) std::sort(v.begin(), v.end());
        for (auto& v : T.col_b1) std::sort(v.begin(), v.end());
    }
    return out;
}

// ---- boundary index -----------------------------------------------------------
// boundary.h:129-148
unsigned BoundaryIndex::add_cohort(std::size_t lb, std::size_t rb, const std::vector<long>& off) {
    unsigned ci = n_cohorts();
    lbrb[lb][rb] = ci;
    offsets.push_back(off);
    cscale.push_back(std::vector<double>(off.size(), 1.0));
    trans.push_back(std::vector<char>(off.size(), 0));
    tr_.push_back(0);
    lsz.push_back(bra[lb].second);
    rsz.push_back(ket[rb].second);
    nb.push_back(unsigned(std::count_if(off.begin(), off.end(), [](long o) { return o > -1; })));
    return ci;
}

// boundary.h:150-179; conjugate_correction is 1 for abelian symmetries (boundary.h:66-71)
void BoundaryIndex::complement_transpose(const std::vector<int>& herm, const std::vector<int>& phase, bool forward) {
    for (std::size_t rb = 0; rb < ket.size(); ++rb)
        for (std::size_t lb = 0; lb < bra.size(); ++lb) {
            if (lbrb[lb][rb] == std::numeric_limits<unsigned>::max()) continue;
            unsigned ciA = lbrb[lb][rb];
            unsigned ciB = cohort_index(ket[rb].first, bra[lb].first);
            if (ciB == n_cohorts()) {
                std::size_t blb = bra.position(ket[rb].first), brb = ket.position(bra[lb].first);
                if (blb == bra.size() || brb == ket.size()) continue;
                ciB = add_cohort(blb, brb, std::vector<long>(herm.size(), -1));
                tr_[ciB] = 1;
            }
            for (unsigned b = 0; b < herm.size(); ++b) {
                if (MPOTensor::skip(herm, b, ket[rb].first, bra[lb].first)) {
                    offsets[ciB][b] = offsets[ciA][herm[b]];
                    cscale[ciB][b] = double(phase[forward ? b : herm[b]]);
                    trans[ciB][b] = 1;
                }
            }
        }
}

Boundary trivial_boundary(const Index& idx, std::size_t aux_dim) {
    Boundary B;
    B.index = BoundaryIndex(idx, idx);
    for (std::size_t i = 0; i < idx.size(); ++i) {
        std::size_t bs = idx[i].second * idx[i].second;
        std::vector<long> off(aux_dim);
        for (std::size_t b = 0; b < aux_dim; ++b) off[b] = long(b * bs);
        B.index.add_cohort(i, i, off);
    }
    B.allocate_all();
    for (auto& v : B.data) std::fill(v.begin(), v.end(), 1.0);
    return B;
}

// ---- BLAS / LAPACK through scipy's OpenBLAS ----------------------------------
namespace {
typedef void (*dgemm_t)(const char*, const char*, const int*, const int*, const int*, const double*, const double*,
                        const int*, const double*, const int*, const double*, double*, const int*);
typedef void (*dgesvd_t)(const char*, const char*, const int*, const int*, double*, const int*, double*, double*,
                         const int*, double*, const int*, double*, const int*, int*);
typedef void (*dsyevx_t)(const char*, const char*, const char*, const int*, double*, const int*, const double*,
                         const double*, const int*, const int*, const double*, int*, double*, double*, const int*,
                         double*, const int*, int*, int*, int*);
typedef void (*dsyevd_t)(const char*, const char*, const int*, double*, const int*, double*, double*, const int*, int*,
                         const int*, int*);
typedef void (*setthreads_t)(int);
dgemm_t p_dgemm = nullptr;
dgesvd_t p_dgesvd = nullptr;
dsyevx_t p_dsyevx = nullptr;
dsyevd_t p_dsyevd = nullptr;
}  // namespace

bool blas_init(const char* path, std::string& err) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (p_dgemm) return true;
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) { err = dlerror(); return false; }
    p_dgemm = (dgemm_t)dlsym(h, "scipy_dgemm_");
    p_dgesvd = (dgesvd_t)dlsym(h, "scipy_dgesvd_");
    p_dsyevx = (dsyevx_t)dlsym(h, "scipy_dsyevx_");
    p_dsyevd = (dsyevd_t)dlsym(h, "scipy_dsyevd_");
    auto st = (setthreads_t)dlsym(h, "scipy_openblas_set_num_threads");
    if (!p_dgemm || !p_dgesvd || !p_dsyevx || !p_dsyevd) {
        err = "missing LAPACK symbol";
        p_dgemm = nullptr;
        return false;
    }
    if (st) st(1);  // parallelism comes from OpenMP over blocks, as in the reference
    return true;
}

void dgemm(char ta, char tb, int m, int n, int k, double alpha, const double* A, int lda, const double* B, int ldb,
           double beta, double* C, int ldc) {
    if (m == 0 || n == 0) return;
    if (k == 0) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < m; ++i) C[i + std::size_t(j) * ldc] = beta == 0.0 ? 0.0 : beta * C[i + std::size_t(j) * ldc];
        return;
    }
    p_dgemm(&ta, &tb, &m, &n, &k, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}

void daxpy(std::size_t n, double a, const double* x, double* y) {
    for (std::size_t i = 0; i < n; ++i) y[i] += a * x[i];
}

// alps/matrix/algorithms.hpp:243-257 (gesvd 'S','S')
void dgesvd_thin(const Mat& A0, Mat& U, std::vector<double>& S, Mat& VT) {
    int m = int(A0.r), n = int(A0.c), k = std::min(m, n);
    Mat A = A0;
    U = Mat(m, k); VT = Mat(k, n); S.assign(k, 0.0);
    if (k == 0) return;
    char jobu = 'S', jobvt = 'S';
    int lwork = -1, info = 0, ldu = std::max(1, m), ldvt = std::max(1, k);
    double wq;
    p_dgesvd(&jobu, &jobvt, &m, &n, A.d.data(), &m, S.data(), U.d.data(), &ldu, VT.d.data(), &ldvt, &wq, &lwork, &info);
    lwork = int(wq);
    std::vector<double> work(lwork);
    p_dgesvd(&jobu, &jobvt, &m, &n, A.d.data(), &m, S.data(), U.d.data(), &ldu, VT.d.data(), &ldvt, work.data(), &lwork, &info);
    if (info != 0) throw std::runtime_error("oracle dgesvd failed");
}

// qr / lq (alps/matrix/algorithms.hpp:259-325: geqrf + orgqr, gelqf + orglq) restated as the
// unblocked Householder method of geqr2 / org2r, with one rule added on both the oracle's and the
// device's side: a column whose remaining part is below 64 eps |A|_F (rounding noise, e.g. every
// column after the first of a rank-1 block) is set to exactly zero and gets no reflector.  The
// orthonormal completion of Q is then H_0 ... H_{k-1} applied to unit vectors, fixed by the
// arithmetic instead of by rounding noise (LAPACK's completion of a rank-deficient block differs
// between implementations, so the reference itself is not reproducible there).
namespace {
// Householder QR of F (m x n, column-major, in place): R above, reflectors below the diagonal, tau
void householder(Mat& F, std::vector<double>& tau) {
    const std::size_t m = F.r, n = F.c, k = std::min(m, n);
    double fro = 0.0;
    for (double x : F.d) fro += x * x;
    const double thr = 64.0 * 2.220446049250313e-16 * std::sqrt(fro);
    tau.assign(k, 0.0);
    for (std::size_t j = 0; j < k; ++j) {
        double s = 0.0;
        for (std::size_t i = j + 1; i < m; ++i) s += F(i, j) * F(i, j);
        const double alpha = F(j, j), xnorm = std::sqrt(s);
        if (std::hypot(alpha, xnorm) <= thr) {
            for (std::size_t i = j; i < m; ++i) F(i, j) = 0.0;
            continue;
        }
        if (xnorm == 0.0) continue;
        const double beta = -std::copysign(std::hypot(alpha, xnorm), alpha);
        const double t = (beta - alpha) / beta, sc = 1.0 / (alpha - beta);
        for (std::size_t i = j + 1; i < m; ++i) F(i, j) *= sc;
        F(j, j) = beta;
        tau[j] = t;
        for (std::size_t c = j + 1; c < n; ++c) {
            double d = F(j, c);
            for (std::size_t i = j + 1; i < m; ++i) d += F(i, j) * F(i, c);
            d *= t;
            F(j, c) -= d;
            for (std::size_t i = j + 1; i < m; ++i) F(i, c) -= d * F(i, j);
        }
    }
}
// Q (m x k) = H_0 ... H_{k-1} I(:, 0:k)
Mat householder_q(const Mat& F, const std::vector<double>& tau) {
    const std::size_t m = F.r, k = tau.size();
    Mat Q(m, k);
    for (std::size_t c = 0; c < k; ++c) Q(c, c) = 1.0;
    for (std::size_t jj = k; jj-- > 0;) {
        if (tau[jj] == 0.0) continue;
        for (std::size_t c = jj; c < k; ++c) {
            double d = Q(jj, c);
            for (std::size_t i = jj + 1; i < m; ++i) d += F(i, jj) * Q(i, c);
            d *= tau[jj];
            Q(jj, c) -= d;
            for (std::size_t i = jj + 1; i < m; ++i) Q(i, c) -= d * F(i, jj);
        }
    }
    return Q;
}
}  // namespace

void qr(const Mat& A0, Mat& Qm, Mat& R) {
    const std::size_t m = A0.r, n = A0.c, k = std::min(m, n);
    Mat F = A0;
    std::vector<double> tau;
    householder(F, tau);
    R = Mat(k, n);
    for (std::size_t j = 0; j < n; ++j)
        for (std::size_t i = 0; i <= std::min(j, k - 1); ++i) R(i, j) = F(i, j);
    Qm = householder_q(F, tau);
}

void lq(const Mat& A0, Mat& Lm, Mat& Qm) {
    const std::size_t m = A0.r, n = A0.c, k = std::min(m, n);
    Mat F(n, m);
    for (std::size_t j = 0; j < n; ++j)
        for (std::size_t i = 0; i < m; ++i) F(j, i) = A0(i, j);
    std::vector<double> tau;
    householder(F, tau);
    Lm = Mat(m, k);
    for (std::size_t j = 0; j < k; ++j)
        for (std::size_t i = j; i < m; ++i) Lm(i, j) = F(j, i);
    const Mat Qt = householder_q(F, tau);  // n x k
    Qm = Mat(k, n);
    for (std::size_t j = 0; j < n; ++j)
        for (std::size_t i = 0; i < k; ++i) Qm(i, j) = Qt(j, i);
}

// ietl/jacobi.h:476-516
void dsyevx_lowest(const double* M, int ldm, int dim, double abstol, double& w, std::vector<double>& z) {
    std::vector<double> A(std::size_t(dim) * dim, 0.0);
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j <= i; ++j) A[j + std::size_t(i) * dim] = M[j + std::size_t(i) * ldm];
    char jobz = 'V', range = 'I', uplo = 'U';
    int n = dim, lda = dim, il = 1, iu = 1, m = 0, ldz = dim, lwork = 8 * dim, info = 0;
    double vl = 0, vu = 0;
    std::vector<double> wv(dim), zv(dim), work(lwork);
    std::vector<int> iwork(5 * dim), ifail(dim);
    p_dsyevx(&jobz, &range, &uplo, &n, A.data(), &lda, &vl, &vu, &il, &iu, &abstol, &m, wv.data(), zv.data(), &ldz,
             work.data(), &lwork, iwork.data(), ifail.data(), &info);
    if (info != 0) throw std::runtime_error("oracle dsyevx failed");
    w = wv[0];
    z.assign(zv.begin(), zv.begin() + dim);
}

void heev_desc(const Mat& M0, Mat& evecs, std::vector<double>& evals) {
    const int n = int(M0.r);
    evals.assign(n, 0.0);
    evecs = Mat(n, n);
    if (n == 0) return;
    Mat A = M0;
    char jobz = 'V', uplo = 'L';
    int lwork = -1, liwork = -1, info = 0, iwq = 0;
    double wq = 0;
    std::vector<double> w(n);
    p_dsyevd(&jobz, &uplo, &n, A.d.data(), &n, w.data(), &wq, &lwork, &iwq, &liwork, &info);
    lwork = std::max(1, int(wq));
    liwork = std::max(1, iwq);
    std::vector<double> work(lwork);
    std::vector<int> iwork(liwork);
    p_dsyevd(&jobz, &uplo, &n, A.d.data(), &n, w.data(), work.data(), &lwork, iwork.data(), &liwork, &info);
    if (info != 0) throw std::runtime_error("oracle dsyevd failed");
    for (int c = 0; c < n; ++c) {
        evals[c] = w[n - 1 - c];
        for (int i = 0; i < n; ++i) evecs(i, c) = A(i, n - 1 - c);
    }
}

}  // namespace orc
