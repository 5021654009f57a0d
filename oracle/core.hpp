// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement (plain C++17, FP64, column-major) of the QCMaquis two-site
// DMRG effective-Hamiltonian path, written to check the B200 product and to
// serve as the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline / --impl reference legs may call it; the product
// never links or executes anything under oracle/.
//
// Every function names the reference code it restates (paths relative to
// the QCMaquis tree's dmrg/ directory).  Parity is pinned by exact
// diagonalisation (oracle/fci.py) and by the reference's own two-site TwoU1
// golden energy (regression/applications/dmrg/test_fermiladder_ts.py:65).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

namespace orc {

// ---- symmetry: TwoU1 charges (block_matrix/symmetry/nu1_tpl.h) -------------
struct Q {
    int n[2] = {0, 0};
    Q() = default;
    Q(int a, int b) { n[0] = a; n[1] = b; }
};
inline Q operator+(Q x, Q y) { return Q(x.n[0] + y.n[0], x.n[1] + y.n[1]); }
inline Q operator-(Q x) { return Q(-x.n[0], -x.n[1]); }
inline bool operator==(Q x, Q y) { return x.n[0] == y.n[0] && x.n[1] == y.n[1]; }
inline bool operator!=(Q x, Q y) { return !(x == y); }
inline bool operator<(Q x, Q y) { return x.n[0] < y.n[0] || (x.n[0] == y.n[0] && x.n[1] < y.n[1]); }
inline bool operator>(Q x, Q y) { return y < x; }
inline int particleNumber(Q x) { return x.n[0] + x.n[1]; }

// ---- Index (block_matrix/indexing_stable.hpp:97-...) -------------------------
struct Index {
    std::vector<std::pair<Q, std::size_t>> v;  // sorted by descending charge
    std::size_t size() const { return v.size(); }
    const std::pair<Q, std::size_t>& operator[](std::size_t i) const { return v[i]; }
    std::pair<Q, std::size_t>& operator[](std::size_t i) { return v[i]; }
    std::size_t position(Q c) const {
        for (std::size_t i = 0; i < v.size(); ++i) if (v[i].first == c) return i;
        return v.size();
    }
    bool has(Q c) const { return position(c) < v.size(); }
    std::size_t size_of_block(Q c) const { std::size_t p = position(c); return p < v.size() ? v[p].second : 0; }
    void insert(Q c, std::size_t s) {
        std::size_t d = 0;
        while (d < v.size() && !(v[d].first < c)) ++d;
        v.insert(v.begin() + d, {c, s});
    }
    void sort() { std::stable_sort(v.begin(), v.end(), [](auto& a, auto& b) { return a.first > b.first; }); }
    std::size_t sum_of_sizes() const { std::size_t s = 0; for (auto& e : v) s += e.second; return s; }
    std::vector<std::size_t> sizes() const { std::vector<std::size_t> r; for (auto& e : v) r.push_back(e.second); return r; }
};
Index operator*(const Index& a, const Index& b);  // indexing_stable.hpp:434-451
Index adjoin(const Index& a);                     // indexing_stable.hpp adjoin()
void common_subset(Index& a, Index& b);           // indexing.h common_subset()

struct ProductBasis {  // indexing_stable.hpp:310-360
    std::map<std::pair<std::pair<int, int>, std::pair<int, int>>, std::size_t> kv;
    std::map<std::pair<int, int>, std::size_t> sz;
    ProductBasis() = default;
    ProductBasis(const Index& a, const Index& b, bool neg_first = false);
    std::size_t operator()(Q a, Q b) const;
    std::size_t size(Q pc) const { auto it = sz.find({pc.n[0], pc.n[1]}); return it == sz.end() ? 0 : it->second; }
};

// ---- dense column-major blocks and block matrices ---------------------------
struct Mat {
    std::size_t r = 0, c = 0;
    std::vector<double> d;
    Mat() = default;
    Mat(std::size_t r_, std::size_t c_, double v = 0.0) : r(r_), c(c_), d(r_ * c_, v) {}
    double& operator()(std::size_t i, std::size_t j) { return d[i + j * r]; }
    double operator()(std::size_t i, std::size_t j) const { return d[i + j * r]; }
};

struct BlockMatrix {  // block_matrix/block_matrix.h:52-172 (blocks with left/right charges)
    std::vector<Q> lc, rc;
    std::vector<Mat> b;
    std::size_t n_blocks() const { return b.size(); }
    std::size_t find(Q l, Q r) const {
        for (std::size_t k = 0; k < b.size(); ++k) if (lc[k] == l && rc[k] == r) return k;
        return b.size();
    }
    std::size_t find_left(Q l) const {
        for (std::size_t k = 0; k < b.size(); ++k) if (lc[k] == l) return k;
        return b.size();
    }
    std::size_t insert(Q l, Q r, Mat m);  // keeps blocks sorted by descending (left charge)
    Index left_basis() const;
    Index right_basis() const;
    double norm2() const { double s = 0; for (auto& m : b) for (double x : m.d) s += x * x; return s; }
};

// ---- MPS tensor (mp_tensors/mpstensor.h/.hpp) -------------------------------
enum Pairing { LeftPaired, RightPaired };
struct MPSTensor {
    Index phys, left, right;
    Pairing pairing = LeftPaired;
    BlockMatrix data;
    void make_left_paired();    // mp_tensors/reshapes.h reshape_right_to_left_new
    void make_right_paired();   // mp_tensors/reshapes.h reshape_left_to_right_new
    double norm() const { return std::sqrt(data.norm2()); }
    void scale(double f) { for (auto& m : data.b) for (auto& x : m.d) x *= f; }
};

// ---- MPO tensor (mp_tensors/mpotensor.h, mpotensor_detail.h) ----------------
struct OpBlock {  // one block of a SparseOperator (block_matrix/sparse_operator.h)
    std::size_t in_sec, out_sec;         // phys sector positions (left = in, right = out)
    std::vector<unsigned> ss1, ss2;      // row (in) / col (out) sub-indices
    std::vector<double> coeff;
};
struct SiteOp { std::vector<OpBlock> blocks; };
struct MPOTensor {
    unsigned rows = 1, cols = 1;
    Index phys;
    std::vector<unsigned> b1, b2, op;
    std::vector<double> scale;
    std::vector<SiteOp> ops;
    std::vector<std::vector<unsigned>> row_b2;       // row(b1): increasing distinct b2
    std::vector<std::vector<unsigned>> col_b1;       // column(b2): increasing distinct b1
    std::map<std::pair<unsigned, unsigned>, std::vector<unsigned>> at;  // (b1,b2) -> entries
    std::vector<int> herm_left, phase_left, herm_right, phase_right;
    // Hermitian::skip (mpotensor_detail.h:147-156)
    static bool skip(const std::vector<int>& herm, unsigned b, Q l, Q r) { return (l < r) && herm[b] >= 0; }
};
std::vector<MPOTensor> load_mpo_blob(const uint8_t* p, std::size_t n, bool& twosite);

// ---- boundary (mp_tensors/boundary.h:76-406, boundary_index_rt.hpp) --------
struct BoundaryIndex {
    Index bra, ket;
    std::vector<std::vector<unsigned>> lbrb;  // [bra pos][ket pos] -> ci or UINT_MAX
    std::vector<std::vector<long>> offsets;
    std::vector<std::vector<double>> cscale;
    std::vector<std::vector<char>> trans;
    std::vector<char> tr_;
    std::vector<std::size_t> lsz, rsz;
    std::vector<unsigned> nb;
    BoundaryIndex() = default;
    BoundaryIndex(const Index& b, const Index& k)
        : bra(b), ket(k), lbrb(b.size(), std::vector<unsigned>(k.size(), std::numeric_limits<unsigned>::max())) {}
    unsigned n_cohorts() const { return unsigned(offsets.size()); }
    long offset(unsigned ci, unsigned b) const { return offsets[ci][b]; }
    bool has_block(unsigned ci, unsigned b) const { return ci < n_cohorts() && offsets[ci][b] > -1; }
    double conjugate_scale(unsigned ci, unsigned b) const { return cscale[ci][b]; }
    bool tr(unsigned ci) const { return tr_[ci]; }
    std::size_t left_size(unsigned ci) const { return lsz[ci]; }
    std::size_t right_size(unsigned ci) const { return rsz[ci]; }
    std::size_t n_blocks(unsigned ci) const { return nb[ci]; }
    std::size_t block_size(unsigned ci) const { return lsz[ci] * rsz[ci]; }
    std::size_t cohort_size(unsigned ci) const { return nb[ci] * block_size(ci); }
    unsigned cohort_index_pos(std::size_t lb, std::size_t rb) const {
        if (lb < lbrb.size() && rb < ket.size() && lbrb[lb][rb] != std::numeric_limits<unsigned>::max()) return lbrb[lb][rb];
        return n_cohorts();
    }
    unsigned cohort_index(Q lc, Q rc) const { return cohort_index_pos(bra.position(lc), ket.position(rc)); }
    unsigned add_cohort(std::size_t lb, std::size_t rb, const std::vector<long>& off);
    void complement_transpose(const std::vector<int>& herm, const std::vector<int>& phase, bool forward);
};

struct Boundary {
    BoundaryIndex index;
    std::vector<std::vector<double>> data;  // per cohort
    void allocate_all() { data.resize(index.n_cohorts()); for (unsigned c = 0; c < index.n_cohorts(); ++c) data[c].assign(index.cohort_size(c), 0.0); }
};
// trivial boundaries (boundary.h:257-283, mps.hpp left_boundary/right_boundary)
Boundary trivial_boundary(const Index& idx, std::size_t aux_dim);

// ---- BLAS / LAPACK (scipy-bundled OpenBLAS, loaded at run time) -------------
bool blas_init(const char* path, std::string& err);
void dgemm(char ta, char tb, int m, int n, int k, double alpha, const double* A, int lda,
           const double* B, int ldb, double beta, double* C, int ldc);
void daxpy(std::size_t n, double a, const double* x, double* y);
// thin SVD of an m x n block: U (m x k), S (k), VT (k x n), k = min(m, n)
void dgesvd_thin(const Mat& A, Mat& U, std::vector<double>& S, Mat& VT);
// QR (geqrf + orgqr): Q m x k, R k x n
void qr(const Mat& A, Mat& Q, Mat& R);
// LQ (gelqf + orglq): L m x k, Q k x n
void lq(const Mat& A, Mat& L, Mat& Qm);
// lowest eigenpair of the leading dim x dim upper triangle of M (ld = ldm), dsyevx range 'I'
void dsyevx_lowest(const double* M, int ldm, int dim, double abstol, double& w, std::vector<double>& z);
// alps/matrix/algorithms.hpp:374-396 (heevd 'V', then reversed to descending order)
void heev_desc(const Mat& M, Mat& evecs, std::vector<double>& evals);

}  // namespace orc
