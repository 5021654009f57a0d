// Dense per-block factorizations on the device, used by the truncation and
// canonisation steps of the sweep:
//   thin SVD   (framework/alps/matrix/algorithms.hpp:243-257, gesvd 'S','S'): one-sided Jacobi,
//              all blocks in one launch (cuSOLVER gesvdj completes a block whose kept singular
//              values include exact zeros)
//   thin QR    (algorithms.hpp:260-291, geqrf + orgqr) and thin LQ (algorithms.hpp:293-325, gelqf
//              + orglq, here QR of the transpose): Householder, all blocks in one launch
//   symmetric eigendecomposition of the density-matrix blocks (algorithms.hpp:374-396, heevd):
//              cuSOLVER syevd on side lanes
// plus the Rayleigh-Ritz eigenproblem of the Jacobi-Davidson solver (host, <= 64 x 64).
#pragma once

#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cstdint>
#include <vector>

#include "device.hpp"

namespace qcm {

struct Solver {
    cusolverDnHandle_t h = nullptr;
    gesvdjInfo_t svdp = nullptr;
    DBuf<int> info;  // one status word per factorization since the last check
    uint32_t n_info = 0;
    // side streams for independent per-block factorizations (fork from / join to a stream)
    static constexpr int LANES = 8;
    struct Lane {
        cudaStream_t s = nullptr;
        cusolverDnHandle_t h = nullptr;
        gesvdjInfo_t svdp = nullptr;
        DBuf<double> a, work;
        cudaEvent_t done = nullptr;
    };
    Lane lane[LANES];
    cudaEvent_t fork_ev = nullptr;
    Solver();
    ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;
    void bind(cudaStream_t s);
    // throws if any factorization since the last call reported a failure (synchronizes s)
    void check(cudaStream_t s);
    // lanes start after the work queued on s so far; s continues after all lanes' work
    void fork(cudaStream_t s);
    void join(cudaStream_t s);
    // n consecutive status words for factorizations issued from several host threads
    int* reserve_info(uint32_t n, cudaStream_t s);
};

// A (m x n, lda = m) is read only.  k = min(m, n).
// U (m x k, ld m), S (k, descending), V (n x k, ld n): A = U diag(S) V^T, by cuSOLVER's gesvdj on side
// lane `l` (between fork and join), status to *info
void svd_thin_lane(Solver& sv, int l, const double* A, int m, int n, double* U, double* S, double* V, int* info);
// Thin SVDs of many small blocks in one launch (one-sided Jacobi, one CTA per block):
// A_j (m x n, ld m) = U_j diag(S_j) V_j^T with U_j (m x k, ld m), S_j descending (k), V_j
// (n x k, ld n), k = min(m, n) -- the layout of gesvdj with econ = 1.  A singular value that
// is exactly zero leaves a zero column in U_j (m >= n) or V_j (m < n); zero_count[id] counts them
// (zero_count has an entry for every id); sweeps_used (optional, same indexing) receives the
// number of Jacobi sweeps each block took.
struct SvdJob {
    uint64_t a_off, u_off, s_off, v_off, w_off;  // w_off: scratch of jacobi_svd_scratch(m, n) doubles
    uint32_t m, n;
    uint32_t id, pad;  // zero_count[id] receives the block's number of zero singular values
};
uint64_t jacobi_svd_scratch(uint32_t m, uint32_t n);
// doubles of the Jacobi kernel's shared-memory work space (blocks larger than it work in L2)
uint64_t jacobi_svd_smem_doubles();
// Symmetric eigendecomposition (divide and conquer, lower triangle) on lane `l`: A (n x n, ld n)
// is overwritten by the eigenvectors, W receives the eigenvalues in ascending order.
// Replaces heevd('V') of alps/matrix/algorithms.hpp:374-396 (which then reverses the order).
void syevd_lane(Solver& sv, int l, double* A, int n, double* W, int* info);
// A, U, S, V, W: base pointers of the offsets in jobs (host list, validated against the lengths)
void batched_jacobi_svd(const std::vector<SvdJob>& jobs, const double* A, uint64_t a_len, double* U, uint64_t u_len, double* S,
                        uint64_t s_len, double* V, uint64_t v_len, double* W, uint64_t w_len, int* zero_count,
                        DBuf<SvdJob>& jobbuf, cudaStream_t s, int* sweeps_used = nullptr);
// Thin QR / LQ of many blocks in one launch (Householder, one CTA per block; qr_batched.cu):
//   lq = 0: A_j (m x n, ld m) = Q_j R_j, Q_j (m x k, ld m), R_j (k x n, ld k);
//   lq = 1: A_j = L_j Q_j, L_j (m x k, ld m) at r_off, Q_j (k x n, ld k) at q_off;
// k = min(m, n); W: scratch of qr_scratch(m, n, lq) doubles per block at w_off.
// flags QR_PIVOT: column pivoting of the factorised matrix F (A, or A^T for an LQ): F P = Q' R' with
//   the column of largest remaining norm taken at every step (ties: the lowest index); perm (at p_off,
//   min(m, n) = the columns of F, which must then be at most 1024) receives column i of F P as perm[i].
// flags QR_RT (lq = 0): R is written transposed, R^T (n x k, ld n).
constexpr uint32_t QR_PIVOT = 1, QR_RT = 2;
// dst[dst_off + perm[p_off + i] + j * ldd] = src[src_off + i + j * n] for i, j < n (rows of an n x n
// block scattered by a permutation), one CTA per job
struct PermJob {
    uint64_t src_off, dst_off, p_off;
    uint32_t n, ldd;
};
void batched_permute_rows(const std::vector<PermJob>& jobs, const double* src, uint64_t src_len, double* dst, uint64_t dst_len,
                          const uint32_t* perm, uint64_t p_len, DBuf<PermJob>& jobbuf, cudaStream_t s);
struct QrJob {
    uint64_t a_off, q_off, r_off, w_off;
    uint32_t m, n, lq, flags;
    uint64_t p_off;
};
uint64_t qr_scratch(uint32_t m, uint32_t n, bool lq);
void batched_qr(const std::vector<QrJob>& jobs, const double* A, uint64_t a_len, double* Q, uint64_t q_len, double* R,
                uint64_t r_len, double* W, uint64_t w_len, DBuf<QrJob>& jobbuf, cudaStream_t s, uint32_t* P = nullptr,
                uint64_t p_len = 0);

// Lowest eigenpair of the symmetric n x n matrix held in the upper triangle of
// M (column-major, leading dimension ldm); cyclic Jacobi rotations, FP64.
// Replaces the dsyevx(range='I', il=iu=1) call of ietl/jacobi.h:476-516.
void sym_lowest_eigenpair(const double* M, int ldm, int n, double& w, std::vector<double>& z);

}  // namespace qcm
