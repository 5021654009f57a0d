// Dense per-block factorizations on the device (see linalg.hpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "linalg.hpp"

#define QCM_SOLVER(call)                                                                                   \
    do {                                                                                                   \
        cusolverStatus_t st_ = (call);                                                                     \
        if (st_ != CUSOLVER_STATUS_SUCCESS)                                                                \
            throw qcm::cuda_error(std::string(#call) + ": cuSOLVER status " + std::to_string(int(st_)));   \
    } while (0)

namespace qcm {
namespace {

constexpr uint32_t INFO_CAP = 4096;

}  // namespace

Solver::Solver() {
    QCM_SOLVER(cusolverDnCreate(&h));
    QCM_SOLVER(cusolverDnCreateGesvdjInfo(&svdp));
    QCM_SOLVER(cusolverDnXgesvdjSetMaxSweeps(svdp, 100));
    QCM_SOLVER(cusolverDnXgesvdjSetSortEig(svdp, 1));
    info.alloc(INFO_CAP);
    QCM_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
    for (Lane& L : lane) {
        QCM_CUDA(cudaStreamCreateWithFlags(&L.s, cudaStreamNonBlocking));
        register_stream(L.s);
        QCM_CUDA(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
        QCM_SOLVER(cusolverDnCreate(&L.h));
        QCM_SOLVER(cusolverDnSetStream(L.h, L.s));
        QCM_SOLVER(cusolverDnCreateGesvdjInfo(&L.svdp));
        QCM_SOLVER(cusolverDnXgesvdjSetMaxSweeps(L.svdp, 100));
        QCM_SOLVER(cusolverDnXgesvdjSetSortEig(L.svdp, 1));
    }
}

Solver::~Solver() {
    for (Lane& L : lane) {
        if (L.s) cudaStreamSynchronize(L.s);
        L.a.reset();
        L.work.reset();
        if (L.s) {
            cudaStreamSynchronize(L.s);
            retire_stream(L.s);
        }
        if (L.svdp) cusolverDnDestroyGesvdjInfo(L.svdp);
        if (L.h) cusolverDnDestroy(L.h);
        if (L.done) cudaEventDestroy(L.done);
        if (L.s) cudaStreamDestroy(L.s);
    }
    if (fork_ev) cudaEventDestroy(fork_ev);
    if (svdp) cusolverDnDestroyGesvdjInfo(svdp);
    if (h) cusolverDnDestroy(h);
}

void Solver::fork(cudaStream_t s) {
    QCM_CUDA(cudaEventRecord(fork_ev, s));
    for (Lane& L : lane) QCM_CUDA(cudaStreamWaitEvent(L.s, fork_ev, 0));
}

int* Solver::reserve_info(uint32_t n, cudaStream_t s) {
    if (n > INFO_CAP) throw std::runtime_error("too many factorizations in one batch");
    if (n_info + n > INFO_CAP) check(s);
    int* p = info.get() + n_info;
    n_info += n;
    return p;
}

void Solver::join(cudaStream_t s) {
    for (Lane& L : lane) {
        QCM_CUDA(cudaEventRecord(L.done, L.s));
        QCM_CUDA(cudaStreamWaitEvent(s, L.done, 0));
    }
}

void Solver::bind(cudaStream_t s) { QCM_SOLVER(cusolverDnSetStream(h, s)); }

void Solver::check(cudaStream_t s) {
    if (!n_info) return;
    std::vector<int> hi(n_info);
    QCM_CUDA(cudaMemcpyAsync(hi.data(), info.get(), n_info * sizeof(int), cudaMemcpyDeviceToHost, s));
    QCM_CUDA(cudaStreamSynchronize(s));
    n_info = 0;
    for (int v : hi)
        if (v != 0) throw std::runtime_error("device factorization failed (info " + std::to_string(v) + ")");
}

void svd_thin_lane(Solver& sv, int l, const double* A, int m, int n, double* U, double* S, double* V, int* info) {
    if (m == 0 || n == 0) return;
    Solver::Lane& L = sv.lane[l];
    AllocStream scope(L.s);  // a lane's buffers are ordered on the lane's stream
    if (L.a.size() < std::size_t(m) * n) L.a.alloc(std::size_t(m) * n);
    QCM_CUDA(cudaMemcpyAsync(L.a.get(), A, std::size_t(m) * n * sizeof(double), cudaMemcpyDeviceToDevice, L.s));
    int lwork = 0;
    QCM_SOLVER(cusolverDnDgesvdj_bufferSize(L.h, CUSOLVER_EIG_MODE_VECTOR, 1, m, n, L.a.get(), m, S, U, m, V, n, &lwork,
                                            L.svdp));
    if (L.work.size() < std::size_t(lwork)) L.work.alloc(std::size_t(lwork));
    QCM_SOLVER(cusolverDnDgesvdj(L.h, CUSOLVER_EIG_MODE_VECTOR, 1, m, n, L.a.get(), m, S, U, m, V, n, L.work.get(), lwork,
                                 info, L.svdp));
}

// ---------------------------------------------------------------------------
// One-sided Jacobi SVD (Hestenes).  G (r x c, ld r) is A when m >= n and A^T otherwise; its
// columns are rotated pairwise until mutually orthogonal, and the rotations accumulate in Q
// (c x c, ld c, starting at I).  Then G = Vg diag(sigma) with sigma_j = |G_j|, and
// A = G Q^T (m >= n: U = G / sigma, V = Q) or A^T = G Q^T (m < n: U = Q, V = G / sigma).
// Column pairs follow the circle (round-robin) ordering, c' - 1 rounds of c'/2 disjoint
// pairs per sweep (c' = c rounded up to even, pairs with the padding column skipped); a
// half-warp takes a pair: gamma = G_p . G_q with alpha = |G_p|^2, beta = |G_q|^2 tracked in
// shared memory (recomputed at the start of every sweep, updated exactly by alpha -= t gamma,
// beta += t gamma after a rotation), and if |gamma| > r eps sqrt(alpha beta) (the rounding
// level of a length-r dot product) the rotation with t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)),
// zeta = (beta - alpha) / (2 gamma), c = rsqrt(1 + t^2), s = c t makes them orthogonal.
// Sweeps end when one performs no rotation (at most JMAX_SWEEPS).
namespace {
constexpr int JTHR = 1024;
constexpr int JMAX_SWEEPS = 40;
constexpr double JEPS = 2.220446049250313e-16;  // unit roundoff of double
constexpr uint32_t JSMEM_DOUBLES = 27000;  // dynamic shared memory (with the 12 KiB static part, under 227 KiB)

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// sum over each aligned group of gs lanes (gs = 8 or 16; all 32 lanes call it)
__device__ __forceinline__ double group_sum(double v, uint32_t gs) {
    for (uint32_t o = gs >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, int(o));
    return v;
}

__global__ void __launch_bounds__(JTHR) k_jacobi_svd(const SvdJob* __restrict__ jobs, const double* __restrict__ A,
                                                     double* __restrict__ U, double* __restrict__ S, double* __restrict__ V,
                                                     double* __restrict__ Wg, uint32_t smem_doubles,
                                                     int* __restrict__ zero_count, int* __restrict__ sweeps_used) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int rotated;
    __shared__ uint32_t rank_of[1024];
    __shared__ double nrm[1024];
    const SvdJob J = jobs[blockIdx.x];
    const bool tall = J.m >= J.n;
    const uint32_t r = tall ? J.m : J.n, c = tall ? J.n : J.m;
    // work matrix G (r x c) and rotations Q (c x c), columns padded to an even length (a zero row, which
    // rotations keep zero) so that every column starts on 16 bytes and is read and written two
    // elements at a time: both in the launch's shared memory when they fit, else G there and Q in the
    // block's global scratch (L2-resident), else both in the scratch
    const uint32_t rp = r + (r & 1u), cq = c + (c & 1u);
    const uint64_t rc = uint64_t(rp) * c;
    double* G;
    double* Q;
    if (rc + uint64_t(cq) * c <= smem_doubles) { G = smem; Q = smem + rc; }
    else if (rc <= smem_doubles) { G = smem; Q = Wg + J.w_off + rc; }
    else { G = Wg + J.w_off; Q = G + rc; }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = JTHR / 32;
    // G = A or A^T, Q = I
    const double* a = A + J.a_off;
    for (uint64_t i = tid; i < uint64_t(rp) * c; i += JTHR) {
        const uint32_t row = uint32_t(i % rp), col = uint32_t(i / rp);
        G[i] = row >= r ? 0.0 : (tall ? a[row + uint64_t(col) * J.m] : a[col + uint64_t(row) * J.m]);
    }
    for (uint64_t i = tid; i < uint64_t(cq) * c; i += JTHR) Q[i] = (i % cq == i / cq) ? 1.0 : 0.0;
    __syncthreads();
    const uint32_t cp = c + (c & 1u);  // players, padded to even
    const double tol2 = (JEPS * double(r)) * (JEPS * double(r));
    // lanes per pair: a round costs about the larger of the CTA's instructions over its four
    // schedulers and one lane group's dependent chain; each active warp pays the fixed part of a pair
    // (indices, reduction, rotation angle: about JFIX instructions) once per pair it holds, and every
    // lane JELEM instructions per element pair of its share of the two columns (dot product, G and Q
    // rotations).  Fewer lanes per pair spread the fixed part over more pairs per warp; more lanes
    // shorten the chain when the columns are long or the pairs few.
    const uint32_t gs = cp / 2 > uint32_t(JTHR / 16) ? 8u : 16u;
    const uint32_t grp = uint32_t(tid) / gs, hl = uint32_t(tid) % gs, ngrp = JTHR / gs;
    for (int sweep = 0; sweep < JMAX_SWEEPS && c > 1; ++sweep) {
        if (tid == 0) rotated = 0;
        for (uint32_t j = warp; j < c; j += nwarp) {
            const double* g = G + uint64_t(j) * rp;
            double x = 0.0;
            for (uint32_t i = lane; i < r; i += 32) x = fma(g[i], g[i], x);
            x = warp_sum(x);
            if (lane == 0) nrm[j] = x;
        }
        __syncthreads();
        const uint32_t rh = rp / 2, ch = cq / 2;  // column lengths in element pairs
        for (uint32_t k = 0; k + 1 < cp; ++k) {
            // one pair per lane group; every lane runs the same number of passes so the group
            // shuffles never diverge
            for (uint32_t pass = 0; pass * ngrp < cp / 2; ++pass) {
                const uint32_t t = pass * ngrp + grp;
                const uint32_t i0 = t, i1 = cp - 1 - t;
                uint32_t p = 0, q = 0;
                bool act = t < cp / 2;
                if (act) {
                    // (i - 1 + k) mod (cp - 1) + 1 with i - 1 + k < 2 (cp - 1)
                    uint32_t xp = i0 - 1 + k, xq = i1 - 1 + k;
                    xp -= xp >= cp - 1 ? cp - 1 : 0u;
                    xq -= xq >= cp - 1 ? cp - 1 : 0u;
                    p = i0 == 0 ? 0 : xp + 1;
                    q = i1 == 0 ? 0 : xq + 1;
                    act = p < c && q < c;
                }
                double2* gp = reinterpret_cast<double2*>(G + uint64_t(p) * rp);
                double2* gq = reinterpret_cast<double2*>(G + uint64_t(q) * rp);
                double ga = 0.0;
                if (act)
                    for (uint32_t i = hl; i < rh; i += gs) {
                        const double2 x = gp[i], y = gq[i];
                        ga = fma(x.x, y.x, ga);
                        ga = fma(x.y, y.y, ga);
                    }
                ga = group_sum(ga, gs);
                const double al = act ? nrm[p] : 0.0, be = act ? nrm[q] : 0.0;
                const bool rot = act && ga * ga > tol2 * (al * be);
                if (rot) {
                    // t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = d / h, d = beta - alpha, h = 2 gamma,
                    // multiplied through by |h| (one square root and one division) unless d^2 + h^2 could
                    // overflow
                    const double d = be - al, h = 2.0 * ga;
                    double tt;
                    if (fabs(d) < 1e150 && fabs(h) < 1e150) {
                        tt = (d >= 0.0 ? h : -h) / (fabs(d) + sqrt(fma(d, d, h * h)));
                    } else {
                        const double zeta = d / h;
                        tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    }
                    const double cs = rsqrt(1.0 + tt * tt), sn = cs * tt;
                    for (uint32_t i = hl; i < rh; i += gs) {
                        const double2 x = gp[i], y = gq[i];
                        gp[i] = make_double2(cs * x.x - sn * y.x, cs * x.y - sn * y.y);
                        gq[i] = make_double2(sn * x.x + cs * y.x, sn * x.y + cs * y.y);
                    }
                    double2* qp = reinterpret_cast<double2*>(Q + uint64_t(p) * cq);
                    double2* qq = reinterpret_cast<double2*>(Q + uint64_t(q) * cq);
                    for (uint32_t i = hl; i < ch; i += gs) {
                        const double2 x = qp[i], y = qq[i];
                        qp[i] = make_double2(cs * x.x - sn * y.x, cs * x.y - sn * y.y);
                        qq[i] = make_double2(sn * x.x + cs * y.x, sn * x.y + cs * y.y);
                    }
                    if (hl == 0) {
                        nrm[p] = al - tt * ga;
                        nrm[q] = be + tt * ga;
                        rotated = 1;
                    }
                }
                __syncwarp();
            }
            __syncthreads();
        }
        const int any = rotated;
        __syncthreads();
        if (sweeps_used && tid == 0) sweeps_used[J.id] = sweep + 1;
        if (!any) break;
    }
    // sigma_j = |G_j| into S (unsorted, temporarily), then ranks by descending sigma (ties by index)
    double* sv = S + J.s_off;
    for (uint32_t j = warp; j < c; j += nwarp) {
        const double* g = G + uint64_t(j) * rp;
        double x = 0.0;
        for (uint32_t i = lane; i < r; i += 32) x = fma(g[i], g[i], x);
        x = warp_sum(x);
        if (lane == 0) sv[j] = sqrt(x);
    }
    __syncthreads();
    for (uint32_t j = tid; j < c; j += JTHR) {
        const double x = sv[j];
        uint32_t rk = 0;
        for (uint32_t i = 0; i < c; ++i) {
            const double y = sv[i];
            rk += (y > x || (y == x && i < j)) ? 1u : 0u;
        }
        rank_of[j] = rk;
    }
    __syncthreads();
    // outputs in sorted order: the normalised G columns and Q's columns
    double* Gout = tall ? U + J.u_off : V + J.v_off;   // r x c, ld r
    double* Qout = tall ? V + J.v_off : U + J.u_off;   // c x c, ld c
    for (uint64_t i = tid; i < uint64_t(r) * c; i += JTHR) {
        const uint32_t row = uint32_t(i % r), col = uint32_t(i / r);
        const double sg = sv[col];
        Gout[row + uint64_t(rank_of[col]) * r] = sg > 0.0 ? G[row + uint64_t(col) * rp] / sg : 0.0;
    }
    for (uint64_t i = tid; i < uint64_t(c) * c; i += JTHR) {
        const uint32_t row = uint32_t(i % c), col = uint32_t(i / c);
        Qout[row + uint64_t(rank_of[col]) * c] = Q[row + uint64_t(col) * cq];
    }
    __syncthreads();
    // sigma in sorted order (through the scratch column space, G is no longer needed)
    for (uint32_t j = tid; j < c; j += JTHR) G[rank_of[j]] = sv[j];
    __syncthreads();
    int zeros = 0;
    for (uint32_t j = tid; j < c; j += JTHR) {
        sv[j] = G[j];
        zeros += G[j] == 0.0 ? 1 : 0;
    }
    if (zeros) atomicAdd(zero_count + J.id, zeros);
}
}  // namespace

void syevd_lane(Solver& sv, int l, double* A, int n, double* W, int* info) {
    if (n == 0) return;
    Solver::Lane& L = sv.lane[l];
    AllocStream scope(L.s);
    int lwork = 0;
    QCM_SOLVER(cusolverDnDsyevd_bufferSize(L.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A, n, W, &lwork));
    if (L.work.size() < std::size_t(lwork)) L.work.alloc(std::size_t(lwork));
    QCM_SOLVER(cusolverDnDsyevd(L.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A, n, W, L.work.get(), lwork, info));
}

uint64_t jacobi_svd_smem_doubles() { return JSMEM_DOUBLES; }

uint64_t jacobi_svd_scratch(uint32_t m, uint32_t n) {
    const uint64_t r = std::max(m, n), c = std::min(m, n);
    const uint64_t d = (r + (r & 1)) * c + (c + (c & 1)) * c;  // the padded columns
    return (d + 31) / 32 * 32;  // whole multiples of 32 doubles: the next block's scratch stays 16-byte aligned
}

void batched_jacobi_svd(const std::vector<SvdJob>& jobs, const double* A, uint64_t a_len, double* U, uint64_t u_len, double* S,
                        uint64_t s_len, double* V, uint64_t v_len, double* W, uint64_t w_len, int* zero_count,
                        DBuf<SvdJob>& jobbuf, cudaStream_t s, int* sweeps_used) {
    // one launch for the blocks whose work matrix G fits in shared memory (their rotations Q too where
    // they fit), one with both in the global scratch for the rest
    std::vector<SvdJob> small, large;
    for (const SvdJob& j : jobs) {
        const uint64_t k = std::min(j.m, j.n);
        if (!j.m || !j.n) continue;
        if (k > 1024) throw std::runtime_error("batched_jacobi_svd: block larger than 1024 in both dimensions");
        if (j.a_off + uint64_t(j.m) * j.n > a_len || j.u_off + uint64_t(j.m) * k > u_len || j.s_off + k > s_len ||
            j.v_off + uint64_t(j.n) * k > v_len || j.w_off + jacobi_svd_scratch(j.m, j.n) > w_len)
            throw std::runtime_error("batched_jacobi_svd: block outside its buffers");
        if (j.w_off % 2) throw std::runtime_error("batched_jacobi_svd: scratch offset not 16-byte aligned");
        // the blocks working in global memory first: they take longest
        if (std::max(j.m, j.n) * uint64_t(k) <= JSMEM_DOUBLES) small.push_back(j);
        else large.push_back(j);
    }
    uint32_t nid = 0;
    for (const SvdJob& j : jobs) nid = std::max(nid, j.id + 1);
    if (nid) QCM_CUDA(cudaMemsetAsync(zero_count, 0, nid * sizeof(int), s));
    std::vector<SvdJob> all(large);
    all.insert(all.end(), small.begin(), small.end());
    if (all.empty()) return;
    jobbuf.upload(all, s);
    // one launch: each CTA places its work matrix and rotations by its own size (one CTA per SM
    // in either case, at 1024 threads)
    const std::size_t bytes = std::size_t(JSMEM_DOUBLES) * sizeof(double);
    QCM_CUDA(cudaFuncSetAttribute(k_jacobi_svd, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    k_jacobi_svd<<<unsigned(all.size()), JTHR, bytes, s>>>(jobbuf.get(), A, U, S, V, W, JSMEM_DOUBLES, zero_count,
                                                           sweeps_used);
    QCM_CUDA(cudaGetLastError());
}

void sym_lowest_eigenpair(const double* M, int ldm, int n, double& w, std::vector<double>& z) {
    std::vector<double> A(std::size_t(n) * n), V(std::size_t(n) * n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) A[i + std::size_t(j) * n] = A[j + std::size_t(i) * n] = M[i + std::size_t(j) * ldm];
    for (int i = 0; i < n; ++i) V[i + std::size_t(i) * n] = 1.0;
    auto a = [&](int i, int j) -> double& { return A[i + std::size_t(j) * n]; };
    // cyclic Jacobi (Golub & Van Loan, Algorithm 8.5.3) until the off-diagonal part is negligible
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) { tot += a(i, j) * a(i, j); if (i != j) off += a(i, j) * a(i, j); }
        if (off <= 1e-32 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = a(p, q);
                if (apq == 0.0) continue;
                double tau = (a(q, q) - a(p, p)) / (2.0 * apq);
                double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
                double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {  // A <- A J
                    double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // A <- J^T A
                    double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {  // V <- V J
                    double vkp = V[k + std::size_t(p) * n], vkq = V[k + std::size_t(q) * n];
                    V[k + std::size_t(p) * n] = c * vkp - s * vkq;
                    V[k + std::size_t(q) * n] = s * vkp + c * vkq;
                }
            }
    }
    int best = 0;
    for (int i = 1; i < n; ++i) if (a(i, i) < a(best, best)) best = i;
    w = a(best, best);
    z.assign(V.begin() + std::size_t(best) * n, V.begin() + std::size_t(best + 1) * n);
}

}  // namespace qcm
