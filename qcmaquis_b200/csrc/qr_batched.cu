// Thin QR and LQ of many blocks in one launch (the canonisation steps of the sweep).
//
// The reference canonises a site tensor block by block with LAPACK: qr / lq
// (framework/alps/matrix/algorithms.hpp:260-325, geqrf + orgqr, gelqf + orglq), called by
// MPSTensor::normalize_left / normalize_right (mp_tensors/mpstensor.hpp:242-300).  Here every
// block of a site tensor is factorised by one CTA of the same launch, with the unblocked Householder
// method LAPACK's geqr2 / org2r define (a published algorithm; Golub & Van Loan, Algorithm 5.2.1):
//   for j < k = min(m, n): alpha = A(j, j), xnorm = |A(j+1:m, j)|;
//     xnorm = 0: tau_j = 0 (H_j = I);
//     else beta = -sign(alpha) hypot(alpha, xnorm), tau_j = (beta - alpha) / beta,
//          v_j = (1, A(j+1:m, j) / (alpha - beta)), A(j, j) = beta;
//     A(j:m, j+1:n) -= tau_j v_j (v_j^T A(j:m, j+1:n));
//   R = the upper triangle (k x n); Q = H_0 ... H_{k-1} applied to the first k columns of I (m x k).
// One rule is added (the oracle's restatement has it too): a column whose remaining part
// |A(j:m, j)| is at most 64 eps |A|_F -- rounding noise, as in every column after the first of a
// rank-1 block -- is set to exactly zero and gets no reflector, so that the orthonormal completion
// of Q is fixed by the arithmetic rather than by that noise (which LAPACK implementations resolve
// differently).
// LQ is the QR of the transpose (the same reflectors as gelqf): L = R'^T, Q = Q'^T.
// The work matrix and the reflectors live in global scratch (L2-resident at these sizes); a warp
// updates one trailing column at a time (its dot product reduced within the warp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

#include "linalg.hpp"

namespace qcm {

namespace {

constexpr int QR_THR = 1024;
constexpr int QR_WARPS = QR_THR / 32;
constexpr uint32_t QR_PIV_MAX = 1024;  // columns of a pivoted factorisation
constexpr uint64_t QR_SMEM_DOUBLES = 27400;  // dynamic shared memory (with the 12.4 KB static part, under 227 KB)

__device__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(QR_THR) k_qr(const QrJob* __restrict__ jobs, const double* __restrict__ A,
                                               double* __restrict__ Q, double* __restrict__ R, double* __restrict__ W,
                                               uint32_t* __restrict__ P, uint32_t smem_doubles) {
    extern __shared__ double qsm[];
    __shared__ double red[QR_WARPS];
    __shared__ uint32_t redi[QR_WARPS];
    __shared__ double sh_tau, sh_scale, sh_thr;
    __shared__ int sh_zero;
    __shared__ uint32_t sh_piv;
    __shared__ double cn[QR_PIV_MAX];
    __shared__ uint32_t perm[QR_PIV_MAX];
    const QrJob J = jobs[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // the matrix factorised: F (mm x nn) = A_j, or A_j^T for an LQ
    const uint32_t mm = J.lq ? J.n : J.m, nn = J.lq ? J.m : J.n, k = mm < nn ? mm : nn;
    const bool pivot = (J.flags & QR_PIVOT) != 0;
    // F, then R above and the reflectors below the diagonal, with the k reflector scales after it: in the
    // launch's shared memory when they fit, else in the block's global scratch (L2-resident)
    const uint64_t fsz = uint64_t(mm) * nn + k;
    double* w = fsz <= smem_doubles ? qsm : W + J.w_off;
    double* taus = w + uint64_t(mm) * nn;
    double* qf = W + J.w_off + fsz;  // Q' (mm x k) for an LQ; the QR writes Q directly
    const double* a = A + J.a_off;
    for (uint64_t e = tid; e < uint64_t(mm) * nn; e += QR_THR) {
        const uint32_t i = uint32_t(e % mm), c = uint32_t(e / mm);
        w[e] = J.lq ? a[c + uint64_t(i) * J.m] : a[i + uint64_t(c) * J.m];
    }
    {
        // the negligible-column threshold 64 eps |A|_F
        double f = 0.0;
        for (uint64_t e = tid; e < uint64_t(J.m) * J.n; e += QR_THR) f = fma(a[e], a[e], f);
        f = warp_sum(f);
        if (lane == 0) red[warp] = f;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int q = 0; q < QR_WARPS; ++q) t += red[q];
            sh_thr = 64.0 * 2.220446049250313e-16 * sqrt(t);
        }
    }
    if (pivot)
        for (uint32_t c = tid; c < nn; c += QR_THR) perm[c] = c;
    __syncthreads();
    for (uint32_t j = 0; j < k; ++j) {
        if (pivot) {
            // the remaining column of largest norm over rows j .. mm-1 (exact norms every step), lowest
            // index on ties, swapped into place
            for (uint32_t c = j + warp; c < nn; c += QR_WARPS) {
                const double* fc = w + uint64_t(c) * mm;
                double x = 0.0;
                for (uint32_t i = j + lane; i < mm; i += 32) x = fma(fc[i], fc[i], x);
                x = warp_sum(x);
                if (lane == 0) cn[c] = x;
            }
            __syncthreads();
            {
                double bv = -1.0;
                uint32_t bi = nn;
                for (uint32_t c = j + tid; c < nn; c += QR_THR)
                    if (cn[c] > bv) { bv = cn[c]; bi = c; }  // c increases: the first maximum is kept
                for (int o = 16; o > 0; o >>= 1) {
                    const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                    const uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
                }
                if (lane == 0) { red[warp] = bv; redi[warp] = bi; }
                __syncthreads();
                if (tid == 0) {
                    double v = red[0];
                    uint32_t b = redi[0];
                    for (int q = 1; q < QR_WARPS; ++q)
                        if (red[q] > v || (red[q] == v && redi[q] < b)) { v = red[q]; b = redi[q]; }
                    sh_piv = b < nn ? b : j;
                }
                __syncthreads();
            }
            const uint32_t pv = sh_piv;
            if (pv != j) {
                double* fa = w + uint64_t(j) * mm;
                double* fb = w + uint64_t(pv) * mm;
                for (uint32_t i = tid; i < mm; i += QR_THR) {
                    const double t = fa[i];
                    fa[i] = fb[i];
                    fb[i] = t;
                }
                if (tid == 0) {
                    const uint32_t t = perm[j];
                    perm[j] = perm[pv];
                    perm[pv] = t;
                }
            }
            __syncthreads();
        }
        double* vj = w + uint64_t(j) * mm;
        double s = 0.0;
        for (uint32_t i = j + 1 + tid; i < mm; i += QR_THR) s = fma(vj[i], vj[i], s);
        s = warp_sum(s);
        if (lane == 0) red[warp] = s;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int q = 0; q < QR_WARPS; ++q) t += red[q];
            const double alpha = vj[j], xnorm = sqrt(t);
            double tau = 0.0, scale = 1.0;
            const int zero = hypot(alpha, xnorm) <= sh_thr;
            if (!zero && xnorm != 0.0) {
                const double beta = -copysign(hypot(alpha, xnorm), alpha);
                tau = (beta - alpha) / beta;
                scale = 1.0 / (alpha - beta);
                vj[j] = beta;
            }
            sh_tau = tau;
            sh_scale = scale;
            sh_zero = zero;
            taus[j] = tau;
        }
        __syncthreads();
        if (sh_zero) {
            // a negligible column: exactly zero in R, no reflector
            for (uint32_t i = j + tid; i < mm; i += QR_THR) vj[i] = 0.0;
            __syncthreads();
            continue;
        }
        const double tau = sh_tau;
        if (tau != 0.0) {
            const double scale = sh_scale;
            for (uint32_t i = j + 1 + tid; i < mm; i += QR_THR) vj[i] *= scale;
            __syncthreads();
            // trailing columns, one warp each: F(j:mm, c) -= tau v (v^T F(j:mm, c)), v_j = 1
            for (uint32_t c = j + 1 + warp; c < nn; c += QR_WARPS) {
                double* fc = w + uint64_t(c) * mm;
                const double fj = fc[j];  // read by every lane before lane 0 writes it
                double d = 0.0;
                for (uint32_t i = j + 1 + lane; i < mm; i += 32) d = fma(vj[i], fc[i], d);
                d = warp_sum(d) + fj;
                d *= tau;
                if (lane == 0) fc[j] -= d;
                for (uint32_t i = j + 1 + lane; i < mm; i += 32) fc[i] = fma(-d, vj[i], fc[i]);
            }
        }
        __syncthreads();
    }
    // R (k x nn, ld k) from the upper triangle; for an LQ, L = R'^T (m x k, ld m)
    double* r = R + J.r_off;
    const bool rt = (J.flags & QR_RT) != 0;
    for (uint64_t e = tid; e < uint64_t(k) * nn; e += QR_THR) {
        const uint32_t i = uint32_t(e % k), c = uint32_t(e / k);
        const double v = i <= c ? w[i + uint64_t(c) * mm] : 0.0;
        if (J.lq) r[c + uint64_t(i) * J.m] = v;
        else if (rt) r[c + uint64_t(i) * nn] = v;
        else r[e] = v;
    }
    if (pivot)
        for (uint32_t c = tid; c < nn; c += QR_THR) P[J.p_off + c] = perm[c];
    // Q' = H_0 ... H_{k-1} I(:, 0:k), the reflectors applied from the last to the first
    double* qo = J.lq ? qf : Q + J.q_off;
    for (uint64_t e = tid; e < uint64_t(mm) * k; e += QR_THR) {
        const uint32_t i = uint32_t(e % mm), c = uint32_t(e / mm);
        qo[e] = i == c ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int jj = int(k) - 1; jj >= 0; --jj) {
        const uint32_t j = uint32_t(jj);
        const double tau = taus[j];
        if (tau != 0.0) {
            const double* vj = w + uint64_t(j) * mm;
            for (uint32_t c = j + warp; c < k; c += QR_WARPS) {
                double* qc = qo + uint64_t(c) * mm;
                const double qj = qc[j];
                double d = 0.0;
                for (uint32_t i = j + 1 + lane; i < mm; i += 32) d = fma(vj[i], qc[i], d);
                d = warp_sum(d) + qj;
                d *= tau;
                if (lane == 0) qc[j] -= d;
                for (uint32_t i = j + 1 + lane; i < mm; i += 32) qc[i] = fma(-d, vj[i], qc[i]);
            }
        }
        __syncthreads();
    }
    if (J.lq) {
        // Q = Q'^T (k x n, ld k)
        double* q = Q + J.q_off;
        for (uint64_t e = tid; e < uint64_t(mm) * k; e += QR_THR) {
            const uint32_t i = uint32_t(e % mm), c = uint32_t(e / mm);
            q[c + uint64_t(i) * k] = qf[e];
        }
    }
}

__global__ void k_permute_rows(const PermJob* __restrict__ jobs, const double* __restrict__ src, double* __restrict__ dst,
                               const uint32_t* __restrict__ perm) {
    const PermJob J = jobs[blockIdx.x];
    const uint64_t n2 = uint64_t(J.n) * J.n;
    for (uint64_t e = threadIdx.x; e < n2; e += blockDim.x) {
        const uint32_t i = uint32_t(e % J.n), j = uint32_t(e / J.n);
        dst[J.dst_off + perm[J.p_off + i] + uint64_t(j) * J.ldd] = src[J.src_off + e];
    }
}

}  // namespace

void batched_permute_rows(const std::vector<PermJob>& jobs, const double* src, uint64_t src_len, double* dst, uint64_t dst_len,
                          const uint32_t* perm, uint64_t p_len, DBuf<PermJob>& jobbuf, cudaStream_t s) {
    if (jobs.empty()) return;
    for (const PermJob& j : jobs) {
        const uint64_t n = j.n;
        if (!n || j.ldd < n || j.src_off + n * n > src_len || j.dst_off + (n - 1) * j.ldd + n > dst_len || j.p_off + n > p_len)
            throw std::runtime_error("row permutation: a block outside its buffers");
    }
    jobbuf.upload(jobs, s);
    k_permute_rows<<<unsigned(jobs.size()), 256, 0, s>>>(jobbuf.get(), src, dst, perm);
    QCM_CUDA(cudaGetLastError());
}

uint64_t qr_scratch(uint32_t m, uint32_t n, bool lq) {
    const uint64_t k = std::min(m, n);
    return uint64_t(m) * n + k + (lq ? uint64_t(m) * n : 0) + 1;
}

void batched_qr(const std::vector<QrJob>& jobs, const double* A, uint64_t a_len, double* Q, uint64_t q_len, double* R,
                uint64_t r_len, double* W, uint64_t w_len, DBuf<QrJob>& jobbuf, cudaStream_t s, uint32_t* P, uint64_t p_len) {
    if (jobs.empty()) return;
    for (const QrJob& j : jobs) {
        const uint64_t k = std::min(j.m, j.n);
        if (!j.m || !j.n || j.a_off + uint64_t(j.m) * j.n > a_len || j.w_off + qr_scratch(j.m, j.n, j.lq != 0) > w_len ||
            j.q_off + k * (j.lq ? j.n : j.m) > q_len || j.r_off + k * (j.lq ? j.m : j.n) > r_len)
            throw std::runtime_error("batched QR: a block outside its buffers");
        const uint32_t nn = j.lq ? j.m : j.n;
        if ((j.flags & QR_RT) && j.lq) throw std::runtime_error("batched QR: a transposed R is for a QR, not an LQ");
        if ((j.flags & QR_PIVOT) && (!P || nn > QR_PIV_MAX || j.p_off + nn > p_len))
            throw std::runtime_error("batched QR: pivoting needs a permutation buffer and at most 1024 columns");
    }
    // shared memory for the largest work matrix that fits (one CTA per SM in either case)
    uint64_t sm = 0;
    for (const QrJob& j : jobs) {
        const uint64_t f = uint64_t(j.m) * j.n + std::min(j.m, j.n);
        if (f <= QR_SMEM_DOUBLES) sm = std::max(sm, f);
    }
    const std::size_t bytes = std::size_t(sm) * sizeof(double);
    if (bytes) QCM_CUDA(cudaFuncSetAttribute(k_qr, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    jobbuf.upload(jobs, s);
    k_qr<<<unsigned(jobs.size()), QR_THR, bytes, s>>>(jobbuf.get(), A, Q, R, W, P, uint32_t(sm));
    QCM_CUDA(cudaGetLastError());
}

}  // namespace qcm
