// Jacobi-Davidson for many independent site problems at once (the batching form of the path).
//
// The reference solves one site problem at a time (solve_ietl_jcd, solver/ietl_jacobi_davidson.h:
// 35-76; jacobi_davidson::calculate_eigenvalue, ietl/jacobi.h:386-474).  Here the problems' plans
// are merged into one plan (merge_plans) and the solves run in lockstep: every iteration applies
// all H_eff at once, and every other step of the iteration runs for all solves in one launch:
//   t = V[it] made orthogonal to V[0..it) (classical Gram-Schmidt applied twice) and normalised;
//   VA[it] = H V[it] (the merged plan);
//   column it of the projected matrix, <V[k], VA[it]> for k <= it;
//   Rayleigh-Ritz on the device (cyclic Jacobi, one thread per solve): theta, s;
//   u = V s, r = VA s - theta u, |r|, r.u, u.u;
//   convergence |r| <= tol |theta| or |r| < tol (ietl/jacobi.h:428-432), the solve's eigenpair kept
//   at its converging iteration (or the last); the next direction t = -r + (r.u)/(u.u) u (zero
//   for a converged solve).
// Nothing in an iteration waits for the host, so each iteration (one per subspace slot) is captured
// once as a CUDA graph and replayed; the host reads one counter per iteration to stop early.
// Vectors live in arenas (solve i's entries at xo[i] .. xo[i] + n[i]; the arena gaps are zero).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "dmrg_dev.hpp"
#include "heff.hpp"

namespace qcm {

namespace {

constexpr int BJ_THR = 256;
constexpr int BJ_MAXIT = 16;  // subspace slots of the batched solve

__device__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < BJ_THR / 32; ++i) r += sh[i];
    __syncthreads();
    return r;  // valid in thread 0
}

// out[k * ns + i] = <A_k, B> over solve i's entries, k < nk (A_k = A + k * ld).  Grid (nk, ns).
__global__ void __launch_bounds__(BJ_THR) k_bdots(const double* __restrict__ A, uint64_t ld, const double* __restrict__ B,
                                                  const uint64_t* __restrict__ xo, const uint64_t* __restrict__ xn,
                                                  int ns, double* __restrict__ out) {
    __shared__ double sh[BJ_THR / 32];
    const int k = blockIdx.x, i = blockIdx.y;
    const double* a = A + uint64_t(k) * ld + xo[i];
    const double* b = B + xo[i];
    const uint64_t n = xn[i];
    double v = 0.0;
    for (uint64_t j = threadIdx.x; j < n; j += BJ_THR) v = fma(a[j], b[j], v);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) out[uint64_t(k) * ns + i] = v;
}

// Y_i = beta * Y_i + sa * sum_{k < nk} c[k * ns + i] * A_k,i  (+ sg * g[i] * G_i if G).  Grid (chunks, ns).
__global__ void __launch_bounds__(BJ_THR) k_blincomb(const double* __restrict__ A, uint64_t ld, int nk,
                                                     const double* __restrict__ c, int ns, double sa, double beta,
                                                     const double* __restrict__ G, const double* __restrict__ g, double sg,
                                                     double* __restrict__ Y, const uint64_t* __restrict__ xo,
                                                     const uint64_t* __restrict__ xn) {
    const int i = blockIdx.y;
    const uint64_t n = xn[i], o = xo[i];
    for (uint64_t j = uint64_t(blockIdx.x) * BJ_THR + threadIdx.x; j < n; j += uint64_t(gridDim.x) * BJ_THR) {
        double acc = 0.0;
        for (int k = 0; k < nk; ++k) acc = fma(c[k * ns + i], A[uint64_t(k) * ld + o + j], acc);
        double v = beta == 0.0 ? sa * acc : fma(sa, acc, beta * Y[o + j]);
        if (G) v = fma(sg * g[i], G[o + j], v);
        Y[o + j] = v;
    }
}

// Y_i *= f[i]; f computed per solve by the first thread of each block from a norm^2: 1/sqrt (0 if 0)
__global__ void __launch_bounds__(BJ_THR) k_bnormalise(double* __restrict__ Y, const double* __restrict__ nrm2,
                                                       const uint64_t* __restrict__ xo, const uint64_t* __restrict__ xn) {
    const int i = blockIdx.y;
    const double q = nrm2[i];
    const double f = q > 0.0 ? 1.0 / sqrt(q) : 0.0;
    const uint64_t n = xn[i], o = xo[i];
    for (uint64_t j = uint64_t(blockIdx.x) * BJ_THR + threadIdx.x; j < n; j += uint64_t(gridDim.x) * BJ_THR) Y[o + j] *= f;
}

// Rayleigh-Ritz of solve i (one thread each): M (column `it` just computed into Mcol) appended to
// the solve's projected matrix Mp (BJ_MAXIT x BJ_MAXIT, column-major); lowest eigenpair of its
// leading (it+1) block by cyclic Jacobi (the same rotations as the host solver) -> theta[i], s[i].
__global__ void k_brr(int ns, int it, const double* __restrict__ Mcol, double* __restrict__ Mp, double* __restrict__ theta,
                      double* __restrict__ s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    double* M = Mp + uint64_t(i) * BJ_MAXIT * BJ_MAXIT;
    for (int k = 0; k <= it; ++k) M[k + it * BJ_MAXIT] = Mcol[uint64_t(k) * ns + i];
    const int n = it + 1;
    double A[BJ_MAXIT][BJ_MAXIT], V[BJ_MAXIT][BJ_MAXIT];
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) {
            A[r][c] = r <= c ? M[r + c * BJ_MAXIT] : M[c + r * BJ_MAXIT];
            V[r][c] = r == c ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int c = 0; c < n; ++c)
            for (int r = 0; r < n; ++r) { tot += A[r][c] * A[r][c]; if (r != c) off += A[r][c] * A[r][c]; }
        if (off <= 1e-32 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p][q];
                if (apq == 0.0) continue;
                const double tau = (A[q][q] - A[p][p]) / (2.0 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double cs = 1.0 / sqrt(1.0 + t * t), sn = t * cs;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = cs * akp - sn * akq;
                    A[k][q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = cs * apk - sn * aqk;
                    A[q][k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = cs * vkp - sn * vkq;
                    V[k][q] = sn * vkp + cs * vkq;
                }
            }
    }
    int best = 0;
    for (int k = 1; k < n; ++k) if (A[k][k] < A[best][best]) best = k;
    theta[i] = A[best][best];
    for (int k = 0; k < BJ_MAXIT; ++k) s[uint64_t(k) * ns + i] = k < n ? V[k][best] : 0.0;
}

// After u and r: convergence, the kept eigenpair, the next direction's coefficients and the count of
// solves still running.  d3[0..ns) = |r|^2, d3[ns..2ns) = r.u, d3[2ns..3ns) = u.u (k_bdots layout).
// cr[i], cu[i]: coefficients of r and u in the next direction (0, 0 for a converged solve).
__global__ void k_bconv(int ns, int it, int last, double tol, const double* __restrict__ d3, const double* __restrict__ theta,
                        int* __restrict__ state, double* __restrict__ ev, int* __restrict__ iters, double* __restrict__ cr,
                        double* __restrict__ cu, int* __restrict__ keep, int* __restrict__ active) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    keep[i] = 0;
    if (state[i]) { cr[i] = 0.0; cu[i] = 0.0; return; }
    const double rn = sqrt(d3[i]), th = theta[i];
    const bool done = rn <= tol * fabs(th) || rn < tol;
    if (done || last) {
        state[i] = 1;
        ev[i] = th;
        iters[i] = it + 1;
        keep[i] = 1;
        cr[i] = 0.0;
        cu[i] = 0.0;
        return;
    }
    atomicAdd(active, 1);  // a count, not a value that feeds the arithmetic
    cr[i] = -1.0;
    cu[i] = d3[uint64_t(ns) + i] / d3[uint64_t(2) * ns + i];
}

// X_i = U_i for the solves whose eigenpair was kept in this iteration
__global__ void __launch_bounds__(BJ_THR) k_bkeep(const double* __restrict__ U, double* __restrict__ X,
                                                  const int* __restrict__ keep, const uint64_t* __restrict__ xo,
                                                  const uint64_t* __restrict__ xn) {
    const int i = blockIdx.y;
    if (!keep[i]) return;
    const uint64_t n = xn[i], o = xo[i];
    for (uint64_t j = uint64_t(blockIdx.x) * BJ_THR + threadIdx.x; j < n; j += uint64_t(gridDim.x) * BJ_THR) X[o + j] = U[o + j];
}

}  // namespace

void jacobi_davidson_batched(HeffPlan& g, const std::vector<uint64_t>& xo, const std::vector<uint64_t>& xn, double* X,
                             double tol, int maxiter, std::vector<double>& ev, std::vector<int>& iters, bool use_graphs,
                             int* applies) {
    if (!g.merged) throw std::runtime_error("batched JD: expects a merged plan group");
    if (maxiter < 1 || maxiter > BJ_MAXIT) throw std::runtime_error("batched JD: maxiter must be in 1..16");
    const int ns = int(xo.size());
    if (ns < 1 || xn.size() != xo.size()) throw std::runtime_error("batched JD: bad solve layout");
    for (int i = 0; i < ns; ++i)
        if (xo[i] + xn[i] > g.x_len || xn[i] == 0) throw std::runtime_error("batched JD: a solve outside the arena");
    cudaStream_t s = g.stream;
    AllocStream scope(s);
    const uint64_t ld = (g.x_len + 31) / 32 * 32;
    // arenas: V[maxiter], VA[maxiter], U, R; per-solve scalars
    DBuf<double> vec(uint64_t(2 * maxiter + 2) * ld);
    double* V = vec.get();
    double* VA = V + uint64_t(maxiter) * ld;
    double* U = VA + uint64_t(maxiter) * ld;
    double* R = U + ld;
    QCM_CUDA(cudaMemsetAsync(V, 0, uint64_t(2 * maxiter + 2) * ld * sizeof(double), s));
    QCM_CUDA(cudaMemcpyAsync(V, X, g.x_len * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const uint64_t nsu = uint64_t(ns);
    // scalars: dots (maxiter x ns), Mcol (maxiter x ns), Mp (ns x 16 x 16), theta, s (16 x ns), d3 (3 ns),
    // ev, cr, cu, nrm2
    DBuf<double> scal(nsu * (2 * BJ_MAXIT + BJ_MAXIT * BJ_MAXIT + 1 + BJ_MAXIT + 3 + 1 + 2 + 1));
    double* dots = scal.get();
    double* Mcol = dots + nsu * BJ_MAXIT;
    double* Mp = Mcol + nsu * BJ_MAXIT;
    double* theta = Mp + nsu * BJ_MAXIT * BJ_MAXIT;
    double* sv = theta + nsu;
    double* d3 = sv + nsu * BJ_MAXIT;
    double* devv = d3 + 3 * nsu;
    double* cr = devv + nsu;
    double* cu = cr + nsu;
    double* nrm2 = cu + nsu;
    DBuf<int> ints(4 * nsu + 1);
    int* state = ints.get();
    int* dit = state + nsu;
    int* keep = dit + nsu;
    int* active = keep + nsu;
    QCM_CUDA(cudaMemsetAsync(scal.get(), 0, scal.size() * sizeof(double), s));
    QCM_CUDA(cudaMemsetAsync(ints.get(), 0, ints.size() * sizeof(int), s));
    DBuf<uint64_t> dxo, dxn;
    dxo.upload(xo, s);
    dxn.upload(xn, s);
    uint64_t nmax = 0;
    for (uint64_t n : xn) nmax = std::max(nmax, n);
    const dim3 eg(unsigned(std::min<uint64_t>((nmax + BJ_THR - 1) / BJ_THR, 1024)), unsigned(ns));
    const unsigned sg = unsigned((ns + 127) / 128);
    auto Vi = [&](int k) { return V + uint64_t(k) * ld; };
    auto VAi = [&](int k) { return VA + uint64_t(k) * ld; };
    auto iteration = [&](int it) {
        double* t = Vi(it);
        // classical Gram-Schmidt against V[0..it), twice
        for (int pass = 0; pass < (it > 0 ? 2 : 0); ++pass) {
            k_bdots<<<dim3(unsigned(it), unsigned(ns)), BJ_THR, 0, s>>>(V, ld, t, dxo.get(), dxn.get(), ns, dots);
            k_blincomb<<<eg, BJ_THR, 0, s>>>(V, ld, it, dots, ns, -1.0, 1.0, nullptr, nullptr, 0.0, t, dxo.get(),
                                             dxn.get());
        }
        k_bdots<<<dim3(1, unsigned(ns)), BJ_THR, 0, s>>>(t, ld, t, dxo.get(), dxn.get(), ns, nrm2);
        k_bnormalise<<<eg, BJ_THR, 0, s>>>(t, nrm2, dxo.get(), dxn.get());
        heff_apply_device(g, t, VAi(it));
        k_bdots<<<dim3(unsigned(it + 1), unsigned(ns)), BJ_THR, 0, s>>>(V, ld, VAi(it), dxo.get(), dxn.get(), ns, Mcol);
        k_brr<<<sg, 128, 0, s>>>(ns, it, Mcol, Mp, theta, sv);
        // u = V s; r = VA s - theta u
        k_blincomb<<<eg, BJ_THR, 0, s>>>(V, ld, it + 1, sv, ns, 1.0, 0.0, nullptr, nullptr, 0.0, U, dxo.get(), dxn.get());
        k_blincomb<<<eg, BJ_THR, 0, s>>>(VA, ld, it + 1, sv, ns, 1.0, 0.0, U, theta, -1.0, R, dxo.get(), dxn.get());
        k_bdots<<<dim3(1, unsigned(ns)), BJ_THR, 0, s>>>(R, ld, R, dxo.get(), dxn.get(), ns, d3);
        k_bdots<<<dim3(1, unsigned(ns)), BJ_THR, 0, s>>>(R, ld, U, dxo.get(), dxn.get(), ns, d3 + nsu);
        k_bdots<<<dim3(1, unsigned(ns)), BJ_THR, 0, s>>>(U, ld, U, dxo.get(), dxn.get(), ns, d3 + 2 * nsu);
        QCM_CUDA(cudaMemsetAsync(active, 0, sizeof(int), s));
        k_bconv<<<sg, 128, 0, s>>>(ns, it, it == maxiter - 1, tol, d3, theta, state, devv, dit, cr, cu, keep, active);
        k_bkeep<<<eg, BJ_THR, 0, s>>>(U, X, keep, dxo.get(), dxn.get());
        // next direction t = cr r + cu u (zero for converged solves)
        if (it + 1 < maxiter)
            k_blincomb<<<eg, BJ_THR, 0, s>>>(R, ld, 1, cr, ns, 1.0, 0.0, U, cu, 1.0, Vi(it + 1), dxo.get(), dxn.get());
        QCM_CUDA(cudaGetLastError());
    };
    std::vector<cudaGraphExec_t> execs;
    int napply = 0;
    for (int it = 0; it < maxiter; ++it) {
        if (use_graphs) {
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            QCM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                iteration(it);
            } catch (...) {
                cudaStreamEndCapture(s, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            QCM_CUDA(cudaStreamEndCapture(s, &graph));
            cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) throw cuda_error(std::string("batched JD: graph instantiation: ") + cudaGetErrorString(e));
            execs.push_back(exec);
            QCM_CUDA(cudaGraphLaunch(exec, s));
        } else {
            iteration(it);
        }
        ++napply;
        int h_active = 0;
        QCM_CUDA(cudaMemcpyAsync(&h_active, active, sizeof(int), cudaMemcpyDeviceToHost, s));
        QCM_CUDA(cudaStreamSynchronize(s));
        if (h_active == 0) break;
    }
    for (auto e : execs) cudaGraphExecDestroy(e);
    ev.assign(nsu, 0.0);
    iters.assign(nsu, 0);
    QCM_CUDA(cudaMemcpyAsync(ev.data(), devv, nsu * sizeof(double), cudaMemcpyDeviceToHost, s));
    QCM_CUDA(cudaMemcpyAsync(iters.data(), dit, nsu * sizeof(int), cudaMemcpyDeviceToHost, s));
    QCM_CUDA(cudaStreamSynchronize(s));
    if (applies) *applies = napply;
}

}  // namespace qcm
