// Generic batched device operations (see dev_ops.hpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>

#include "dev_ops.hpp"
#include "dmma.cuh"

namespace qcm {
namespace {
using namespace dm;

struct GTile { uint32_t job, m0, n0, pad; };

// One CTA per (job, 64x64 tile); operands may be transposed (ta/tb)
__global__ void __launch_bounds__(NTHR) k_bgemm(const GemmJob* __restrict__ jobs, const GTile* __restrict__ tiles,
                                                const double* __restrict__ A, const double* __restrict__ B,
                                                double* __restrict__ C) {
    using S = Sh64;
    __shared__ Stage<S> st[2];
    const GTile tile = tiles[blockIdx.x];
    const GemmJob J = jobs[tile.job];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto issue = [&](int sidx, uint32_t k0) {
        Stage<S>& s = st[sidx];
#pragma unroll
        for (int rr = 0; rr < S::A_PER; ++rr) {
            int e = tid + rr * NTHR;
            int m, k;
            if (!J.ta) { m = e % S::BM; k = e / S::BM; } else { k = e % BK; m = e / BK; }
            uint32_t gm = tile.m0 + m, gk = k0 + k;
            bool ok = gm < J.M && gk < J.K;
            uint64_t base = J.a_off;
            if (J.arb) { const uint32_t blk = gm / J.arb; base += uint64_t(blk) * J.a_bs; gm -= blk * J.arb; }
            const double* src = J.ta ? A + base + gk + uint64_t(gm) * J.lda : A + base + gm + uint64_t(gk) * J.lda;
            cp8(&s.A[k][m], ok ? src : A, ok);
        }
#pragma unroll
        for (int rr = 0; rr < S::B_PER; ++rr) {
            int e = tid + rr * NTHR;
            int k, n;
            if (!J.tb) { k = e % BK; n = e / BK; } else { n = e % S::BN; k = e / S::BN; }
            uint32_t gn = tile.n0 + n, gk = k0 + k;
            bool ok = gn < J.N && gk < J.K;
            const double* src = J.tb ? B + J.b_off + gn + uint64_t(gk) * J.ldb : B + J.b_off + gk + uint64_t(gn) * J.ldb;
            cp8(&s.B[k][n], ok ? src : B, ok);
        }
        cp_commit();
    };
    Acc<S> acc;
    acc.zero();
    const uint32_t nk = (J.K + BK - 1) / BK;
    if (nk) issue(0, 0);
    for (uint32_t kc = 0; kc < nk; ++kc) {
        cp_wait_all();
        __syncthreads();
        if (kc + 1 < nk) issue((kc + 1) & 1, (kc + 1) * BK);
        mma_stage<S>(st[kc & 1].A, st[kc & 1].B, acc, warp, lane);
    }
    // the thread's FM rows (row-blocked C: block gm / crb) and FN x 2 columns, each offset once
    const int r = lane >> 2, q = lane & 3;
    const int wm = warp % S::WM, wn = warp / S::WM;
#pragma unroll
    for (int i = 0; i < S::FM; ++i) {
        uint32_t gm = tile.m0 + wm * S::FM * 8 + i * 8 + r;
        if (gm >= J.M) continue;
        uint64_t base = J.c_off;
        if (J.crb) {
            const uint32_t blk = gm / J.crb;
            base += uint64_t(blk) * J.c_bs;
            gm -= blk * J.crb;
        }
        double* crow = C + base + gm;
#pragma unroll
        for (int j = 0; j < S::FN; ++j)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const uint32_t gn = tile.n0 + wn * S::FN * 8 + j * 8 + q * 2 + cc;
                if (gn >= J.N) continue;
                double* c = crow + uint64_t(gn) * J.ldc;
                const double v = acc.c[i][j][cc];
                *c = (J.beta == 0.0) ? J.alpha * v : J.alpha * v + J.beta * *c;
            }
    }
}

__global__ void k_bcopy(const CopyJob* __restrict__ jobs, uint32_t njobs, const double* __restrict__ src,
                        double* __restrict__ dst) {
    const CopyJob J = jobs[blockIdx.x];
    const uint64_t n = uint64_t(J.rows) * J.cols;
    for (uint64_t e = threadIdx.x; e < n; e += blockDim.x) {
        uint32_t j = uint32_t(e / J.rows), i = uint32_t(e - uint64_t(j) * J.rows);
        double v = src[J.src_off + i + uint64_t(J.rev ? J.cols - 1 - j : j) * J.src_ld];
        if (!J.trans) dst[J.dst_off + i + uint64_t(j) * J.dst_ld] = v;
        else dst[J.dst_off + j + uint64_t(i) * J.dst_ld] = v;
    }
}

// out[j] = <V_j, w>; one CTA per j, fixed-order tree reduction (deterministic)
// partial sums of <V_j, w>: block (b, j) takes i = b*256 + t (+ k * DOT_PARTS*256), two
// interleaved accumulators per thread, then a tree over the block
__global__ void __launch_bounds__(256) k_dots_part(const double* __restrict__ V, uint64_t ldv, const double* __restrict__ w,
                                                   uint64_t n, double* __restrict__ part) {
    __shared__ double red[256];
    const double* v = V + uint64_t(blockIdx.y) * ldv;
    const uint64_t stride = uint64_t(DOT_PARTS) * 256;
    double s0 = 0.0, s1 = 0.0;
    uint64_t i = uint64_t(blockIdx.x) * 256 + threadIdx.x;
    for (; i + stride < n; i += 2 * stride) {
        s0 = fma(v[i], w[i], s0);
        s1 = fma(v[i + stride], w[i + stride], s1);
    }
    if (i < n) s0 = fma(v[i], w[i], s0);
    red[threadIdx.x] = s0 + s1;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[uint64_t(blockIdx.y) * DOT_PARTS + blockIdx.x] = red[0];
}

// out[j] = tree sum of the DOT_PARTS partials of product j
__global__ void __launch_bounds__(DOT_PARTS) k_dots_sum(const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double red[DOT_PARTS];
    red[threadIdx.x] = part[uint64_t(blockIdx.x) * DOT_PARTS + threadIdx.x];
    __syncthreads();
    for (int h = DOT_PARTS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

__global__ void k_lincomb(const double* __restrict__ V, uint64_t ldv, uint32_t m, const double* __restrict__ c, uint64_t n,
                          double* __restrict__ y, int acc) {
    __shared__ double cs[64];
    if (threadIdx.x < m) cs[threadIdx.x] = c[threadIdx.x];
    __syncthreads();
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        double s = acc ? y[i] : 0.0;
        for (uint32_t j = 0; j < m; ++j) s = fma(cs[j], V[j * ldv + i], s);
        y[i] = s;
    }
}

__global__ void k_axpby(double a, const double* x, double b, double* y, uint64_t n) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        y[i] = (b == 0.0) ? a * x[i] : fma(a, x[i], b * y[i]);
}

__global__ void k_axpy_d(const double* __restrict__ a, double sa, const double* __restrict__ x, double* __restrict__ y,
                         uint64_t n) {
    const double f = sa * a[0];
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        y[i] = fma(f, x[i], y[i]);
}

__global__ void k_fill(double* p, uint64_t n, double v) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) p[i] = v;
}

__global__ void k_scale(double* A, uint32_t rows, uint32_t cols, uint32_t lda, const double* __restrict__ d, int by_row) {
    const uint64_t n = uint64_t(rows) * cols;
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < n; e += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t j = uint32_t(e / rows), i = uint32_t(e - uint64_t(j) * rows);
        A[i + uint64_t(j) * lda] *= by_row ? d[i] : d[j];
    }
}

unsigned grid_for(uint64_t n, unsigned bs = 256) {
    uint64_t g = (n + bs - 1) / bs;
    return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(g, 148 * 16)));
}

}  // namespace

void check_extent(uint64_t off, uint64_t rows, uint64_t cols, uint64_t ld, uint64_t len, const char* what) {
    if (!rows || !cols) return;
    if (ld < rows || off + (rows - 1) + (cols - 1) * ld >= len)
        throw std::runtime_error(std::string("device work list out of bounds: ") + what);
}

void batched_gemm(const std::vector<GemmJob>& jobs, const double* A, uint64_t a_len, const double* B, uint64_t b_len,
                  double* C, uint64_t c_len, DBuf<GemmJob>& jobbuf, DBuf<uint32_t>& tilebuf, cudaStream_t s) {
    if (jobs.empty()) return;
    for (const GemmJob& j : jobs) {
        if (!j.M || !j.N) continue;
        const uint32_t arb = j.arb ? j.arb : j.M, crb = j.crb ? j.crb : j.M;
        if (j.M % arb || j.M % crb) throw std::runtime_error("gemm: rows are not a whole number of row blocks");
        const uint64_t alast = j.a_off + uint64_t(j.M / arb - 1) * j.a_bs, clast = j.c_off + uint64_t(j.M / crb - 1) * j.c_bs;
        for (uint64_t ao : {j.a_off, alast}) {
            if (j.ta) check_extent(ao, j.K, arb, j.lda, a_len, "gemm A");
            else check_extent(ao, arb, j.K, j.lda, a_len, "gemm A");
        }
        if (j.tb) check_extent(j.b_off, j.N, j.K, j.ldb, b_len, "gemm B");
        else check_extent(j.b_off, j.K, j.N, j.ldb, b_len, "gemm B");
        for (uint64_t co : {j.c_off, clast}) check_extent(co, crb, j.N, j.ldc, c_len, "gemm C");
    }
    std::vector<GTile> tiles;
    for (uint32_t j = 0; j < jobs.size(); ++j)
        for (uint32_t n0 = 0; n0 < jobs[j].N; n0 += 64)
            for (uint32_t m0 = 0; m0 < jobs[j].M; m0 += 64) tiles.push_back(GTile{j, m0, n0, 0});
    if (tiles.empty()) return;
    jobbuf.upload(jobs, s);
    tilebuf.upload(reinterpret_cast<const uint32_t*>(tiles.data()), tiles.size() * 4, s);
    k_bgemm<<<unsigned(tiles.size()), NTHR, 0, s>>>(jobbuf.get(), reinterpret_cast<const GTile*>(tilebuf.get()), A, B, C);
    QCM_CUDA(cudaGetLastError());
    // job/tile buffers are reused by the next call: keep the host order simple by finishing here
    QCM_CUDA(cudaStreamSynchronize(s));
}

void batched_copy(const std::vector<CopyJob>& jobs, const double* src, uint64_t src_len, double* dst, uint64_t dst_len,
                  DBuf<CopyJob>& jobbuf, cudaStream_t s) {
    if (jobs.empty()) return;
    for (const CopyJob& j : jobs) {
        check_extent(j.src_off, j.rows, j.cols, j.src_ld, src_len, "copy source");
        if (j.trans) check_extent(j.dst_off, j.cols, j.rows, j.dst_ld, dst_len, "copy destination");
        else check_extent(j.dst_off, j.rows, j.cols, j.dst_ld, dst_len, "copy destination");
    }
    uint64_t mx = 0;
    for (auto& j : jobs) mx = std::max<uint64_t>(mx, uint64_t(j.rows) * j.cols);
    if (mx == 0) return;
    jobbuf.upload(jobs, s);
    k_bcopy<<<unsigned(jobs.size()), 256, 0, s>>>(jobbuf.get(), unsigned(jobs.size()), src, dst);
    QCM_CUDA(cudaGetLastError());
    QCM_CUDA(cudaStreamSynchronize(s));
}

void dev_dots(const double* V, uint64_t ldv, uint32_t m, const double* w, uint64_t n, double* out, double* scratch,
              cudaStream_t s) {
    if (!m) return;
    if (m > 65535) throw std::runtime_error("dev_dots: too many products");
    k_dots_part<<<dim3(DOT_PARTS, m), 256, 0, s>>>(V, ldv, w, n, scratch);
    k_dots_sum<<<m, DOT_PARTS, 0, s>>>(scratch, out);
    QCM_CUDA(cudaGetLastError());
}

void dev_lincomb(const double* V, uint64_t ldv, uint32_t m, const double* c, uint64_t n, double* y, bool accumulate,
                 cudaStream_t s) {
    if (m > 64) throw std::runtime_error("dev_lincomb: at most 64 vectors");
    k_lincomb<<<grid_for(n), 256, 0, s>>>(V, ldv, m, c, n, y, accumulate ? 1 : 0);
    QCM_CUDA(cudaGetLastError());
}

void dev_axpby(double a, const double* x, double b, double* y, uint64_t n, cudaStream_t s) {
    k_axpby<<<grid_for(n), 256, 0, s>>>(a, x, b, y, n);
    QCM_CUDA(cudaGetLastError());
}

void dev_axpy_dscalar(const double* a_dev, double sa, const double* x, double* y, uint64_t n, cudaStream_t s) {
    if (!n) return;
    k_axpy_d<<<grid_for(n), 256, 0, s>>>(a_dev, sa, x, y, n);
    QCM_CUDA(cudaGetLastError());
}

void dev_fill(double* p, uint64_t n, double v, cudaStream_t s) {
    if (!n) return;
    k_fill<<<grid_for(n), 256, 0, s>>>(p, n, v);
    QCM_CUDA(cudaGetLastError());
}

void dev_scale_rows(double* A, uint32_t rows, uint32_t cols, uint32_t lda, const double* d, cudaStream_t s) {
    if (!rows || !cols) return;
    k_scale<<<grid_for(uint64_t(rows) * cols), 256, 0, s>>>(A, rows, cols, lda, d, 1);
    QCM_CUDA(cudaGetLastError());
}

void dev_scale_cols(double* A, uint32_t rows, uint32_t cols, uint32_t lda, const double* d, cudaStream_t s) {
    if (!rows || !cols) return;
    k_scale<<<grid_for(uint64_t(rows) * cols), 256, 0, s>>>(A, rows, cols, lda, d, 0);
    QCM_CUDA(cudaGetLastError());
}

}  // namespace qcm
