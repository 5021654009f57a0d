// FP64 H_eff kernels for sm_100a.
//
// tcgen05.mma has no f64 kind, so the plain (FP64) form runs its sector GEMMs on
// the double-precision tensor path: mma.sync.aligned.m8n8k4 .f64 (DMMA).
// One CTA = 64 x 64 output tile, 4 warps each owning a 32 x 32 warp tile
// (4 x 4 DMMA fragments), K staged through shared memory 16 deep.
//
//   k_tgemm : T[ti] = psi_slab * R[ci_eff] (per-block transposed when the R
//             cohort is stored as its Hermitian partner)      (tasks.cpp:707-752)
//   k_gather: S = sum alpha * T slices                        (gpu_dgemm_ddot.cu:282-359)
//   k_lsgemm: y[lb_out] = sum over cohorts L[ci_eff] * S, one K loop over all
//             cohorts of the output block -> deterministic, no atomics
//                                                             (tasks.cpp:315-344 + atomic_add)
#include <cuda_runtime.h>

#include <cstdint>

#include "heff.hpp"

namespace qcm {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, PAD = 4, NTHR = 128;

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// Shared-memory tile pair and the warp-level DMMA product over one BK chunk.
struct Tiles {
    double A[BK][BM + PAD];
    double B[BK][BN + PAD];
};

__device__ __forceinline__ void mma_chunk(const Tiles& t, double (&acc)[4][4][2], int wm, int wn, int lane) {
    const int r = lane >> 2, q = lane & 3;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = t.A[kk + q][wm * 32 + i * 8 + r];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = t.B[kk + q][wn * 32 + j * 8 + r];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma(acc[i][j], a[i], b[j]);
    }
}

__device__ __forceinline__ void store_tile(double* __restrict__ C, uint64_t c_off, uint32_t ldc, uint32_t M, uint32_t N,
                                           uint32_t m0, uint32_t n0, const double (&acc)[4][4][2], int wm, int wn,
                                           int lane) {
    const int r = lane >> 2, q = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                uint32_t m = m0 + wm * 32 + i * 8 + r;
                uint32_t n = n0 + wn * 32 + j * 8 + q * 2 + c;
                if (m < M && n < N) C[c_off + m + uint64_t(n) * ldc] = acc[i][j][c];
            }
}

// T-GEMM: one CTA per (job, 64x64 tile)
__global__ void __launch_bounds__(NTHR) k_tgemm(const TJobD* __restrict__ jobs, const TileD* __restrict__ tiles,
                                                const double* __restrict__ x, const double* __restrict__ R,
                                                double* __restrict__ T) {
    __shared__ Tiles t;
    __shared__ uint64_t colbase[BN];
    const TileD tile = tiles[blockIdx.x];
    const TJobD J = jobs[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp & 1, wn = warp >> 1;
    if (tid < BN) {
        uint32_t n = tile.n0 + tid;
        uint64_t cb = 0;
        if (n < J.N) {
            uint32_t b = n / J.brs, j = n - b * J.brs;
            cb = J.b_off + uint64_t(b) * J.K * J.brs + (J.tr ? uint64_t(j) : uint64_t(j) * J.K);
        }
        colbase[tid] = cb;
    }
    const uint64_t kstride = J.tr ? J.brs : 1;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    __syncthreads();
    for (uint32_t k0 = 0; k0 < J.K; k0 += BK) {
#pragma unroll
        for (int rr = 0; rr < (BM * BK) / NTHR; ++rr) {
            int e = tid + rr * NTHR;
            int m = e & (BM - 1), k = e >> 6;
            uint32_t gm = tile.m0 + m, gk = k0 + k;
            t.A[k][m] = (gm < J.M && gk < J.K) ? x[J.a_off + gm + uint64_t(gk) * J.lda] : 0.0;
        }
        if (!J.tr) {
#pragma unroll
            for (int rr = 0; rr < (BN * BK) / NTHR; ++rr) {
                int e = tid + rr * NTHR;
                int k = e & (BK - 1), n = e >> 4;
                uint32_t gn = tile.n0 + n, gk = k0 + k;
                t.B[k][n] = (gn < J.N && gk < J.K) ? R[colbase[n] + gk] : 0.0;
            }
        } else {
#pragma unroll
            for (int rr = 0; rr < (BN * BK) / NTHR; ++rr) {
                int e = tid + rr * NTHR;
                int n = e & (BN - 1), k = e >> 6;
                uint32_t gn = tile.n0 + n, gk = k0 + k;
                t.B[k][n] = (gn < J.N && gk < J.K) ? R[colbase[n] + uint64_t(gk) * kstride] : 0.0;
            }
        }
        __syncthreads();
        mma_chunk(t, acc, wm, wn, lane);
        __syncthreads();
    }
    store_tile(T, J.c_off, J.M, J.M, J.N, tile.m0, tile.n0, acc, wm, wn, lane);
}

// S gather: one CTA per (cohort, unit, L block row) line
__global__ void __launch_bounds__(256) k_gather(const GTaskD* __restrict__ tasks, const double* __restrict__ alpha,
                                                const uint64_t* __restrict__ aoff, const double* __restrict__ T,
                                                double* __restrict__ S) {
    __shared__ double sa[64];
    __shared__ uint64_t so[64];
    const GTaskD g = tasks[blockIdx.x];
    const uint32_t n = g.rows * g.cols;
    for (uint32_t a0 = 0; a0 < g.a_count; a0 += 64) {
        uint32_t na = min(64u, g.a_count - a0);
        __syncthreads();
        if (threadIdx.x < na) {
            sa[threadIdx.x] = alpha[g.a_start + a0 + threadIdx.x];
            so[threadIdx.x] = aoff[g.a_start + a0 + threadIdx.x];
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) {
            uint32_t c = e / g.rows, r = e - c * g.rows;
            uint64_t rel = r + uint64_t(c) * g.rows;
            double s = 0.0;
            for (uint32_t a = 0; a < na; ++a) s = fma(sa[a], T[so[a] + rel], s);
            double* dst = &S[g.s_off + r + uint64_t(c) * g.ldS];
            *dst = (a0 == 0) ? s : *dst + s;
        }
    }
}

// L.S GEMM: one CTA per (output block, 64x64 tile); K runs over every cohort segment
__global__ void __launch_bounds__(NTHR) k_lsgemm(const OutD* __restrict__ outs, const SegD* __restrict__ segs,
                                                 const TileD* __restrict__ tiles, const double* __restrict__ Lb,
                                                 const double* __restrict__ S, double* __restrict__ y) {
    __shared__ Tiles t;
    __shared__ uint64_t kbase[BK];
    const TileD tile = tiles[blockIdx.x];
    const OutD O = outs[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp & 1, wn = warp >> 1;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const uint32_t M = O.M;
    for (uint32_t sgi = 0; sgi < O.seg_count; ++sgi) {
        const SegD sg = segs[O.seg_start + sgi];
        const uint32_t Kc = sg.nS * sg.ls_in;
        const uint64_t blk = uint64_t(M) * sg.ls_in;
        for (uint32_t k0 = 0; k0 < Kc; k0 += BK) {
            if (tid < BK) {
                uint32_t kk = k0 + tid;
                uint64_t kb = 0;
                if (kk < Kc) {
                    uint32_t b = kk / sg.ls_in, j = kk - b * sg.ls_in;
                    kb = sg.l_off + b * blk + (sg.tr ? uint64_t(j) : uint64_t(j) * M);
                }
                kbase[tid] = kb;
            }
            __syncthreads();
            if (!sg.tr) {
#pragma unroll
                for (int rr = 0; rr < (BM * BK) / NTHR; ++rr) {
                    int e = tid + rr * NTHR;
                    int m = e & (BM - 1), k = e >> 6;
                    uint32_t gm = tile.m0 + m, gk = k0 + k;
                    t.A[k][m] = (gm < M && gk < Kc) ? Lb[kbase[k] + gm] : 0.0;
                }
            } else {
#pragma unroll
                for (int rr = 0; rr < (BM * BK) / NTHR; ++rr) {
                    int e = tid + rr * NTHR;
                    int k = e & (BK - 1), m = e >> 4;
                    uint32_t gm = tile.m0 + m, gk = k0 + k;
                    t.A[k][m] = (gm < M && gk < Kc) ? Lb[kbase[k] + uint64_t(gm) * sg.ls_in] : 0.0;
                }
            }
#pragma unroll
            for (int rr = 0; rr < (BN * BK) / NTHR; ++rr) {
                int e = tid + rr * NTHR;
                int k = e & (BK - 1), n = e >> 4;
                uint32_t gn = tile.n0 + n, gk = k0 + k;
                t.B[k][n] = (gn < O.N && gk < Kc) ? S[sg.s_off + gk + uint64_t(gn) * Kc] : 0.0;
            }
            __syncthreads();
            mma_chunk(t, acc, wm, wn, lane);
            __syncthreads();
        }
    }
    store_tile(y, O.y_off, M, M, O.N, tile.m0, tile.n0, acc, wm, wn, lane);
}

}  // namespace

void heff_apply_device(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev) {
    cudaStream_t s = p.stream;
    if (ev) QCM_CUDA(cudaEventRecord(ev[0], s));
    QCM_CUDA(cudaMemsetAsync(y, 0, p.x_len * sizeof(double), s));
    if (!p.ttiles.empty())
        k_tgemm<<<unsigned(p.ttiles.size()), NTHR, 0, s>>>(p.d_tjobs.get(), p.d_ttiles.get(), x, p.R->data.get(), p.d_T.get());
    if (ev) QCM_CUDA(cudaEventRecord(ev[1], s));
    if (p.s_len) QCM_CUDA(cudaMemsetAsync(p.d_S.get(), 0, p.s_len * sizeof(double), s));
    if (!p.gtasks.empty())
        k_gather<<<unsigned(p.gtasks.size()), 256, 0, s>>>(p.d_gtasks.get(), p.d_alpha.get(), p.d_aoff.get(), p.d_T.get(), p.d_S.get());
    if (ev) QCM_CUDA(cudaEventRecord(ev[2], s));
    if (!p.otiles.empty())
        k_lsgemm<<<unsigned(p.otiles.size()), NTHR, 0, s>>>(p.d_outs.get(), p.d_segs.get(), p.d_otiles.get(), p.L->data.get(), p.d_S.get(), y);
    if (ev) QCM_CUDA(cudaEventRecord(ev[3], s));
    QCM_CUDA(cudaGetLastError());
}

void upload_plan(HeffPlan& p) {
    cudaStream_t s = p.stream;
    p.d_tjobs.upload(p.tjobs, s);
    p.d_ttiles.upload(p.ttiles, s);
    p.d_gtasks.upload(p.gtasks, s);
    p.d_alpha.upload(p.alpha, s);
    p.d_aoff.upload(p.aoff, s);
    p.d_segs.upload(p.segs, s);
    p.d_outs.upload(p.outs, s);
    p.d_otiles.upload(p.otiles, s);
    p.d_T.alloc(p.t_len);
    p.d_S.alloc(p.s_len);
    QCM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace qcm
