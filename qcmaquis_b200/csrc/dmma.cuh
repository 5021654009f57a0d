// DMMA (mma.sync m8n8k4 .f64) tile machinery shared by the FP64 kernels: CTA
// tile shapes, a two-stage cp.async staging buffer, warp-level fragments.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace qcm {
namespace dm {

constexpr int BK = 16, PAD = 4, NTHR = 128;

static __device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// 8-byte asynchronous global->shared copy; a false predicate writes zeros (src-size 0)
static __device__ __forceinline__ void cp8(double* smem, const double* gmem, bool pred) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(pred ? 8 : 0));
}
// 16-byte asynchronous copy (both addresses 16-byte aligned); a false predicate writes zeros
static __device__ __forceinline__ void cp16(void* smem, const void* gmem, bool pred) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(pred ? 16 : 0));
}
static __device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
static __device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// CTA tile = WM x WN warps, each warp FM x FN DMMA fragments of 8 x 8.
template <int WM_, int WN_, int FM_, int FN_>
struct Shape {
    static constexpr int WM = WM_, WN = WN_, FM = FM_, FN = FN_;
    static constexpr int BM = WM * FM * 8, BN = WN * FN * 8;
    static constexpr int A_PER = BM * BK / NTHR, B_PER = BN * BK / NTHR;
    static_assert(WM * WN * 32 == NTHR, "4 warps per CTA");
};
using Sh16 = Shape<1, 4, 2, 4>;  // 16 x 128
using Sh32 = Shape<1, 4, 4, 4>;  // 32 x 128
using Sh64 = Shape<2, 2, 4, 4>;  // 64 x 64
using Sh128 = Shape<4, 1, 4, 4>; // 128 x 32

template <class S>
struct __align__(16) Stage {
    double A[BK][S::BM + PAD];
    double B[BK][S::BN + PAD];
};

template <class S>
struct Acc {
    double c[S::FM][S::FN][2];
    __device__ void zero() {
#pragma unroll
        for (int i = 0; i < S::FM; ++i)
#pragma unroll
            for (int j = 0; j < S::FN; ++j) c[i][j][0] = c[i][j][1] = 0.0;
    }
};

template <class S>
static __device__ __forceinline__ void mma_stage(const double (*A)[S::BM + PAD], const double (*B)[S::BN + PAD], Acc<S>& acc,
                                          int warp, int lane) {
    const int r = lane >> 2, q = lane & 3;
    const int wm = warp % S::WM, wn = warp / S::WM;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
        double a[S::FM], b[S::FN];
#pragma unroll
        for (int i = 0; i < S::FM; ++i) a[i] = A[kk + q][wm * S::FM * 8 + i * 8 + r];
#pragma unroll
        for (int j = 0; j < S::FN; ++j) b[j] = B[kk + q][wn * S::FN * 8 + j * 8 + r];
#pragma unroll
        for (int i = 0; i < S::FM; ++i)
#pragma unroll
            for (int j = 0; j < S::FN; ++j) dmma(acc.c[i][j], a[i], b[j]);
    }
}

// Same, skipping the 4-slice k groups whose bit in mask is clear (all-zero coefficients)
template <class S>
static __device__ __forceinline__ void mma_stage_masked(const double (*A)[S::BM + PAD], const double (*B)[S::BN + PAD],
                                                 Acc<S>& acc, int warp, int lane, uint32_t mask) {
    const int r = lane >> 2, q = lane & 3;
    const int wm = warp % S::WM, wn = warp / S::WM;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
        if (!((mask >> (kk / 4)) & 1u)) continue;
        double a[S::FM], b[S::FN];
#pragma unroll
        for (int i = 0; i < S::FM; ++i) a[i] = A[kk + q][wm * S::FM * 8 + i * 8 + r];
#pragma unroll
        for (int j = 0; j < S::FN; ++j) b[j] = B[kk + q][wn * S::FN * 8 + j * 8 + r];
#pragma unroll
        for (int i = 0; i < S::FM; ++i)
#pragma unroll
            for (int j = 0; j < S::FN; ++j) dmma(acc.c[i][j], a[i], b[j]);
    }
}

// Visit every accumulator element: f(m, n, value) with tile-local (m, n).
template <class S, class F>
static __device__ __forceinline__ void for_acc(const Acc<S>& acc, int warp, int lane, F f) {
    const int r = lane >> 2, q = lane & 3;
    const int wm = warp % S::WM, wn = warp / S::WM;
#pragma unroll
    for (int i = 0; i < S::FM; ++i)
#pragma unroll
        for (int j = 0; j < S::FN; ++j)
#pragma unroll
            for (int c = 0; c < 2; ++c) f(wm * S::FM * 8 + i * 8 + r, wn * S::FN * 8 + j * 8 + q * 2 + c, acc.c[i][j][c]);
}


}  // namespace dm
}  // namespace qcm
