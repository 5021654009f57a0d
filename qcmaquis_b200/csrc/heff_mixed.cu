// Mixed-precision S build of H_eff: the unit GEMMs S_u = W_u * T slices with FP32 operands in
// HBM and three TF32 tensor-core products per term (3xTF32: a = a_hi + a_lo, b = b_hi + b_lo,
// a*b ~ a_lo*b_hi + a_hi*b_lo + a_hi*b_hi), accumulated in FP32 and written to S as FP64.
// The relative error of a product is ~2^-21 instead of TF32's 2^-11, so the S build carries
// FP32-level accuracy at tensor-core throughput.  Two forms:
//  * QCM_PRECISION_MIXED: FP32 operands (coefficient blocks copied once per plan, T written in
//    FP32 by the T-GEMM epilogue), split into hi and lo at the mma.sync fragment loads;
//  * QCM_PRECISION_MIXED_TC: operands split once, in HBM (coefficient blocks per plan by
//    k_split, T by the T-GEMM epilogue; hi and lo are TF32 values rounded to nearest, stored as
//    FP32 bit patterns), the 16- and 32-line tiles on tcgen05, the others on mma.sync.
// Measured at the L=24 M=512 middle bond the first is the faster: every form is bound by the
// element-wise gathers of T slices into shared memory, which the pre-split doubles.
//
// Same work lists as the FP64 kernel (k_sgemm): one CTA per (unit, line tile, element tile),
// the tile shapes of the plan, the per m-tile k-step lists with their 4-slice masks (a k8 step
// runs if either of its two groups holds a coefficient), cp.async staging with the slice
// offsets loaded a stage ahead.
//
// k_sgemm_tc (16 x 128 and 32 x 128 tiles): tcgen05.mma kind::tf32 with the accumulator in
// tensor memory.  The tile is computed transposed, D^T (128 elements x BM lines) =
// T_slices^T (128 x 16 per stage) * W_u^T (16 x BM), so M = 128 and N = BM; both operands are
// staged K-major (the element-wise copies transpose them on the way) in the canonical
// no-swizzle layout: 8 MN rows x 4 consecutive slices = one 128-byte core matrix, groups of 8
// MN rows 128 B apart (SBO), 4-slice chunks MN/8 * 128 B apart (LBO), two chunks per K = 8
// MMA.  (A standalone probe of the MN-major encoding of these descriptors on B200 returned
// zeros, the K-major one the exact product, so the K-major form is the one used.)  One
// thread issues the MMAs of a stage and commits them to the stage's mbarrier; a stage buffer
// is refilled only after that mbarrier completes.
//
// k_sgemm_x3 (64 x 64 and 128 x 32 tiles): mma.sync m16n8k8 .tf32 fragments: A (16 x 8) a0
// (g, t) a1 (g+8, t) a2 (g, t+4) a3 (g+8, t+4), B (8 x 8) b0 (t, g) b1 (t+4, g), C c0 (g, 2t)
// c1 (g, 2t+1) c2 (g+8, 2t) c3 (g+8, 2t+1), g = lane / 4, t = lane % 4.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>

#include "heff.hpp"

namespace qcm {
namespace {

constexpr int XTHR = 128;  // 4 warps
constexpr int XBK = 16;    // slices per pipeline stage (the plan's k-step)

template <int WM_, int WN_, int FM_, int FN_>
struct XShape {
    static constexpr int WM = WM_, WN = WN_, FM = FM_, FN = FN_;
    static constexpr int BM = WM * FM * 16, BN = WN * FN * 8;
    // row padding: fragment reads of 4 k-rows x 8 consecutive m/n fall in 32 distinct banks
    static constexpr int PA = (BM % 32 == 0) ? 8 : 24, PB = (BN % 32 == 0) ? 8 : 24;
    static constexpr int A_PER = BM * XBK / XTHR, B_PER = BN * XBK / XTHR;
    static_assert(WM * WN == 4, "4 warps per CTA");
    static_assert(A_PER * XTHR == BM * XBK && B_PER * XTHR == BN * XBK, "whole elements per thread");
};
using X16 = XShape<1, 4, 1, 4>;   // 16 x 128
using X32 = XShape<1, 4, 2, 4>;   // 32 x 128
using X64 = XShape<2, 2, 2, 4>;   // 64 x 64
using X128 = XShape<4, 1, 2, 4>;  // 128 x 32

// PRE: operands pre-split in HBM (hi and lo arrays); otherwise single FP32 values split at the
// fragment loads
template <class S, bool PRE>
struct __align__(16) XStage {
    float Ah[XBK][S::BM + S::PA], Al[PRE ? XBK : 1][S::BM + S::PA];
    float Bh[XBK][S::BN + S::PB], Bl[PRE ? XBK : 1][S::BN + S::PB];
};

// x = hi + lo with hi, lo TF32 (round to nearest)
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(hi) : "f"(x));
    const float r = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void cp4(float* smem, const float* gmem, bool pred) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(pred ? 4 : 0));
}
__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool pred) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(pred ? 16 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }



__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <class S, bool PRE>
__global__ void __launch_bounds__(XTHR) k_sgemm_x3(const UnitD* __restrict__ units, const TileD* __restrict__ tiles,
                                                   const uint32_t* __restrict__ line_b1, const uint64_t* __restrict__ slice_off,
                                                   const uint16_t* __restrict__ klist, const float* __restrict__ Wh,
                                                   const float* __restrict__ Wl, const float* __restrict__ Th,
                                                   const float* __restrict__ Tl, double* __restrict__ Sm) {
    __shared__ XStage<S, PRE> st[2];
    const TileD tile = tiles[blockIdx.x];
    const UnitD U = units[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp % S::WM, wn = warp / S::WM;
    const uint16_t* ks = klist + tile.pad;
    const uint32_t nsteps = ks[0];
    // 16-byte chunks (4 floats) along the W_u columns (ld wld, rows nl .. wld - 1 zero) and the
    // T slices (16-byte aligned); a chunk past a slice's ne elements is not read, one that
    // straddles ne reads the slice's padding into columns the epilogue drops
    constexpr int ACH = S::BM / 4 * XBK, BCH = S::BN / 4 * XBK;
    constexpr int ARND = (ACH + XTHR - 1) / XTHR, BRND = BCH / XTHR;
    static_assert(BCH % XTHR == 0, "whole B chunks per thread");
    uint64_t boff[BRND];
    auto load_offs = [&](uint32_t k0) {
#pragma unroll
        for (int rr = 0; rr < BRND; ++rr) {
            const uint32_t gk = k0 + uint32_t(tid + rr * XTHR) / (S::BN / 4);
            boff[rr] = gk < U.nk ? __ldg(slice_off + U.slice0 + gk) : 0;
        }
    };
    auto issue = [&](int sidx, uint32_t k0) {
        XStage<S, PRE>& s = st[sidx];
#pragma unroll
        for (int rr = 0; rr < ARND; ++rr) {
            const int c = tid + rr * XTHR;
            if (ACH % XTHR != 0 && c >= ACH) break;
            const int m = 4 * (c % (S::BM / 4)), k = c / (S::BM / 4);
            const uint32_t gm = tile.m0 + m, gk = k0 + k;
            const bool ok = gm < U.wld && gk < U.nk;
            const uint64_t o = ok ? U.w_off + gm + uint64_t(gk) * U.wld : 0;
            cp16(&s.Ah[k][m], Wh + o, ok);
            if (PRE) cp16(&s.Al[k][m], Wl + o, ok);
        }
#pragma unroll
        for (int rr = 0; rr < BRND; ++rr) {
            const int c = tid + rr * XTHR;
            const int n = 4 * (c % (S::BN / 4)), k = c / (S::BN / 4);
            const uint32_t gn = tile.n0 + n, gk = k0 + k;
            const bool ok = gn < U.ne && gk < U.nk;
            const uint64_t o = ok ? boff[rr] + gn : 0;
            cp16(&s.Bh[k][n], Th + o, ok);
            if (PRE) cp16(&s.Bl[k][n], Tl + o, ok);
        }
        cp_commit();
    };
    float acc[S::FM][S::FN][4];
#pragma unroll
    for (int i = 0; i < S::FM; ++i)
#pragma unroll
        for (int j = 0; j < S::FN; ++j) acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0.0f;
    uint32_t knext = nsteps > 1 ? uint32_t(ks[2] >> 4) * XBK : 0;
    if (nsteps) {
        load_offs(uint32_t(ks[1] >> 4) * XBK);
        issue(0, uint32_t(ks[1] >> 4) * XBK);
        if (nsteps > 1) load_offs(knext);
    }
    uint32_t mcur = nsteps ? (ks[1] & 15u) : 0;
    for (uint32_t it = 0; it < nsteps; ++it) {
        cp_wait_all();
        __syncthreads();
        const uint32_t mask = mcur;
        if (it + 1 < nsteps) {
            mcur = ks[2 + it] & 15u;
            issue((it + 1) & 1, knext);
            if (it + 2 < nsteps) {
                knext = uint32_t(ks[3 + it] >> 4) * XBK;
                load_offs(knext);
            }
        }
        const XStage<S, PRE>& s = st[it & 1];
#pragma unroll
        for (int kk = 0; kk < XBK; kk += 8) {
            if (!((mask >> (kk / 4)) & 3u)) continue;  // both 4-slice groups of this k8 step empty
            uint32_t ah[S::FM][4], al[S::FM][4], bh[S::FN][2], bl[S::FN][2];
#pragma unroll
            for (int i = 0; i < S::FM; ++i) {
                const int m = wm * S::FM * 16 + i * 16 + g;
                const int ra[4] = {kk + t, kk + t, kk + t + 4, kk + t + 4}, ca[4] = {m, m + 8, m, m + 8};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (PRE) {
                        ah[i][q] = __float_as_uint(s.Ah[ra[q]][ca[q]]);
                        al[i][q] = __float_as_uint(s.Al[PRE ? ra[q] : 0][ca[q]]);
                    } else {
                        split_tf32(s.Ah[ra[q]][ca[q]], ah[i][q], al[i][q]);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < S::FN; ++j) {
                const int n = wn * S::FN * 8 + j * 8 + g;
                const int rb[2] = {kk + t, kk + t + 4};
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    if (PRE) {
                        bh[j][q] = __float_as_uint(s.Bh[rb[q]][n]);
                        bl[j][q] = __float_as_uint(s.Bl[PRE ? rb[q] : 0][n]);
                    } else {
                        split_tf32(s.Bh[rb[q]][n], bh[j][q], bl[j][q]);
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < S::FM; ++i)
#pragma unroll
                for (int j = 0; j < S::FN; ++j) {
                    mma_tf32(acc[i][j], al[i], bh[j]);
                    mma_tf32(acc[i][j], ah[i], bl[j]);
                    mma_tf32(acc[i][j], ah[i], bh[j]);
                }
        }
    }
    // the thread's outputs: FN x 2 columns (element gn % erows of column block gn / erows) and FM x 2 lines,
    // each offset computed once
    uint32_t cof[S::FN][2];
#pragma unroll
    for (int j = 0; j < S::FN; ++j)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const uint32_t gn = tile.n0 + wn * S::FN * 8 + j * 8 + 2 * t + c;
            const uint32_t cb = gn / U.erows;
            cof[j][c] = gn < U.ne ? (gn - cb * U.erows) + cb * U.col_stride : 0xffffffffu;
        }
#pragma unroll
    for (int i = 0; i < S::FM; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t gl = tile.m0 + wm * S::FM * 16 + i * 16 + g + h * 8;
            if (gl >= U.nl) continue;
            double* srow = Sm + U.s_off + uint64_t(line_b1[U.line0 + gl]) * U.line_stride;
#pragma unroll
            for (int j = 0; j < S::FN; ++j)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (cof[j][c] != 0xffffffffu) srow[cof[j][c]] = double(acc[i][j][2 * h + c]);
        }
}

// ---------------------------------------------------------------------------
// tcgen05 path (16 x 128 and 32 x 128 tiles)

constexpr int TCM = 128;               // MMA M: elements of the tile
constexpr uint32_t TC_WAIT = 1u << 22;  // bounded mbarrier waits (~1 s); past that the tile gives up

// no-swizzle K-major shared-memory descriptor (start, LBO = 4-slice chunk stride, SBO = 8-row group stride)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) | (uint64_t((sbo >> 4) & 0x3FFFu) << 32) |
           (uint64_t(1) << 46);  // descriptor version 1, base offset 0, no swizzle
}
// instruction descriptor: D f32, A and B tf32, both K-major, N, M
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t i = 0; i < TC_WAIT; ++i)
        if (mbar_try(mbar, parity)) return true;
    return false;
}
__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// float index of (mn, k) in a stage operand of MN rows x 16 k: [4-slice chunk][8-row group][row][4]
template <int MN>
__device__ __forceinline__ int tc_idx(int mn, int k) {
    return (k >> 2) * (MN / 8) * 32 + (mn >> 3) * 32 + (mn & 7) * 4 + (k & 3);
}

template <int BML>  // lines per tile (MMA N)
struct TcStage {
    float Ah[TCM * XBK], Al[TCM * XBK];  // T slices^T: 128 elements x 16 slices
    float Bh[BML * XBK], Bl[BML * XBK];  // W_u^T: 16 slices x BML lines
};

template <int BML>
__global__ void __launch_bounds__(XTHR) k_sgemm_tc(const UnitD* __restrict__ units, const TileD* __restrict__ tiles,
                                                   const uint32_t* __restrict__ line_b1, const uint64_t* __restrict__ slice_off,
                                                   const uint16_t* __restrict__ klist, const float* __restrict__ Wh,
                                                   const float* __restrict__ Wl, const float* __restrict__ Th,
                                                   const float* __restrict__ Tl, double* __restrict__ Sm,
                                                   uint32_t* __restrict__ err) {
    static_assert(BML == 16 || BML == 32, "tile lines = MMA N (16 or 32; one 32-column TMEM allocation)");
    __shared__ __align__(128) TcStage<BML> st[2];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;
    const TileD tile = tiles[blockIdx.x];
    const UnitD U = units[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint16_t* ks = klist + tile.pad;
    const uint32_t nsteps = ks[0];
    if (nsteps == 0) return;  // S stays zero (cleared before the launch)
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(saddr(&mbar[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;\n" ::"r"(saddr(&tmem_base)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;

    // copies: thread tid owns element tid of every slice (T), and (line, slice) pairs of W_u
    uint64_t boff[XBK];
    auto load_offs = [&](uint32_t k0) {
#pragma unroll
        for (int k = 0; k < XBK; ++k) {
            const uint32_t gk = k0 + k;
            boff[k] = gk < U.nk ? __ldg(slice_off + U.slice0 + gk) : 0;
        }
    };
    auto issue = [&](int b, uint32_t k0) {
        TcStage<BML>& s = st[b];
        const uint32_t gn = tile.n0 + tid;
#pragma unroll
        for (int k = 0; k < XBK; ++k) {
            const bool ok = gn < U.ne && k0 + k < U.nk;
            const uint64_t o = ok ? boff[k] + gn : 0;
            const int i = tc_idx<TCM>(tid, k);
            cp4(&s.Ah[i], Th + o, ok);
            cp4(&s.Al[i], Tl + o, ok);
        }
#pragma unroll
        for (int r = 0; r < BML * XBK / XTHR; ++r) {
            const int e = tid + r * XTHR;
            const int l = e % BML, k = e / BML;
            const uint32_t gl = tile.m0 + l, gk = k0 + k;
            const bool ok = gl < U.nl && gk < U.nk;
            const uint64_t o = ok ? U.w_off + gl + uint64_t(gk) * U.wld : 0;
            const int i = tc_idx<BML>(l, k);
            cp4(&s.Bh[i], Wh + o, ok);
            cp4(&s.Bl[i], Wl + o, ok);
        }
        cp_commit();
    };
    constexpr uint32_t idesc = tc_idesc(TCM, BML);
    constexpr uint32_t lbo_a = (TCM / 8) * 128, lbo_b = (BML / 8) * 128, sbo = 128;
    bool ok = true;
    uint32_t first = 1;  // the tile's first MMA overwrites the accumulator
    uint32_t knext = nsteps > 1 ? uint32_t(ks[2] >> 4) * XBK : 0;
    load_offs(uint32_t(ks[1] >> 4) * XBK);
    issue(0, uint32_t(ks[1] >> 4) * XBK);
    if (nsteps > 1) load_offs(knext);
    uint32_t mcur = ks[1] & 15u;
    for (uint32_t it = 0; it < nsteps && ok; ++it) {
        const int b = it & 1;
        cp_wait_all();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // cp.async data -> tensor-core reads
        __syncthreads();
        const uint32_t mask = mcur;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const TcStage<BML>& s = st[b];
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                if (!((mask >> (2 * g)) & 3u)) continue;
                // k8 group g = 4-slice chunks 2g and 2g + 1
                const uint32_t oa = 2 * g * lbo_a, ob = 2 * g * lbo_b;
                const uint64_t ah = tc_desc(saddr(s.Ah) + oa, lbo_a, sbo), al = tc_desc(saddr(s.Al) + oa, lbo_a, sbo);
                const uint64_t bh = tc_desc(saddr(s.Bh) + ob, lbo_b, sbo), bl = tc_desc(saddr(s.Bl) + ob, lbo_b, sbo);
                tc_mma(tmem, al, bh, idesc, first ? 0u : 1u);
                tc_mma(tmem, ah, bl, idesc, 1u);
                tc_mma(tmem, ah, bh, idesc, 1u);
                first = 0;
            }
            tc_commit(saddr(&mbar[b]));
        }
        __syncwarp();
        if (it + 1 < nsteps) {
            mcur = ks[2 + it] & 15u;
            // the other buffer was read by the MMAs of step it - 1: wait for them before refilling it
            // (the outcome is made uniform, so every thread leaves the loop at the same barrier)
            if (it >= 1) {
                const bool w = mbar_wait(saddr(&mbar[(it + 1) & 1]), ((it - 1) >> 1) & 1u);
                if (!__syncthreads_and(w)) { ok = false; break; }
            }
            issue((it + 1) & 1, knext);
            if (it + 2 < nsteps) {
                knext = uint32_t(ks[3 + it] >> 4) * XBK;
                load_offs(knext);
            }
        }
    }
    // the last step's commit covers every MMA of the tile
    if (ok && !mbar_wait(saddr(&mbar[(nsteps - 1) & 1]), ((nsteps - 1) >> 1) & 1u)) ok = false;
    cp_wait_all();
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicOr(err, 1u);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        // warp w holds TMEM lanes 32w .. 32w + 31 = elements; columns = lines
        uint32_t v[BML];
#pragma unroll
        for (int c = 0; c < BML; c += 16) {
            const uint32_t ta = tmem + (uint32_t(32 * warp) << 16) + uint32_t(c);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                : "=r"(v[c + 0]), "=r"(v[c + 1]), "=r"(v[c + 2]), "=r"(v[c + 3]), "=r"(v[c + 4]), "=r"(v[c + 5]),
                  "=r"(v[c + 6]), "=r"(v[c + 7]), "=r"(v[c + 8]), "=r"(v[c + 9]), "=r"(v[c + 10]), "=r"(v[c + 11]),
                  "=r"(v[c + 12]), "=r"(v[c + 13]), "=r"(v[c + 14]), "=r"(v[c + 15])
                : "r"(ta));
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        const uint32_t gn = tile.n0 + 32 * warp + lane;
        if (gn < U.ne) {
            const uint32_t col = gn / U.erows, row = gn - col * U.erows;
            const uint64_t base = U.s_off + row + uint64_t(col) * U.col_stride;
#pragma unroll
            for (int l = 0; l < BML; ++l) {
                const uint32_t gl = tile.m0 + l;
                if (gl < U.nl) Sm[base + uint64_t(line_b1[U.line0 + gl]) * U.line_stride] = double(__uint_as_float(v[l]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;\n" ::"r"(tmem) : "memory");
}

// x (FP64) -> hi, lo: TF32 values (round to nearest) with hi + lo = x to ~2^-22 relative
__global__ void k_to_f32(const double* __restrict__ x, float* __restrict__ y, uint64_t n) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        y[i] = float(x[i]);
}

__global__ void k_split(const double* __restrict__ x, float* __restrict__ hi, float* __restrict__ lo, uint64_t n) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t h, l;
        asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(h) : "f"(float(x[i])));
        asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(l) : "f"(float(x[i] - double(__uint_as_float(h)))));
        hi[i] = __uint_as_float(h);
        lo[i] = __uint_as_float(l);
    }
}

template <class S, bool PRE>
void launch_x3(const HeffPlan& p, int sh, const float* Wh, const float* Wl, const float* Th, const float* Tl, double* Sm,
               cudaStream_t s) {
    if (p.utiles[sh].empty()) return;
    k_sgemm_x3<S, PRE><<<unsigned(p.utiles[sh].size()), XTHR, 0, s>>>(p.d_units.get(), p.d_utiles[sh].get(), p.d_line_b1.get(),
                                                                  p.d_slice_off.get(), p.d_klist.get(), Wh, Wl, Th, Tl, Sm);
}

template <int BML>
void launch_tc(const HeffPlan& p, int sh, const float* Wh, const float* Wl, const float* Th, const float* Tl, double* Sm,
               uint32_t* err, cudaStream_t s) {
    if (p.utiles[sh].empty()) return;
    k_sgemm_tc<BML><<<unsigned(p.utiles[sh].size()), XTHR, 0, s>>>(p.d_units.get(), p.d_utiles[sh].get(), p.d_line_b1.get(),
                                                                    p.d_slice_off.get(), p.d_klist.get(), Wh, Wl, Th, Tl, Sm, err);
}

}  // namespace

void to_f32(const double* x, float* y, uint64_t n, cudaStream_t s) {
    if (!n) return;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 16);
    k_to_f32<<<unsigned(blocks), 256, 0, s>>>(x, y, n);
    QCM_CUDA(cudaGetLastError());
}

void split_tf32(const double* x, float* hi, float* lo, uint64_t n, cudaStream_t s) {
    if (!n) return;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 16);
    k_split<<<unsigned(blocks), 256, 0, s>>>(x, hi, lo, n);
    QCM_CUDA(cudaGetLastError());
}

void run_sgemm_mixed(const HeffPlan& p, bool tc, const float* Wh, const float* Wl, const float* Th, const float* Tl, double* Sm,
                     uint32_t* err, cudaStream_t s) {
    static_assert(X16::BM == 16 && X16::BN == 128 && X32::BM == 32 && X32::BN == 128, "tile shapes of the plan");
    static_assert(X64::BM == 64 && X64::BN == 64 && X128::BM == 128 && X128::BN == 32, "tile shapes of the plan");
    if (tc) {
        // hi / lo operands: tcgen05 for the 16- and 32-line tiles, mma.sync for the others
        launch_tc<16>(p, SHAPE_16, Wh, Wl, Th, Tl, Sm, err, s);
        launch_tc<32>(p, SHAPE_32, Wh, Wl, Th, Tl, Sm, err, s);
        launch_x3<X64, true>(p, SHAPE_64, Wh, Wl, Th, Tl, Sm, s);
        launch_x3<X128, true>(p, SHAPE_128, Wh, Wl, Th, Tl, Sm, s);
    } else {
        // single FP32 operands, split at the fragment loads
        launch_x3<X16, false>(p, SHAPE_16, Wh, nullptr, Th, nullptr, Sm, s);
        launch_x3<X32, false>(p, SHAPE_32, Wh, nullptr, Th, nullptr, Sm, s);
        launch_x3<X64, false>(p, SHAPE_64, Wh, nullptr, Th, nullptr, Sm, s);
        launch_x3<X128, false>(p, SHAPE_128, Wh, nullptr, Th, nullptr, Sm, s);
    }
    QCM_CUDA(cudaGetLastError());
}

}  // namespace qcm
