// FP64 H_eff kernels for sm_100a.
//
// tcgen05.mma has no f64 kind, so the plain (FP64) form runs every contraction
// on the double-precision tensor path, mma.sync.aligned.m8n8k4 .f64 (DMMA).  A
// CTA of 4 warps owns a BM x BN tile (16x128, 32x128 or 64x64, picked from the
// row count so short sectors do not waste rows).  K is staged 16 deep through a
// two-stage cp.async pipeline (the operands are gathered through per-column /
// per-row base tables, so bulk tensor copies do not apply).
//
//   k_tgemm   : T[ti] = psi_slab * R[ci_eff] (per-block transposed when the R
//               cohort is stored as its Hermitian partner)         (tasks.cpp:707-752)
//   k_sgemm   : S rows of a cohort unit = W_u (lines x slices, the unit's MPO
//               coefficients as a dense block, scattered once per plan by
//               k_wfill) * T slices.
//               Replaces the alpha-weighted gather (gpu_dgemm_ddot.cu:282-359,
//               tasks.cpp:466-494) by a tensor-core GEMM.
//   k_lspart  : split-K partial tiles of y[lb_out] = sum_cohorts L[ci_eff] * S
//   k_lsreduce: partials of each output tile summed in a fixed order -> y
//               (deterministic; replaces cublasDgemm + atomic_add, tasks.cpp:315-344)
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>

#include "dmma.cuh"
#include "heff.hpp"

namespace qcm {
namespace {

using namespace dm;

// ---------------------------------------------------------------------------
// T-GEMM: one CTA per (job, tile)
template <class S>
__global__ void __launch_bounds__(NTHR) k_tgemm(const TJobD* __restrict__ jobs, const TileD* __restrict__ tiles,
                                                const double* __restrict__ x, const double* __restrict__ R,
                                                double* __restrict__ T) {
    __shared__ Stage<S> st[2];
    __shared__ uint64_t colbase[S::BN];
    const TileD tile = tiles[blockIdx.x];
    const TJobD J = jobs[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int c = tid; c < S::BN; c += NTHR) {
        uint32_t n = tile.n0 + c;
        uint64_t cb = J.b_off;
        if (n < J.N) {
            uint32_t b = n / J.brs, j = n - b * J.brs;
            cb = J.b_off + uint64_t(b) * J.K * J.brs + (J.tr ? uint64_t(j) : uint64_t(j) * J.K);
        }
        colbase[c] = cb;
    }
    __syncthreads();
    const uint64_t kstride = J.tr ? J.brs : 1;
    auto issue = [&](int sidx, uint32_t k0) {
        Stage<S>& s = st[sidx];
#pragma unroll
        for (int rr = 0; rr < S::A_PER; ++rr) {
            int e = tid + rr * NTHR;
            int m = e % S::BM, k = e / S::BM;
            uint32_t gm = tile.m0 + m, gk = k0 + k;
            bool ok = gm < J.M && gk < J.K;
            cp8(&s.A[k][m], ok ? x + J.a_off + gm + uint64_t(gk) * J.lda : x, ok);
        }
        if (!J.tr) {
#pragma unroll
            for (int rr = 0; rr < S::B_PER; ++rr) {
                int e = tid + rr * NTHR;
                int k = e % BK, n = e / BK;
                uint32_t gn = tile.n0 + n, gk = k0 + k;
                bool ok = gn < J.N && gk < J.K;
                cp8(&s.B[k][n], ok ? R + colbase[n] + gk : R, ok);
            }
        } else {
#pragma unroll
            for (int rr = 0; rr < S::B_PER; ++rr) {
                int e = tid + rr * NTHR;
                int n = e % S::BN, k = e / S::BN;
                uint32_t gn = tile.n0 + n, gk = k0 + k;
                bool ok = gn < J.N && gk < J.K;
                cp8(&s.B[k][n], ok ? R + colbase[n] + uint64_t(gk) * kstride : R, ok);
            }
        }
        cp_commit();
    };
    Acc<S> acc;
    acc.zero();
    const uint32_t nk = (J.K + BK - 1) / BK;
    issue(0, 0);
    for (uint32_t kc = 0; kc < nk; ++kc) {
        cp_wait_all();
        __syncthreads();
        if (kc + 1 < nk) issue((kc + 1) & 1, (kc + 1) * BK);
        mma_stage<S>(st[kc & 1].A, st[kc & 1].B, acc, warp, lane);
    }
    for_acc<S>(acc, warp, lane, [&](int m, int n, double v) {
        uint32_t gm = tile.m0 + m, gn = tile.n0 + n;
        if (gm < J.M && gn < J.N) T[J.c_off + gm + uint64_t(gn) * J.M] = v;
    });
}

// ---------------------------------------------------------------------------
// S build: one CTA per (unit, line tile, element tile)
template <class S>
__global__ void __launch_bounds__(NTHR) k_sgemm(const UnitD* __restrict__ units, const TileD* __restrict__ tiles,
                                                const uint32_t* __restrict__ line_b1, const uint64_t* __restrict__ slice_off,
                                                const uint16_t* __restrict__ klist, const double* __restrict__ W,
                                                const double* __restrict__ T, double* __restrict__ Sm) {
    __shared__ Stage<S> st[2];
    const TileD tile = tiles[blockIdx.x];
    const UnitD U = units[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // only the k-steps whose coefficient block (this tile's lines x 16 slices) holds an entry
    const uint16_t* ks = klist + tile.pad;
    const uint32_t nsteps = ks[0];
    const double* Wu = W + U.w_off;
    // T offsets of the slices this thread copies, loaded one stage ahead of their use
    uint64_t boff[S::B_PER];
    auto load_offs = [&](uint32_t k0) {
#pragma unroll
        for (int rr = 0; rr < S::B_PER; ++rr) {
            const uint32_t gk = k0 + uint32_t(tid + rr * NTHR) / S::BN;
            boff[rr] = gk < U.nk ? __ldg(slice_off + U.slice0 + gk) : 0;
        }
    };
    auto issue = [&](int sidx, uint32_t k0) {
        Stage<S>& s = st[sidx];
        // A = W_u (lines x slices, column-major, ld nl)
#pragma unroll
        for (int rr = 0; rr < S::A_PER; ++rr) {
            int e = tid + rr * NTHR;
            int m = e % S::BM, k = e / S::BM;
            uint32_t gm = tile.m0 + m, gk = k0 + k;
            bool ok = gm < U.nl && gk < U.nk;
            cp8(&s.A[k][m], ok ? Wu + gm + uint64_t(gk) * U.nl : W, ok);
        }
        // B row k = T slice k (ne contiguous elements)
#pragma unroll
        for (int rr = 0; rr < S::B_PER; ++rr) {
            int e = tid + rr * NTHR;
            int n = e % S::BN, k = e / S::BN;
            uint32_t gn = tile.n0 + n, gk = k0 + k;
            bool ok = gn < U.ne && gk < U.nk;
            cp8(&s.B[k][n], ok ? T + boff[rr] + gn : T, ok);
        }
        cp_commit();
    };
    Acc<S> acc;
    acc.zero();
    // step entries: k-step index << 4 | mask of its non-empty 4-slice groups
    uint32_t knext = nsteps > 1 ? uint32_t(ks[2] >> 4) * BK : 0;
    if (nsteps) {
        load_offs(uint32_t(ks[1] >> 4) * BK);
        issue(0, uint32_t(ks[1] >> 4) * BK);
        if (nsteps > 1) load_offs(knext);
    }
    uint32_t mcur = nsteps ? (ks[1] & 15u) : 0;
    for (uint32_t i = 0; i < nsteps; ++i) {
        cp_wait_all();
        __syncthreads();
        const uint32_t mask = mcur;
        if (i + 1 < nsteps) {
            mcur = ks[2 + i] & 15u;
            issue((i + 1) & 1, knext);
            if (i + 2 < nsteps) {
                knext = uint32_t(ks[3 + i] >> 4) * BK;
                load_offs(knext);
            }
        }
        mma_stage_masked<S>(st[i & 1].A, st[i & 1].B, acc, warp, lane, mask);
    }
    for_acc<S>(acc, warp, lane, [&](int m, int n, double v) {
        uint32_t gl = tile.m0 + m, gn = tile.n0 + n;
        if (gl < U.nl && gn < U.ne) {
            uint32_t b1 = line_b1[U.line0 + gl];
            uint32_t c = gn / U.erows, r = gn - c * U.erows;
            Sm[U.s_off + uint64_t(b1) * U.line_stride + r + uint64_t(c) * U.col_stride] = v;
        }
    });
}

// One CTA per unit: its coefficient entries into the dense block W_u (duplicates were merged on the host)
__global__ void k_wfill(const UnitD* __restrict__ units, const uint32_t* __restrict__ sptr, const WEntD* __restrict__ went,
                        double* __restrict__ W) {
    const UnitD U = units[blockIdx.x];
    const uint32_t e0 = sptr[U.sptr0], e1 = sptr[U.sptr0 + U.nk];
    for (uint32_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const WEntD w = went[e];
        W[U.w_off + w.line + uint64_t(w.k) * U.nl] = w.a;
    }
}

// ---------------------------------------------------------------------------
// L.S GEMM, split-K: item = (output tile, segment, K range) -> partial tile P[item]
template <class S>
__global__ void __launch_bounds__(NTHR) k_lspart(const KItemD* __restrict__ items, const OTileD* __restrict__ otiles,
                                                 const OutD* __restrict__ outs, const SegD* __restrict__ segs,
                                                 const double* __restrict__ Lb, const double* __restrict__ Sm,
                                                 double* __restrict__ P) {
    __shared__ Stage<S> st[2];
    __shared__ uint64_t kbase[2][BK];
    const KItemD it = items[blockIdx.x];
    const OTileD ot = otiles[it.tile];
    const OutD O = outs[ot.out];
    const SegD sg = segs[it.seg];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t M = O.M, Kc = sg.nS * sg.ls_in;
    const uint64_t blk = uint64_t(M) * sg.ls_in;
    auto issue = [&](int sidx, uint32_t k0) {
        if (tid < BK) {
            uint32_t kk = k0 + tid;
            uint64_t kb = sg.l_off;
            if (kk < it.k1) {
                uint32_t b = kk / sg.ls_in, j = kk - b * sg.ls_in;
                kb = sg.l_off + b * blk + (sg.tr ? uint64_t(j) : uint64_t(j) * M);
            }
            kbase[sidx][tid] = kb;
        }
        __syncthreads();
        Stage<S>& s = st[sidx];
        if (!sg.tr) {
#pragma unroll
            for (int rr = 0; rr < S::A_PER; ++rr) {
                int e = tid + rr * NTHR;
                int m = e % S::BM, k = e / S::BM;
                uint32_t gm = ot.m0 + m, gk = k0 + k;
                bool ok = gm < M && gk < it.k1;
                cp8(&s.A[k][m], ok ? Lb + kbase[sidx][k] + gm : Lb, ok);
            }
        } else {
#pragma unroll
            for (int rr = 0; rr < S::A_PER; ++rr) {
                int e = tid + rr * NTHR;
                int k = e % BK, m = e / BK;
                uint32_t gm = ot.m0 + m, gk = k0 + k;
                bool ok = gm < M && gk < it.k1;
                cp8(&s.A[k][m], ok ? Lb + kbase[sidx][k] + uint64_t(gm) * sg.ls_in : Lb, ok);
            }
        }
#pragma unroll
        for (int rr = 0; rr < S::B_PER; ++rr) {
            int e = tid + rr * NTHR;
            int k = e % BK, n = e / BK;
            uint32_t gn = ot.n0 + n, gk = k0 + k;
            bool ok = gn < O.N && gk < it.k1;
            cp8(&s.B[k][n], ok ? Sm + sg.s_off + gk + uint64_t(gn) * Kc : Sm, ok);
        }
        cp_commit();
    };
    Acc<S> acc;
    acc.zero();
    const uint32_t nk = (it.k1 - it.k0 + BK - 1) / BK;
    issue(0, it.k0);
    for (uint32_t kc = 0; kc < nk; ++kc) {
        cp_wait_all();
        __syncthreads();
        if (kc + 1 < nk) issue((kc + 1) & 1, it.k0 + (kc + 1) * BK);
        mma_stage<S>(st[kc & 1].A, st[kc & 1].B, acc, warp, lane);
    }
    double* Pt = P + uint64_t(blockIdx.x) * S::BM * S::BN;
    for_acc<S>(acc, warp, lane, [&](int m, int n, double v) { Pt[m + n * S::BM] = v; });
}

// Sum the partial tiles of each output tile in item order and write y.
template <class S>
__global__ void __launch_bounds__(256) k_lsreduce(const OTileD* __restrict__ otiles, const OutD* __restrict__ outs,
                                                  const double* __restrict__ P, double* __restrict__ y) {
    const OTileD ot = otiles[blockIdx.x];
    const OutD O = outs[ot.out];
    for (int e = threadIdx.x; e < S::BM * S::BN; e += blockDim.x) {
        const int m = e % S::BM, n = e / S::BM;
        const uint32_t gm = ot.m0 + m, gn = ot.n0 + n;
        if (gm >= O.M || gn >= O.N) continue;
        double s = 0.0;
        for (uint32_t p = 0; p < ot.nparts; ++p) s += P[uint64_t(ot.part0 + p) * S::BM * S::BN + e];
        y[O.y_off + gm + uint64_t(gn) * O.M] = s;
    }
}

template <class S>
void launch_t(HeffPlan& p, int sh, const double* x, double* Tb, cudaStream_t s) {
    if (!p.ttiles[sh].empty())
        k_tgemm<S><<<unsigned(p.ttiles[sh].size()), NTHR, 0, s>>>(p.d_tjobs.get(), p.d_ttiles[sh].get(), x,
                                                                  p.R->data.get(), Tb);
}

template <class S>
void launch_s(HeffPlan& p, int sh, const double* Tb, double* Sb, cudaStream_t s) {
    if (!p.utiles[sh].empty())
        k_sgemm<S><<<unsigned(p.utiles[sh].size()), NTHR, 0, s>>>(p.d_units.get(), p.d_utiles[sh].get(), p.d_line_b1.get(),
                                                                  p.d_slice_off.get(), p.d_klist.get(), p.d_W.get(), Tb, Sb);
}

template <class S>
void launch_ls(HeffPlan& p, int sh, const double* Sb, double* Pb, double* y, cudaStream_t s) {
    if (p.kitems[sh].empty()) return;
    k_lspart<S><<<unsigned(p.kitems[sh].size()), NTHR, 0, s>>>(p.d_kitems[sh].get(), p.d_otiles[sh].get(), p.d_outs.get(),
                                                               p.d_segs.get(), p.L->data.get(), Sb, Pb);
    k_lsreduce<S><<<unsigned(p.otiles[sh].size()), 256, 0, s>>>(p.d_otiles[sh].get(), p.d_outs.get(), Pb, y);
}

}  // namespace

namespace {
// One H.psi: T-GEMM -> S build -> split-K L.S, with the scratch buffers T, S and P given
// explicitly (the plan's own buffers, or caller-provided memory of the same sizes).
void apply_impl(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev, double* Tb, double* Sb, double* Pb) {
    cudaStream_t s = p.stream;
    if (ev) QCM_CUDA(cudaEventRecord(ev[0], s));
    QCM_CUDA(cudaMemsetAsync(y, 0, p.x_len * sizeof(double), s));
    launch_t<Sh16>(p, SHAPE_16, x, Tb, s);
    launch_t<Sh32>(p, SHAPE_32, x, Tb, s);
    launch_t<Sh64>(p, SHAPE_64, x, Tb, s);
    if (ev) QCM_CUDA(cudaEventRecord(ev[1], s));
    if (p.s_len) QCM_CUDA(cudaMemsetAsync(Sb, 0, p.s_len * sizeof(double), s));  // rows without lines stay 0
    launch_s<Sh16>(p, SHAPE_16, Tb, Sb, s);
    launch_s<Sh32>(p, SHAPE_32, Tb, Sb, s);
    launch_s<Sh64>(p, SHAPE_64, Tb, Sb, s);
    launch_s<Sh128>(p, SHAPE_128, Tb, Sb, s);
    if (ev) QCM_CUDA(cudaEventRecord(ev[2], s));
    launch_ls<Sh16>(p, SHAPE_16, Sb, Pb, y, s);
    launch_ls<Sh32>(p, SHAPE_32, Sb, Pb, y, s);
    launch_ls<Sh64>(p, SHAPE_64, Sb, Pb, y, s);
    if (ev) QCM_CUDA(cudaEventRecord(ev[3], s));
    QCM_CUDA(cudaGetLastError());
}
}  // namespace

void heff_apply_device(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev) {
    apply_impl(p, x, y, ev, p.d_T.get(), p.d_S.get(), p.d_P.get());
}

void heff_apply_device_scratch(HeffPlan& p, const double* x, double* y, double* Tb, double* Sb, double* Pb) {
    apply_impl(p, x, y, nullptr, Tb, Sb, Pb);
}

void run_tgemm(const TJobD* jobs, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const double* x,
               const double* R, double* T, cudaStream_t s) {
    if (!htiles[SHAPE_16].empty())
        k_tgemm<Sh16><<<unsigned(htiles[SHAPE_16].size()), NTHR, 0, s>>>(jobs, dtiles[SHAPE_16].get(), x, R, T);
    if (!htiles[SHAPE_32].empty())
        k_tgemm<Sh32><<<unsigned(htiles[SHAPE_32].size()), NTHR, 0, s>>>(jobs, dtiles[SHAPE_32].get(), x, R, T);
    if (!htiles[SHAPE_64].empty())
        k_tgemm<Sh64><<<unsigned(htiles[SHAPE_64].size()), NTHR, 0, s>>>(jobs, dtiles[SHAPE_64].get(), x, R, T);
    QCM_CUDA(cudaGetLastError());
}

void run_sgemm(const UnitD* units, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const uint32_t* line_b1,
               const uint64_t* slice_off, const uint16_t* klist, const double* W, const double* T, double* S,
               cudaStream_t s) {
    if (!htiles[SHAPE_16].empty())
        k_sgemm<Sh16><<<unsigned(htiles[SHAPE_16].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_16].get(), line_b1, slice_off, klist, W, T, S);
    if (!htiles[SHAPE_32].empty())
        k_sgemm<Sh32><<<unsigned(htiles[SHAPE_32].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_32].get(), line_b1, slice_off, klist, W, T, S);
    if (!htiles[SHAPE_64].empty())
        k_sgemm<Sh64><<<unsigned(htiles[SHAPE_64].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_64].get(), line_b1, slice_off, klist, W, T, S);
    if (!htiles[SHAPE_128].empty())
        k_sgemm<Sh128><<<unsigned(htiles[SHAPE_128].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_128].get(), line_b1, slice_off, klist, W, T, S);
    QCM_CUDA(cudaGetLastError());
}

void fill_coefficients(const UnitD* units, uint32_t n_units, const uint32_t* sptr, const WEntD* went, double* W,
                       uint64_t w_len, cudaStream_t s) {
    if (w_len) QCM_CUDA(cudaMemsetAsync(W, 0, w_len * sizeof(double), s));
    if (n_units) k_wfill<<<n_units, 128, 0, s>>>(units, sptr, went, W);
    QCM_CUDA(cudaGetLastError());
}

int heff_launches_per_apply(const HeffPlan& p) {
    int n = 0;
    for (int sh = 0; sh < N_SHAPES; ++sh) {
        n += !p.ttiles[sh].empty();
        n += !p.utiles[sh].empty();
        n += p.kitems[sh].empty() ? 0 : 2;
    }
    return n;
}

void upload_plan(HeffPlan& p) {
    cudaStream_t s = p.stream;
    for (const UnitD& u : p.units)
        if (u.w_off + uint64_t(u.nl) * u.nk > p.w_len || (u.nk && u.slice0 + u.nk > p.slice_off.size()))
            throw std::runtime_error("heff plan: unit outside its work lists");
    for (int sh = 0; sh < N_SHAPES; ++sh)
        for (const TileD& t : p.utiles[sh]) {
            if (t.item >= p.units.size() || std::size_t(t.pad) >= p.klist.size() ||
                std::size_t(t.pad) + 1 + p.klist[t.pad] > p.klist.size())
                throw std::runtime_error("heff plan: S tile outside its work lists");
            for (uint32_t i = 0; i < p.klist[t.pad]; ++i)
                if (uint32_t(p.klist[t.pad + 1 + i] >> 4) * BK >= p.units[t.item].nk) throw std::runtime_error("heff plan: S tile k-step out of range");
        }
    p.d_tjobs.upload(p.tjobs, s);
    for (int sh = 0; sh < N_SHAPES; ++sh) {
        p.d_ttiles[sh].upload(p.ttiles[sh], s);
        p.d_utiles[sh].upload(p.utiles[sh], s);
        p.d_otiles[sh].upload(p.otiles[sh], s);
        p.d_kitems[sh].upload(p.kitems[sh], s);
    }
    p.d_units.upload(p.units, s);
    p.d_line_b1.upload(p.line_b1, s);
    p.d_slice_off.upload(p.slice_off, s);
    p.d_sptr.upload(p.sptr, s);
    p.d_went.upload(p.went, s);
    p.d_klist.upload(p.klist, s);
    p.d_segs.upload(p.segs, s);
    p.d_outs.upload(p.outs, s);
    p.d_T.alloc(p.t_len);
    p.d_S.alloc(p.s_len);
    p.d_P.alloc(p.p_len);
    // dense coefficient blocks, built once per plan and reused by every apply
    p.d_W.alloc(p.w_len ? p.w_len : 1);
    fill_coefficients(p.d_units.get(), uint32_t(p.units.size()), p.d_sptr.get(), p.d_went.get(), p.d_W.get(), p.w_len, s);
    QCM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace qcm
