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
//   k_wgen    : W_u (lines x slices) = the unit's MPO coefficient terms summed into
//               a dense block, once per plan, from the MPO, operator and boundary
//               tables (one thread per line)
//   k_sgemm   : S rows of a cohort unit = W_u * T slices.
//               Replaces the alpha-weighted gather (gpu_dgemm_ddot.cu:282-359,
//               tasks.cpp:466-494) by a tensor-core GEMM.
//   k_lspart  : split-K partial tiles of y[lb_out] = sum_cohorts L[ci_eff] * S
//   k_lsreduce: partials of each output tile summed in a fixed order -> y
//               (deterministic; replaces cublasDgemm + atomic_add, tasks.cpp:315-344)
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

#include "dmma.cuh"
#include "heff.hpp"

namespace qcm {
namespace {

using namespace dm;

// ---------------------------------------------------------------------------
// T-GEMM: one CTA per (job, tile)
template <class S>
__global__ void __launch_bounds__(NTHR, 5) k_tgemm(const TJobD* __restrict__ jobs, const TileD* __restrict__ tiles,
                                                const double* __restrict__ x, const double* __restrict__ R,
                                                double* __restrict__ T, float* __restrict__ Thi, float* __restrict__ Tlo) {
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
    // the thread's output columns: FN fragments x 2 columns each; their T offsets once (slice
    // blk at blk * sst, column within it at (n % brs) * M)
    const int r = lane >> 2, q = lane & 3;
    const int wm = warp % S::WM, wn = warp / S::WM;
    uint64_t cof[S::FN][2];
    bool cok[S::FN][2];
#pragma unroll
    for (int j = 0; j < S::FN; ++j)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const uint32_t gn = tile.n0 + wn * S::FN * 8 + j * 8 + q * 2 + c;
            cok[j][c] = gn < J.N;
            const uint32_t blk = cok[j][c] ? gn / J.brs : 0;
            cof[j][c] = J.c_off + uint64_t(blk) * J.sst + uint64_t(gn - blk * J.brs) * J.M;
        }
#pragma unroll
    for (int i = 0; i < S::FM; ++i) {
        const uint32_t gm = tile.m0 + wm * S::FM * 8 + i * 8 + r;
        if (gm >= J.M) continue;
#pragma unroll
        for (int j = 0; j < S::FN; ++j)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                if (!cok[j][c]) continue;
                const double v = acc.c[i][j][c];
                const uint64_t o = cof[j][c] + gm;
                if (Thi && !Tlo) {
                    Thi[o] = float(v);  // mixed form: T in FP32, split by the S build
                } else if (Thi) {
                    // mixed form (tensor-memory path): T as TF32 hi + lo (round to nearest)
                    uint32_t h, l;
                    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(h) : "f"(float(v)));
                    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(l) : "f"(float(v - double(__uint_as_float(h)))));
                    Thi[o] = __uint_as_float(h);
                    Tlo[o] = __uint_as_float(l);
                } else {
                    T[o] = v;
                }
            }
    }
}

// ---------------------------------------------------------------------------
// S build: one CTA per (unit, line tile, element tile)
template <class S>
__global__ void __launch_bounds__(NTHR, 5) k_sgemm(const UnitD* __restrict__ units, const TileD* __restrict__ tiles,
                                                const uint32_t* __restrict__ line_b1, const uint64_t* __restrict__ slice_off,
                                                const uint16_t* __restrict__ klist, const double* __restrict__ W,
                                                const double* __restrict__ T, double* __restrict__ Sm, uint64_t w0) {
    __shared__ Stage<S> st[2];
    const TileD tile = tiles[blockIdx.x];
    const UnitD U = units[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // only the k-steps whose coefficient block (this tile's lines x 16 slices) holds an entry
    const uint16_t* ks = klist + tile.pad;
    const uint32_t nsteps = ks[0];
    const double* Wu = W + (U.w_off - w0);  // W holds the coefficient blocks from element w0 on
    // 16-byte chunks (2 doubles): W_u columns (ld wld, rows nl .. wld - 1 zero) and T slices (sst
    // apart, 16-byte aligned) are read 16 bytes at a time; a chunk past the slice's ne elements
    // is not read, one that straddles ne reads the slice's padding into columns the epilogue drops
    constexpr int ACH = S::BM / 2 * BK, BCH = S::BN / 2 * BK;
    static_assert(ACH % NTHR == 0 && BCH % NTHR == 0, "whole chunks per thread");
    // T offsets of the slices this thread copies, loaded one stage ahead of their use
    uint64_t boff[BCH / NTHR];
    auto load_offs = [&](uint32_t k0) {
#pragma unroll
        for (int rr = 0; rr < BCH / NTHR; ++rr) {
            const uint32_t gk = k0 + uint32_t(tid + rr * NTHR) / (S::BN / 2);
            boff[rr] = gk < U.nk ? __ldg(slice_off + U.slice0 + gk) : 0;
        }
    };
    auto issue = [&](int sidx, uint32_t k0) {
        Stage<S>& s = st[sidx];
        // A = W_u (lines x slices, column-major, ld wld)
#pragma unroll
        for (int rr = 0; rr < ACH / NTHR; ++rr) {
            const int c = tid + rr * NTHR;
            const int m = 2 * (c % (S::BM / 2)), k = c / (S::BM / 2);
            const uint32_t gm = tile.m0 + m, gk = k0 + k;
            const bool ok = gm < U.wld && gk < U.nk;
            cp16(&s.A[k][m], ok ? Wu + gm + uint64_t(gk) * U.wld : W, ok);
        }
        // B row k = T slice k (ne contiguous elements)
#pragma unroll
        for (int rr = 0; rr < BCH / NTHR; ++rr) {
            const int c = tid + rr * NTHR;
            const int n = 2 * (c % (S::BN / 2)), k = c / (S::BN / 2);
            const uint32_t gn = tile.n0 + n, gk = k0 + k;
            const bool ok = gn < U.ne && gk < U.nk;
            cp16(&s.B[k][n], ok ? T + boff[rr] + gn : T, ok);
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
    // the thread's outputs: its FN x 2 columns (element gn % erows of column block gn / erows) and FM
    // lines (S row block of line_b1), each offset computed once
    const int r = lane >> 2, q = lane & 3;
    const int wm = warp % S::WM, wn = warp / S::WM;
    uint32_t cof[S::FN][2];
#pragma unroll
    for (int j = 0; j < S::FN; ++j)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const uint32_t gn = tile.n0 + wn * S::FN * 8 + j * 8 + q * 2 + c;
            const uint32_t cb = gn / U.erows;
            cof[j][c] = gn < U.ne ? (gn - cb * U.erows) + cb * U.col_stride : 0xffffffffu;
        }
#pragma unroll
    for (int i = 0; i < S::FM; ++i) {
        const uint32_t gl = tile.m0 + wm * S::FM * 8 + i * 8 + r;
        if (gl >= U.nl) continue;
        double* srow = Sm + U.s_off + uint64_t(line_b1[U.line0 + gl]) * U.line_stride;
#pragma unroll
        for (int j = 0; j < S::FN; ++j)
#pragma unroll
            for (int c = 0; c < 2; ++c)
                if (cof[j][c] != 0xffffffffu) srow[cof[j][c]] = acc.c[i][j][c];
    }
}

// One CTA per unit, one thread per line: the line's coefficient terms (CoefGen), in MPO-entry
// then operator-term order, summed into W_u.  Products and sums are rounded separately (no
// contraction), so W_u holds the same values as a host evaluation of the same terms.
constexpr int WG_THR = 256;  // 256 against 128: streamed applies 3-11 % faster
constexpr uint32_t WG_SMAP = 4096;  // (slice id, slot) pairs staged in shared memory
constexpr uint32_t WG_NST = 64;     // physical states of the basis
__global__ void __launch_bounds__(WG_THR) k_wgen(const WGenUnitD* __restrict__ units, const WGenInD* __restrict__ gin,
                                                 uint32_t nst, const uint32_t* __restrict__ line_major,
                                                 const double* __restrict__ line_scale,
                                                 const uint32_t* __restrict__ smap_id, const uint32_t* __restrict__ smap_slot,
                                                 const uint32_t* __restrict__ m_ptr, const uint32_t* __restrict__ m_other,
                                                 const uint32_t* __restrict__ m_op, const double* __restrict__ m_scale,
                                                 const uint32_t* __restrict__ o_ptr, const uint32_t* __restrict__ o_in,
                                                 const double* __restrict__ o_val, const int32_t* __restrict__ b_pos,
                                                 const double* __restrict__ b_cs, uint32_t b_aux, double* __restrict__ W,
                                                 uint64_t w0, uint32_t* __restrict__ err) {
    __shared__ uint32_t sid[WG_SMAP], sslot[WG_SMAP];
    __shared__ WGenInD sin[WG_NST];
    const WGenUnitD U = units[blockIdx.x];
    const bool staged = U.nk <= WG_SMAP;
    if (staged)
        for (uint32_t i = threadIdx.x; i < U.nk; i += blockDim.x) {
            sid[i] = smap_id[U.map0 + i];
            sslot[i] = smap_slot[U.map0 + i];
        }
    for (uint32_t i = threadIdx.x; i < nst; i += blockDim.x) sin[i] = gin[std::size_t(blockIdx.x) * nst + i];
    __syncthreads();
    const uint32_t* ids = staged ? sid : smap_id + U.map0;
    const uint32_t* slots = staged ? sslot : smap_slot + U.map0;
    for (uint32_t line = threadIdx.x; line < U.nl; line += blockDim.x) {
        const uint32_t m = line_major[U.line0 + line];
        const double lsc = line_scale[U.line0 + line];
        double* Wl = W + (U.w_off - w0) + line;
        for (uint32_t e = m_ptr[m]; e < m_ptr[m + 1]; ++e) {
            const uint32_t x = m_other[e], op = m_op[e];
            const double wsc = __dmul_rn(m_scale[e], lsc);
            const std::size_t q = std::size_t(op) * nst + U.st_out;
            for (uint32_t k = o_ptr[q]; k < o_ptr[q + 1]; ++k) {
                const WGenInD g = sin[o_in[k]];
                if (g.c == WGEN_NONE) continue;
                const std::size_t bq = std::size_t(g.c) * b_aux + x;
                const int32_t pos = b_pos[bq];
                if (pos < 0) continue;
                const double a = __dmul_rn(__dmul_rn(o_val[k], b_cs[bq]), wsc);
                const uint32_t id = g.jbase + uint32_t(pos);
                uint32_t lo = 0, hi = U.nk;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (ids[mid] < id) lo = mid + 1;
                    else hi = mid;
                }
                if (lo >= U.nk || ids[lo] != id) { atomicOr(err, 1u); continue; }
                double* w = Wl + uint64_t(slots[lo]) * U.wld;
                *w = __dadd_rn(*w, a);
            }
        }
    }
}

}  // namespace

void CoefGen::validate() const {
    const std::size_t nu = units.size();
    auto bad = [](const char* what) { throw std::runtime_error(std::string("coefficient tables: ") + what); };
    if (!mt || mt->nst != nst) bad("MPO tables");
    if (nst > WG_NST || gin.size() != nu * nst || line_scale.size() != line_major.size() || smap_slot.size() != smap_id.size())
        bad("unit tables");
    // the MPO tables were checked when built (indices inside the tensor); here: against the boundary
    const uint32_t nmaj = by_row ? mt->rows : mt->cols, nother = by_row ? mt->cols : mt->rows;
    if (nother > b_aux) bad("MPO index outside the boundary");
    if (!b_cs || b_cs->size() != b_pos.size() || (b_aux && b_pos.size() % b_aux)) bad("boundary tables");
    const std::size_t ncoh = b_aux ? b_pos.size() / b_aux : 0;
    for (const WGenInD& g : gin)
        if (g.c != WGEN_NONE && g.c >= ncoh) bad("boundary cohort");
    for (const WGenUnitD& g : units) {
        if (g.st_out >= nst || std::size_t(g.line0) + g.nl > line_major.size() || std::size_t(g.map0) + g.nk > smap_id.size() ||
            g.wld < g.nl || g.w_off + uint64_t(g.wld) * g.nk > w_len)
            bad("unit extent");
        for (uint32_t l = 0; l < g.nl; ++l)
            if (line_major[g.line0 + l] >= nmaj) bad("line index");
        for (uint32_t i = 0; i < g.nk; ++i) {
            if (smap_slot[g.map0 + i] >= g.nk) bad("slot");
            if (i && smap_id[g.map0 + i - 1] >= smap_id[g.map0 + i]) bad("slice ids not sorted");
        }
    }
}

void CoefGen::upload(cudaStream_t s) {
    validate();
    d_units.upload(units, s);
    d_gin.upload(gin, s);
    d_line_major.upload(line_major, s);
    d_line_scale.upload(line_scale, s);
    d_smap_id.upload(smap_id, s);
    d_smap_slot.upload(smap_slot, s);
    d_m_ptr.upload(by_row ? mt->row_ptr : mt->col_ptr, s);
    d_m_other.upload(by_row ? mt->row_other : mt->col_other, s);
    d_m_op.upload(by_row ? mt->row_op : mt->col_op, s);
    d_m_scale.upload(by_row ? mt->row_scale : mt->col_scale, s);
    d_o_ptr.upload(mt->o_ptr, s);
    d_o_in.upload(mt->o_in, s);
    d_o_val.upload(mt->o_val, s);
    d_b_pos.upload(b_pos, s);
    d_b_cs.upload(*b_cs, s);
}

void CoefGen::generate(double* W, cudaStream_t s) {
    generate_range(W, 0, uint32_t(units.size()), 0, w_len, s);
    check_generated(s);
}

void CoefGen::generate_range(double* W, uint32_t u0, uint32_t u1, uint64_t w0, uint64_t w1, cudaStream_t s) {
    if (w1 > w0) QCM_CUDA(cudaMemsetAsync(W, 0, (w1 - w0) * sizeof(double), s));
    if (u1 <= u0) return;
    if (d_units.size() < units.size()) throw std::runtime_error("coefficient tables: not uploaded");
    if (u1 > units.size()) throw std::runtime_error("coefficient tables: unit range outside the plan");
    if (d_err.size() < 1) {
        d_err.alloc(1);
        QCM_CUDA(cudaMemsetAsync(d_err.get(), 0, sizeof(uint32_t), s));
    }
    k_wgen<<<unsigned(u1 - u0), WG_THR, 0, s>>>(d_units.get() + u0, d_gin.get() + std::size_t(u0) * nst, nst, d_line_major.get(),
                                                d_line_scale.get(), d_smap_id.get(), d_smap_slot.get(), d_m_ptr.get(),
                                                d_m_other.get(), d_m_op.get(), d_m_scale.get(), d_o_ptr.get(), d_o_in.get(),
                                                d_o_val.get(), d_b_pos.get(), d_b_cs.get(), b_aux, W, w0, d_err.get());
    QCM_CUDA(cudaGetLastError());
}

void CoefGen::check_generated(cudaStream_t s) {
    if (units.empty() || d_err.size() < 1) return;
    uint32_t h = 0;
    QCM_CUDA(cudaMemcpyAsync(&h, d_err.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    QCM_CUDA(cudaStreamSynchronize(s));
    QCM_CUDA(cudaMemsetAsync(d_err.get(), 0, sizeof(uint32_t), s));
    if (h) throw std::runtime_error("coefficient tables: a term has no slice slot");
}

namespace {

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
    // L column bases of a stage's 16 k rows, written two stages ahead so that the loop's barrier
    // publishes them before their stage is issued
    auto bases = [&](int sidx, uint32_t k0) {
        if (tid < BK) {
            uint32_t kk = k0 + tid;
            uint64_t kb = sg.l_off;
            if (kk < it.k1) {
                uint32_t b = kk / sg.ls_in, j = kk - b * sg.ls_in;
                kb = sg.l_off + b * blk + (sg.tr ? uint64_t(j) : uint64_t(j) * M);
            }
            kbase[sidx][tid] = kb;
        }
    };
    auto issue = [&](int sidx, uint32_t k0) {
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
    bases(0, it.k0);
    bases(1, it.k0 + BK);
    __syncthreads();
    issue(0, it.k0);
    for (uint32_t kc = 0; kc < nk; ++kc) {
        cp_wait_all();
        __syncthreads();
        if (kc + 1 < nk) issue((kc + 1) & 1, it.k0 + (kc + 1) * BK);
        // stage kc's bases were consumed when it was issued: the buffer takes stage kc + 2's
        if (kc + 2 < nk) bases(kc & 1, it.k0 + (kc + 2) * BK);
        mma_stage<S>(st[kc & 1].A, st[kc & 1].B, acc, warp, lane);
    }
    double* Pt = P + uint64_t(it.slot) * S::BM * S::BN;
    for_acc<S>(acc, warp, lane, [&](int m, int n, double v) { Pt[m + n * S::BM] = v; });
}

// Sum the partial tiles of each output tile in item order and write y.  Grid: (output tile, 256-element
// chunk of the tile).
template <class S>
__global__ void __launch_bounds__(256) k_lsreduce(const OTileD* __restrict__ otiles, const OutD* __restrict__ outs,
                                                  const double* __restrict__ P, double* __restrict__ y) {
    // one thread per tile element (blockIdx.y: the tile's 256-element chunk): the element's partials are
    // added in item order; the unrolled loop keeps several of its loads in flight
    const OTileD ot = otiles[blockIdx.x];
    const OutD O = outs[ot.out];
    const int e = int(blockIdx.y) * int(blockDim.x) + int(threadIdx.x);
    if (e >= S::BM * S::BN) return;
    const int m = e % S::BM, n = e / S::BM;
    const uint32_t gm = ot.m0 + m, gn = ot.n0 + n;
    if (gm >= O.M || gn >= O.N) return;
    const double* Pe = P + uint64_t(ot.part0) * S::BM * S::BN + e;
    double s = 0.0;
#pragma unroll 8
    for (uint32_t p = 0; p < ot.nparts; ++p) s += Pe[uint64_t(p) * S::BM * S::BN];
    y[O.y_off + gm + uint64_t(gn) * O.M] = s;
}

template <class S>
void launch_t(HeffPlan& p, int sh, const double* x, double* Tb, cudaStream_t s, float* Thi = nullptr,
              float* Tlo = nullptr) {
    if (!p.ttiles[sh].empty())
        k_tgemm<S><<<unsigned(p.ttiles[sh].size()), NTHR, 0, s>>>(p.d_tjobs.get(), p.d_ttiles[sh].get(), x,
                                                                  p.r_data(), Tb, Thi, Tlo);
}

template <class S>
void launch_s(HeffPlan& p, int sh, const double* Tb, double* Sb, cudaStream_t s) {
    if (!p.utiles[sh].empty())
        k_sgemm<S><<<unsigned(p.utiles[sh].size()), NTHR, 0, s>>>(p.d_units.get(), p.d_utiles[sh].get(), p.d_line_b1.get(),
                                                                  p.d_slice_off.get(), p.d_klist.get(), p.w_data(), Tb, Sb, 0);
}

// one ket-sector chunk's T-GEMM tiles, S-GEMM tiles and L.S items (T, S and the coefficient blocks from
// their chunk bases on)
template <class S>
void launch_t_chunk(HeffPlan& p, int sh, const HeffPlan::SChunk& c, const double* x, double* Tb, cudaStream_t s) {
    const uint32_t a = c.tt[0][sh], b = c.tt[1][sh];
    if (b > a)
        k_tgemm<S><<<unsigned(b - a), NTHR, 0, s>>>(p.d_tjobs.get(), p.d_ttiles[sh].get() + a, x, p.r_data(), Tb, nullptr,
                                                    nullptr);
}

template <class S>
void launch_s_chunk(HeffPlan& p, int sh, const HeffPlan::SChunk& c, uint64_t w0, const double* Tb, double* Sb,
                    cudaStream_t s) {
    const uint32_t a = c.ut[0][sh], b = c.ut[1][sh];
    if (b > a)
        k_sgemm<S><<<unsigned(b - a), NTHR, 0, s>>>(p.d_units.get(), p.d_utiles[sh].get() + a, p.d_line_b1.get(),
                                                    p.d_slice_off.get(), p.d_klist.get(), p.d_W.get(), Tb, Sb, w0);
}

template <class S>
void launch_ls_chunk(HeffPlan& p, int sh, const HeffPlan::SChunk& c, const double* Sb, double* Pb, cudaStream_t s) {
    const uint32_t a = c.kt[0][sh], b = c.kt[1][sh];
    if (b > a)
        k_lspart<S><<<unsigned(b - a), NTHR, 0, s>>>(p.d_kitems[sh].get() + a, p.d_otiles[sh].get(), p.d_outs.get(),
                                                     p.d_segs.get(), p.l_data(), Sb, Pb + p.pc_off[sh]);
}

template <class S>
void launch_lsreduce(HeffPlan& p, int sh, const double* Pb, double* y, cudaStream_t s) {
    if (p.kitems[sh].empty()) return;
    const dim3 rg(unsigned(p.otiles[sh].size()), unsigned((S::BM * S::BN + 255) / 256));
    k_lsreduce<S><<<rg, 256, 0, s>>>(p.d_otiles[sh].get(), p.d_outs.get(), Pb + p.pc_off[sh], y);
}

// the S-GEMM tiles of one coefficient chunk, reading the chunk's blocks from the plan's scratch
template <class S>
void launch_s_range(HeffPlan& p, int sh, const HeffPlan::WChunk& ch, const double* Tb, double* Sb, cudaStream_t s) {
    if (ch.t1[sh] > ch.t0[sh])
        k_sgemm<S><<<unsigned(ch.t1[sh] - ch.t0[sh]), NTHR, 0, s>>>(p.d_units.get(), p.d_utiles[sh].get() + ch.t0[sh],
                                                                    p.d_line_b1.get(), p.d_slice_off.get(), p.d_klist.get(),
                                                                    p.d_W.get(), Tb, Sb, ch.w0);
}

template <class S>
void launch_ls(HeffPlan& p, int sh, const double* Sb, double* Pb, double* y, cudaStream_t s) {
    if (p.kitems[sh].empty()) return;
    k_lspart<S><<<unsigned(p.kitems[sh].size()), NTHR, 0, s>>>(p.d_kitems[sh].get(), p.d_otiles[sh].get(), p.d_outs.get(),
                                                               p.d_segs.get(), p.l_data(), Sb, Pb);
    const dim3 rg(unsigned(p.otiles[sh].size()), unsigned((S::BM * S::BN + 255) / 256));
    k_lsreduce<S><<<rg, 256, 0, s>>>(p.d_otiles[sh].get(), p.d_outs.get(), Pb, y);
}

}  // namespace

namespace {
// One H.psi: T-GEMM -> S build -> split-K L.S, with the scratch buffers T, S and P given
// explicitly (the plan's own buffers, or caller-provided memory of the same sizes).
void apply_impl(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev, double* Tb, double* Sb, double* Pb) {
    cudaStream_t s = p.stream;
    if (!p.lists_staged) throw std::runtime_error("heff apply: the plan's work lists are not on the device");
    if (ev) QCM_CUDA(cudaEventRecord(ev[0], s));
    QCM_CUDA(cudaMemsetAsync(y, 0, p.x_len * sizeof(double), s));
    if (p.sector_chunked()) {
        // chunk by chunk: T, coefficient blocks, S and the L.S partials of its ket sectors; the partials
        // of all chunks summed at the end (the phase events mark the chunk loop and the sum)
        for (const HeffPlan::SChunk& c : p.schunks) {
            launch_t_chunk<Sh16>(p, SHAPE_16, c, x, Tb, s);
            launch_t_chunk<Sh32>(p, SHAPE_32, c, x, Tb, s);
            launch_t_chunk<Sh64>(p, SHAPE_64, c, x, Tb, s);
            if (c.s1 > c.s0) QCM_CUDA(cudaMemsetAsync(Sb, 0, (c.s1 - c.s0) * sizeof(double), s));
            const uint64_t w0 = p.chunk_keeps_w ? 0 : c.w0;  // kept blocks: the whole, from element 0
            if (!p.chunk_keeps_w) p.cg.generate_range(p.d_W.get(), c.u0, c.u1, c.w0, c.w1, s);
            launch_s_chunk<Sh16>(p, SHAPE_16, c, w0, Tb, Sb, s);
            launch_s_chunk<Sh32>(p, SHAPE_32, c, w0, Tb, Sb, s);
            launch_s_chunk<Sh64>(p, SHAPE_64, c, w0, Tb, Sb, s);
            launch_s_chunk<Sh128>(p, SHAPE_128, c, w0, Tb, Sb, s);
            launch_ls_chunk<Sh16>(p, SHAPE_16, c, Sb, Pb, s);
            launch_ls_chunk<Sh32>(p, SHAPE_32, c, Sb, Pb, s);
            launch_ls_chunk<Sh64>(p, SHAPE_64, c, Sb, Pb, s);
        }
        if (ev) QCM_CUDA(cudaEventRecord(ev[1], s));
        if (ev) QCM_CUDA(cudaEventRecord(ev[2], s));
        launch_lsreduce<Sh16>(p, SHAPE_16, Pb, y, s);
        launch_lsreduce<Sh32>(p, SHAPE_32, Pb, y, s);
        launch_lsreduce<Sh64>(p, SHAPE_64, Pb, y, s);
        if (ev) QCM_CUDA(cudaEventRecord(ev[3], s));
        QCM_CUDA(cudaGetLastError());
        return;
    }
    launch_t<Sh16>(p, SHAPE_16, x, Tb, s);
    launch_t<Sh32>(p, SHAPE_32, x, Tb, s);
    launch_t<Sh64>(p, SHAPE_64, x, Tb, s);
    if (ev) QCM_CUDA(cudaEventRecord(ev[1], s));
    if (p.s_len) QCM_CUDA(cudaMemsetAsync(Sb, 0, p.s_len * sizeof(double), s));  // rows without lines stay 0
    if (p.streamed()) {
        for (const HeffPlan::WChunk& ch : p.wchunks) {
            p.cg.generate_range(p.d_W.get(), ch.u0, ch.u1, ch.w0, ch.w1, s);
            launch_s_range<Sh16>(p, SHAPE_16, ch, Tb, Sb, s);
            launch_s_range<Sh32>(p, SHAPE_32, ch, Tb, Sb, s);
            launch_s_range<Sh64>(p, SHAPE_64, ch, Tb, Sb, s);
            launch_s_range<Sh128>(p, SHAPE_128, ch, Tb, Sb, s);
        }
    } else {
        launch_s<Sh16>(p, SHAPE_16, Tb, Sb, s);
        launch_s<Sh32>(p, SHAPE_32, Tb, Sb, s);
        launch_s<Sh64>(p, SHAPE_64, Tb, Sb, s);
        launch_s<Sh128>(p, SHAPE_128, Tb, Sb, s);
    }
    if (ev) QCM_CUDA(cudaEventRecord(ev[2], s));
    launch_ls<Sh16>(p, SHAPE_16, Sb, Pb, y, s);
    launch_ls<Sh32>(p, SHAPE_32, Sb, Pb, y, s);
    launch_ls<Sh64>(p, SHAPE_64, Sb, Pb, y, s);
    if (ev) QCM_CUDA(cudaEventRecord(ev[3], s));
    QCM_CUDA(cudaGetLastError());
}
// Mixed form: the T-GEMM (FP64 DMMA) writes T in FP32, the S build runs 3xTF32 on the tensor
// cores from the FP32 coefficient blocks, the L.S GEMM stays FP64.
void apply_mixed_impl(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev, bool tc) {
    cudaStream_t s = p.stream;
    if (!p.lists_staged) throw std::runtime_error("heff apply: the plan's work lists are not on the device");
    prepare_mixed(p, tc);
    if (ev) QCM_CUDA(cudaEventRecord(ev[0], s));
    QCM_CUDA(cudaMemsetAsync(y, 0, p.x_len * sizeof(double), s));
    // T in FP32, or its hi and lo, lives in the bytes of the FP64 T buffer (t_len doubles = 2 t_len floats)
    double* Tb = p.d_T.get();
    float* Thi = reinterpret_cast<float*>(Tb);
    float* Tlo = tc ? Thi + p.t_len : nullptr;
    launch_t<Sh16>(p, SHAPE_16, x, Tb, s, Thi, Tlo);
    launch_t<Sh32>(p, SHAPE_32, x, Tb, s, Thi, Tlo);
    launch_t<Sh64>(p, SHAPE_64, x, Tb, s, Thi, Tlo);
    if (ev) QCM_CUDA(cudaEventRecord(ev[1], s));
    double* Sb = p.d_S.get();
    if (p.s_len) QCM_CUDA(cudaMemsetAsync(Sb, 0, p.s_len * sizeof(double), s));
    if (tc) run_sgemm_mixed(p, true, p.d_W32s.get(), p.d_W32s.get() + p.w_len, Thi, Tlo, Sb, p.d_merr.get(), s);
    else run_sgemm_mixed(p, false, p.d_W32.get(), nullptr, Thi, nullptr, Sb, p.d_merr.get(), s);
    if (ev) QCM_CUDA(cudaEventRecord(ev[2], s));
    launch_ls<Sh16>(p, SHAPE_16, Sb, p.d_P.get(), y, s);
    launch_ls<Sh32>(p, SHAPE_32, Sb, p.d_P.get(), y, s);
    launch_ls<Sh64>(p, SHAPE_64, Sb, p.d_P.get(), y, s);
    if (ev) QCM_CUDA(cudaEventRecord(ev[3], s));
    QCM_CUDA(cudaGetLastError());
}
}  // namespace

void heff_apply_device(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev) {
    apply_impl(p, x, y, ev, p.d_T.get(), p.d_S.get(), p.d_P.get());
}

void heff_tgemm_device(HeffPlan& p, const double* x, double* T) {
    if (!p.lists_staged) throw std::runtime_error("heff T-GEMM: the plan's work lists are not on the device");
    if (p.sector_chunked()) throw std::runtime_error("heff T-GEMM: the plan's apply is chunked by ket sector");
    launch_t<Sh16>(p, SHAPE_16, x, T, p.stream);
    launch_t<Sh32>(p, SHAPE_32, x, T, p.stream);
    launch_t<Sh64>(p, SHAPE_64, x, T, p.stream);
    QCM_CUDA(cudaGetLastError());
}

void prepare_mixed(HeffPlan& p, bool tc) {
    if (p.merged) throw std::runtime_error("a merged plan group applies in FP64 only");
    if (p.streamed() || p.sector_chunked())
        throw std::runtime_error("a plan with streamed coefficient blocks or a chunked apply applies in FP64 only");
    AllocStream scope(p.stream);
    if (!p.d_merr.size()) {
        p.d_merr.alloc(1);
        QCM_CUDA(cudaMemsetAsync(p.d_merr.get(), 0, sizeof(uint32_t), p.stream));
    }
    if (tc && !p.d_W32s.size()) {
        p.d_W32s.alloc(2 * std::max<uint64_t>(p.w_len, 1));
        split_tf32(p.d_W.get(), p.d_W32s.get(), p.d_W32s.get() + p.w_len, p.w_len, p.stream);
    }
    if (!tc && !p.d_W32.size()) {
        p.d_W32.alloc(std::max<uint64_t>(p.w_len, 1));
        to_f32(p.d_W.get(), p.d_W32.get(), p.w_len, p.stream);
    }
}

void check_mixed(HeffPlan& p) {
    if (!p.d_merr.size()) return;
    uint32_t h = 0;
    QCM_CUDA(cudaMemcpyAsync(&h, p.d_merr.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, p.stream));
    QCM_CUDA(cudaStreamSynchronize(p.stream));
    if (h) throw std::runtime_error("mixed H_eff: an S-build tile gave up waiting for its tensor-core MMAs");
}

void heff_apply_device_mixed(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev, bool tc) {
    apply_mixed_impl(p, x, y, ev, tc);
}

void heff_apply_device_scratch(HeffPlan& p, const double* x, double* y, double* Tb, double* Sb, double* Pb) {
    apply_impl(p, x, y, nullptr, Tb, Sb, Pb);
}

void run_tgemm(const TJobD* jobs, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const double* x,
               const double* R, double* T, cudaStream_t s) {
    if (!htiles[SHAPE_16].empty())
        k_tgemm<Sh16><<<unsigned(htiles[SHAPE_16].size()), NTHR, 0, s>>>(jobs, dtiles[SHAPE_16].get(), x, R, T, nullptr, nullptr);
    if (!htiles[SHAPE_32].empty())
        k_tgemm<Sh32><<<unsigned(htiles[SHAPE_32].size()), NTHR, 0, s>>>(jobs, dtiles[SHAPE_32].get(), x, R, T, nullptr, nullptr);
    if (!htiles[SHAPE_64].empty())
        k_tgemm<Sh64><<<unsigned(htiles[SHAPE_64].size()), NTHR, 0, s>>>(jobs, dtiles[SHAPE_64].get(), x, R, T, nullptr, nullptr);
    QCM_CUDA(cudaGetLastError());
}

void run_sgemm(const UnitD* units, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const uint32_t* line_b1,
               const uint64_t* slice_off, const uint16_t* klist, const double* W, const double* T, double* S,
               cudaStream_t s) {
    if (!htiles[SHAPE_16].empty())
        k_sgemm<Sh16><<<unsigned(htiles[SHAPE_16].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_16].get(), line_b1, slice_off, klist, W, T, S, 0);
    if (!htiles[SHAPE_32].empty())
        k_sgemm<Sh32><<<unsigned(htiles[SHAPE_32].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_32].get(), line_b1, slice_off, klist, W, T, S, 0);
    if (!htiles[SHAPE_64].empty())
        k_sgemm<Sh64><<<unsigned(htiles[SHAPE_64].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_64].get(), line_b1, slice_off, klist, W, T, S, 0);
    if (!htiles[SHAPE_128].empty())
        k_sgemm<Sh128><<<unsigned(htiles[SHAPE_128].size()), NTHR, 0, s>>>(units, dtiles[SHAPE_128].get(), line_b1, slice_off, klist, W, T, S, 0);
    QCM_CUDA(cudaGetLastError());
}


int heff_launches_per_apply(const HeffPlan& p) {
    int n = 0;
    for (int sh = 0; sh < N_SHAPES; ++sh) {
        n += !p.ttiles[sh].empty();
        if (!p.streamed()) n += !p.utiles[sh].empty();
        n += p.kitems[sh].empty() ? 0 : 2;
    }
    for (const HeffPlan::WChunk& ch : p.wchunks) {
        n += ch.u1 > ch.u0;  // the chunk's coefficient generation
        for (int sh = 0; sh < N_SHAPES; ++sh) n += ch.t1[sh] > ch.t0[sh];
    }
    if (p.sector_chunked()) {
        n = 0;
        for (const HeffPlan::SChunk& c : p.schunks) {
            n += !p.chunk_keeps_w && c.u1 > c.u0;
            for (int sh = 0; sh < N_SHAPES; ++sh)
                n += (c.tt[1][sh] > c.tt[0][sh]) + (c.ut[1][sh] > c.ut[0][sh]) + (c.kt[1][sh] > c.kt[0][sh]);
        }
        for (int sh = 0; sh < N_SHAPES; ++sh) n += !p.kitems[sh].empty();  // the partial sums
    }
    return n;
}

void release_plan_device(HeffPlan& p) {
    p.d_tjobs.reset();
    for (int sh = 0; sh < N_SHAPES; ++sh) {
        p.d_ttiles[sh].reset(); p.d_utiles[sh].reset(); p.d_otiles[sh].reset(); p.d_kitems[sh].reset();
    }
    p.d_P.reset(); p.d_units.reset(); p.d_line_b1.reset(); p.d_slice_off.reset(); p.d_W.reset(); p.d_klist.reset();
    p.d_segs.reset(); p.d_outs.reset(); p.d_T.reset(); p.d_S.reset(); p.d_W32.reset(); p.d_W32s.reset();
    p.d_merr.reset(); p.d_x.reset(); p.d_y.reset();
    p.adj.reset();
    CoefGen& g = p.cg;
    g.d_units.reset(); g.d_gin.reset(); g.d_line_major.reset(); g.d_smap_id.reset(); g.d_smap_slot.reset();
    g.d_m_ptr.reset(); g.d_m_other.reset(); g.d_m_op.reset(); g.d_o_ptr.reset(); g.d_o_in.reset(); g.d_err.reset();
    g.d_line_scale.reset(); g.d_m_scale.reset(); g.d_o_val.reset(); g.d_b_cs.reset(); g.d_b_pos.reset();
    p.lists_staged = false;
}

void release_plan_scratch(HeffPlan& p) {
    p.d_T.reset(); p.d_S.reset(); p.d_P.reset(); p.d_x.reset(); p.d_y.reset();
    p.d_W32.reset(); p.d_W32s.reset(); p.d_merr.reset();
    p.adj.reset();
    CoefGen& g = p.cg;
    g.d_units.reset(); g.d_gin.reset(); g.d_line_major.reset(); g.d_smap_id.reset(); g.d_smap_slot.reset();
    g.d_m_ptr.reset(); g.d_m_other.reset(); g.d_m_op.reset(); g.d_o_ptr.reset(); g.d_o_in.reset(); g.d_err.reset();
    g.d_line_scale.reset(); g.d_m_scale.reset(); g.d_o_val.reset(); g.d_b_cs.reset(); g.d_b_pos.reset();
}

uint64_t plan_resident_bytes(const HeffPlan& p) {
    uint64_t b = p.d_W.size() * sizeof(double) + p.d_tjobs.size() * sizeof(TJobD) + p.d_units.size() * sizeof(UnitD) +
                 p.d_line_b1.size() * 4 + p.d_slice_off.size() * 8 + p.d_klist.size() * 2 + p.d_segs.size() * sizeof(SegD) +
                 p.d_outs.size() * sizeof(OutD);
    for (int sh = 0; sh < N_SHAPES; ++sh)
        b += (p.d_ttiles[sh].size() + p.d_utiles[sh].size()) * sizeof(TileD) + p.d_otiles[sh].size() * sizeof(OTileD) +
             p.d_kitems[sh].size() * sizeof(KItemD);
    return b;
}

namespace {
void stage_lists(HeffPlan& p);
uint64_t chunk_t_len(const HeffPlan& p);
uint64_t chunk_s_len(const HeffPlan& p);
}

void restage_plan(HeffPlan& p) {
    AllocStream scope(p.stream);
    if (p.streamed() || p.sector_chunked()) {
        // the generation tables of every apply, and its error word (applies allocate nothing)
        p.cg.upload(p.stream);
        if (!p.cg.d_err.size()) {
            p.cg.d_err.alloc(1);
            QCM_CUDA(cudaMemsetAsync(p.cg.d_err.get(), 0, sizeof(uint32_t), p.stream));
        }
    }
    if (!p.lists_staged) {
        stage_lists(p);
        QCM_CUDA(cudaStreamSynchronize(p.stream));
        return;
    }
    p.d_T.alloc(chunk_t_len(p));
    p.d_S.alloc(chunk_s_len(p));
    p.d_P.alloc(p.sector_chunked() ? p.pc_len : p.p_len);
}

void rebind_plan(HeffPlan& p, const DevBoundary& L, const DevBoundary& R) {
    p.L = &L;
    p.R = &R;
    p.cg.b_cs = &R.idx.cscale;  // the coefficient generation reads the right boundary's conjugate scales
}

// The merged plan's work lists (member plans validated each against their own buffers when staged;
// here the merged T, S and k-step lists are checked again) and its own T, S and partial buffers.
void upload_merged(HeffPlan& p) {
    cudaStream_t s = p.stream;
    for (const TJobD& j : p.tjobs)
        if (j.brs == 0 || j.N % j.brs || j.sst < j.brs * j.M || j.sst % 4 || j.c_off % 4 ||
            j.c_off + uint64_t(j.N / j.brs) * j.sst > p.t_len || j.a_off + uint64_t(j.K ? j.K - 1 : 0) * j.lda + j.M > p.x_len)
            throw std::runtime_error("plan group: T job outside the merged buffers");
    for (const UnitD& u : p.units)
        if (u.nk && u.slice0 + u.nk > p.slice_off.size()) throw std::runtime_error("plan group: unit outside its slices");
    for (std::size_t k = 0; k < p.slice_off.size(); ++k)
        if (p.slice_off[k] % 4 || p.slice_off[k] > p.t_len) throw std::runtime_error("plan group: T slice misplaced");
    for (int sh = 0; sh < N_SHAPES; ++sh)
        for (const TileD& t : p.utiles[sh])
            if (t.item >= p.units.size() || std::size_t(t.pad) >= p.klist.size() ||
                std::size_t(t.pad) + 1 + p.klist[t.pad] > p.klist.size())
                throw std::runtime_error("plan group: S tile outside its work lists");
    for (const OutD& o : p.outs)
        if (o.y_off + uint64_t(o.M) * o.N > p.x_len || o.seg_start + o.seg_count > p.segs.size())
            throw std::runtime_error("plan group: output block outside the arena");
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
    p.d_klist.upload(p.klist, s);
    p.d_segs.upload(p.segs, s);
    p.d_outs.upload(p.outs, s);
    p.d_T.alloc(p.t_len);
    p.d_S.alloc(p.s_len);
    p.d_P.alloc(p.p_len);
    p.lists_staged = true;
    QCM_CUDA(cudaStreamSynchronize(s));
}

namespace {

// T and S scratch of one apply: the whole buffers, or the largest ket-sector chunk's
uint64_t chunk_t_len(const HeffPlan& p) {
    if (!p.sector_chunked()) return p.t_len;
    uint64_t m = 1;
    for (const HeffPlan::SChunk& c : p.schunks) m = std::max(m, c.t1 - c.t0);
    return m;
}
uint64_t chunk_s_len(const HeffPlan& p) {
    if (!p.sector_chunked()) return p.s_len;
    uint64_t m = 1;
    for (const HeffPlan::SChunk& c : p.schunks) m = std::max(m, c.s1 - c.s0);
    return m;
}

// the work lists and the scratch of one plan on the device
void stage_lists(HeffPlan& p) {
    cudaStream_t s = p.stream;
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
    p.d_klist.upload(p.klist, s);
    p.d_segs.upload(p.segs, s);
    p.d_outs.upload(p.outs, s);
    p.d_T.alloc(chunk_t_len(p));
    p.d_S.alloc(chunk_s_len(p));
    p.d_P.alloc(p.sector_chunked() ? p.pc_len : p.p_len);
    p.lists_staged = true;
}

}  // namespace

void upload_plan(HeffPlan& p, bool lists) {
    cudaStream_t s = p.stream;
    for (const UnitD& u : p.units)
        if (u.wld < u.nl || u.wld % 4 || u.w_off % 4 || u.w_off + uint64_t(u.wld) * u.nk > p.w_len ||
            (u.nk && u.slice0 + u.nk > p.slice_off.size()))
            throw std::runtime_error("heff plan: unit outside its work lists");
    for (const TJobD& j : p.tjobs)
        if (j.brs == 0 || j.N % j.brs || j.sst < j.brs * j.M || j.sst % 4 || j.c_off % 4 ||
            j.c_off + uint64_t(j.N / j.brs) * j.sst > p.t_len)
            throw std::runtime_error("heff plan: T job outside the T buffer");
    for (std::size_t k = 0; k < p.slice_off.size(); ++k)
        if (p.slice_off[k] % 4) throw std::runtime_error("heff plan: T slice not 16-byte aligned");
    for (int sh = 0; sh < N_SHAPES; ++sh)
        for (const TileD& t : p.utiles[sh]) {
            if (t.item >= p.units.size() || std::size_t(t.pad) >= p.klist.size() ||
                std::size_t(t.pad) + 1 + p.klist[t.pad] > p.klist.size())
                throw std::runtime_error("heff plan: S tile outside its work lists");
            for (uint32_t i = 0; i < p.klist[t.pad]; ++i)
                if (uint32_t(p.klist[t.pad + 1 + i] >> 4) * BK >= p.units[t.item].nk) throw std::runtime_error("heff plan: S tile k-step out of range");
        }
    if (lists) stage_lists(p);
    p.cg.upload(s);
    // dense coefficient blocks, built once per plan and reused by every apply
    if (p.streamed() || (p.sector_chunked() && !p.chunk_keeps_w)) {
        // one chunk's scratch; every chunk generated once here so that a term without a slot is found
        // when the plan is staged (each apply generates them again, unchecked)
        uint64_t mx = 1;
        for (const HeffPlan::WChunk& ch : p.wchunks) mx = std::max(mx, ch.w1 - ch.w0);
        for (const HeffPlan::SChunk& c : p.schunks) mx = std::max(mx, c.w1 - c.w0);
        p.d_W.alloc(mx);
        for (const HeffPlan::WChunk& ch : p.wchunks) p.cg.generate_range(p.d_W.get(), ch.u0, ch.u1, ch.w0, ch.w1, s);
        for (const HeffPlan::SChunk& c : p.schunks) p.cg.generate_range(p.d_W.get(), c.u0, c.u1, c.w0, c.w1, s);
        p.cg.check_generated(s);
        return;
    }
    p.d_W.alloc(p.w_len ? p.w_len : 1);
    static const bool tdbg = std::getenv("QCM_PLAN_TIMING") != nullptr;
    auto now = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    double t0 = 0;
    if (tdbg) {
        QCM_CUDA(cudaStreamSynchronize(s));
        t0 = now();
    }
    p.cg.generate(p.d_W.get(), s);
    QCM_CUDA(cudaStreamSynchronize(s));
    if (tdbg)
        std::fprintf(stderr, "plan upload: coefficient generation %.4f s (%llu terms, %llu coefficients)\n", now() - t0,
                     (unsigned long long)p.n_alpha, (unsigned long long)p.w_len);
}

}  // namespace qcm

namespace qcm {

void stream_coefficients(HeffPlan& p, uint64_t max_doubles) {
    p.wchunks.clear();
    if (p.merged) throw std::runtime_error("stream_coefficients: a merged plan group keeps its members' blocks");
    if (!max_doubles || p.w_len <= max_doubles || p.units.empty()) return;
    if (p.cg.units.size() != p.units.size()) throw std::runtime_error("stream_coefficients: generation units differ from the plan's");
    for (std::size_t i = 0; i < p.units.size(); ++i)
        if (p.cg.units[i].w_off != p.units[i].w_off || (i && p.units[i].w_off < p.units[i - 1].w_off))
            throw std::runtime_error("stream_coefficients: coefficient blocks out of unit order");
    auto wend = [&](std::size_t i) { return p.units[i].w_off + uint64_t(p.units[i].wld) * p.units[i].nk; };
    HeffPlan::WChunk ch;
    ch.u0 = 0;
    ch.w0 = p.units[0].w_off;
    for (std::size_t i = 1; i <= p.units.size(); ++i) {
        if (i < p.units.size() && wend(i) - ch.w0 <= max_doubles) continue;
        ch.u1 = uint32_t(i);
        ch.w1 = i < p.units.size() ? p.units[i].w_off : p.w_len;
        p.wchunks.push_back(ch);
        if (i < p.units.size()) { ch = HeffPlan::WChunk(); ch.u0 = uint32_t(i); ch.w0 = p.units[i].w_off; }
    }
    // each shape's tiles are in unit order: a chunk's are one range
    for (int sh = 0; sh < N_SHAPES; ++sh) {
        const std::vector<TileD>& t = p.utiles[sh];
        for (std::size_t k = 1; k < t.size(); ++k)
            if (t[k].item < t[k - 1].item) throw std::runtime_error("stream_coefficients: S tiles out of unit order");
        std::size_t k = 0;
        for (HeffPlan::WChunk& c : p.wchunks) {
            while (k < t.size() && t[k].item < c.u0) ++k;
            c.t0[sh] = uint32_t(k);
            while (k < t.size() && t[k].item < c.u1) ++k;
            c.t1[sh] = uint32_t(k);
        }
    }
}

}  // namespace qcm

namespace qcm {

namespace {

// adds (sign +1) or removes (-1) the chunk bases of a chunked plan's T and S offsets
void rebase_chunks(HeffPlan& p, int sign) {
    for (std::size_t c = 0; c < p.schunks.size(); ++c) {
        const HeffPlan::SChunk& ch = p.schunks[c];
        const uint64_t t0 = ch.t0, s0 = ch.s0;
        auto shift = [sign](uint64_t& v, uint64_t b) { v = sign > 0 ? v + b : v - b; };
        for (uint32_t j = p.part_job[ch.p0]; j < p.part_job[ch.p1]; ++j) shift(p.tjobs[j].c_off, t0);
        for (uint32_t u = ch.u0; u < ch.u1; ++u) {
            UnitD& U = p.units[u];
            shift(U.s_off, s0);
            for (uint32_t k = 0; k < U.nk; ++k) shift(p.slice_off[U.slice0 + k], t0);
        }
        for (std::size_t g = 0; g < p.segs.size(); ++g)
            if (p.seg_chunk[g] == c) shift(p.segs[g].s_off, s0);
    }
}

}  // namespace

void chunk_sectors(HeffPlan& p, uint64_t max_doubles) {
    if (p.sector_chunked()) rebase_chunks(p, +1);  // back to whole-buffer offsets first
    p.schunks.clear();
    p.seg_chunk.clear();
    if (p.merged) throw std::runtime_error("chunk_sectors: a merged plan group");
    if (!max_doubles || p.t_len + p.s_len + p.w_len <= max_doubles) return;
    if (p.part_t.size() < 2) throw std::runtime_error("chunk_sectors: the plan has no ket-sector prefixes");
    p.wchunks.clear();  // the chunks below generate their own coefficient blocks
    const std::size_t np = p.part_t.size() - 1;
    p.chunk_keeps_w = p.w_len <= max_doubles / 2;
    const uint64_t room = p.chunk_keeps_w ? max_doubles - p.w_len : max_doubles;
    auto size = [&](std::size_t a, std::size_t b) {
        return (p.part_t[b] - p.part_t[a]) + (p.part_s[b] - p.part_s[a]) +
               (p.chunk_keeps_w ? 0 : p.part_w[b] - p.part_w[a]);
    };
    std::vector<uint32_t> chunk_of(np);
    std::size_t a = 0;
    for (std::size_t i = 1; i <= np; ++i) {
        if (i < np && size(a, i + 1) <= room) continue;
        HeffPlan::SChunk c;
        c.p0 = uint32_t(a); c.p1 = uint32_t(i);
        c.u0 = p.part_unit[a]; c.u1 = p.part_unit[i];
        c.t0 = p.part_t[a]; c.t1 = p.part_t[i];
        c.s0 = p.part_s[a]; c.s1 = p.part_s[i];
        c.w0 = p.part_w[a]; c.w1 = p.part_w[i];
        for (std::size_t k = a; k < i; ++k) chunk_of[k] = uint32_t(p.schunks.size());
        p.schunks.push_back(c);
        a = i;
    }
    const std::size_t nc = p.schunks.size();
    // the ket sector of a T job, an S unit and an L.S segment (by its S rows)
    auto part_of = [](const auto& pre, uint64_t v) {
        return std::size_t(std::upper_bound(pre.begin(), pre.end(), v) - pre.begin()) - 1;
    };
    for (int sh = 0; sh < N_SHAPES; ++sh) {
        // each list grouped by chunk, in its order within a chunk (the tiles write disjoint parts of T and
        // S, and an L.S item its own partial slot, so the order of the launches does not matter)
        // returns the chunk boundaries in the regrouped list
        auto regroup = [&](auto& list, auto chunk_fn) {
            std::vector<std::size_t> cnt(nc + 1, 0);
            for (const auto& e : list) ++cnt[chunk_fn(e) + 1];
            for (std::size_t c = 0; c < nc; ++c) cnt[c + 1] += cnt[c];
            std::remove_reference_t<decltype(list)> out(list.size());
            std::vector<std::size_t> pos(cnt.begin(), cnt.end() - 1);
            for (const auto& e : list) out[pos[chunk_fn(e)]++] = e;
            list.swap(out);
            return cnt;
        };
        auto tcnt = regroup(p.ttiles[sh], [&](const TileD& t) { return chunk_of[part_of(p.part_job, t.item)]; });
        auto ucnt = regroup(p.utiles[sh], [&](const TileD& t) { return chunk_of[part_of(p.part_unit, t.item)]; });
        auto kcnt = regroup(p.kitems[sh], [&](const KItemD& k) { return chunk_of[part_of(p.part_s, p.segs[k.seg].s_off)]; });
        for (std::size_t c = 0; c < nc; ++c) {
            HeffPlan::SChunk& ch = p.schunks[c];
            ch.tt[0][sh] = uint32_t(tcnt[c]); ch.tt[1][sh] = uint32_t(tcnt[c + 1]);
            ch.ut[0][sh] = uint32_t(ucnt[c]); ch.ut[1][sh] = uint32_t(ucnt[c + 1]);
            ch.kt[0][sh] = uint32_t(kcnt[c]); ch.kt[1][sh] = uint32_t(kcnt[c + 1]);
        }
    }
    p.seg_chunk.resize(p.segs.size());
    for (std::size_t g = 0; g < p.segs.size(); ++g) p.seg_chunk[g] = chunk_of[part_of(p.part_s, p.segs[g].s_off)];
    // each shape's partials in a region of its own
    p.pc_len = 0;
    for (int sh = 0; sh < N_SHAPES; ++sh) {
        p.pc_off[sh] = p.pc_len;
        p.pc_len += uint64_t(p.kitems[sh].size()) * shape_bm(sh) * shape_bn(sh);
    }
    p.pc_len = std::max<uint64_t>(p.pc_len, 1);
    // every chunk's T slices, S rows and coefficient blocks lie in its ranges
    for (std::size_t c = 0; c < nc; ++c) {
        const HeffPlan::SChunk& ch = p.schunks[c];
        for (int sh = 0; sh < N_SHAPES; ++sh) {
            for (uint32_t i = ch.tt[0][sh]; i < ch.tt[1][sh]; ++i) {
                const TJobD& j = p.tjobs[p.ttiles[sh][i].item];
                if (j.c_off < ch.t0 || j.c_off + uint64_t(j.N / j.brs) * j.sst > ch.t1)
                    throw std::runtime_error("chunk_sectors: T job outside its chunk");
            }
            for (uint32_t i = ch.ut[0][sh]; i < ch.ut[1][sh]; ++i) {
                const UnitD& u = p.units[p.utiles[sh][i].item];
                if (u.s_off < ch.s0 || u.s_off > ch.s1 || u.w_off < ch.w0 || u.w_off + uint64_t(u.wld) * u.nk > ch.w1)
                    throw std::runtime_error("chunk_sectors: S unit outside its chunk");
                for (uint32_t k = 0; k < u.nk; ++k)
                    if (p.slice_off[u.slice0 + k] < ch.t0 || p.slice_off[u.slice0 + k] >= ch.t1)
                        throw std::runtime_error("chunk_sectors: T slice outside its chunk");
            }
            for (uint32_t i = ch.kt[0][sh]; i < ch.kt[1][sh]; ++i) {
                const SegD& g = p.segs[p.kitems[sh][i].seg];
                if (g.s_off < ch.s0 || g.s_off > ch.s1) throw std::runtime_error("chunk_sectors: L.S segment outside its chunk");
            }
        }
    }
    rebase_chunks(p, -1);
}

}  // namespace qcm
