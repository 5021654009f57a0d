// Adjoint of the H_eff apply (the differentiation form of the path).  For f = ybar . H_eff(W) x:
//   psi_bar   = H_eff^T ybar = H_eff ybar: the two-site H_eff of a Hermitian MPO is symmetric;
//   coeff_bar = df / d scale_e for every entry e of the plan's two-site MPO tensor.
// f is linear in every scale.  Each coefficient term that k_wgen sums into the dense block W_u
// (lines x slots) of an S-build unit is alpha = o_val * b_cs * (scale_e * line_scale), and the unit's
// S rows are S_u = W_u T_u (create_s_r, tasks.cpp:466-494, as a dense GEMM).  So
//   Sbar      = L_eff^T ybar per L.S segment       (transpose of contract, tasks.cpp:286-313),
//   Wbar_u    = Sbar_u T_u^T per unit              (k_wbar, DMMA, in the coefficient-block layout),
//   coeff_bar = sum over the terms of entry e of Wbar_u(line, slot) * o_val * b_cs * line_scale.
// The last runs k_wgen's traversal backwards.  One thread per line writes the line's partial sum for
// every entry of its MPO row (k_wadj).  Then one thread per entry adds the partials of the lines of
// its row in increasing line order (k_entry_sum).  There are no atomics, so the result does not
// vary from run to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "dev_ops.hpp"
#include "dmma.cuh"
#include "heff.hpp"

namespace qcm {

struct HeffAdjointWork {
    std::vector<TileD> tiles;  // k_wbar: (unit, first line, first slot) per 64 x 64 tile of Wbar
    DBuf<TileD> d_tiles;
    DBuf<double> d_Wb;          // Wbar, the coefficient-block layout (w_len doubles)
    DBuf<double> d_P;           // per line, one partial per entry of its MPO row
    DBuf<uint64_t> d_pofs;      // per line: offset of its partials in P
    DBuf<uint32_t> d_rl_ptr, d_rl_line, d_e_row;  // lines grouped by MPO row (CSR); MPO row per entry
    DBuf<uint32_t> d_err;
    std::vector<GemmJob> sjobs;  // Sbar = L^T ybar per segment
    DBuf<GemmJob> d_jobs;
    DBuf<uint32_t> d_jtiles;
    uint64_t p_len = 0, n_terms = 0;
};

namespace {

using namespace dm;
using SW = Sh64;

// Wbar_u(line, slot) = sum_e Sbar(S row block line_b1[line], element e) * T(slice of slot, e); one CTA
// per 64 x 64 tile, K = the unit's elements.
__global__ void __launch_bounds__(NTHR) k_wbar(const UnitD* __restrict__ units, const TileD* __restrict__ tiles,
                                               const uint32_t* __restrict__ line_b1, const uint64_t* __restrict__ slice_off,
                                               const double* __restrict__ Sb, const double* __restrict__ T,
                                               double* __restrict__ Wb) {
    __shared__ Stage<SW> st[2];
    __shared__ uint64_t soff[SW::BN], lrow[SW::BM];
    const TileD tile = tiles[blockIdx.x];
    const UnitD U = units[tile.item];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int c = tid; c < SW::BN; c += NTHR) {
        const uint32_t n = tile.n0 + c;
        soff[c] = n < U.nk ? slice_off[U.slice0 + n] : 0;
    }
    // S row block of each line of the tile (the rows k_sgemm writes for it)
    for (int c = tid; c < SW::BM; c += NTHR) {
        const uint32_t l = tile.m0 + c;
        lrow[c] = l < U.nl ? U.s_off + uint64_t(line_b1[U.line0 + l]) * U.line_stride : 0;
    }
    __syncthreads();
    auto issue = [&](int sidx, uint32_t k0) {
        Stage<SW>& s = st[sidx];
        // element-fastest thread order: consecutive threads read consecutive rows of a slice column
#pragma unroll
        for (int rr = 0; rr < SW::A_PER; ++rr) {
            const int e = tid + rr * NTHR;
            const int k = e % BK, m = e / BK;
            const uint32_t gm = tile.m0 + m, ge = k0 + k;
            const bool ok = gm < U.nl && ge < U.ne;
            uint64_t a = 0;
            if (ok) {
                const uint32_t c = ge / U.erows, r = ge - c * U.erows;
                a = lrow[m] + r + uint64_t(c) * U.col_stride;
            }
            cp8(&s.A[k][m], Sb + a, ok);
        }
#pragma unroll
        for (int rr = 0; rr < SW::B_PER; ++rr) {
            const int e = tid + rr * NTHR;
            const int k = e % BK, n = e / BK;
            const uint32_t gn = tile.n0 + n, ge = k0 + k;
            const bool ok = gn < U.nk && ge < U.ne;
            cp8(&s.B[k][n], ok ? T + soff[n] + ge : T, ok);
        }
        cp_commit();
    };
    Acc<SW> acc;
    acc.zero();
    const uint32_t nk = (U.ne + BK - 1) / BK;
    if (nk) issue(0, 0);
    for (uint32_t kc = 0; kc < nk; ++kc) {
        cp_wait_all();
        __syncthreads();
        if (kc + 1 < nk) issue((kc + 1) & 1, (kc + 1) * BK);
        mma_stage<SW>(st[kc & 1].A, st[kc & 1].B, acc, warp, lane);
    }
    for_acc<SW>(acc, warp, lane, [&](int m, int n, double v) {
        const uint32_t gm = tile.m0 + m, gn = tile.n0 + n;
        if (gm < U.nl && gn < U.nk) Wb[U.w_off + gm + uint64_t(gn) * U.wld] = v;
    });
}

constexpr int WA_THR = 128;
constexpr uint32_t WA_SMAP = 4096;  // (slice id, slot) pairs staged in shared memory
constexpr uint32_t WA_NST = 64;     // physical states of the basis (CoefGen::validate bounds nst)

// Per line: P[pofs[line] + (e - m_ptr[m])] = sum over the terms of entry e (row m of the line) of
// Wbar(line, slot) * o_val * b_cs * line_scale; the traversal and slot lookup of k_wgen.
__global__ void __launch_bounds__(WA_THR) k_wadj(const WGenUnitD* __restrict__ units, const WGenInD* __restrict__ gin,
                                                 uint32_t nst, const uint32_t* __restrict__ line_major,
                                                 const double* __restrict__ line_scale,
                                                 const uint32_t* __restrict__ smap_id, const uint32_t* __restrict__ smap_slot,
                                                 const uint32_t* __restrict__ m_ptr, const uint32_t* __restrict__ m_other,
                                                 const uint32_t* __restrict__ m_op, const uint32_t* __restrict__ o_ptr,
                                                 const uint32_t* __restrict__ o_in, const double* __restrict__ o_val,
                                                 const int32_t* __restrict__ b_pos, const double* __restrict__ b_cs,
                                                 uint32_t b_aux, const double* __restrict__ Wb,
                                                 const uint64_t* __restrict__ pofs, double* __restrict__ P,
                                                 uint32_t* __restrict__ err) {
    __shared__ uint32_t sid[WA_SMAP], sslot[WA_SMAP];
    __shared__ WGenInD sin[WA_NST];
    const WGenUnitD U = units[blockIdx.x];
    const bool staged = U.nk <= WA_SMAP;
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
        const uint32_t gl = U.line0 + line;
        const uint32_t m = line_major[gl];
        const double lsc = line_scale[gl];
        const double* Wl = Wb + U.w_off + line;
        double* Pl = P + pofs[gl];
        const uint32_t e0 = m_ptr[m];
        for (uint32_t e = e0; e < m_ptr[m + 1]; ++e) {
            const uint32_t x = m_other[e], op = m_op[e];
            const std::size_t q = std::size_t(op) * nst + U.st_out;
            double acc = 0.0;
            for (uint32_t k = o_ptr[q]; k < o_ptr[q + 1]; ++k) {
                const WGenInD g = sin[o_in[k]];
                if (g.c == WGEN_NONE) continue;
                const std::size_t bq = std::size_t(g.c) * b_aux + x;
                const int32_t pos = b_pos[bq];
                if (pos < 0) continue;
                const uint32_t id = g.jbase + uint32_t(pos);
                uint32_t lo = 0, hi = U.nk;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (ids[mid] < id) lo = mid + 1;
                    else hi = mid;
                }
                if (lo >= U.nk || ids[lo] != id) { atomicOr(err, 1u); continue; }
                const double d = __dmul_rn(__dmul_rn(o_val[k], b_cs[bq]), lsc);  // d alpha / d scale_e
                acc = fma(Wl[uint64_t(slots[lo]) * U.wld], d, acc);
            }
            Pl[e - e0] = acc;
        }
    }
}

// out[e] = sum over the lines of e's MPO row (increasing line order) of their partial for e
__global__ void k_entry_sum(uint64_t n_terms, const uint32_t* __restrict__ e_row, const uint32_t* __restrict__ m_ptr,
                            const uint32_t* __restrict__ rl_ptr, const uint32_t* __restrict__ rl_line,
                            const uint64_t* __restrict__ pofs, const double* __restrict__ P, double* __restrict__ out) {
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < n_terms; e += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t m = e_row[e];
        const uint64_t j = e - m_ptr[m];
        double s = 0.0;
        for (uint32_t t = rl_ptr[m]; t < rl_ptr[m + 1]; ++t) s += P[pofs[rl_line[t]] + j];
        out[e] = s;
    }
}

HeffAdjointWork& adjoint_work(HeffPlan& p) {
    if (p.adj) return *p.adj;
    const CoefGen& cg = p.cg;
    if (!cg.by_row || !cg.mt) throw std::runtime_error("heff adjoint: plan without row-major coefficient tables");
    if (!p.L || !p.R) throw std::runtime_error("heff adjoint: plan without boundaries");
    const MPOTables& mt = *cg.mt;
    auto w = std::make_shared<HeffAdjointWork>();
    w->n_terms = mt.row_other.size();
    for (uint32_t i = 0; i < uint32_t(p.units.size()); ++i) {
        const UnitD& u = p.units[i];
        // every Sbar element and T slice element k_wbar reads lies in its buffer
        if (u.nl && u.ne) {
            if (!u.erows) throw std::runtime_error("heff adjoint: unit without element rows");
            auto at = [&](uint32_t e) { return uint64_t(e % u.erows) + uint64_t(e / u.erows) * u.col_stride; };
            uint64_t emax = at(u.ne - 1);
            if (u.ne > u.erows) emax = std::max(emax, at((u.ne - 1) / u.erows * u.erows - 1));
            uint32_t bmax = 0;
            for (uint32_t l = 0; l < u.nl; ++l) bmax = std::max(bmax, p.line_b1.at(std::size_t(u.line0) + l));
            if (u.s_off + uint64_t(bmax) * u.line_stride + emax >= p.s_len)
                throw std::runtime_error("heff adjoint: unit rows outside the S buffer");
            for (uint32_t k = 0; k < u.nk; ++k)
                if (p.slice_off[u.slice0 + k] + u.ne > p.t_len) throw std::runtime_error("heff adjoint: slice outside T");
        }
        for (uint32_t m0 = 0; m0 < u.nl; m0 += SW::BM)
            for (uint32_t n0 = 0; n0 < u.nk; n0 += SW::BN) w->tiles.push_back(TileD{i, m0, n0, 0});
    }
    // partials: per line (global line order), one per entry of its MPO row
    const std::size_t nlines = cg.line_major.size();
    const uint32_t rows = uint32_t(mt.row_ptr.size() - 1);
    std::vector<uint64_t> pofs(nlines);
    std::vector<uint32_t> rl_ptr(std::size_t(rows) + 1, 0), rl_line(nlines), e_row(w->n_terms);
    uint64_t acc = 0;
    for (std::size_t gl = 0; gl < nlines; ++gl) {
        const uint32_t m = cg.line_major[gl];
        if (m >= rows) throw std::runtime_error("heff adjoint: line outside the MPO rows");
        pofs[gl] = acc;
        acc += mt.row_ptr[m + 1] - mt.row_ptr[m];
        rl_ptr[m + 1]++;
    }
    w->p_len = acc;
    for (uint32_t m = 0; m < rows; ++m) rl_ptr[m + 1] += rl_ptr[m];
    {
        std::vector<uint32_t> fill(rl_ptr.begin(), rl_ptr.end() - 1);
        for (std::size_t gl = 0; gl < nlines; ++gl) rl_line[fill[cg.line_major[gl]]++] = uint32_t(gl);
    }
    for (uint32_t m = 0; m < rows; ++m)
        for (uint32_t e = mt.row_ptr[m]; e < mt.row_ptr[m + 1]; ++e) e_row[e] = m;
    // Sbar = L^T ybar per segment (the L.S GEMM's operands, transposed)
    for (const OutD& o : p.outs)
        for (uint32_t k = 0; k < o.seg_count; ++k) {
            const SegD& sg = p.segs[o.seg_start + k];
            GemmJob j{};
            j.a_off = sg.l_off; j.b_off = o.y_off; j.c_off = sg.s_off;
            j.M = sg.nS * sg.ls_in; j.N = o.N; j.K = o.M;
            j.ldb = o.M; j.ldc = sg.nS * sg.ls_in;
            j.tb = 0; j.alpha = 1.0; j.beta = 0.0;
            if (!sg.tr) {
                // L_eff = the cohort's nS blocks (M x ls_in each) side by side: Sbar = L_eff^T ybar
                j.lda = o.M; j.ta = 1;
            } else {
                // a transposed cohort reads its Hermitian partner's blocks (ls_in x M each), so block b of
                // L_eff^T is the stored block itself: row blocks of ls_in rows, block b at b * M * ls_in
                j.lda = sg.ls_in; j.ta = 0;
                j.arb = sg.ls_in; j.a_bs = uint64_t(o.M) * sg.ls_in;
            }
            w->sjobs.push_back(j);
        }
    cudaStream_t s = p.stream;
    w->d_tiles.upload(w->tiles, s);
    w->d_Wb.alloc(p.w_len ? p.w_len : 1);
    w->d_P.alloc(w->p_len ? w->p_len : 1);
    w->d_pofs.upload(pofs, s);
    w->d_rl_ptr.upload(rl_ptr, s);
    w->d_rl_line.upload(rl_line, s);
    w->d_e_row.upload(e_row, s);
    w->d_err.alloc(1);
    p.adj = w;
    return *w;
}

}  // namespace

uint64_t heff_adjoint_terms(const HeffPlan& p) { return p.cg.mt ? p.cg.mt->row_other.size() : 0; }

void heff_adjoint_device(HeffPlan& p, const double* x, const double* ybar, double* psi_bar, double* coeff_bar) {
    cudaStream_t s = p.stream;
    if (p.sector_chunked()) throw std::runtime_error("heff adjoint: the plan's apply is chunked by ket sector");
    if (psi_bar) heff_apply_device(p, ybar, psi_bar);
    if (!coeff_bar) return;
    HeffAdjointWork& w = adjoint_work(p);
    if (!w.n_terms) return;
    double* T = p.d_T.get();
    double* Sb = p.d_S.get();
    heff_tgemm_device(p, x, T);
    if (p.s_len) QCM_CUDA(cudaMemsetAsync(Sb, 0, p.s_len * sizeof(double), s));
    if (!w.sjobs.empty())
        batched_gemm(w.sjobs, p.L->data.get(), p.L->data.size(), ybar, p.x_len, Sb, p.s_len, w.d_jobs, w.d_jtiles, s);
    if (!w.tiles.empty())
        k_wbar<<<unsigned(w.tiles.size()), NTHR, 0, s>>>(p.d_units.get(), w.d_tiles.get(), p.d_line_b1.get(),
                                                         p.d_slice_off.get(), Sb, T, w.d_Wb.get());
    QCM_CUDA(cudaGetLastError());
    const CoefGen& cg = p.cg;
    QCM_CUDA(cudaMemsetAsync(w.d_err.get(), 0, sizeof(uint32_t), s));
    if (!cg.units.empty())
        k_wadj<<<unsigned(cg.units.size()), WA_THR, 0, s>>>(
            cg.d_units.get(), cg.d_gin.get(), cg.nst, cg.d_line_major.get(), cg.d_line_scale.get(), cg.d_smap_id.get(),
            cg.d_smap_slot.get(), cg.d_m_ptr.get(), cg.d_m_other.get(), cg.d_m_op.get(), cg.d_o_ptr.get(), cg.d_o_in.get(),
            cg.d_o_val.get(), cg.d_b_pos.get(), cg.d_b_cs.get(), cg.b_aux, w.d_Wb.get(), w.d_pofs.get(), w.d_P.get(),
            w.d_err.get());
    QCM_CUDA(cudaGetLastError());
    const unsigned grid = unsigned(std::min<uint64_t>((w.n_terms + 255) / 256, 148 * 16));
    k_entry_sum<<<grid, 256, 0, s>>>(w.n_terms, w.d_e_row.get(), cg.d_m_ptr.get(), w.d_rl_ptr.get(), w.d_rl_line.get(),
                                     w.d_pofs.get(), w.d_P.get(), coeff_bar);
    QCM_CUDA(cudaGetLastError());
    uint32_t h = 0;
    QCM_CUDA(cudaMemcpyAsync(&h, w.d_err.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    QCM_CUDA(cudaStreamSynchronize(s));
    if (h) throw std::runtime_error("heff adjoint: a coefficient term has no slice slot");
}

}  // namespace qcm
