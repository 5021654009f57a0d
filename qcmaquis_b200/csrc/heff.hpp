// Two-site effective Hamiltonian on one B200: boundaries resident in HBM and the
// flattened contraction schedule ("plan").
//
// Reference path (solver/tasks.cpp, solver/super_hamil_mv.hpp): per ket sector
// lb_in, T[ti] = psi_slab * R[ci_eff] (create_T, :650-705); per (lb_in, lb_out)
// cohort, S = sum alpha * T-slices (create_s_r, :466-494) and out[lb_out] +=
// L[ci_eff] * S (contract, :286-313), with the output accumulated under a
// mutex (CPU) or with atomics (GPU).
//
// B200 form: the whole H.psi is three launches over flat work lists --
//   (1) one grouped FP64 GEMM over every T job of every sector,
//   (2) one gather launch building every cohort's S (HBM-bound),
//   (3) one grouped FP64 GEMM per output tile whose K loop runs over all
//       cohorts writing that output block (deterministic, no atomics).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <unordered_map>
#include <vector>

#include "device.hpp"
#include "mpo.hpp"
#include "symm.hpp"

namespace qcm {

// Boundary index (mp_tensors/boundary.h:76-234): cohorts keyed by (bra, ket)
// sector positions; per cohort aux_dim block offsets (-1 = absent), conjugate
// scales, the transposed-storage flag tr and block shapes lsz x rsz.
struct BoundaryIndexH {
    Index bra, ket;
    uint32_t aux = 0;
    std::vector<uint32_t> cbra, cket, lsz, rsz, nb;
    std::vector<uint8_t> tr;
    std::vector<int64_t> offsets;  // ncoh * aux
    std::vector<double> cscale;    // ncoh * aux
    std::vector<uint64_t> data_off;  // element offset of each cohort in the device buffer
    uint64_t total = 0;
    std::vector<std::vector<uint32_t>> lbrb;

    uint32_t n_cohorts() const { return uint32_t(cbra.size()); }
    uint32_t cohort_index(Charge l, Charge r) const {
        std::size_t a = bra.position(l), b = ket.position(r);
        if (a >= bra.size() || b >= ket.size()) return n_cohorts();
        return lbrb[a][b];
    }
    bool has_block(uint32_t ci, uint32_t b) const { return ci < n_cohorts() && b < aux && offsets[std::size_t(ci) * aux + b] > -1; }
    int64_t offset(uint32_t ci, uint32_t b) const { return offsets[std::size_t(ci) * aux + b]; }
    double conj_scale(uint32_t ci, uint32_t b) const { return cscale[std::size_t(ci) * aux + b]; }
    uint64_t cohort_size(uint32_t ci) const { return uint64_t(nb[ci]) * lsz[ci] * rsz[ci]; }
    void finish();  // builds lbrb, data offsets
};

struct DevBoundary {
    BoundaryIndexH idx;
    DBuf<double> data;
};

// Flattened plan.  All offsets are element offsets into the device buffers.
struct TJobD {        // T[c_off] (M x N) = psi[a_off] (M x K, lda) * Rop (K x N)
    uint64_t a_off, b_off, c_off;
    uint32_t M, K, N, lda, brs, tr;  // Rop(k, n) = R[b_off + (n/brs)*K*brs + (tr ? n%brs + k*brs : k + (n%brs)*K)]
};
struct GTaskD {       // S[s_off + r + c*ldS] (r < rows, c < cols) = sum_a alpha[a] * T[toff[a] + r + c*rows]
    uint64_t s_off;
    uint32_t ldS, rows, cols, a_start, a_count, pad;
};
struct SegD {         // K segment of an output block: L cohort (M x nS*ls_in, maybe tile-transposed) times S (ldS = nS*ls_in)
    uint64_t l_off, s_off;
    uint32_t ls_in, nS, tr, pad;
};
struct OutD {
    uint64_t y_off;
    uint32_t M, N, seg_start, seg_count;
};
struct TileD { uint32_t item, m0, n0, pad; };

struct HeffPlan {
    Index phys, left, right;
    std::vector<uint64_t> x_off;  // block offset per left sector (right-paired blocks, ls x stripe)
    std::vector<uint32_t> x_cols;
    uint64_t x_len = 0;

    std::vector<TJobD> tjobs;
    std::vector<TileD> ttiles;
    uint64_t t_len = 0;

    std::vector<GTaskD> gtasks;
    std::vector<double> alpha;
    std::vector<uint64_t> aoff;
    uint64_t s_len = 0;

    std::vector<SegD> segs;
    std::vector<OutD> outs;
    std::vector<TileD> otiles;

    // reference work count ScheduleNew::total_flops (tasks.cpp:388-398, 777-796)
    double flops = 0, flops_t = 0, flops_ls = 0, flops_s = 0;
    // gather volume: S elements written, T elements read (one per alpha per element)
    uint64_t g_elems = 0, g_reads = 0;
    // bookkeeping export rows: (lb_in, lb_out, ci, ci_eff, unit offset, ms, b1, mps_offset, ci_right, col) + alpha
    std::vector<uint32_t> bk_int;
    std::vector<double> bk_alpha;

    // device copies
    DBuf<TJobD> d_tjobs;
    DBuf<TileD> d_ttiles, d_otiles;
    DBuf<GTaskD> d_gtasks;
    DBuf<double> d_alpha;
    DBuf<uint64_t> d_aoff;
    DBuf<SegD> d_segs;
    DBuf<OutD> d_outs;
    DBuf<double> d_T, d_S;
    DBuf<double> d_x, d_y;  // staging for host-buffer applies

    const DevBoundary* L = nullptr;
    const DevBoundary* R = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    const double* graph_x = nullptr;
    double* graph_y = nullptr;
    ~HeffPlan();
};

std::unique_ptr<HeffPlan> build_heff_plan(const DevBoundary& L, const DevBoundary& R, const MPOTensor& W,
                                          const Index& phys, const Index& left, const Index& right, bool bookkeeping);
void upload_plan(HeffPlan& p);

// y = H_eff x on device (x, y device pointers of length x_len), launched on p.stream.
// ev (optional, 4 events) is recorded before the T-GEMM, after it, after the S
// gather and after the L.S GEMM.
void heff_apply_device(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev = nullptr);

}  // namespace qcm
