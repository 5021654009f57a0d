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

#include <algorithm>
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
struct UnitD {        // S rows of one cohort unit: S_u (lines x elements) = W_u (lines x slices) * slices
    uint64_t s_off;        // S offset of (line 0, element 0) of the unit
    uint64_t line_stride;  // S offset step per line
    uint32_t erows;        // element e of a slice is (r, c) = (e % erows, e / erows) ...
    uint32_t col_stride;   // ... and lands at s_off + line*line_stride + r + c*col_stride
    uint32_t ne;           // elements per slice
    uint32_t nl;           // lines (boundary blocks with coefficients)
    uint32_t line0;        // first entry in line_b1[]
    uint32_t nk;           // distinct T slices referenced
    uint32_t slice0;       // first entry in slice_off[]
    uint32_t sptr0;        // first of nk + 1 entry pointers in sptr[]
    uint64_t w_off;        // dense coefficient block W_u (nl x nk, column-major) in the W buffer
};
struct WEntD {        // coefficient alpha at (line, slice) of a unit; entries sorted by slice
    uint32_t line, k;
    double a;
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
struct KItemD {       // split-K work item of the L.S GEMM: output tile, one segment, K range
    uint32_t tile, seg, k0, k1;
};
struct OTileD {       // output tile of the L.S GEMM and its contiguous range of split-K partials
    uint32_t out, m0, n0, part0, nparts, pad0, pad1, pad2;
};

// Appends one unit's coefficient entries (line, slice k, alpha) to went, sorted by
// (slice, line), with entries that share (line, slice) summed in their input order --
// several MPO terms may couple the same boundary block, input state and output state,
// and the densified coefficient tile holds their sum -- and the unit's nk + 1 slice
// pointers to sptr.
template <class WV, class PV>
inline void pack_unit_entries(std::vector<WEntD> ents, uint32_t nk, WV& went, PV& sptr) {
    // counting sort by slice; entries arrive in line order, so each slice's lines stay ascending
    std::vector<uint32_t> cnt(std::size_t(nk) + 1, 0);
    for (const WEntD& e : ents) cnt[e.k + 1]++;
    for (uint32_t k = 0; k < nk; ++k) cnt[k + 1] += cnt[k];
    std::vector<WEntD> sorted(ents.size());
    {
        std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
        for (const WEntD& e : ents) sorted[fill[e.k]++] = e;
    }
    for (uint32_t k = 0; k < nk; ++k)  // a slice's lines need not arrive sorted when lines repeat out of order
        if (!std::is_sorted(sorted.begin() + cnt[k], sorted.begin() + cnt[k + 1],
                            [](const WEntD& x, const WEntD& y) { return x.line < y.line; }))
            std::stable_sort(sorted.begin() + cnt[k], sorted.begin() + cnt[k + 1],
                             [](const WEntD& x, const WEntD& y) { return x.line < y.line; });
    const uint32_t w0 = uint32_t(went.size());
    sptr.push_back(w0);
    for (uint32_t k = 0; k < nk; ++k) {
        for (uint32_t i = cnt[k]; i < cnt[k + 1]; ++i) {
            const WEntD& e = sorted[i];
            if (went.size() > w0 && went.back().k == e.k && went.back().line == e.line) went.back().a += e.a;
            else went.push_back(e);
        }
        sptr.push_back(uint32_t(went.size()));
    }
}

// DMMA tile shapes (rows x cols of the CTA tile).  GEMM jobs pick the class from their row
// count (16 x 128, 32 x 128, 64 x 64); S-build units also use 128 x 32 (see add_unit_tiles).
enum { SHAPE_16 = 0, SHAPE_32 = 1, SHAPE_64 = 2, SHAPE_128 = 3, N_SHAPES = 4 };
inline int shape_for_rows(uint32_t M) { return M <= 16 ? SHAPE_16 : (M <= 32 ? SHAPE_32 : SHAPE_64); }
inline uint32_t shape_bm(int s) { return s == SHAPE_16 ? 16 : (s == SHAPE_32 ? 32 : (s == SHAPE_64 ? 64 : 128)); }
inline uint32_t shape_bn(int s) { return s == SHAPE_64 ? 64 : (s == SHAPE_128 ? 32 : 128); }

// S-GEMM tiles of one unit.  ents[0..n) are the unit's coefficient entries.  The tile shape
// is the one with the least tensor work counting only the (BM lines x 4 slices) coefficient
// groups that hold an entry; every m-tile's non-empty k-steps go to klist as (count, steps...),
// a step being (k-step index << 4 | mask of its non-empty 4-slice groups), and its tiles carry
// that list's offset in TileD::pad.
void add_unit_tiles(const UnitD& u, uint32_t item, const WEntD* ents, std::size_t n, std::vector<TileD>* utiles,
                    std::vector<uint16_t>& klist);

struct HeffPlan {
    Index phys, left, right;
    std::vector<uint64_t> x_off;  // block offset per left sector (right-paired blocks, ls x stripe)
    std::vector<uint32_t> x_cols;
    uint64_t x_len = 0;

    hvec<TJobD> tjobs;
    std::vector<TileD> ttiles[N_SHAPES];
    uint64_t t_len = 0;

    hvec<UnitD> units;
    std::vector<TileD> utiles[N_SHAPES];   // (unit, line tile m0, element tile n0)
    hvec<uint32_t> line_b1, sptr;
    hvec<uint64_t> slice_off;
    hvec<WEntD> went;
    uint64_t s_len = 0;
    uint64_t w_len = 0;  // dense coefficient blocks of all units (doubles)
    std::vector<uint16_t> klist;  // non-empty k-steps per S-GEMM m-tile

    std::vector<SegD> segs;
    std::vector<OutD> outs;
    std::vector<OTileD> otiles[N_SHAPES];
    std::vector<KItemD> kitems[N_SHAPES];
    uint64_t p_len = 0;  // split-K partial tiles (doubles)

    // reference work count ScheduleNew::total_flops (tasks.cpp:388-398, 777-796)
    double flops = 0, flops_t = 0, flops_ls = 0, flops_s = 0;
    // S build volume: S elements written, T elements read (one per alpha per element),
    // dense tensor-core work of the unit GEMMs (2 * lines * slices * elements)
    uint64_t g_elems = 0, g_reads = 0;
    double flops_sdense = 0;
    double flops_sexec = 0;  // tensor work the S-GEMM tiles execute (active k-steps x tile area)
    // bookkeeping export rows: (lb_in, lb_out, ci, ci_eff, unit offset, ms, b1, mps_offset, ci_right, col) + alpha
    std::vector<uint32_t> bk_int;
    std::vector<double> bk_alpha;

    // device copies
    DBuf<TJobD> d_tjobs;
    DBuf<TileD> d_ttiles[N_SHAPES];
    DBuf<OTileD> d_otiles[N_SHAPES];
    DBuf<KItemD> d_kitems[N_SHAPES];
    DBuf<double> d_P;
    DBuf<UnitD> d_units;
    DBuf<TileD> d_utiles[N_SHAPES];
    DBuf<uint32_t> d_line_b1, d_sptr;
    DBuf<uint64_t> d_slice_off;
    DBuf<WEntD> d_went;
    DBuf<double> d_W;
    DBuf<uint16_t> d_klist;
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
int heff_launches_per_apply(const HeffPlan& p);
// Grouped T-GEMM and unit S-GEMM launches over prepared work lists (three tile shapes each).
void run_tgemm(const TJobD* jobs, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const double* x,
               const double* R, double* T, cudaStream_t s);
void run_sgemm(const UnitD* units, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const uint32_t* line_b1,
               const uint64_t* slice_off, const uint16_t* klist, const double* W, const double* T, double* S,
               cudaStream_t s);
// Scatters every unit's coefficient entries into its dense block of W (w_len doubles, zeroed first).
void fill_coefficients(const UnitD* units, uint32_t n_units, const uint32_t* sptr, const WEntD* went, double* W,
                       uint64_t w_len, cudaStream_t s);
// Same apply with caller-provided scratch: Tb (t_len), Sb (s_len) and Pb (p_len) doubles.
void heff_apply_device_scratch(HeffPlan& p, const double* x, double* y, double* Tb, double* Sb, double* Pb);

}  // namespace qcm
