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
#include <cstring>
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
    // structure hash of idx (boundary_key), computed on first use: the index of a boundary is not
    // changed after the boundary is made
    mutable uint64_t key = 0;
    // a copy in pinned host memory (host_len doubles), made when the boundary is moved out of device
    // memory (its data released until it is fetched back); a boundary's values never change, so the
    // copy stays valid and a later eviction only releases the device data
    std::shared_ptr<double> host;
    uint64_t host_len = 0;
    bool on_device() const { return data.get() != nullptr || !host; }
};

// Hash of structure (sectors, cohorts, block offsets, conjugate scales) for the plan caches
struct KeyHash {
    uint64_t h = 0x243F6A8885A308D3ull;
    void word(uint64_t v) {
        h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 31;
    }
    template <class T> void vec(const std::vector<T>& v) {
        word(v.size());
        for (const T& x : v) {
            uint64_t u = 0;
            std::memcpy(&u, &x, sizeof(T) < 8 ? sizeof(T) : 8);
            word(u);
        }
    }
    void index(const Index& I) {
        word(I.size());
        for (auto& e : I.d) { word(uint64_t(uint32_t(e.first.a))); word(uint64_t(uint32_t(e.first.b))); word(e.second); }
    }
    void boundary(const BoundaryIndexH& B) {
        index(B.bra); index(B.ket); word(B.aux);
        vec(B.cbra); vec(B.cket); vec(B.lsz); vec(B.rsz); vec(B.nb); vec(B.tr); vec(B.offsets); vec(B.cscale);
    }
};
// B's structure hash, cached in B
uint64_t boundary_key(const DevBoundary& B);

// Flattened plan.  All offsets are element offsets into the device buffers.
struct TJobD {        // T[c_off] (M x N) = psi[a_off] (M x K, lda) * Rop (K x N)
    uint64_t a_off, b_off, c_off;
    uint32_t M, K, N, lda, brs, tr;  // Rop(k, n) = R[b_off + (n/brs)*K*brs + (tr ? n%brs + k*brs : k + (n%brs)*K)]
    // T is stored as N / brs slices (blocks of brs columns, M x brs column-major) sst elements
    // apart: column n at c_off + (n / brs) * sst + (n % brs) * M; sst = brs * M rounded up to 4
    // elements, so every slice starts on a 16-byte boundary (FP32 and FP64)
    uint32_t sst, pad;
};
// slice stride of a T job: brs * M rounded up to a multiple of 4 elements
inline uint32_t slice_stride(uint32_t brs, uint32_t M) { return (brs * M + 3u) / 4u * 4u; }
// leading dimension of a dense coefficient block: lines rounded up to a multiple of 4
inline uint32_t coef_ld(uint32_t nl) { return (nl + 3u) / 4u * 4u; }
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
    uint32_t wld;          // leading dimension of W_u (nl rounded up to 4; rows nl .. wld - 1 are zero)
    uint64_t w_off;        // dense coefficient block W_u (nl x nk, column-major) in the W buffer
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
struct KItemD {       // split-K work item of the L.S GEMM: output tile, one segment, K range, partial slot
    uint32_t tile, seg, k0, k1, slot;
};
struct OTileD {       // output tile of the L.S GEMM and its contiguous range of split-K partials
    uint32_t out, m0, n0, part0, nparts, pad0, pad1, pad2;
};

// DMMA tile shapes (rows x cols of the CTA tile).  GEMM jobs pick the class from their row
// count (16 x 128, 32 x 128, 64 x 64); S-build units also use 128 x 32 (see add_unit_tiles).
// (An 8 x 128 shape for GEMM jobs of at most 8 rows measured slower at L=24, M=512: T-GEMM +7 us,
// L.S +36 us; the 16-row tile's padding rows cost less than the extra B traffic of half-height tiles.)
enum { SHAPE_16 = 0, SHAPE_32 = 1, SHAPE_64 = 2, SHAPE_128 = 3, N_SHAPES = 4 };
inline int shape_for_rows(uint32_t M) { return M <= 16 ? SHAPE_16 : (M <= 32 ? SHAPE_32 : SHAPE_64); }
inline uint32_t shape_bm(int s) { return s == SHAPE_16 ? 16 : (s == SHAPE_32 ? 32 : (s == SHAPE_64 ? 64 : 128)); }
inline uint32_t shape_bn(int s) { return s == SHAPE_64 ? 64 : (s == SHAPE_128 ? 32 : 128); }

struct LKD { uint32_t line, k; };  // (line, slice) position of one coefficient term

// S-GEMM tiles of one unit.  ents[0..n) are the unit's coefficient entries.  The tile shape
// is the one with the least tensor work counting only the (BM lines x 4 slices) coefficient
// groups that hold an entry; every m-tile's non-empty k-steps go to klist as (count, steps...),
// a step being (k-step index << 4 | mask of its non-empty 4-slice groups), and its tiles carry
// that list's offset in TileD::pad.
void add_unit_tiles(const UnitD& u, uint32_t item, const LKD* ents, std::size_t n, std::vector<TileD>* utiles,
                    std::vector<uint16_t>& klist);


// Dense coefficient blocks W_u of S units, computed on the device (k_wgen).  Line l of a
// unit iterates the MPO entries of its line index m = line_major[line0 + l] (a row b1 or a
// column b2, depending on how m_ptr groups the entries), and every operator term of an entry
// with the unit's output state adds
//     alpha = op value * boundary conj scale(c, x) * (MPO scale * line_scale[line0 + l])
// at W[w_off + l + slot * nl], where x is the entry's other MPO index, c the boundary cohort
// of (unit, input state), and slot the unit's slot of slice id jbase(unit, input state) +
// block position of x in cohort c.  Terms of one line are summed in entry, then operator-term
// order by one thread, with products and sums rounded separately.
struct WGenUnitD {
    uint64_t w_off;
    uint32_t st_out;   // output physical state of the unit
    uint32_t line0, nl;
    uint32_t map0, nk;  // sorted (slice id, slot) pairs at smap_id/smap_slot[map0 .. map0 + nk)
    uint32_t wld;       // leading dimension of the unit's coefficient block
};
struct WGenInD { uint32_t c, jbase; };  // per (unit, input state): boundary cohort and slice-id base, or WGEN_NONE
constexpr uint32_t WGEN_NONE = 0xffffffffu;

struct MPOTables {
    uint32_t nst = 0;     // states of the physical index
    std::size_t nops = 0;
    // operator terms, CSR per operator: (input state, output state, value)
    std::vector<uint32_t> optr, oin, oout;
    std::vector<double> oval;
    // the same grouped by (operator, output state), in their order within the operator
    std::vector<uint32_t> o_ptr, o_in;
    std::vector<double> o_val;
    // per (operator, output state): the input state of its only term, O_NONE without a term, O_MANY with
    // several; and per entry in row order (op * nst) << 32 | b2, the entry's two lookups in one word
    static constexpr uint32_t O_NONE = 0xfffffffeu, O_MANY = 0xffffffffu;
    std::vector<uint32_t> o_one;
    std::vector<uint64_t> row_qb;
    // MPO entries by row b1 (other index b2) and by column b2 (other index b1, increasing b1)
    std::vector<uint32_t> row_ptr, row_other, row_op, col_ptr, col_other, col_op;
    std::vector<double> row_scale, col_scale;
    uint32_t rows = 0, cols = 0;
};
std::shared_ptr<const MPOTables> build_mpo_tables(const MPOTensor& W);

struct CoefGen {
    hvec<WGenUnitD> units;
    hvec<WGenInD> gin;  // units x nst
    hvec<uint32_t> line_major;
    hvec<double> line_scale;
    hvec<uint32_t> smap_id, smap_slot;
    uint32_t nst = 0;
    std::shared_ptr<const MPOTables> mt;  // MPO entries (by row or column) and operator terms
    bool by_row = true;
    std::vector<int32_t> b_pos;  // boundary cohort x aux: block position of the MPO index, or -1
    const std::vector<double>* b_cs = nullptr;  // boundary conj scales (cohort x aux)
    uint32_t b_aux = 0;
    uint64_t w_len = 0;

    DBuf<WGenUnitD> d_units;
    DBuf<WGenInD> d_gin;
    DBuf<uint32_t> d_line_major, d_smap_id, d_smap_slot, d_m_ptr, d_m_other, d_m_op, d_o_ptr, d_o_in, d_err;
    DBuf<double> d_line_scale, d_m_scale, d_o_val, d_b_cs;
    DBuf<int32_t> d_b_pos;

    // MPO entries by row b1 (other index b2) or by column b2 (other index b1, in increasing b1),
    // and the operator terms
    void set_mpo(const MPOTensor& W, bool by_row);
    void set_boundary(const BoundaryIndexH& B);
    // appends one unit: its lines (MPO index and scale each), slot -> slice id, and the
    // (cohort, slice-id base) of each of the nst input states
    void add_unit(uint64_t w_off, uint32_t wld, uint32_t st_out, const uint32_t* majors, const double* scales, uint32_t nl,
                  const std::vector<uint32_t>& slices, const WGenInD* in_row);
    // appends the per-unit tables of another builder (part) with its lines, slice-map and
    // coefficient-block bases
    void append_units(const CoefGen& part, uint32_t line_base, uint32_t map_base, uint64_t w_base);
    void validate() const;  // throws unless every index k_wgen derives stays in its buffer
    void upload(cudaStream_t s);
    // W (w_len doubles) = coefficient blocks; waits for the stream and throws if a term had no slot
    void generate(double* W, cudaStream_t s);
    // the blocks of units [u0, u1) (elements [w0, w1) of the whole, written from W on), without the
    // check of generate; check_generated reads and clears the error flag of the generations so far
    void generate_range(double* W, uint32_t u0, uint32_t u1, uint64_t w0, uint64_t w1, cudaStream_t s);
    void check_generated(cudaStream_t s);
};

struct HeffAdjointWork;  // work lists and buffers of the adjoint, made on its first call

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
    hvec<uint32_t> line_b1;
    hvec<uint64_t> slice_off;
    uint64_t s_len = 0;
    uint64_t n_alpha = 0;  // coefficient terms (before terms of one (line, slice) are summed)
    CoefGen cg;            // coefficient blocks of the units (lines iterate MPO rows b1)
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
    DBuf<uint32_t> d_line_b1;
    DBuf<uint64_t> d_slice_off;
    DBuf<double> d_W;  // the coefficient blocks (w_len doubles), or one chunk of them when streamed
    // coefficient blocks generated chunk by chunk inside every apply instead of kept
    // (stream_coefficients): units [u0, u1) with their blocks [w0, w1) and, per tile shape, their
    // S-GEMM tiles [t0, t1)
    struct WChunk {
        uint32_t u0 = 0, u1 = 0;
        uint64_t w0 = 0, w1 = 0;
        uint32_t t0[N_SHAPES] = {}, t1[N_SHAPES] = {};
    };
    std::vector<WChunk> wchunks;
    bool streamed() const { return !wchunks.empty(); }
    // where each ket sector's share starts in the plan's lists (prefixes over the ket sectors: T jobs,
    // S units, T and S elements, coefficient elements), for the ket-sector chunks
    std::vector<uint32_t> part_job, part_unit;
    std::vector<uint64_t> part_t, part_s, part_w;
    // the apply cut by ket sector (chunk_sectors): chunk c covers ket sectors [p0, p1), whose T slices
    // [t0, t1), S rows [s0, s1) and coefficient blocks [w0, w1) (units [u0, u1)) are made and used by
    // the chunk alone; per tile shape, its T-GEMM tiles, S-GEMM tiles and L.S items (the lists are
    // ordered by chunk) are the ranges [a, b)
    struct SChunk {
        uint32_t p0 = 0, p1 = 0, u0 = 0, u1 = 0;
        uint64_t t0 = 0, t1 = 0, s0 = 0, s1 = 0, w0 = 0, w1 = 0;
        uint32_t tt[2][N_SHAPES] = {}, ut[2][N_SHAPES] = {}, kt[2][N_SHAPES] = {};
    };
    std::vector<SChunk> schunks;
    bool sector_chunked() const { return !schunks.empty(); }
    // a chunked apply sums every shape's partials at the end, so each shape has its own partial region
    // (from pc_off[sh] on; pc_len in all) instead of the one region the shapes take in turn
    uint64_t pc_off[N_SHAPES] = {}, pc_len = 0;
    // in a chunked plan the T offsets of its T jobs and slices and the S offsets of its units and L.S
    // segments count from their chunk's t0 and s0 (the kernels address one chunk's scratch); seg_chunk
    // is each segment's chunk, for undoing it
    std::vector<uint32_t> seg_chunk;
    // the chunks share the whole coefficient blocks, generated once (they take at most half the budget),
    // instead of generating their own in every apply
    bool chunk_keeps_w = false;
    DBuf<uint16_t> d_klist;
    DBuf<SegD> d_segs;
    DBuf<OutD> d_outs;
    DBuf<double> d_T, d_S;
    // mixed forms: the coefficient blocks in FP32 (w_len floats) and split into TF32 hi and lo
    // (2 w_len floats), each made on the first apply that needs it; T in FP32 (or its hi and lo)
    // is written into the bytes of d_T; error word of the tensor-memory path's waits
    DBuf<float> d_W32, d_W32s;
    DBuf<uint32_t> d_merr;
    DBuf<double> d_x, d_y;  // staging for host-buffer applies

    std::shared_ptr<HeffAdjointWork> adj;

    const DevBoundary* L = nullptr;
    const DevBoundary* R = nullptr;
    // a merged plan (merge_plans): the boundaries and coefficient blocks of its member plans are
    // addressed from these bases (its job offsets are relative to them); FP64 applies only
    bool merged = false;
    bool lists_staged = false;  // the work lists are on the device (upload_plan with lists, restage_plan)
    const double* base_L = nullptr;
    const double* base_R = nullptr;
    const double* base_W = nullptr;
    const double* l_data() const { return merged ? base_L : L->data.get(); }
    const double* r_data() const { return merged ? base_R : R->data.get(); }
    const double* w_data() const { return merged ? base_W : d_W.get(); }
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    const double* graph_x = nullptr;
    double* graph_y = nullptr;
    ~HeffPlan();
};

std::unique_ptr<HeffPlan> build_heff_plan(const DevBoundary& L, const DevBoundary& R, const MPOTensor& W,
                                          const Index& phys, const Index& left, const Index& right, bool bookkeeping);
// Stages a plan on the device: its coefficient blocks (generated on the device) and, with lists, its
// work lists and scratch.  A plan staged without lists is applied only inside a merged plan group
// (merge_plans, which stages the group's own lists); restage_plan adds the lists when it is reused alone.
void upload_plan(HeffPlan& p, bool lists = true);
// Bounds a plan's coefficient blocks to max_doubles on the device (0 or w_len <= max_doubles: kept
// whole): the units are cut into consecutive chunks of at most max_doubles of blocks (a larger unit
// is a chunk of its own) and every FP64 apply generates each chunk into one scratch and runs its
// S-GEMM tiles from it, in the same order and with the same arithmetic as the kept blocks (the apply's
// result is the same to the bit).  Set before upload_plan; the mixed forms and plan groups need the
// blocks kept.
void stream_coefficients(HeffPlan& p, uint64_t max_doubles);
// Bounds the device memory of an apply: the ket sectors are cut into consecutive chunks whose T slices,
// S rows and coefficient blocks together take at most max_doubles (a larger sector is a chunk of its
// own; when the whole coefficient blocks take at most half of max_doubles they are kept, generated once,
// and the chunks' T and S share the rest), and every FP64 apply runs chunk by chunk: the chunk's T-GEMM
// into one T scratch, its coefficient blocks (unless kept) generated into one scratch, its S-GEMM into
// one S scratch and its split-K L.S partials; the
// partials of all chunks are summed at the end in the fixed order, so the result is the whole apply's
// to the bit.  0 (or a plan that fits) undoes it.  Set before upload_plan; supersedes
// stream_coefficients; the mixed forms, the adjoint and plan groups need the whole apply.
void chunk_sectors(HeffPlan& p, uint64_t max_doubles);
// Frees a plan's device buffers (work lists, coefficient blocks, scratch) and keeps its host work lists:
// upload_plan stages it again, against boundaries of the same structure (rebind_plan).
void release_plan_device(HeffPlan& p);
// Frees only the scratch (T, S, partials, staging, mixed-form copies, coefficient-generation tables):
// the work lists and coefficient blocks stay on the device (plan_resident_bytes of them), and
// restage_plan makes the plan applicable again, against boundaries of the same structure (staging the
// work lists first when the plan was staged without them).
void release_plan_scratch(HeffPlan& p);
uint64_t plan_resident_bytes(const HeffPlan& p);
void restage_plan(HeffPlan& p);
void rebind_plan(HeffPlan& p, const DevBoundary& L, const DevBoundary& R);
// 64-bit fingerprint of what a plan's work lists depend on besides the MPO tensor: the two boundaries'
// sectors, cohorts, block offsets, conjugate scales and transposition flags, and the site indices.
uint64_t plan_structure_key(const BoundaryIndexH& L, const BoundaryIndexH& R, const Index& phys, const Index& left,
                            const Index& right);
// the same from the boundaries' cached hashes
uint64_t plan_structure_key(const DevBoundary& L, const DevBoundary& R, const Index& phys, const Index& left,
                            const Index& right);

// y = H_eff x on device (x, y device pointers of length x_len), launched on p.stream.
// ev (optional, 4 events) is recorded before the T-GEMM, after it, after the S
// gather and after the L.S GEMM.
void heff_apply_device(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev = nullptr);
// The apply's T-GEMM alone: T (t_len doubles, the plan's slice layout) from x, FP64.
void heff_tgemm_device(HeffPlan& p, const double* x, double* T);
// Adjoint of the apply (the differentiation form) for f = ybar . H_eff x, device pointers on
// p.stream: psi_bar = H_eff ybar (H_eff is symmetric for a Hermitian MPO) and coeff_bar[e] =
// df / d scale_e for the heff_adjoint_terms(p) entries of the plan's two-site MPO tensor, in the
// tensor's entry order; either output may be null.  Uses the plan's T and S buffers.
void heff_adjoint_device(HeffPlan& p, const double* x, const double* ybar, double* psi_bar, double* coeff_bar);
uint64_t heff_adjoint_terms(const HeffPlan& p);
int heff_launches_per_apply(const HeffPlan& p);
// Mixed-precision H.psi (same layout and stream as heff_apply_device): the S build in 3xTF32 on
// the tensor cores from FP32 operands, T-GEMM and L.S in FP64.  The first call makes the FP32
// copy of the coefficient blocks (prepare_mixed).
// tc: the tensor-memory (tcgen05) S build for the 16- and 32-line tiles from pre-split operands
void heff_apply_device_mixed(HeffPlan& p, const double* x, double* y, cudaEvent_t* ev = nullptr, bool tc = false);
void prepare_mixed(HeffPlan& p, bool tc);
// waits for the plan's stream and throws if a mixed S-build tile gave up on a bounded wait
void check_mixed(HeffPlan& p);
void run_sgemm_mixed(const HeffPlan& p, bool tc, const float* Wh, const float* Wl, const float* Th, const float* Tl, double* S,
                     uint32_t* err, cudaStream_t s);
void split_tf32(const double* x, float* hi, float* lo, uint64_t n, cudaStream_t s);
void to_f32(const double* x, float* y, uint64_t n, cudaStream_t s);
// Grouped T-GEMM and unit S-GEMM launches over prepared work lists (three tile shapes each).
void run_tgemm(const TJobD* jobs, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const double* x,
               const double* R, double* T, cudaStream_t s);
void run_sgemm(const UnitD* units, const DBuf<TileD>* dtiles, const std::vector<TileD>* htiles, const uint32_t* line_b1,
               const uint64_t* slice_off, const uint16_t* klist, const double* W, const double* T, double* S,
               cudaStream_t s);
// Many plans as one (the batching form): the work lists of `plans` concatenated into one merged
// plan whose vector is the arena of the plans' vectors (plan i's at xo[i], each rounded up to 32
// doubles); T, S and the split-K partials get merged buffers, the boundaries and coefficient blocks
// stay in the plans' buffers (which must outlive the merged plan).  heff_apply_device on the merged
// plan applies every member's H_eff in one launch sequence, with each member's arithmetic unchanged.
std::unique_ptr<HeffPlan> merge_plans(const std::vector<HeffPlan*>& plans, std::vector<uint64_t>& xo, cudaStream_t s);
void upload_merged(HeffPlan& g);
// Same apply with caller-provided scratch: Tb (t_len), Sb (s_len) and Pb (p_len) doubles.
void heff_apply_device_scratch(HeffPlan& p, const double* x, double* y, double* Tb, double* Sb, double* Pb);

}  // namespace qcm
