// Device-resident MPS tensors, boundary steps and the two-site sweep on one B200.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <vector>

#include "dev_ops.hpp"
#include "device.hpp"
#include "heff.hpp"
#include "linalg.hpp"
#include "mpo.hpp"
#include "symm.hpp"

namespace qcm {

// Block matrix in HBM: block k has charges (lc[k], rc[k]), rows x cols, column-major at off[k].
struct DBlocks {
    std::vector<Charge> lc, rc;
    std::vector<uint32_t> rows, cols;
    std::vector<uint64_t> off;
    uint64_t total = 0;
    DBuf<double> d;
    std::size_t n() const { return lc.size(); }
    std::size_t find_l(Charge c) const {
        for (std::size_t k = 0; k < lc.size(); ++k) if (lc[k] == c) return k;
        return lc.size();
    }
    std::size_t find_r(Charge c) const {
        for (std::size_t k = 0; k < rc.size(); ++k) if (rc[k] == c) return k;
        return rc.size();
    }
    // blocks start on 32-element boundaries unless packed (the H_eff vector layout is packed)
    void add(Charge l, Charge r, uint32_t nr, uint32_t nc, bool packed = false) {
        lc.push_back(l); rc.push_back(r); rows.push_back(nr); cols.push_back(nc);
        off.push_back(total);
        total += packed ? uint64_t(nr) * nc : (uint64_t(nr) * nc + 31) / 32 * 32;
    }
    uint64_t elems(std::size_t k) const { return uint64_t(rows[k]) * cols[k]; }
    void allocate(cudaStream_t s, bool zero) {
        d.alloc(total ? total : 1);
        if (zero) QCM_CUDA(cudaMemsetAsync(d.get(), 0, (total ? total : 1) * sizeof(double), s));
    }
    Index left_basis() const { Index r; for (std::size_t k = 0; k < n(); ++k) r.d.push_back({lc[k], rows[k]}); return r; }
    Index right_basis() const { Index r; for (std::size_t k = 0; k < n(); ++k) r.d.push_back({rc[k], cols[k]}); return r; }
};

// MPSTensor (mp_tensors/mpstensor.h): blocks keyed by the left charge when
// right-paired (ls x stripe, columns ProductBasis(phys, right, -p + r)) and by
// the right charge when left-paired (rows ProductBasis(phys, left), rs columns).
struct DMPS {
    Index phys, left, right;
    bool right_paired = false;
    DBlocks b;
};

// Work lists of the unit S-GEMM (shared by H_eff and the boundary steps)
// T slices of a schedule part: job j owns slice ids [pos0[j], pos0[j + 1]); slice id
// pos0[j] + b starts at T offset c_off[j] + b * bsize[j].
struct JobSlices {
    std::vector<uint32_t> pos0{0};
    std::vector<uint64_t> c_off, bsize;
    uint32_t add(uint64_t off, uint64_t bs, uint32_t nblocks) {  // returns the job's first id
        const uint32_t first = pos0.back();
        pos0.push_back(first + nblocks); c_off.push_back(off); bsize.push_back(bs);
        return first;
    }
    uint64_t offset(uint32_t id) const;
};

struct SBuild {
    hvec<UnitD> units;
    std::vector<TileD> utiles[N_SHAPES];
    hvec<uint32_t> line_b1;  // S row block of each line
    hvec<uint64_t> slice_off;
    uint64_t w_len = 0;  // dense coefficient blocks (doubles)
    std::vector<uint16_t> klist;  // non-empty k-steps per S-GEMM m-tile
    CoefGen cg;  // coefficient generation: per-unit tables here, MPO and boundary tables on the merged build
    DBuf<UnitD> d_units;
    DBuf<uint16_t> d_klist;
    DBuf<TileD> d_utiles[N_SHAPES];
    DBuf<uint32_t> d_line_b1;
    DBuf<uint64_t> d_slice_off;
    // One unit: local line i writes S row block rows[i] and iterates MPO index majors[i]; terms
    // are (local line, slice id) and leave as (local line, slot).  slot is a scratch table over
    // the part's slice ids, all NONE on entry and on return; in_row = the nst (cohort, id base)
    // pairs of the unit's input states.
    void add_unit(uint64_t s_off, uint64_t line_stride, uint32_t erows, uint32_t col_stride, uint32_t ne, uint32_t st_out,
                  const std::vector<uint32_t>& rows, const std::vector<uint32_t>& majors, std::vector<LKD>& ents,
                  std::vector<uint32_t>& slot, const JobSlices& js, const WGenInD* in_row);
    void upload(cudaStream_t s);
    // throws unless every unit's S writes and T slice reads lie inside [0, s_len) and [0, t_len)
    void validate(uint64_t t_len, uint64_t s_len) const;
};

// Engine context: stream, cuSOLVER handle and scratch buffers reused across steps.
struct Ctx {
    cudaStream_t s = nullptr;
    int device = 0;
    std::unique_ptr<Solver> sv;
    DBuf<double> T, S, W, work, tmp, jd, scal, coef;
    DBuf<GemmJob> gjobs;
    DBuf<uint32_t> gtiles;
    DBuf<CopyJob> cjobs;
    DBuf<SvdJob> sjobs;
    DBuf<QrJob> qjobs;
    DBuf<PermJob> pjobs;
    DBuf<double> qrw;  // QR / LQ scratch
    DBuf<TJobD> tjobs;
    DBuf<TileD> ttiles[N_SHAPES];
    DBuf<int> info;
    static void ensure(DBuf<double>& b, uint64_t n) { if (b.size() < n) b.alloc(n); }
};

// ---- MPS tensors on the device (mp_tensors/mpstensor.hpp, reshapes.h) ----
DBlocks layout_right_paired(const Index& phys, const Index& left, const Index& right, bool packed = false);
DBlocks layout_left_paired(const Index& phys, const Index& left, const Index& right);
void make_left_paired(Ctx& c, DMPS& t);
void make_right_paired(Ctx& c, DMPS& t);
DMPS right_paired_copy(Ctx& c, const DMPS& t);
DMPS left_paired_copy(Ctx& c, const DMPS& t);

// ---- excited states (mp_tensors/mps.h:175-219, contractions/special.hpp:38-62) ----
// Overlap boundaries between the current MPS (bra) and an ortho state (ket): one block per charge,
// rows on the bra's sector, columns on the ket's.
// unit blocks of an end index (left_boundary_bm / right_boundary_bm, mps.hpp:241-264)
DBlocks unit_blocks(Ctx& c, const Index& i);
// overlap_left_step: bra left-paired, ket right-paired; returns the boundary one site further right
DBlocks ortho_left_step(Ctx& c, const DMPS& bra, const DMPS& ket, const DBlocks& left);
// overlap_right_step: bra right-paired, ket left-paired; returns the boundary one site further left
DBlocks ortho_right_step(Ctx& c, const DMPS& bra, const DMPS& ket, const DBlocks& right);
// site_ortho_boundaries: the ortho twin projected onto the current twin's basis, written to v (device,
// twin.b.total doubles, the twin's right-paired block layout); zero where the ortho product has no block
void ortho_vector(Ctx& c, const DMPS& twin, const DMPS& ortho_twin, const DBlocks& left, const DBlocks& right, double* v);
double norm2(Ctx& c, const DBlocks& b);
void scale(Ctx& c, DBlocks& b, double f);
// normalize_left/right (mpstensor.hpp:242-300): QR / LQ per block; returns R / L as a block matrix
DBlocks normalize_left(Ctx& c, DMPS& t);
DBlocks normalize_right(Ctx& c, DMPS& t);
void multiply_from_left(Ctx& c, DMPS& t, const DBlocks& N);   // t = N * t (right-paired)
void multiply_from_right(Ctx& c, DMPS& t, const DBlocks& N);  // t = t * N (left-paired)

// block_matrix_algorithms.h:48-63
struct TruncResults {
    uint64_t bond_dimension = 0;
    double truncated_weight = 0, truncated_fraction = 0, smallest_ev = 0;
};

// svd_truncate (block_matrix_algorithms.h:185-240) of device blocks: per block a thin SVD (U
// rows x k at uo, S k descending at so, V cols x k at vo, k = min(rows, cols)), then
// estimate_truncation over all singular values: keep[k] of block k are kept.
struct BlockSVD {
    std::vector<uint64_t> uo, so, vo;
    std::vector<uint32_t> kk, keep;
    std::vector<std::vector<double>> vals;  // singular values per block, descending
    DBuf<double> U, S, V;
    uint64_t u_len = 0, s_len = 0, v_len = 0;
    TruncResults tr;
    std::vector<TruncResults> gtr;  // per group (svd_truncate_groups)
};
BlockSVD svd_truncate(Ctx& c, const DBlocks& M, uint64_t Mmax, double cutoff);
// The blocks of several independent matrices in one decomposition (one QR, one Jacobi and one assembly
// launch for all), each group of blocks [g0[g], g0[g+1]) cut by its own Mmax and cutoff: keep[] per
// block, gtr[] per group.
BlockSVD svd_truncate_groups(Ctx& c, const DBlocks& M, const std::vector<std::size_t>& g0,
                             const std::vector<uint64_t>& Mmax, const std::vector<double>& cutoff);
// heev_truncate (block_matrix_algorithms.h:299-355) of device symmetric blocks: dm is
// overwritten by its eigenvectors (ascending eigenvalue order, so the kept ones are the last
// keep[k] columns read backwards); the cut is on sqrt of the positive eigenvalues and the
// truncated fraction is reported in both fields.
struct BlockHeev {
    std::vector<uint32_t> keep;
    std::vector<std::vector<double>> evals;  // eigenvalues per block, descending
    TruncResults tr;
};
BlockHeev heev_truncate(Ctx& c, DBlocks& dm, uint64_t Mmax, double cutoff);

// TwoSiteTensor (mp_tensors/twositetensor.hpp:29-199, ts_reshape.h)
struct DTwoSite {
    Index phys1, phys2, phys, left, right;
    DBlocks both;               // rows ProductBasis(phys1, left), cols ProductBasis(phys2, right, -p + r), per middle charge
    std::vector<uint8_t> prod;  // block is a product block of a * b (the rest are created by the back-reshape)
    DMPS twin;                  // right-paired over phys1 x phys2, packed (H_eff vector layout)
    void build(Ctx& c, const DMPS& a_lp, const DMPS& b_rp);
    void twin_to_both(Ctx& c);  // reshape_right_to_both
    // split_mps_l2r / split_mps_r2l with svd_truncate (block_matrix_algorithms.h:136-240)
    TruncResults split(Ctx& c, bool l2r, uint64_t Mmax, double cutoff, DMPS& m1, DMPS& m2);
    // the same from a decomposition already made: this tensor's blocks are sv's blocks b0 .. b0 + n,
    // cut as sv's group g
    TruncResults split_from(Ctx& c, bool l2r, const BlockSVD& sv, std::size_t b0, std::size_t g, DMPS& m1, DMPS& m2);
    // predict_split_l2r / _r2l (contractions/boundary_ops/prediction.hpp:152-236): reduced density
    // matrix plus alpha times the boundary noise (B = L[site1] with W = mpo[site1] for l2r,
    // R[site2+1] with mpo[site2] for r2l), truncated by heev; alpha = 0 is the SVD split
    TruncResults predict_split(Ctx& c, bool l2r, uint64_t Mmax, double cutoff, double alpha, const DevBoundary& B,
                               const MPOTensor& W, DMPS& m1, DMPS& m2);
};

// Single-site growth (grow_l2r_sweep / grow_r2l_sweep, contractions/engine.hpp:85-123): the optimised
// site tensor a becomes the kept eigenvectors of its reduced density matrix plus alpha times the boundary
// noise (predict_new_state_*_sweep, contractions/boundary_ops/prediction.hpp:77-131; L = left boundary of
// a's site for l2r, R = right boundary of the site after a for r2l, W = a's MPO tensor), and the
// neighbour b takes the projection of the old a (predict_lanczos_*_sweep, :93-148): l2r a = U
// (left-paired), b = (U^T a) b; r2l a = U^T (right-paired), b = b (a U).
TruncResults grow_l2r(Ctx& c, DMPS& a, DMPS& b, const DevBoundary& L, const MPOTensor& W, double alpha, uint64_t Mmax,
                      double cutoff);
TruncResults grow_r2l(Ctx& c, DMPS& a, DMPS& b, const DevBoundary& R, const MPOTensor& W, double alpha, uint64_t Mmax,
                      double cutoff);

// Jacobi-Davidson for the lowest eigenpair (solve_ietl_jcd, solver/ietl_jacobi_davidson.h:35-76;
// ietl/jacobi.h:386-474): x (device, plan vector layout) holds the start vector and receives the
// eigenvector.
// mixed: every H.psi in the mixed form (heff_apply_device_mixed), stopping by the FP64 rule (and, with
// mixed_floor > 0, once the residual is below mixed_floor |theta| and no longer halves); then the FP64
// residual correction: one FP64 H.psi gives the
// Rayleigh quotient and the FP64 residual of the final vector, and up to mixed_refine Jacobi-Davidson
// steps in FP64 (the correction t = -r + (r.u)/(u.u) u, Rayleigh-Ritz on span{u, t}, one FP64 H.psi
// each) improve it while its FP64 residual is above tol |theta|.  The returned eigenvalue is FP64.
constexpr double MIXED_RESIDUAL_FLOOR = 1e-7;  // the mixed H.psi's relative error: a floor worth setting
// Beyond the plain solve: the correction equation (I - uu*)(A - theta)(I - uu*) t = -r solved by
// GMRES with `gmres` iterations from t0 = -r + (r.u)/(u.u) u (jcd_gmres_solver, ietl/jacobi.h:126-164;
// ietl_gmres, ietl/gmres.h:78-146; 0 = t0 itself), and the search space kept orthogonal to n_ortho
// vectors (excited states; DavidsonVS::project, solver/ietl_interface_dv.h:94-99), device pointers in
// the plan vector layout, ortho_ld doubles apart, Gram-Schmidt'd among themselves first.
struct JDOptions {
    int gmres = 0;
    const double* ortho = nullptr;
    int n_ortho = 0;
    uint64_t ortho_ld = 0;
    double mixed_floor = 0.0;  // mixed form: residual floor of its own iterations (0: none)
    int mixed_refine = 0;      // mixed form: FP64 correction steps after them
    int fp64_applies = 0;                       // out: FP64 applies of a mixed solve
};
constexpr int JD_MAX_GMRES = 64;
// precision: 0 FP64, 1 mixed, 2 mixed with the tensor-memory S build (QCM_PRECISION_*).
// *applies (may be null): the H_eff applies of the solve in its own form (the mixed form's FP64
// Rayleigh quotient not included).
double jacobi_davidson(Ctx& c, HeffPlan& p, double* x, double tol, int maxiter, int& iters, int precision = 0,
                       const JDOptions* opt = nullptr, int* applies = nullptr);

// Jacobi-Davidson for many independent site problems in lockstep on a merged plan group (the batching
// form): X (device, the group's vector arena) holds the start vectors and receives the eigenvectors;
// solve i's entries are X[xo[i] .. xo[i] + xn[i]).  Every iteration applies all H_eff in one launch
// sequence and runs the rest (classical Gram-Schmidt twice, device Rayleigh-Ritz, residuals,
// convergence, next direction) for all solves at once; with use_graphs each iteration is captured as a
// CUDA graph and replayed.  maxiter <= 16; ev / iters per solve; *applies: group applies run.
void jacobi_davidson_batched(HeffPlan& g, const std::vector<uint64_t>& xo, const std::vector<uint64_t>& xn, double* X,
                             double tol, int maxiter, std::vector<double>& ev, std::vector<int>& iters, bool use_graphs,
                             int* applies);

// Boundary steps (contractions/boundary_ops/move_boundary.hpp:147-404): new left boundary
// from L[site] and mps[site]; new right boundary from R[site+1] and mps[site].
// A step's schedule (T jobs, S-build units and their coefficient tables, the new boundary's index,
// the projection GEMMs) depends only on structure: the old boundary's index, the site tensors' sectors
// and block layouts, the MPO tensor.  With a cache, a step whose structure matches the cached
// schedule's runs that schedule again (its device lists stay on the device) instead of building it.
struct BStepPlan;
struct BStepCache {
    uint64_t key = 0;
    std::shared_ptr<BStepPlan> plan;
    uint64_t bytes = 0;  // device bytes the cached schedule holds
    bool hit = false;    // the last step ran the cached schedule
};
std::unique_ptr<DevBoundary> boundary_step_left(Ctx& c, const DevBoundary& L, const DMPS& ket_rp, const DMPS& bra_lp,
                                                const MPOTensor& W, bool symmetric, BStepCache* cache = nullptr);
std::unique_ptr<DevBoundary> boundary_step_right(Ctx& c, const DevBoundary& R, const DMPS& ket, const MPOTensor& W,
                                                 bool symmetric, BStepCache* cache = nullptr);

// trivial boundary: one cohort per sector, aux_dim blocks of ones (boundary.h / optimize.h:158-195)
std::unique_ptr<DevBoundary> trivial_boundary(const Index& idx, uint32_t aux_dim, cudaStream_t s);

// Density-matrix noise of the heev truncation (contractions/boundary_ops/move_boundary.hpp:37-145):
// the boundary step's S build without Hermitian skipping, then dm[k] += alpha S S^T (lbtm, dm keyed
// by the ket's right sectors) or alpha S^T S (rbtm, keyed by its left sectors), summed in cohort order.
struct DensityNoise {
    DBlocks* dm;
    double alpha;
};
void lbtm_accumulate(Ctx& c, const DevBoundary& L, const DMPS& ket_rp, const DMPS& bra_lp, const MPOTensor& W, DBlocks& dm,
                     double alpha);
void rbtm_accumulate(Ctx& c, const DevBoundary& R, const DMPS& ket_rp, const MPOTensor& W, DBlocks& dm, double alpha);

// complement_transpose of a boundary index (boundary.h:150-179; abelian conjugate correction 1)
void complement_transpose(BoundaryIndexH& x, const std::vector<int32_t>& herm, const std::vector<int32_t>& phase, bool forward);

// Two-site DMRG sweep on the device (optimize/ts_optimize.hpp:114-362, optimize.h:134-233).
struct DMRGParams {
    uint64_t Mmax = 64;
    uint64_t init_bond_dimension = 64;
    double cutoff = 1e-16;
    double jcd_tol = 1e-10;
    int jcd_maxiter = 8;
    int jcd_gmres = 0;  // ietl_jcd_gmres
    double ecore = 0.0;
    // twosite_truncation = heev with its noise per sweep (ts_optimize.hpp:275-296)
    bool heev = false;
    double alpha_initial = 1e-2, alpha_main = 1e-4, alpha_final = 1e-8;
    int ngrowsweeps = 0, nmainsweeps = 0;
    int precision = 0;  // H.psi form of the JD (QCM_PRECISION_*); mixed: FP64 Rayleigh quotient per step
    double mixed_floor = 0.0;  // mixed JD: residual floor of its mixed iterations (0: none)
    int mixed_refine = 0;      // mixed JD: FP64 correction steps at most
    // optimization = singlesite (ss_optimize.hpp:59-186): 2L steps per sweep over sites 0 .. L-1, L-1 .. 0,
    // each solved with the single-site MPO tensor and grown with the alphas above (heev does not apply)
    bool single_site = false;
};

struct DMRGStats {
    uint64_t plans_built = 0, plans_reused = 0;  // step plans built from scratch / re-staged from the cache
    uint64_t bsteps_built = 0, bsteps_reused = 0;  // boundary-step schedules built / run again from the cache
    uint64_t hpsi_count = 0;
    uint64_t hpsi_count64 = 0;   // mixed form: the extra FP64 applies (Rayleigh quotients)
    double hpsi_flops64 = 0;
    double hpsi_flops = 0, hpsi_ms = 0;  // reference flop count and device time of the H.psi applies
    double plan_s = 0, jd_s = 0, trunc_s = 0, boundary_s = 0, total_s = 0;
    uint64_t boundary_bytes_peak = 0;  // device bytes of the sweep's boundaries, largest after a step
    uint64_t boundaries_offloaded = 0, boundaries_fetched = 0;  // moves to and from pinned host memory
};

// One two-site step between its phases: the two-site tensor and its staged plan (step_prepare), then
// the eigenvector in tst.twin and the eigenvalue (the JD), then truncation and boundary step (step_finish)
struct StepState {
    int step = 0, lr = 0, site1 = 0, site2 = 0;
    DTwoSite tst;
    std::unique_ptr<HeffPlan> plan;
    uint64_t key = 0;
    bool resident = false;  // the plan's device buffers were kept from the previous sweep
    bool timing = false;
    bool pre_done = false;  // step_finish_pre ran
    double t0 = 0, t1 = 0, t2 = 0, tt[8] = {};
};

struct DevDMRG {
    int L = 0;
    std::vector<MPOTensor> mpo, ts_mpo;
    std::vector<DMPS> mps;
    std::vector<std::unique_ptr<DevBoundary>> left_, right_;
    DMRGParams p;
    DMRGStats st;
    Ctx c;
    // const MPS over the allowed sectors of (nup, ndown), canonised to site 0
    DevDMRG(const std::vector<MPOTensor>& single, const std::vector<MPOTensor>& twosite, int nup, int ndown,
            const DMRGParams& prm, cudaStream_t s);
    // given MPS (right-normalised on sites 1 .. L-1, as after canonize(0)); initial_site > 0 resumes the
    // sweep at that site (ts_optimize's initial site): left boundaries over sites 0 .. site-1, right
    // boundaries over L-1 .. site (init_left_right(mpo, site), optimize.h:158-195), next step = site
    DevDMRG(const std::vector<MPOTensor>& single, const std::vector<MPOTensor>& twosite, std::vector<DMPS> sites,
            const DMRGParams& prm, cudaStream_t s, int initial_site = 0);
    // excited states (ts_optimize.hpp:217-223, optimize.h:134-172): ortho states in both pairings and
    // their overlap boundaries with the current MPS
    std::vector<std::vector<DMPS>> ortho_lp, ortho_rp;
    std::vector<std::vector<DBlocks>> ortho_left_, ortho_right_;
    // sets the ortho states (right-paired site tensors, one vector per state) at the start of a sweep
    // and builds their right boundaries
    void set_ortho(std::vector<std::vector<DMPS>> states_rp);
    // <Psi|W|Psi> / <Psi|Psi> of the current MPS between sweeps (the MPS canonised to site 0) for an MPO W
    // of the same physical basis: left boundary steps through every site
    double expectation(const std::vector<MPOTensor>& W);
    // dE/d scale_e, E = <Psi|W|Psi> / <Psi|Psi>, for every entry e of every site tensor of a single-site
    // MPO W of the same physical basis (grad[k] in the entry order of W[k]), between sweeps: the adjoint
    // of the single-site H_eff apply at each site, the orthogonality centre moved through a copy of the MPS
    std::vector<std::vector<double>> mpo_gradient(const std::vector<MPOTensor>& W);
    int next_step = 0;  // step index (0 .. steps_per_sweep() - 1) the sweep continues with
    int steps_per_sweep() const { return p.single_site ? 2 * L : 2 * L - 2; }
    int sweep_count = 0;  // completed sweeps
    void sweep(std::vector<double>& energies, std::vector<TruncResults>& trunc);
    // run the current sweep up to (not including) step `stop`; appends energies / truncations
    void run_until(int stop, std::vector<double>& energies, std::vector<TruncResults>& trunc);
    // H_eff plan of the pending step (boundaries and MPS of this object; valid until the sweep continues),
    // the twin vector on the host, and the twin's indices
    std::unique_ptr<HeffPlan> pending_plan(std::vector<double>* twin, Index* phys, Index* left, Index* right);
    // start vector of the pending step (right-paired twin, H_eff vector layout)
    void pending_twin(std::vector<double>& twin);
    void step_sites(int step, int& lr, int& site1, int& site2) const;

    // the phases of a two-site step (step = prepare, the JD on the plan and twin, finish)
    // device bytes allowed for the sweep's boundaries (0: no limit); over it, boundaries move to pinned
    // host memory and back (the reference's boundary storage, storage.h, as host offload)
    uint64_t boundary_budget = 0;
    // doubles of coefficient blocks a plan keeps on the device (0: no limit); larger plans stream them
    uint64_t coefficient_budget = 0;
    // doubles of T, S and coefficient blocks one apply chunk may hold (0: whole applies)
    uint64_t apply_budget = 0;
    // boundary residency: the boundaries a step uses are brought to the device (bnd_use); after a step,
    // those no later step reads before the next half-sweep rebuilds them are released, and over the
    // budget the device copies farthest from the next step's two are moved to pinned host memory
    // (bnd_trim, with the step that comes next)
    void bnd_use(DevBoundary* b);
    void bnd_trim(int next_step);
    void step_prepare(StepState& S, int step);
    // step_prepare in parts: the two-site tensor (device), the plan (host only: built, or re-bound from
    // the previous sweep; runs of a group build theirs concurrently), the plan staged on the device (a
    // group member's coefficient blocks only)
    void step_prepare_site(StepState& S, int step);
    void step_prepare_plan(StepState& S);
    void step_prepare_stage(StepState& S, bool group);
    // step_finish_pre: the plan kept for the next sweep and the eigenvector reshaped to the two-site
    // blocks (the first part of step_finish); step_finish with sv: the truncation from a decomposition
    // made for many runs at once, this run's blocks from b0 on, cut as its group g
    void step_finish_pre(StepState& S);
    void step_finish(StepState& S, double eigenvalue, double& energy, TruncResults& tr, const BlockSVD* sv = nullptr,
                     std::size_t b0 = 0, std::size_t g = 0);
    int last_iters = 0;  // JD iterations of the last step

  private:
    // H_eff plans of the previous sweep's steps, kept on the host with their device buffers released:
    // a step whose boundaries and site indices have the same structure (the same sectors, cohorts,
    // block offsets and conjugate scales) as its cached plan's re-stages that plan (work lists
    // uploaded, coefficient blocks regenerated on the device) instead of rebuilding the schedule.
    // Plans whose work lists and coefficient blocks fit in the device budget keep them on the device (a
    // reuse then only re-binds the boundaries); the others keep their host lists only.
    struct CachedPlan {
        std::unique_ptr<HeffPlan> plan;
        uint64_t key = 0;
        uint64_t resident = 0;  // device bytes kept with the plan
    };
    std::vector<CachedPlan> plan_cache_;
    uint64_t plan_cache_budget_ = 0, plan_cache_bytes_ = 0;
    // boundary-step schedules of the previous sweep's steps (one per step), their device lists within
    // a budget of a sixteenth of the device's memory
    std::vector<BStepCache> bstep_cache_;
    uint64_t bstep_cache_bytes_ = 0, bstep_cache_budget_ = 0;
    BStepCache* bstep_cache_for(int step);
    void bstep_cache_done(int step);

    std::unique_ptr<HeffPlan> plan_for(int step, const DevBoundary& Lb, const DevBoundary& Rb, const MPOTensor& W,
                                       const Index& phys, const Index& left, const Index& right, uint64_t& key,
                                       bool& resident);
    void keep_plan(int step, std::unique_ptr<HeffPlan> plan, uint64_t key);
    void init_boundaries(int site = 0);
    void step(int step, double& energy, TruncResults& tr);
    void step_single(int step, double& energy, TruncResults& tr);
    // JD of one step's plan with this object's ortho vectors (built by make_ortho) and its statistics
    double solve(HeffPlan& plan, DMPS& x, const std::function<void(std::size_t, double*)>& make_ortho);
};

// Many independent two-site FP64 runs (same length and JD settings, one stream, at the start of a sweep)
// swept in lockstep, the batching form for whole solves: at every step each run builds or re-binds its
// plan, the plans are merged into one group (merge_plans) and one lockstep Jacobi-Davidson
// (jacobi_davidson_batched, a CUDA graph per iteration) solves every run's two-site problem, then each
// run truncates and moves its boundary.  energies[run][step], trunc[run][step].
void dmrg_group_sweep(const std::vector<DevDMRG*>& runs, std::vector<std::vector<double>>& energies,
                      std::vector<std::vector<TruncResults>>& trunc);

}  // namespace qcm
