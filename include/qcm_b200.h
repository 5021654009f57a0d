/*
 * qcm_b200.h -- C-ABI of the B200-native two-site DMRG effective-Hamiltonian path.
 *
 * Plain C: opaque handles, host pointers and sizes, int status codes.  No
 * entry point exits the process; on failure it returns a negative code and
 * qcm_last_error() describes the cause (thread-local).
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the QCMaquis tree's dmrg/ directory).
 */
#ifndef QCM_B200_H
#define QCM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define QCM_OK 0
#define QCM_ERR_ARG (-1)      /* invalid argument (std::runtime_error in the reference) */
#define QCM_ERR_CUDA (-2)     /* CUDA runtime / launch failure (reference: exit(EXIT_FAILURE)) */
#define QCM_ERR_NOMEM (-3)    /* host or device allocation failed */
#define QCM_ERR_INTERNAL (-4) /* internal consistency error */
#define QCM_ERR_NODEV (-5)    /* no CUDA device: there is no CPU fallback */

/* Human-readable description of the last failure on this thread. */
const char* qcm_last_error(void);

/* Library version string. */
const char* qcm_version(void);

/* ------------------------------------------------------------------------ */
/* MPO (input preparation)                                                    */
/* ------------------------------------------------------------------------ */

typedef struct qcm_mpo qcm_mpo;

/* Exact TwoU1 QC Hamiltonian MPO from integrals h[L*L] and V[L^4] (chemist
 * notation (pq|rs), row-major), terms with |coefficient| <= cutoff dropped.
 * Replaces qc_model::create_terms + make_mpo
 * (framework/dmrg/models/chem/2u1/model.hpp:184, models/generate_mpo.hpp:37). */
int qcm_mpo_build_qc(int L, const double* h, const double* V, double cutoff, qcm_mpo** out);

/* The same Hamiltonian with its integral provenance (the differentiation form): every term the spin
 * structure allows is kept whatever its value (no cutoff), and for every entry the builder records which
 * integrals its scale sums.  qcm_mpo_provenance: site tensor `site`'s records, scale of entry e =
 * sum_{j in [ptr[e], ptr[e+1])} val[j] * x[id[j]] with x = (h[0 .. L^2), V[0 .. L^4)) as passed; ptr has
 * entries + 1 elements, *n = the record count (every array NULL: only *n); pass-through entries have no
 * records (scale 1).  Chain rule for host codes: dE/dx[id] = sum val * dE/d scale (qcm_dmrg_mpo_gradient). */
int qcm_mpo_build_qc_tracked(int L, const double* h, const double* V, qcm_mpo** out);
int qcm_mpo_provenance(const qcm_mpo* m, int site, uint64_t* ptr, uint64_t* id, double* val, uint64_t cap, uint64_t* n);

/* Two-site MPO W_ts[p] = W[p] (x) W[p+1] contracted over the shared bond.
 * Replaces make_ts_cache_mpo / make_twosite_mpo
 * (framework/dmrg/mp_tensors/ts_ops.hpp:97-185). */
int qcm_mpo_make_twosite(const qcm_mpo* m, qcm_mpo** out);

/* Number of site tensors (L, or L-1 for a two-site MPO); -1 for NULL. */
int qcm_mpo_length(const qcm_mpo* m);

/* Binary interchange blob ("QMPO" v1).  Call with buf == NULL to get *len. */
int qcm_mpo_serialize(const qcm_mpo* m, void* buf, size_t cap, size_t* len);
int qcm_mpo_deserialize(const void* buf, size_t len, qcm_mpo** out);
void qcm_mpo_free(qcm_mpo* m);

/* Entries of MPO tensor `site`, in the tensor's entry order (sorted by (b1, b2); an entry is one
 * operator term: row b1, column b2, operator index op, scale), as MPOTensor stores them
 * (mp_tensors/mpotensor.h; the scale is the coefficient the adjoint differentiates).  *n = entry
 * count; with every array NULL only *n is set; otherwise cap must be >= *n. */
int qcm_mpo_tensor_terms(const qcm_mpo* m, int site, uint32_t* b1, uint32_t* b2, uint32_t* op, double* scale, uint64_t cap,
                         uint64_t* n);
/* Replace the scales of MPO tensor `site` (n = its entry count, finite values).  Plans made from
 * the MPO before the call keep their coefficients. */
int qcm_mpo_set_scales(qcm_mpo* m, int site, const double* scale, uint64_t n);

/* One MPO tensor as the reference's MPOTensor holds it (mp_tensors/mpotensor.h:46-135 with
 * mpotensor_detail.h:141-186), in flat arrays:
 *   rows, cols          row_dim() / col_dim();
 *   terms               one per (b1, b2, operator) summand: row b1 < rows, column b2 < cols,
 *                       operator index op < n_ops and its scale (the term_descriptor of
 *                       at(b1, b2)); any order, several terms may share (b1, b2);
 *   site operators      operator k has the entries op_ptr[k] .. op_ptr[k+1]-1, each
 *                       <op_out|O|op_in> = op_val over the physical basis's flat states (state =
 *                       first state of its sector + sub-index, sectors in phys order);
 *   physical index      n_phys sectors (phys_charge[2*s], phys_charge[2*s+1]) = (N_up, N_down)
 *                       of size phys_size[s], in strictly descending charge order;
 *   Hermitian pairs     herm_left[b] (b < rows) / herm_right[b] (b < cols): the partner index of
 *                       b, b itself for a self-adjoint index, or -1 (Hermitian::conj; bond
 *                       properties leftBond().conj() / rightBond().conj()); phase_* the +-1 phase
 *                       of the pair (Hermitian::phase).  NULL arrays mean no pairs on that bond.
 * The two tensors on either side of a bond must give it the same dimension and pairs. */
typedef struct qcm_mpo_tensor_desc {
    uint32_t rows, cols;
    uint64_t n_terms;
    const uint32_t* b1;
    const uint32_t* b2;
    const uint32_t* op;
    const double* scale;
    uint32_t n_ops;
    const uint64_t* op_ptr;
    const uint32_t* op_in;
    const uint32_t* op_out;
    const double* op_val;
    uint32_t n_phys;
    const int32_t* phys_charge;
    const uint32_t* phys_size;
    const int32_t* herm_left;
    const int32_t* phase_left;
    const int32_t* herm_right;
    const int32_t* phase_right;
} qcm_mpo_tensor_desc;

/* An MPO of `length` tensors to be filled by qcm_mpo_set_tensor (twosite != 0: the tensors are
 * two-site tensors, as make_twosite_mpo returns them).  This is the seam through which a host
 * code hands its own MPO<Matrix, SymmGroup> (mp_tensors/mpo.h) to this library, e.g. each tensor
 * of ts_cache_mpo (optimize/ts_optimize.hpp:98-101) for the H_eff plans.  An unset tensor is an
 * error when the MPO is used. */
int qcm_mpo_create(int length, int twosite, qcm_mpo** out);
/* Sets tensor `site` from d (copied; validated: indices in range, pairs symmetric
 * (herm[herm[b]] == b), phases +-1, operator entries inside the physical basis). */
int qcm_mpo_set_tensor(qcm_mpo* m, int site, const qcm_mpo_tensor_desc* d);
/* rows, cols, operator count and physical sector count of tensor `site` (any may be NULL). */
int qcm_mpo_tensor_info(const qcm_mpo* m, int site, uint32_t* rows, uint32_t* cols, uint32_t* n_ops, uint32_t* n_phys);
/* Hermitian pairs and phases of tensor `site`'s left (rows entries) and right (cols entries)
 * bonds, as described above (any may be NULL). */
int qcm_mpo_tensor_hermitian(const qcm_mpo* m, int site, int32_t* herm_left, int32_t* phase_left, int32_t* herm_right,
                             int32_t* phase_right);

/* ------------------------------------------------------------------------ */
/* Context, resident boundaries, H_eff plan                                   */
/* ------------------------------------------------------------------------ */

typedef struct qcm_ctx qcm_ctx;
typedef struct qcm_boundary qcm_boundary;
typedef struct qcm_heff qcm_heff;

/* One charge sector of an Index: TwoU1 charge (a, b) = (N_up, N_down) and size.
 * Sector lists are in strictly descending lexicographic charge order, as the
 * reference's sorted Index (block_matrix/indexing_stable.hpp:97-300). */
typedef struct {
    int32_t a, b;
    uint32_t size;
} qcm_sector;

/* Boundary (environment) tensor: the reference's Boundary + BoundaryIndex
 * (mp_tensors/boundary.h:76-406).  Cohort ci couples bra sector cohort_bra[ci]
 * and ket sector cohort_ket[ci]; it holds n_blocks[ci] column-major blocks of
 * size(bra) x size(ket); offsets[ci*aux_dim + b] is the element offset of MPO
 * index b inside the cohort (-1 = absent), cscale the conjugate scale, tr[ci]
 * = 1 if the cohort is stored as its Hermitian partner's transpose.
 * n_blocks may be NULL (then counted from offsets; 0 for tr cohorts).
 * data + data_offset[ci] holds the cohort's values (host memory). */
typedef struct {
    uint32_t n_bra, n_ket;
    const qcm_sector* bra;
    const qcm_sector* ket;
    uint32_t n_cohorts, aux_dim;
    const uint32_t* cohort_bra;
    const uint32_t* cohort_ket;
    const uint8_t* tr;
    const uint32_t* n_blocks;
    const int64_t* offsets;
    const double* cscale;
    const uint64_t* data_offset;
    const double* data;
} qcm_boundary_desc;

/* Indices of the right-paired two-site tensor (twin MPS, twositetensor.hpp:131-150). */
typedef struct {
    uint32_t n_phys, n_left, n_right;
    const qcm_sector* phys;
    const qcm_sector* left;
    const qcm_sector* right;
} qcm_mps_desc;

typedef struct {
    uint64_t vec_len, t_len, s_len;
    uint64_t n_tjobs, n_ttiles, n_gtasks /* S-build units */, n_alpha, n_segs, n_outs, n_otiles;
    double flops, flops_t, flops_ls, flops_s; /* ScheduleNew::total_flops per H.psi (solver/tasks.cpp:388-398, 777-796) */
    uint64_t g_elems, g_reads;                /* S elements written / T elements read by the gather */
    uint64_t l_len, r_len;                    /* boundary elements resident in HBM */
    uint64_t n_kitems;                        /* split-K items of the L.S GEMM */
    double flops_sdense;                      /* tensor-core work of the S build (dense unit GEMMs) */
    uint64_t launches;                        /* own kernels launched per apply */
    uint64_t w_len;                           /* doubles of the dense coefficient blocks of the S build */
    double flops_sexec;                       /* tensor work the S-build tiles execute (padding included) */
    uint64_t p_len;                           /* doubles of the L.S split-K partial tiles */
} qcm_heff_info;

#define QCM_PLAN_BOOKKEEPING 1 /* keep the (cohort, unit, line, alpha) list for parity checks */
#define QCM_PLAN_HOST_ONLY 2   /* build the schedule on the host only (ctx may be NULL; no apply) */

/* Context on one CUDA device with its own stream.  Replaces accelerator::gpu
 * setup (solver/accelerator.cpp:52-330); QCM_ERR_NODEV without a GPU. */
int qcm_ctx_create(int device, qcm_ctx** out);
void qcm_ctx_destroy(qcm_ctx* ctx);
int qcm_ctx_synchronize(qcm_ctx* ctx);

/* Copy a boundary into HBM (resident).  Replaces storage::gpu::broadcast::fetch
 * of Boundary cohorts (utils/storage.h:441-519, 594-615). */
int qcm_boundary_upload(qcm_ctx* ctx, const qcm_boundary_desc* desc, qcm_boundary** out);
/* Index-only boundary (no device data) for host-only schedule construction. */
int qcm_boundary_index_create(const qcm_boundary_desc* desc, qcm_boundary** out);
void qcm_boundary_free(qcm_boundary* b);

/* Build the flattened contraction schedule of H_eff for the two-site tensor
 * `twin` between L and R with two-site MPO tensor ts_mpo[site] and stage it in
 * HBM.  Replaces create_contraction_schedule + ScheduleNew::stage_gpu
 * (contractions/create_schedule/site_hamil_schedule.hpp:42-93,
 * solver/tasks.cpp:918-977). */
int qcm_heff_plan_create(qcm_ctx* ctx, const qcm_boundary* L, const qcm_boundary* R, const qcm_mpo* ts_mpo, int site,
                         const qcm_mps_desc* twin, int flags, qcm_heff** out);
int qcm_heff_get_info(const qcm_heff* h, qcm_heff_info* info);

/* y = H_eff x.  x, y: host buffers of vec_len doubles, the twin's right-paired
 * blocks (ls x stripe, column-major) concatenated in left-sector order;
 * synchronous.  Replaces ietl::mult -> super_hamil_mv
 * (solver/ietl_interface_dv.h:112-118, solver/super_hamil_mv.hpp:100-155). */
int qcm_heff_apply(qcm_heff* h, const double* x, double* y);
/* Bounds the plan's coefficient blocks (the dense S-build operands, qcm_heff_info.w_len doubles) to
 * max_bytes of device memory: every FP64 apply then generates them chunk by chunk (consecutive S-build
 * units, at most max_bytes each unless one unit is larger) and runs each chunk's S-GEMM tiles from one
 * scratch, with the same result to the bit; the plan is staged again.  max_bytes = 0 keeps them
 * whole.  For problems whose blocks do not fit (they grow with the MPO bond dimension times the
 * squared sector sizes).  Mixed-form applies and plan groups need them whole (QCM_ERR_ARG). */
int qcm_heff_stream_coefficients(qcm_heff* h, uint64_t max_bytes);
/* Bounds the device memory of the plan's applies to about max_bytes of T slices, S rows and coefficient
 * blocks: the ket sectors are cut into consecutive chunks (a larger sector is a chunk of its own) and
 * every FP64 apply runs them in turn (T-GEMM, coefficient generation, S-GEMM and split-K L.S of the
 * chunk, in scratch buffers the size of the largest chunk), with the split-K partials of all chunks
 * summed at the end in the fixed order: the result equals the whole apply's to the bit.  The plan is
 * staged again.  max_bytes = 0 undoes it.  For problems whose T and S buffers (which grow with the MPO
 * bond dimension and the squared bond dimension) do not fit.  Supersedes qcm_heff_stream_coefficients;
 * mixed-form applies, the adjoint and plan groups need the whole apply (QCM_ERR_ARG). */
int qcm_heff_chunk_apply(qcm_heff* h, uint64_t max_bytes);
/* Same with device pointers, enqueued on the context stream (asynchronous). */
int qcm_heff_apply_device(qcm_heff* h, const double* x_dev, double* y_dev);

/* Precision forms of H_eff . psi (the reference has only the FP64 one):
 * QCM_PRECISION_FP64  -- the plain form, every contraction in FP64 (DMMA).
 * QCM_PRECISION_MIXED -- the S build (the coefficient-weighted sum over T slices, ~3/4 of the
 *   work) runs on the tensor cores as 3xTF32 (hi/lo split of FP32 operands, three TF32
 *   products per term, FP32 accumulation): relative error ~1e-7 instead of ~1e-16; T-GEMM,
 *   L.S GEMM, input and output stay FP64.  mma.sync m16n8k8 TF32 fragments, FP32 operands split
 *   at the fragment loads; the first mixed apply of a plan copies its coefficient blocks to FP32
 *   (HBM: half the FP64 blocks again); T in FP32 reuses the FP64 T buffer.
 * QCM_PRECISION_MIXED_TC -- the same arithmetic with the 16- and 32-line S tiles on tcgen05
 *   (TF32 MMAs issued by one thread from shared-memory descriptors, accumulator in tensor memory)
 *   from operands split in HBM (coefficient blocks: as much again as the FP64 ones).  A tile
 *   that gives up on a bounded wait is reported as an error by the next synchronising call
 *   (qcm_heff_apply_mode, qcm_heff_profile_mode, qcm_jd_solve_mode). */
#define QCM_PRECISION_FP64 0
#define QCM_PRECISION_MIXED 1
#define QCM_PRECISION_MIXED_TC 2
int qcm_heff_apply_mode(qcm_heff* h, const double* x, double* y, int precision);
int qcm_heff_apply_device_mode(qcm_heff* h, const double* x_dev, double* y_dev, int precision);

/* Bookkeeping rows (parity checks; plan built with QCM_PLAN_BOOKKEEPING):
 * ints[10*i..] = (lb_in, lb_out, ci, ci_eff, unit_offset, ms, b1_row,
 * mps_offset, ci_right, column), alpha[i].  Call with ints == NULL for *n. */
int qcm_heff_bookkeeping(const qcm_heff* h, uint32_t* ints, double* alpha, uint64_t cap, uint64_t* n);
/* One device apply with CUDA events between the phases, synchronous:
 * ms[0] T-GEMM, ms[1] S gather, ms[2] L.S GEMM, ms[3] whole H.psi. */
int qcm_heff_profile(qcm_heff* h, const double* x_dev, double* y_dev, float* ms);
int qcm_heff_profile_mode(qcm_heff* h, const double* x_dev, double* y_dev, float* ms, int precision);
void qcm_heff_free(qcm_heff* h);

/* Groups of independent plans (the batching form; no counterpart in the reference, which runs one
 * schedule per solve and splits a schedule's ket sectors over devices and threads,
 * solver/tasks.cpp:884-977).  A group merges the work lists of n plans of one context into one plan:
 * one apply of the group runs every member's H_eff in one launch sequence (T-GEMM, S build and
 * split-K L.S per tile shape), each member's arithmetic unchanged, so member i's result equals
 * qcm_heff_apply on that plan bit for bit.  The members' vectors live in one arena of arena_len
 * doubles: member i's vector (its vec_len doubles, the qcm_heff_apply layout) at offsets[i]; the
 * gaps between them are ignored on input and zero on output.  The members must outlive the group;
 * FP64 only.  Typical use: many small independent site problems (for example one step of each of many
 * independent DMRG solves), whose separate applies would be bound by launch latency. */
typedef struct qcm_heff_group qcm_heff_group;
int qcm_heff_group_create(qcm_ctx* ctx, qcm_heff* const* plans, int n, qcm_heff_group** out);
/* *arena_len, and offsets[n] / lengths[n] of the members (any may be NULL). */
int qcm_heff_group_layout(const qcm_heff_group* g, uint64_t* arena_len, uint64_t* offsets, uint64_t* lengths);
/* vec_len (the arena length), buffer sizes, flop counts (summed over the members) and launches. */
int qcm_heff_group_get_info(const qcm_heff_group* g, qcm_heff_info* info);
/* y = H_eff x for every member; host arenas (synchronous) or device arenas (enqueued on the context
 * stream). */
int qcm_heff_group_apply(qcm_heff_group* g, const double* x, double* y);
int qcm_heff_group_apply_device(qcm_heff_group* g, const double* x_dev, double* y_dev);
/* Lowest eigenpair of every member by Jacobi-Davidson in lockstep (host arenas x0 -> out; evals[n],
 * iters[n]; *applies: group applies run).  Each iteration applies all members at once and runs the
 * rest of the iteration (classical Gram-Schmidt twice, Rayleigh-Ritz on the device, residuals,
 * convergence |r| <= tol |theta| or |r| < tol, next direction -r + (r.u)/(u.u) u as in
 * ietl/jacobi.h:386-474) for all members in single launches; with use_graphs each iteration is
 * captured once as a CUDA graph and replayed.  A converged member keeps its eigenpair; the group
 * stops when every member has converged or after maxiter (1..16) iterations. */
int qcm_jd_solve_batched(qcm_heff_group* g, const double* x0, double tol, int maxiter, int use_graphs, double* out,
                         double* evals, int* iters, int* applies);
void qcm_heff_group_free(qcm_heff_group* g);

/* No counterpart in the reference.  For callers that cannot allocate device memory
 * when they need H.psi -- a host code whose HBM is owned by its own caching
 * allocator (a cudaMalloc here may fail or fragment it) or a solver loop that
 * must not stall on cudaFree's device-wide synchronisation -- this variant of
 * qcm_heff_apply_device calls no cudaMalloc/cudaFree and no allocating library
 * routine.  It is the FP64 form only (QCM_PRECISION_FP64), whatever precision
 * the plan's other applies use.  Its scratch (T slices, S, split-K partials,
 * qcm_heff_info t_len + s_len + p_len, each rounded up to 32) lives in one
 * fixed static device array of QCM_NOALLOC_SCRATCH_DOUBLES doubles (64 MiB),
 * which every GPU that loads this library holds until the process exits.  Plans
 * needing more scratch are rejected with QCM_ERR_ARG.  qcm_ctx_create looks the
 * array's device address up on its device (cudaGetSymbolAddress, which also
 * makes the device load the array): create the context before the host
 * allocator reserves HBM and before any stream capture.  The address belongs to
 * the context: after cudaDeviceReset the context and its plans are invalid.
 * All calls on a device share the array and it keeps the last call's contents
 * (S is cleared inside each call): calls that overlap on the GPU -- other
 * streams, other threads -- race.  Makes the context's device current for the
 * call and restores the caller's.  Enqueued on the context stream
 * (asynchronous). */
#define QCM_NOALLOC_SCRATCH_DOUBLES (8u * 1024u * 1024u)
int qcm_heff_apply_device_noalloc(qcm_heff* h, const double* x_dev, double* y_dev);

/* Adjoint of the H_eff apply (the differentiation form; no counterpart in the reference, which has
 * no derivative of its schedule).  For f = ybar . H_eff x (host buffers of vec_len doubles):
 *   psi_bar   = H_eff^T ybar, which is H_eff ybar: the two-site H_eff of a Hermitian MPO is symmetric;
 *   coeff_bar[e] = df / d scale_e for every entry e of the plan's two-site MPO tensor, in the tensor's
 *                  entry order (qcm_mpo_tensor_terms on the two-site MPO at the plan's site), with the
 *                  boundaries held fixed; qcm_heff_adjoint_terms gives the count.
 * f is linear in the scales: the schedule's coefficients alpha (site_hamil_tasks.hpp:41-137) are
 * scale_e times a product of operator and conjugation factors, and S = sum alpha T (tasks.cpp:466-494).
 * The gradient runs the apply's contractions transposed on the device: Sbar = L^T ybar, per S-build
 * unit Wbar = Sbar T^T (FP64 tensor cores), then a fixed-order sum per entry (deterministic).
 * psi_bar or coeff_bar may be NULL (x is read only for coeff_bar). */
int qcm_heff_adjoint(qcm_heff* h, const double* x, const double* ybar, double* psi_bar, double* coeff_bar);
int qcm_heff_adjoint_terms(const qcm_heff* h, uint64_t* n_terms);

/* ------------------------------------------------------------------------ */
/* Eigensolver, boundary propagation and the two-site sweep                   */
/* ------------------------------------------------------------------------ */

/* Lowest eigenpair of H_eff by Jacobi-Davidson (no GMRES inner solve, no ortho vectors), start
 * vector x0, eigenvector to out (host buffers of vec_len doubles, the
 * qcm_heff_apply layout); search space and updates in HBM.  Replaces
 * solve<double>(out, initial, SH, ortho = {}, jcd_gmres = 0, tol, maxiter)
 * (solver/solver.cpp:14-28 -> solve_ietl_jcd, ietl_jacobi_davidson.h:35-76,
 * ietl/jacobi.h:386-474).  Returns the eigenvalue in *eval (no core energy). */
int qcm_jd_solve(qcm_heff* h, const double* x0, double tol, int maxiter, double* out, double* eval, int* iters);
/* Same with a precision form of the H.psi (QCM_PRECISION_*).  Mixed: every iteration uses the
 * mixed H.psi and stops once |r| <= max(tol, 1e-7) |theta| (or at maxiter); the returned
 * eigenvalue is the FP64 Rayleigh quotient of the final vector (one more FP64 H.psi), whose
 * error is of second order in the vector's. */
int qcm_jd_solve_mode(qcm_heff* h, const double* x0, double tol, int maxiter, int precision, double* out, double* eval,
                      int* iters);
/* The full solver seam: solve<double>(out, initial, SH, ortho_vecs, jcd_gmres, jcd_tol, jcd_max_iter)
 * (solver/solver.h:64-68, solver.cpp:14-28 -> solve_ietl_jcd, ietl_jacobi_davidson.h:35-76).
 * ortho[i] (i < n_ortho; host, vec_len doubles each) are states the solution is kept orthogonal to
 * (excited states): they are Gram-Schmidt'd among themselves, then projected out of the start
 * vector, of every new search direction and of A u (DavidsonVS::project, ietl_interface_dv.h:94-99);
 * at most vec_len - 1 are used.  gmres (0..64, ietl_jcd_gmres) is the GMRES iteration count of each
 * correction equation (I - uu*)(A - theta)(I - uu*) t = -r, started from t0 = -r + (r.u)/(u.u) u with
 * absolute tolerance 2^-(it+1) (jcd_gmres_solver, ietl/jacobi.h:126-164; ietl_gmres,
 * ietl/gmres.h:78-146); 0 uses t0.  As in the reference, GMRES keeps only the directions before its
 * last inner step, so gmres = 1 gives the same result as 0 at one more H.psi per correction.
 * *applies (may be NULL): H.psi applies made (the mixed form's FP64 Rayleigh quotient excluded). */
int qcm_jd_solve_ex(qcm_heff* h, const double* x0, const double* const* ortho, int n_ortho, int gmres, double tol,
                    int maxiter, int precision, double* out, double* eval, int* iters, int* applies);

/* New environment from one MPS site tensor, given right-paired (its blocks
 * ls x stripe, column-major, concatenated in left-sector order, as for
 * qcm_heff_apply), with bra = ket.  mpo: single-site MPO, tensor `site`.
 * symmetric != 0 applies the Hermitian complement (complement_transpose).
 * Replace contraction::Engine::overlap_mpo_left_step / overlap_mpo_right_step
 * (contractions/engine.hpp:54-71, boundary_ops/move_boundary.hpp:147-404). */
int qcm_boundary_step_left(qcm_ctx* ctx, const qcm_boundary* L, const qcm_mpo* mpo, int site, const qcm_mps_desc* mps,
                           const double* data_rp, int symmetric, qcm_boundary** out);
int qcm_boundary_step_right(qcm_ctx* ctx, const qcm_boundary* R, const qcm_mpo* mpo, int site, const qcm_mps_desc* mps,
                            const double* data_rp, int symmetric, qcm_boundary** out);

typedef struct {
    uint32_t n_bra, n_ket, n_cohorts, aux_dim;
    uint64_t total;    /* doubles in the device buffer (cohorts start on 32-element boundaries) */
    uint32_t resident; /* 1 if the boundary holds device data */
} qcm_boundary_info;
int qcm_boundary_get_info(const qcm_boundary* b, qcm_boundary_info* info);
/* Copy the index and data of a boundary to host arrays sized from
 * qcm_boundary_get_info (n_cohorts, n_cohorts * aux_dim, total); any pointer
 * may be NULL.  Same fields as qcm_boundary_desc. */
int qcm_boundary_download(const qcm_boundary* b, qcm_sector* bra, qcm_sector* ket, uint32_t* cohort_bra,
                          uint32_t* cohort_ket, uint8_t* tr, uint32_t* n_blocks, int64_t* offsets, double* cscale,
                          uint64_t* data_offset, double* data);

/* Two-site ground-state DMRG with the whole step on the device (H_eff plan,
 * JD, SVD truncation, QR/LQ canonisation, boundary step).  Replaces
 * ts_optimize<Matrix, SymmGroup, Storage> (optimize/ts_optimize.hpp:62-362)
 * with init_state = const (mp_tensors/mps_initializers.h:84-100). */
typedef struct qcm_dmrg qcm_dmrg;
typedef struct {
    uint64_t max_bond_dimension;  /* max_bond_dimension */
    uint64_t init_bond_dimension; /* init_bond_dimension */
    double truncation_cutoff;     /* truncation_final */
    double jcd_tol;               /* ietl_jcd_tol */
    int32_t jcd_maxiter;          /* ietl_jcd_maxiter (1..64) */
    double ecore;                 /* added to the reported energies */
    int32_t twosite_truncation;   /* 0: svd, 1: heev on the reduced density matrix with noise alpha */
    double alpha_initial, alpha_main, alpha_final; /* noise of sweeps < ngrowsweeps, < + nmainsweeps, later */
    int32_t ngrowsweeps, nmainsweeps;
    int32_t hpsi_precision;       /* QCM_PRECISION_FP64, or QCM_PRECISION_MIXED: JD with the mixed H.psi
                                     and an FP64 Rayleigh quotient of each step's final vector */
    int32_t jcd_gmres;            /* ietl_jcd_gmres (0..64): GMRES iterations per JD correction */
    int32_t optimization;         /* QCM_OPTIMIZATION_TWOSITE (ts_optimize) or QCM_OPTIMIZATION_SINGLESITE
                                     (ss_optimize.hpp:59-186: 2L steps per sweep, sites 0 .. L-1 then
                                     L-1 .. 0, each solved with the single-site MPO tensor and grown by
                                     the density-matrix prediction with noise alpha_*; twosite_truncation
                                     does not apply) */
    double mixed_residual_floor;  /* QCM_PRECISION_MIXED*: the mixed iterations of a step's JD stop as the
                                     FP64 ones do (|r| <= jcd_tol |theta| or jcd_maxiter), so that the sweep
                                     follows the FP64 sweep's path; > 0: they also stop once |r| <= this
                                     |theta| and |r| no longer halves (below the mixed H.psi's relative
                                     error, ~1e-7, the residual is noise): fewer applies in converged
                                     sweeps, a path that can leave the FP64 one by ~1e-5 Eh early on */
    int32_t mixed_fp64_refine;    /* QCM_PRECISION_MIXED*: FP64 residual-correction steps after them (0: only
                                     the FP64 Rayleigh quotient of the final vector); each is one FP64
                                     H.psi and one Jacobi-Davidson step while |r| > jcd_tol |theta| */
} qcm_dmrg_params;
#define QCM_OPTIMIZATION_TWOSITE 0
#define QCM_OPTIMIZATION_SINGLESITE 1
/* block_matrix_algorithms.h:48-63 */
typedef struct {
    uint64_t bond_dimension;
    double truncated_weight, truncated_fraction, smallest_ev;
} qcm_trunc_result;
typedef struct {
    uint64_t hpsi_count;
    double hpsi_flops; /* reference flop count (ScheduleNew::total_flops) summed over the applies */
    double plan_s, jd_s, trunc_s, boundary_s, total_s; /* wall time per phase, summed over sweeps */
    uint64_t hpsi_count_fp64;  /* mixed form: the FP64 applies of the residual correction (not in hpsi_count) */
    double hpsi_flops_fp64;
    /* step plans built from scratch, and re-staged from the previous sweep's plan of the same step
     * (whose boundaries and site indices had the same structure: sectors, cohorts, block offsets,
     * conjugate scales), which skips the host schedule construction
     * (create_contraction_schedule, site_hamil_schedule.hpp:42-93) */
    uint64_t plans_built, plans_reused;
    /* boundary steps whose schedule was built, and those that ran the previous sweep's schedule of the
     * same step again (same structure: old boundary, site tensor sectors and block layouts) */
    uint64_t bsteps_built, bsteps_reused;
    /* device bytes of the sweep's boundaries after a step (the largest since the run was created or
     * its boundary budget last set), and the boundaries moved to pinned host memory and back under
     * qcm_dmrg_set_boundary_budget */
    uint64_t boundary_bytes_peak, boundaries_offloaded, boundaries_fetched;
} qcm_dmrg_stats;

/* mpo: single-site QC MPO; nup/ndown: u1_total_charge1/2.  Builds the const
 * MPS, canonises it to site 0 and the right boundaries. */
int qcm_dmrg_create(qcm_ctx* ctx, const qcm_mpo* mpo, int nup, int ndown, const qcm_dmrg_params* params, qcm_dmrg** out);
/* Same with a given MPS (restart): sites[i] / data[i] describe site tensor i
 * right-paired, as for qcm_boundary_step_*; sites 1 .. L-1 right-normalised
 * (the state canonize(0) leaves).  The right boundaries are built on the device. */
int qcm_dmrg_create_from_mps(qcm_ctx* ctx, const qcm_mpo* mpo, const qcm_dmrg_params* params, const qcm_mps_desc* sites,
                             const double* const* data, qcm_dmrg** out);
/* Same, resuming the sweep at initial_site (ts_optimize initial_site_, optimize/ts_optimize.hpp:50-57):
 * left boundaries over sites 0 .. initial_site-1 and right boundaries over L-1 .. initial_site, as
 * init_left_right(mpo, initial_site) builds them (optimize/optimize.h:158-195); the next step is
 * initial_site of the left-to-right half-sweep (qcm_dmrg_pending_plan gives its site problem).  The
 * boundaries are built from the given MPS as it is (no optimisation or canonisation). */
int qcm_dmrg_create_from_mps_at(qcm_ctx* ctx, const qcm_mpo* mpo, const qcm_dmrg_params* params, const qcm_mps_desc* sites,
                                const double* const* data, int initial_site, qcm_dmrg** out);
int qcm_dmrg_length(const qcm_dmrg* d);
/* Steps of one sweep: 2L - 2 (two-site) or 2L (single-site). */
int qcm_dmrg_steps_per_sweep(const qcm_dmrg* d);
/* Excited states (ts_optimize.hpp:217-223, optimize.h:134-172): n_states ortho states (for example
 * converged lower states), each given as L site tensors sites[o*L + i] / data[o*L + i] (right-paired, as
 * for qcm_dmrg_create_from_mps; same physical basis and end sectors as the DMRG state).  From then on
 * every step's Jacobi-Davidson keeps its solution orthogonal to the ortho states' projections onto the
 * step's two-site basis (site_ortho_boundaries, contractions/special.hpp:38-62), and the overlap
 * boundaries with each ortho state (mps.h:175-219) move with the sweep.  Call between sweeps, before
 * the first step of a sweep; replaces earlier ortho states (n_states = 0 clears them). */
int qcm_dmrg_set_ortho(qcm_dmrg* d, int n_states, const qcm_mps_desc* sites, const double* const* data);
/* Site tensor `site` of the current MPS as a "QMPS" v1 blob: u32 magic 0x53504D51, u32 1; Index phys,
 * left, right (u32 count, then i32 a, i32 b, u32 dim per sector); u32 blocks, then per block i32 a, i32 b
 * (left charge), u32 rows, u32 cols and rows x cols doubles (right-paired, column-major).  Call with
 * buf == NULL for *len.  Between steps the MPS is the state the sweep has reached (checkpoints, ortho
 * states for a later excited-state run). */
int qcm_dmrg_export_site(qcm_dmrg* d, int site, void* buf, size_t cap, size_t* len);
/* Spin-summed one-particle density matrix of the current MPS, gamma[i + j*L] = <Psi| sum_s a+_is a_js |Psi>
 * (L x L, symmetric; the oneptdm measurement, lib/interface/cpp_maquis.cpp:235-366), which is the energy
 * derivative dE/dh_ij of the Hamiltonian sum_ij h_ij sum_s a+_is a_js + ... (Hellmann-Feynman).  Computed
 * between sweeps as the expectation values of the one-body operators of h = e_ij + e_ji (their QC MPOs,
 * bond dimension <= 6) through left boundary steps over the whole MPS: L(L+1)/2 contractions. */
int qcm_dmrg_measure_1rdm(qcm_dmrg* d, double* gamma);
/* Two-body energy gradient of the current MPS (the twoptdm measurement in the form the integrals enter):
 * G[p + q L + r L^2 + s L^3] (L^4 doubles) with E_2 = sum_pqrs V_pqrs G_pqrs for every V of the 8-fold
 * symmetry of real (pq|rs), i.e. dE/dV_pqrs; G is 1/2 the spin-summed two-particle density matrix
 * symmetrised over the 8 index permutations.  One expectation value per unique integral (the QC MPO of
 * the integral's orbit): about L^4 / 8 contractions, for small and moderate L. */
int qcm_dmrg_measure_2rdm_grad(qcm_dmrg* d, double* G);
/* Differentiation form: the energy's gradient through the adjoint of the apply (heff_adjoint; the
 * reference has no counterpart, its oneptdm / twoptdm measurements, lib/interface/cpp_maquis.cpp:235-366,
 * are what the gradients are checked against).  E = <Psi|W|Psi> / <Psi|Psi> of the current MPS is linear
 * in each site tensor of W, so dE/d scale_e for an entry of site k is the adjoint of the single-site
 * H_eff of site k (boundaries of W) with x = ybar = the orthogonality centre at k; the centre moves
 * through a copy of the MPS by QR, with one left boundary step of W per site (the boundaries of W are
 * recomputed for the gradient, not kept from the sweep).  Between sweeps.
 * qcm_dmrg_mpo_gradient: W any single-site MPO of the state's physical basis and length; grad[k] receives
 * qcm_mpo_tensor_terms(W, k) doubles, dE/d scale in W[k]'s entry order. */
int qcm_dmrg_mpo_gradient(qcm_dmrg* d, const qcm_mpo* W, double* const* grad);
/* qcm_dmrg_integral_gradient: dE/dh and dE/dV of the QC Hamiltonian of qcm_mpo_build_qc(L, h, V) (the
 * integrals of the state's own Hamiltonian, or any others) through the MPO's integral provenance: the
 * builder keeps every term the spin structure allows, whatever its value, and records which integrals
 * each entry's scale sums; the entry gradients of qcm_dmrg_mpo_gradient are then summed per integral.
 * dh[p*L + q] = dE/dh[p*L + q] and dV[((p*L + q)*L + r)*L + s] = dE/dV[((p*L + q)*L + r)*L + s], every
 * array element as its own variable (dV may be NULL): dh is the spin-summed 1-RDM <a+_p a_q>, and
 * averaging dV over the 8 index permutations of real (pq|rs) gives qcm_dmrg_measure_2rdm_grad.
 * E - ecore = sum h dh + sum V dV (E is linear in the integrals). */
int qcm_dmrg_integral_gradient(qcm_dmrg* d, const double* h, const double* V, double* dh, double* dV);
/* One sweep (qcm_dmrg_steps_per_sweep steps: 2L - 2 two-site, 2L single-site): energies[steps],
 * trunc[steps] (may be NULL); only between sweeps (see qcm_dmrg_run).  Single-site steps that end a
 * half-sweep (site L-1 left to right, site 0 right to left) canonise without truncation and report
 * zero truncation results. */
int qcm_dmrg_sweep(qcm_dmrg* d, double* energies, qcm_trunc_result* trunc);
/* One sweep of n independent runs in lockstep (the batching form for whole DMRG solves; the reference
 * runs one solve per process, sim.h / dmrg_sim.cpp): at every step each run builds (or re-binds) its
 * H_eff plan and two-site tensor, the n plans are merged into one plan group and one lockstep
 * Jacobi-Davidson (as qcm_jd_solve_batched, CUDA graphs) finds every run's ground state, then each run
 * truncates and moves its boundary as qcm_dmrg_sweep does.  Every run: two-site, FP64, no GMRES
 * corrections, no ortho states, jcd_maxiter <= 16, the same length, jcd_tol, jcd_maxiter and context,
 * between sweeps.  energies[n * steps] and trunc[n * steps] (may be NULL) run-major.  Each run's
 * energies agree with its own qcm_dmrg_sweep to the JD tolerance (the lockstep JD orthogonalises its
 * subspace by classical Gram-Schmidt twice instead of the single solve's modified Gram-Schmidt). */
int qcm_dmrg_group_sweep(qcm_dmrg* const* runs, int n, double* energies, qcm_trunc_result* trunc);
int qcm_dmrg_get_stats(const qcm_dmrg* d, qcm_dmrg_stats* stats);
/* Boundary residency (the reference keeps only the active boundaries in memory and moves the others
 * to its storage directory, utils/storage.h:88-330, ts_optimize.hpp:151-182): after every step the
 * boundaries no later step reads before the next half-sweep rebuilds them are released, and with
 * bytes > 0 the device copies of the others, farthest from the next step's two first, move to pinned
 * host memory until the device holds at most bytes of boundaries (the next step's two always stay);
 * a step brings its two back before it runs.  bytes = 0: no limit (the default).  Energies and
 * truncations do not depend on the budget. */
int qcm_dmrg_set_boundary_budget(qcm_dmrg* d, uint64_t bytes);
/* Coefficient blocks of the H_eff plans the run builds from here on bounded to max_bytes each
 * (qcm_heff_stream_coefficients); 0 keeps them whole (the default).  FP64 runs only, not in
 * qcm_dmrg_group_sweep.  Energies and truncations do not depend on it. */
int qcm_dmrg_set_coefficient_budget(qcm_dmrg* d, uint64_t max_bytes);
/* The H_eff plans the run builds from here on apply in ket-sector chunks of at most max_bytes of T, S and
 * coefficient blocks each (qcm_heff_chunk_apply; it supersedes the coefficient budget); 0 for whole
 * applies (the default).  FP64 runs only, not in qcm_dmrg_group_sweep.  Energies and truncations do not
 * depend on it. */
int qcm_dmrg_set_apply_budget(qcm_dmrg* d, uint64_t max_bytes);
/* Run the current sweep up to (not including) step stop_step (steps_per_sweep
 * completes it); energies / trunc receive one entry per step run (may be NULL),
 * *n_steps their count. */
int qcm_dmrg_run(qcm_dmrg* d, int stop_step, double* energies, qcm_trunc_result* trunc, int* n_steps);
/* Step index (0 .. steps_per_sweep - 1) the current sweep continues with. */
int qcm_dmrg_next_step(const qcm_dmrg* d);
/* (Two-site sweeps.)  H_eff plan of the pending step (its boundaries are the sweep's own: the plan
 * is valid until the sweep continues) and, if twin != NULL, its start vector
 * (vec_len doubles, cap = buffer length).  Replaces the snapshot of the site
 * problem that ts_optimize hands to solve_site_problem (ts_optimize.hpp:185-240). */
int qcm_dmrg_pending_plan(qcm_dmrg* d, double* twin, uint64_t cap, qcm_heff** out);
/* Start vector of the pending step (*n = vec_len; twin may be NULL to query). */
int qcm_dmrg_pending_twin(qcm_dmrg* d, double* twin, uint64_t cap, uint64_t* n);
/* The pending step's frozen site problem as a "QSPB" v1 blob (twin + L + R, the
 * interchange format read by the test oracle).  Call with buf == NULL for *len.
 * QCM_EXPORT_INDEX_ONLY: sectors and boundary indices only (blocks of width 0, cohorts
 * without values), enough to rebuild the H_eff schedule on a host. */
#define QCM_EXPORT_INDEX_ONLY 1
int qcm_dmrg_pending_export(qcm_dmrg* d, int flags, void* buf, size_t cap, size_t* len);
/* Current bond dimensions (right basis size of sites 0 .. L-2). */
int qcm_dmrg_bond_dimensions(const qcm_dmrg* d, uint64_t* dims);
void qcm_dmrg_free(qcm_dmrg* d);

/* ---- block-matrix truncation ----------------------------------------------
 * Replaces svd_truncate (block_matrix_algorithms.h:185-240 with estimate_truncation,
 * :136-183) and heev_truncate (:299-355) for a block matrix given as n_blocks
 * column-major host blocks concatenated in block order.
 *
 * qcm_truncate_svd: thin SVD of every block on the device, then the largest singular
 * values over all blocks are kept (at most max_bond_dimension of them plus ties, none
 * below cutoff * s_max).  Outputs per block k, packed in block order with keep[k]
 * columns: U_k (rows x keep, ld rows), S_k (keep, descending), Vt_k (keep x cols, ld keep).
 * Size U, S, Vt for keep = min(rows, cols).  A block larger than 1024 in both
 * dimensions is refused. */
int qcm_truncate_svd(qcm_ctx* ctx, uint32_t n_blocks, const uint32_t* rows, const uint32_t* cols, const double* blocks,
                     uint64_t max_bond_dimension, double cutoff, uint32_t* keep, double* U, double* S, double* Vt,
                     qcm_trunc_result* result);
/* Thin QR (lq = 0) or LQ (lq = 1) of every block, all blocks in one launch (one CTA each, Householder
 * reflectors as geqrf / orgqr and gelqf / orglq define them): replaces qr / lq of
 * framework/alps/matrix/algorithms.hpp:260-325, which MPSTensor::normalize_left / normalize_right
 * (mp_tensors/mpstensor.hpp:242-300) call per block.  With k = min(rows, cols), outputs packed in block
 * order: QR -- Q_k (rows x k) in Q, R_k (k x cols, upper triangular) in R; LQ -- Q_k (k x cols) in Q,
 * L_k (rows x k, lower triangular) in R; all column-major. */
int qcm_qr_blocks(qcm_ctx* ctx, uint32_t n_blocks, const uint32_t* rows, const uint32_t* cols, const double* blocks,
                  int lq, double* Q, double* R);
/* qcm_truncate_heev: symmetric blocks (density matrices, dims[k] x dims[k]); the cut is on
 * sqrt of the positive eigenvalues and the truncated fraction is reported in both
 * truncated_weight and truncated_fraction (as heev_truncate does).  Outputs per block:
 * U_k (dims x keep, the kept eigenvectors in descending eigenvalue order) and evals
 * (the kept eigenvalues, descending). */
int qcm_truncate_heev(qcm_ctx* ctx, uint32_t n_blocks, const uint32_t* dims, const double* blocks, uint64_t max_bond_dimension,
                      double cutoff, uint32_t* keep, double* U, double* evals, qcm_trunc_result* result);

/* FP64 throughput probes on the current device (TFLOP/s): DMMA (mma.sync
 * m8n8k4 .f64) and DFMA loops.  Roofline denominators of the FP64 form. */
int qcm_probe_fp64_peaks(double* dmma_tflops, double* dfma_tflops);

#ifdef __cplusplus
}
#endif

#endif /* QCM_B200_H */
