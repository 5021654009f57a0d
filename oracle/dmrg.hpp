// ORACLE -- TEST INFRASTRUCTURE ONLY.  DMRG layer of the CPU restatement.
#pragma once

#include <functional>

#include "engine.hpp"

namespace orc {

// block_matrix/block_matrix_algorithms.h:48-63
struct TruncationResults {
    std::size_t bond_dimension = 0;
    double truncated_weight = 0, truncated_fraction = 0, smallest_ev = 0;
};

// two-site MPO (mp_tensors/ts_ops.hpp:97-168)
MPOTensor make_twosite_mpo(const MPOTensor& W1, const MPOTensor& W2);

// two-site tensor (mp_tensors/twositetensor.hpp)
struct TwoSite {
    Index phys1, phys2, phys, left, right;
    BlockMatrix both;  // both-paired: rows phys1 x left, cols phys2 x right
    TwoSite(MPSTensor a, MPSTensor b);
    MPSTensor make_mps() const;                      // reshape_both_to_right
    void set_from_mps(const MPSTensor& twin);        // reshape_right_to_both
    void split_l2r(std::size_t Mmax, double cutoff, MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const;
    void split_r2l(std::size_t Mmax, double cutoff, MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const;
    // predict_split_l2r / _r2l (contractions/boundary_ops/prediction.hpp:152-236): the reduced
    // density matrix plus alpha times the boundary noise term, truncated by heev_truncate;
    // alpha = 0 falls back to the SVD split
    void predict_split_l2r(std::size_t Mmax, double cutoff, double alpha, const Boundary& left, const MPOTensor& mpo,
                           MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const;
    void predict_split_r2l(std::size_t Mmax, double cutoff, double alpha, const Boundary& right, const MPOTensor& mpo,
                           MPSTensor& m1, MPSTensor& m2, TruncationResults& tr) const;
};

// estimate_truncation (block_matrix_algorithms.h:136-183) on per-block descending values
TruncationResults estimate_truncation(const std::vector<std::vector<double>>& vals, std::size_t Mmax, double cutoff,
                                      std::vector<std::size_t>& keeps);
// heev_truncate (block_matrix_algorithms.h:299-355): U = kept eigenvectors (descending), weight = fraction
TruncationResults heev_truncate(const BlockMatrix& dm, BlockMatrix& U, double cutoff, std::size_t Mmax);

// per-block SVD + estimate_truncation (block_matrix_algorithms.h:136-240)
TruncationResults svd_truncate(const BlockMatrix& M, BlockMatrix& U, BlockMatrix& V, std::vector<std::vector<double>>& S,
                               double cutoff, std::size_t Mmax);

// MPSTensor normalisation (mpstensor.hpp:242-352)
BlockMatrix normalize_left(MPSTensor& t);
BlockMatrix normalize_right(MPSTensor& t);
void multiply_from_left(MPSTensor& t, const BlockMatrix& N);
void multiply_from_right(MPSTensor& t, const BlockMatrix& N);

// Jacobi-Davidson for the lowest eigenpair (solve_ietl_jcd, ietl_jacobi_davidson.h:35-76; ietl/jacobi.h:386-474):
// correction equation by GMRES(gmres) (ietl/gmres.h:78-146; 0 = the projected residual only), search space
// kept orthogonal to `ortho`; *applies = mult calls
double jacobi_davidson(const std::function<void(const std::vector<double>&, std::vector<double>&)>& mult,
                       const std::vector<double>& x0, double tol, int maxiter, std::vector<double>& out, int& iters,
                       int gmres = 0, const std::vector<std::vector<double>>& ortho = {}, int* applies = nullptr);

struct DMRGParams {
    std::size_t Mmax = 64;
    std::size_t init_bond_dimension = 64;
    double cutoff = 1e-16;
    double jcd_tol = 1e-10;
    int jcd_maxiter = 8;
    int jcd_gmres = 0;  // ietl_jcd_gmres
    double ecore = 0.0;
    // twosite_truncation = heev and its noise (ts_optimize.hpp:275-296)
    bool heev = false;
    double alpha_initial = 1e-2, alpha_main = 1e-4, alpha_final = 1e-8;
    int ngrowsweeps = 0, nmainsweeps = 0;
    // optimization = singlesite (ss_optimize.hpp:59-186): 2L steps per sweep, every step grown by the
    // density-matrix prediction with the alpha above
    bool single_site = false;
};

// grow_l2r_sweep / grow_r2l_sweep (contractions/engine.hpp:85-123): the optimised site tensor a is
// replaced by the kept eigenvectors of its reduced density matrix plus alpha times the boundary noise
// (predict_new_state_*_sweep, contractions/boundary_ops/prediction.hpp:77-131), and the neighbour b takes
// the projection of the old a onto them (predict_lanczos_*_sweep, :93-148).  l2r: a left-paired result,
// b = (U^T a) b; r2l: a = U^T right-paired, b = b (a U).
TruncationResults grow_l2r(MPSTensor& a, MPSTensor& b, const Boundary& left, const MPOTensor& mpo, double alpha,
                           double cutoff, std::size_t Mmax);
TruncationResults grow_r2l(MPSTensor& a, MPSTensor& b, const Boundary& right, const MPOTensor& mpo, double alpha,
                           double cutoff, std::size_t Mmax);

struct DMRG {
    int L;
    std::vector<MPOTensor> mpo, ts_mpo;
    std::vector<MPSTensor> mps;
    std::vector<Boundary> left_, right_;
    DMRGParams p;
    std::size_t hpsi_count = 0;
    double hpsi_time = 0, jd_time = 0, schedule_time = 0, trunc_time = 0, boundary_time = 0;
    std::size_t hpsi_flops = 0;

    DMRG(std::vector<MPOTensor> mpo_single, int nup, int ndown, const DMRGParams& prm);
    // excited states (ts_optimize.hpp:217-223, optimize.h:134-172): ortho states the solution is kept
    // orthogonal to, and per state the overlap boundaries with the current MPS (rows current, columns
    // ortho).  set_ortho expects the sweep to start (the MPS canonised to site 0) and builds the right
    // boundaries.
    std::vector<std::vector<MPSTensor>> ortho_mps;
    std::vector<std::vector<BlockMatrix>> ortho_left_, ortho_right_;
    void set_ortho(std::vector<std::vector<MPSTensor>> states);
    // one full two-site sweep (ts_optimize.hpp:114-362); energies per step.
    // If stop_step >= 0 the sweep stops before solving that step and the
    // frozen site problem is written to *snap.
    void sweep(int sweep_no, std::vector<double>& energies, std::vector<TruncationResults>& trunc, int stop_step = -1,
               std::vector<uint8_t>* snap = nullptr);
    // one single-site sweep (ss_optimize.hpp:59-186): sites 0 .. L-1 left to right, then L-1 .. 0
    void sweep_single(int sweep_no, std::vector<double>& energies, std::vector<TruncationResults>& trunc);
    int steps_per_sweep() const { return p.single_site ? 2 * L : 2 * L - 2; }
};

// frozen site problem ("QSPB" v1): twin MPS (right-paired) + L + R boundaries
std::vector<uint8_t> save_site_problem(const MPSTensor& twin, const Boundary& L, const Boundary& R);
// The two-site problem at (site1, site1 + 1) of a given MPS: left boundaries over sites 0 .. site1-1 and
// right boundaries over L-1 .. site1+2, as init_left_right(mpo, site1) builds them (optimize.h:158-195;
// symmetric steps, optimize.h:134-156), and the fused two-site tensor; exported as "QSPB".
std::vector<uint8_t> site_problem_from_mps(const std::vector<MPOTensor>& mpo, const std::vector<MPSTensor>& mps, int site1);
void load_site_problem(const uint8_t* p, std::size_t n, MPSTensor& twin, Boundary& L, Boundary& R);

// one site tensor ("QMPS" v1): Index phys, left, right; right-paired blocks as in QSPB
std::vector<uint8_t> save_mps_tensor(const MPSTensor& m);
MPSTensor load_mps_tensor(const uint8_t* p, std::size_t n);

// overlap boundaries of the excited-state sweep (mp_tensors/mps.h:175-219), bra = the current MPS, ket =
// an ortho state, and an ortho state's projection onto the current two-site basis in the twin's block
// layout (contractions/special.hpp:38-62)
BlockMatrix ortho_left_step(const MPSTensor& bra, const MPSTensor& ket, const BlockMatrix& left);
BlockMatrix ortho_right_step(const MPSTensor& bra, const MPSTensor& ket, const BlockMatrix& right);
std::vector<double> ortho_vector(const MPSTensor& twin, const MPSTensor& ortho_twin, const BlockMatrix& left,
                                 const BlockMatrix& right);

// boundary step case ("QBSP" v1): side (0 left, 1 right), site; the site tensor (right-paired,
// same block layout as QSPB); the input boundary; the oracle's output boundary
std::vector<uint8_t> save_boundary_step(int side, int site, const MPSTensor& m, const Boundary& in, const Boundary& out);

}  // namespace orc
