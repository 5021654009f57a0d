// MPO tensors for the two-site DMRG path (host side).
//
// Mirrors the parts of framework/dmrg/mp_tensors/mpotensor.h the contraction
// schedule uses: row_dim/col_dim, row(b1) iteration in increasing b2
// (std::set row_index), column(b2) iteration in increasing b1 (CSC col_tags),
// at(b1,b2) -> list of (operator, scale) (term_descriptor), and the bond
// Hermitian-conjugate map (mpotensor_detail.h:141-186).
//
// Site operators use the reference's W(in, out) convention (a block
// (left_charge = phys_in, right_charge = phys_out) holds <out|O|in>, see
// site_hamil_tasks.hpp:109-110 and op_iterate.hpp:54-66); entries are stored
// as flat (in_state, out_state, value) over the physical Index's state order.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "symm.hpp"

namespace qcm {

struct SparseOp {
    std::vector<uint32_t> in, out;
    std::vector<double> val;
};

struct MPOTables;  // lookup tables derived from a finalized tensor (operator terms, entry layouts)

struct MPOTensor {
    uint32_t rows = 1, cols = 1;
    // entries sorted by (b1, b2); several consecutive entries may share (b1, b2)
    std::vector<uint32_t> b1, b2, op;
    std::vector<double> scale;
    std::shared_ptr<std::vector<SparseOp>> ops;
    Index phys;
    // Hermitian pairs on the left and right bond: herm[b] = partner or -1
    std::vector<int32_t> herm_left, phase_left, herm_right, phase_right;

    // derived lookup structures
    std::vector<uint32_t> row_ptr;   // CSR over entries (entries already row sorted)
    std::vector<uint32_t> col_ptr, col_ent;  // CSC: entries of column b2, increasing b1
    void finalize();
    // derived tables, built (and checked) on first use and shared by every schedule built
    // from this tensor; finalize() drops them
    std::shared_ptr<const MPOTables> tables() const;
    mutable std::shared_ptr<const MPOTables> tables_;
};

struct MPO {
    std::vector<MPOTensor> t;
    bool twosite = false;
};

// Integral provenance of a QC MPO: the scale of entry e of site tensor k is
//   sum_{j in [ptr[k][e], ptr[k][e + 1])} val[k][j] * x[id[k][j]],
// x = (h[0 .. L^2), V[0 .. L^4)) as passed to build_qc_mpo, every array element a variable of its
// own (pass-through entries have no provenance: their scale is 1).
struct IntegralProvenance {
    std::vector<std::vector<uint64_t>> ptr, id;
    std::vector<std::vector<double>> val;
};

// Builds the exact QC Hamiltonian MPO (TwoU1) from integrals h (L x L) and
// V (L^4, chemist notation (pq|rs)).  The core energy is not part of the MPO.
// With prov, every term the spin structure allows is kept whatever its value (cutoff is not
// applied) and the provenance of every entry is recorded: the MPO then holds an entry for every
// integral the energy depends on, zero-valued ones included.
MPO build_qc_mpo(int L, const double* h, const double* V, double cutoff, IntegralProvenance* prov = nullptr);

// dE/dx over the integrals from dE/d scale of every entry (grad[k][e], entry order of site k):
// dx[id] += val * grad for every provenance record; dx has L^2 + L^4 elements (h, then V).
void integral_gradient(const IntegralProvenance& prov, const std::vector<std::vector<double>>& grad, double* dx,
                       uint64_t n);

// Two-site MPO: W_ts[p](b1,b3) = sum_b2 kron(W[p](b1,b2), W[p+1](b2,b3))
// (mp_tensors/ts_ops.hpp:97-168).
MPO make_twosite_mpo(const MPO& m);

std::vector<uint8_t> serialize_mpo(const MPO& m);
MPO deserialize_mpo(const uint8_t* p, std::size_t n);

}  // namespace qcm
