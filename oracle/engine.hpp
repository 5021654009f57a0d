// ORACLE -- TEST INFRASTRUCTURE ONLY.  Contraction schedule (solver/tasks.h) restated.
#pragma once

#include <mutex>

#include "core.hpp"

namespace orc {

constexpr std::size_t BUFFER_ALIGNMENT = 128;  // solver/constants.h:6
inline std::size_t round_up(std::size_t x) { return (x + BUFFER_ALIGNMENT - 1) / BUFFER_ALIGNMENT * BUFFER_ALIGNMENT; }

// solver/tasks.h:59-85, tasks.cpp:72-97
struct SUnit {
    unsigned offset = 0, ms = 0;
    std::vector<unsigned> tidx;
    std::vector<double> alpha;
    std::vector<unsigned> b2s, b1;
    unsigned b2count = 0;
    // H_eff schedules only: per alpha, its MPO entry and d alpha / d (entry scale)
    std::vector<unsigned> term;
    std::vector<double> dalpha;
    void push_back(double s, unsigned ti, unsigned col) { alpha.push_back(s); b2count++; tidx.push_back(ti); tidx.push_back(col); }
    unsigned add_line(unsigned b) {
        unsigned ret = b2count;
        if (b2count) { b2s.push_back(b2count); b1.push_back(b); b2count = 0; }
        return ret;
    }
};

using TList = std::vector<std::vector<double>>;

// solver/tasks.h:50-190, tasks.cpp:141-526
struct Cohort {
    unsigned lb = 0, rb = 0, ls = 0, rs = 0, ci = 0, ci_eff = 0;
    unsigned sblock = 0, nSrows = 0, stripe = 0;
    std::vector<long> mpo_offsets;
    std::vector<unsigned> sfold;
    std::vector<SUnit> suv;

    Cohort(const std::vector<std::size_t>& phys_i, unsigned l_block, unsigned r_block, unsigned l_size, unsigned r_size,
           unsigned ci_, unsigned ci_eff_, unsigned mpodim, bool left = false);
    void push_back(unsigned s, unsigned ss2, double scale, unsigned ti, unsigned col) { suv[sfold[s] + ss2].push_back(scale, ti, col); }
    void push_term(unsigned s, unsigned ss2, unsigned e, double d) {
        suv[sfold[s] + ss2].term.push_back(e);
        suv[sfold[s] + ss2].dalpha.push_back(d);
    }
    void add_line(unsigned b1) { for (auto& su : suv) mpo_offsets[b1] += su.add_line(b1); }
    void add_unit(unsigned s, unsigned ss, unsigned m_size, unsigned offset) {
        for (unsigned i = 0; i < ss; ++i) { suv[sfold[s] + i].offset = i * m_size + offset; suv[sfold[s] + i].ms = m_size; stripe += m_size; }
    }
    void finalize();
    std::size_t n_tasks() const { std::size_t n = 0; for (auto& s : suv) n += s.alpha.size(); return n; }
    std::size_t n_flops() const;
    std::size_t S_size() const { return std::size_t(nSrows) * stripe * sblock; }
    std::vector<double> create_s(const TList& T) const;    // tasks.cpp:425-454
    std::vector<double> create_s_r(const TList& T) const;  // tasks.cpp:466-494
    void contract(const std::vector<const double*>& left, const TList& T, double* out, std::mutex& mu) const;  // :286-313
    std::vector<double> contract_buf(const std::vector<const double*>& left, const TList& T) const;     // same, no accumulation
    void prop_l(const double* bra, const TList& T, double* new_left) const;   // :198-209
    void prop_r(const double* bra, const TList& T, double* new_right) const;  // :243-260
    void lbtm(const TList& T, double* out, double alpha) const;               // :346-362
    void rbtm(const TList& T, double* out, double alpha) const;               // :364-380
};

// (mps_offset, ci, ci_eff, lb_ket, aligned size)  solver/tasks.h:234-239
struct TJob { unsigned mps_offset, ci, ci_eff, lb_ket; std::size_t sza; };

// solver/tasks.h:193-268
struct MPSBlock {
    std::vector<TJob> t_schedule;
    std::size_t buf_size = 0;
    std::vector<Cohort> data;
    const std::vector<std::size_t>* lr_ket_sizes = nullptr;
    const BoundaryIndex* left_rt = nullptr;
    const BoundaryIndex* right_rt = nullptr;
    unsigned rb_ket = 0;
    unsigned get_ti(unsigned mps_offset, unsigned ci_virt) const;
    TList create_T(const std::vector<const double*>& right, const std::vector<const double*>& mps) const;       // :650-705
    TList create_T_left(const std::vector<const double*>& left, const std::vector<const double*>& mps) const;  // :545-601
    std::size_t n_flops(const BoundaryIndex& right) const;  // :777-796
};

// solver/tasks.h:287-348
struct Schedule {
    std::vector<std::size_t> lr_ket_sizes;
    std::vector<MPSBlock> blocks;
    std::size_t total_flops = 0;
    std::vector<std::size_t> mps_block_sizes;
};

// create_contraction_schedule (create_schedule/site_hamil_schedule.hpp:42-93) for a
// right-paired ket; the schedule holds pointers to L and R indices.
std::unique_ptr<Schedule> create_contraction_schedule(MPSTensor& initial, const Boundary& left, const Boundary& right,
                                                      const MPOTensor& mpo);

// super_hamil_mv (solver/super_hamil_mv.hpp:100-155), CPU branch; x, y = right-paired block data
void super_hamil_mv(const Schedule& sched, const Boundary& left, const Boundary& right,
                    const std::vector<const double*>& x, const std::vector<double*>& y);
// Adjoint of super_hamil_mv with respect to the scales of the MPO entries (the differentiation form):
// grad[e] = d (ybar . H x) / d scale_e for every entry e of the schedule's MPO tensor (n_terms entries)
void scale_gradient(const Schedule& sched, const Boundary& left, const Boundary& right, const std::vector<const double*>& x,
                    const std::vector<const double*>& ybar, std::size_t n_terms, std::vector<double>& grad);

// boundary steps (contractions/boundary_ops/move_boundary.hpp:147-404)
Boundary overlap_mpo_left_step(const MPSTensor& bra, const MPSTensor& ket, const Boundary& left, const MPOTensor& mpo,
                               bool symmetric);
Boundary overlap_mpo_right_step(const MPSTensor& bra, const MPSTensor& ket, const Boundary& right, const MPOTensor& mpo,
                                bool symmetric);

// density-matrix noise (contractions/boundary_ops/move_boundary.hpp:37-145): dm[rb] += alpha S S^T
// (left, blocks of dm keyed by the ket's right sectors) / dm[lb] += alpha S^T S (right)
void alpha_dm_direct(const MPSTensor& ket, const Boundary& left, const MPOTensor& mpo, BlockMatrix& dm, double alpha);
void alpha_dm_direct_right(const MPSTensor& ket, const Boundary& right, const MPOTensor& mpo, BlockMatrix& dm, double alpha);

}  // namespace orc
