// Host-side contraction schedule: builder structures and builders.
//
// The three-level schedule (schedule -> per-input-block task group -> cohort)
// follows the reference's ScheduleNew / MPSBlock / Cohort
// (dmrg/framework/dmrg/solver/tasks.h:50-348, tasks.cpp:72-526):
//   * a task group owns the "T tasks" (stage 1: one boundary cohort times one
//     column slice of an MPS block),
//   * a cohort (one per (input block, output block) pair) owns S-units, one per
//     output physical sub-sector; a unit holds "lines", one per MPO row b1
//     (or column b2 for the left step), each a list of (alpha, T index, column).
// The builders restate the reference's symbolic enumeration:
//   create_contraction_schedule  site_hamil_schedule.hpp:40-93
//   rshtm_t_tasks / rshtm_tasks  right_tasks.hpp:39-167
//   shtm_tasks                   site_hamil_tasks.hpp:41-137
//   lshtm_t_tasks / lshtm_tasks  left_tasks.hpp:38-172
//   op_iterate                   op_iterate.hpp:37-69
#pragma once

#include <cstdint>
#include <unordered_map>
#include <vector>

#include "boundary_index.hpp"
#include "mpo.hpp"
#include "symm.hpp"

namespace dmrgb200 {

struct SUnit {
    unsigned offset = 0, ms = 0;
    std::vector<unsigned> tidx;  // pairs (T index, column)
    std::vector<double> alpha;
    std::vector<unsigned> b2s;   // terms per line
    std::vector<unsigned> b1;    // S row-block of each line
    // provenance of each term: the MPO term it comes from and d alpha / d (MPO term scale)
    std::vector<unsigned> src;
    std::vector<double> dscale;
    unsigned b2count = 0;

    void push_back(double scale, unsigned ti, unsigned col, unsigned from, double dsc) {
        alpha.push_back(scale);
        src.push_back(from);
        dscale.push_back(dsc);
        ++b2count;
        tidx.push_back(ti);
        tidx.push_back(col);
    }
    unsigned add_line(unsigned b) {
        unsigned n = b2count;
        if (b2count) {
            b2s.push_back(b2count);
            b1.push_back(b);
            b2count = 0;
        }
        return n;
    }
    size_t n_tasks() const { return alpha.size(); }
};

class Cohort {
public:
    // lb/rb: input/output block, ls/rs: their sizes; left selects the left-step S layout
    Cohort(std::vector<unsigned> const& phys_sizes, unsigned lb, unsigned rb, unsigned ls, unsigned rs, unsigned ci,
           unsigned ci_eff, unsigned mpodim, bool left = false);

    void push_back(unsigned s, unsigned ss2, double scale, unsigned ti, unsigned col, unsigned from, double dsc) {
        suv_[sfold_[s] + ss2].push_back(scale, ti, col, from, dsc);
    }
    void add_line(unsigned b1) {
        for (auto& u : suv_) mpo_offsets_[b1] += u.add_line(b1);
    }
    void add_unit(unsigned s, unsigned ss, unsigned m_size, unsigned offset) {
        for (unsigned i = 0; i < ss; ++i) {
            suv_[sfold_[s] + i].offset = i * m_size + offset;
            suv_[sfold_[s] + i].ms = m_size;
            stripe_ += m_size;
        }
    }
    // compress the MPO index to the rows that carry tasks (tasks.cpp:506-526)
    void finalize();

    size_t n_tasks() const;
    size_t n_flops() const;

    unsigned lb, rb, ls, rs, ci, ci_eff, sblock, nSrows, stripe_ = 0;
    std::vector<long> mpo_offsets_;
    std::vector<unsigned> sfold_;
    std::vector<SUnit> suv_;
};

struct TTask {
    unsigned mps_offset, ci, ci_eff, lb_ket;
};

struct MPSBlock {
    std::vector<TTask> t_schedule;
    std::vector<Cohort> cohorts;
    std::unordered_map<uint64_t, unsigned> ti_lookup;

    void push_t(TTask t) {
        ti_lookup.emplace((uint64_t(t.mps_offset) << 32) | t.ci, unsigned(t_schedule.size()));
        t_schedule.push_back(t);
    }
    // index of the T task for (column offset, cohort), UINT_MAX if none (tasks.cpp:766-775)
    unsigned get_ti(unsigned mps_offset, unsigned ci) const {
        auto it = ti_lookup.find((uint64_t(mps_offset) << 32) | ci);
        return it == ti_lookup.end() ? 0xFFFFFFFFu : it->second;
    }
};

struct Schedule {
    std::vector<MPSBlock> blocks;  // one per input (H psi, right step) or ket-right (left step) block
};

// --- builders -----------------------------------------------------------------

// H psi schedule for a right-paired two-site (or one-site) MPS tensor
Schedule create_contraction_schedule(Symm symm, Index const& phys_i, Index const& left_i, Index const& right_i,
                                     BoundaryIndex const& left, BoundaryIndex const& right, MPOTensor const& mpo);

// left boundary step: ket right-paired, bra left-paired; returns the new boundary index
Schedule left_step_schedule(Symm symm, Index const& phys_i, Index const& bra_left_i, Index const& bra_right_i,
                            Index const& ket_left_i, Index const& ket_right_i, BoundaryIndex const& left,
                            MPOTensor const& mpo, bool symmetric, BoundaryIndex& out_index);

// right boundary step: ket and bra right-paired
Schedule right_step_schedule(Symm symm, Index const& phys_i, Index const& bra_left_i, Index const& bra_right_i,
                             Index const& ket_left_i, BoundaryIndex const& right, MPOTensor const& mpo, bool symmetric,
                             BoundaryIndex& out_index);

}  // namespace dmrgb200
