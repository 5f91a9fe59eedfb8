// Flat, symmetry-agnostic execution plan shared by the C ABI, the library's
// schedule builder and the device program compiler.  Field meanings are those
// of dmrgb200_plan_desc in include/dmrgb200.h.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "boundary_index.hpp"
#include "schedule.hpp"

namespace dmrgb200 {

enum PlanKind : int { KIND_HPSI = 0, KIND_LEFT = 1, KIND_RIGHT = 2 };

struct FlatPlan {
    int kind = KIND_HPSI;
    std::vector<uint32_t> g_t, g_c;  // task-group ranges (n_groups + 1 entries each)
    std::vector<uint32_t> in_rows, in_cols;
    std::vector<uint64_t> in_off;
    uint64_t in_size = 0;
    std::vector<uint32_t> out_rows, out_cols;
    std::vector<uint64_t> out_off;
    uint64_t out_size = 0;

    std::vector<uint32_t> t_lb, t_col, t_ci, t_nb, t_brows, t_bcols, t_width;
    std::vector<uint8_t> t_trans;

    std::vector<uint32_t> c_lb, c_rb, c_ls, c_rs, c_ci, c_nsrows, c_stripe, c_out_ci, c_unit;
    std::vector<uint8_t> c_trans;

    std::vector<uint32_t> u_offset, u_ms, u_line;
    std::vector<uint32_t> l_b1, l_term;
    std::vector<double> term_alpha;
    std::vector<uint32_t> term_t, term_col;
    // builder provenance (empty for plans from a caller's description): MPO term
    // of each plan term and d alpha / d (that term's scale); H psi plans only
    std::vector<uint32_t> term_src;
    std::vector<double> term_dscale;

    uint32_t n_groups() const { return g_t.empty() ? 0 : uint32_t(g_t.size() - 1); }
    uint32_t n_t() const { return uint32_t(t_lb.size()); }
    uint32_t n_cohorts() const { return uint32_t(c_lb.size()); }
    uint32_t n_units() const { return uint32_t(u_offset.size()); }
    uint32_t n_lines() const { return uint32_t(l_b1.size()); }
    uint32_t n_terms() const { return uint32_t(term_alpha.size()); }

    // reference flop formula (tasks.cpp:388-398, :777-796)
    uint64_t flops() const;
    // the same formula split into stage 1 (T), stage 2 (S build), stage 3 (contract)
    void stage_flops(uint64_t out[3]) const;
    // T rows / T-block columns per task, following the plan kind
    uint64_t t_rows(uint32_t t) const { return kind == KIND_LEFT ? t_brows[t] : in_rows[t_lb[t]]; }
    uint64_t t_block_cols(uint32_t t) const { return kind == KIND_LEFT ? t_width[t] : t_bcols[t]; }
    uint64_t t_size(uint32_t t) const { return uint64_t(t_nb[t]) * t_rows(t) * t_block_cols(t); }

    // Structural validation; returns an empty string when consistent.
    std::string validate() const;
};

// 128-element padded block layout of an MPS tensor (davidson_vector.cpp:96-97)
struct TensorLayout {
    std::vector<uint32_t> rows, cols;
    std::vector<uint64_t> off;
    uint64_t total = 0;
};
TensorLayout right_paired_layout(Index const& phys, Index const& left, Index const& right);
TensorLayout left_paired_layout(Index const& phys, Index const& left, Index const& right);

inline uint64_t round_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

// Concatenate independent H psi plans into one: instance i's in/out blocks are
// shifted by in_base[i] / out_base[i] (returned), its T tasks, cohorts, units,
// lines, terms and groups are renumbered, and its boundary cohort indices are
// shifted by the given per-instance offsets into the concatenated views.
FlatPlan merge_plans(std::vector<FlatPlan> const& plans, std::vector<uint32_t> const& left_ci_base,
                     std::vector<uint32_t> const& right_ci_base, std::vector<uint64_t>& in_base,
                     std::vector<uint64_t>& out_base);

// Flatten a built schedule.  `other` is the boundary read by the T tasks
// (R for H psi and the right step, L for the left step); `lbnd` is L for H psi.
FlatPlan flatten_hpsi(Schedule const& s, TensorLayout const& psi, BoundaryIndex const& L, BoundaryIndex const& R);
FlatPlan flatten_left_step(Schedule const& s, TensorLayout const& ket_rp, TensorLayout const& bra_lp,
                           Index const& ket_right_i, BoundaryIndex const& L, BoundaryIndex const& out_index);
FlatPlan flatten_right_step(Schedule const& s, TensorLayout const& ket_rp, TensorLayout const& bra_rp,
                            BoundaryIndex const& R, BoundaryIndex const& out_index);

}  // namespace dmrgb200
