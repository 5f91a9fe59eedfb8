// ORACLE — test infrastructure only.  The reference-side half of the drop-in
// boundary: a ScheduleNew<double> built through the reference's own Cohort /
// MPSBlock API (dmrg/framework/dmrg/solver/tasks.h:50-348) is flattened into the
// flat plan description that dmrgb200_plan_create takes (include/dmrgb200.h).
// This is the loop a maintainer adds beside create_contraction_schedule
// (site_hamil_schedule.hpp:40-93) to hand the schedule to libdmrgb200.
//
// Cohort keeps its geometry and S units private (tasks.h:57-95, 186-202) and the
// reference has no accessors for them; this file reads them by compiling the
// header with its access specifiers opened (the `private` macro below), which
// leaves the class layout unchanged.  In the reference tree the equivalent is a
// set of const getters on Cohort (lb, rb, ls, rs, ci, ci_eff, nSrows, stripe and
// the SUnit vector).
#include <cstdint>
#include <iostream>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

// everything tasks.h includes, first and unchanged, so that the macro below only
// opens the classes declared in tasks.h itself
#include "utils/timings.h"
#include "dmrg/utils/utils.hpp"
#include "dmrg/solver/accelerator.h"
#include "dmrg/solver/constants.h"
#include "dmrg/solver/vector_stage.h"
#include "dmrg/mp_tensors/boundary_index_rt.hpp"
#define private public
#include "dmrg/solver/tasks.h"
#undef private
#include "../include/dmrgb200.h"

using contraction::common::Cohort;
using contraction::common::MPSBlock;
using contraction::common::ScheduleNew;

// Flat arrays of one H psi schedule (owned here; the desc points into them).
struct RefFlat {
    std::vector<uint32_t> g_t, g_c, in_rows, in_cols, out_rows, out_cols;
    std::vector<uint64_t> in_off, out_off;
    std::vector<uint32_t> t_lb, t_col, t_ci, t_nb, t_brows, t_bcols;
    std::vector<uint8_t> t_trans, c_trans;
    std::vector<uint32_t> c_lb, c_rb, c_ls, c_rs, c_ci, c_nsrows, c_stripe, c_out_ci, c_unit;
    std::vector<uint32_t> u_offset, u_ms, u_line, l_b1, l_term, term_t, term_col;
    std::vector<double> term_alpha;
    dmrgb200_plan_desc desc{};
};

template <class T>
static const T* ptr(std::vector<T> const& v) {
    return v.empty() ? nullptr : v.data();
}

// Flatten `sched` (task group g = MPSBlock g, input block g).  The T-task shapes come
// from the right boundary's runtime index: rt cohorts 0 .. n_right-1 are the stored
// cohorts, a task whose cohort index differs from its storage cohort (ci != ci_eff)
// reads the Hermitian complement, i.e. the stored blocks transposed
// (tasks.cpp:650-705).  The vector layout (block rows, columns and 128-element
// padded offsets) is the DavidsonVector's, given by the caller.
// C linkage: the adapter declares these inside its extern "C" block
extern "C" void ref_flatten_hpsi(ScheduleNew<double> const& sched, BoundaryIndexRT const& right_rt,
                      std::vector<uint32_t> const& in_rows, std::vector<uint32_t> const& in_cols,
                      std::vector<uint64_t> const& in_off, uint64_t in_size, std::vector<uint32_t> const& out_rows,
                      std::vector<uint32_t> const& out_cols, std::vector<uint64_t> const& out_off, uint64_t out_size,
                      RefFlat& f) {
    f = RefFlat();
    f.in_rows = in_rows;
    f.in_cols = in_cols;
    f.in_off = in_off;
    f.out_rows = out_rows;
    f.out_cols = out_cols;
    f.out_off = out_off;
    f.g_t.push_back(0);
    f.g_c.push_back(0);
    f.c_unit.push_back(0);
    f.u_line.push_back(0);
    f.l_term.push_back(0);
    for (size_t g = 0; g < sched.size(); ++g) {
        MPSBlock<double> const& mb = sched[g];
        const uint32_t t0 = uint32_t(f.t_lb.size());
        for (auto const& t : mb.t_schedule) {
            const unsigned col = std::get<0>(t), ci = std::get<1>(t), ci_eff = std::get<2>(t), lb = std::get<3>(t);
            const bool tr = ci != ci_eff;
            f.t_lb.push_back(lb);
            f.t_col.push_back(col);
            f.t_ci.push_back(ci_eff);
            f.t_trans.push_back(tr ? 1 : 0);
            f.t_nb.push_back(uint32_t(right_rt.n_blocks(ci_eff)));
            f.t_brows.push_back(uint32_t(tr ? right_rt.right_size(ci_eff) : right_rt.left_size(ci_eff)));
            f.t_bcols.push_back(uint32_t(tr ? right_rt.left_size(ci_eff) : right_rt.right_size(ci_eff)));
        }
        for (auto it = mb.begin(); it != mb.end(); ++it) {
            Cohort<double> const& c = *it;
            f.c_lb.push_back(c.lb);
            f.c_rb.push_back(c.rb);
            f.c_ls.push_back(c.ls);
            f.c_rs.push_back(c.rs);
            f.c_ci.push_back(c.ci_eff);
            f.c_trans.push_back(c.ci != c.ci_eff ? 1 : 0);
            f.c_nsrows.push_back(c.nSrows);
            f.c_stripe.push_back(c.stripe);
            f.c_out_ci.push_back(0);
            for (auto const& u : c.suv) {
                f.u_offset.push_back(u.offset);
                f.u_ms.push_back(u.ms);
                size_t k = 0;
                for (size_t l = 0; l < u.b2s.size(); ++l) {
                    f.l_b1.push_back(u.b1[l]);
                    for (unsigned j = 0; j < u.b2s[l]; ++j, ++k) {
                        f.term_alpha.push_back(u.alpha[k]);
                        f.term_t.push_back(t0 + u.tidx[2 * k]);
                        f.term_col.push_back(u.tidx[2 * k + 1]);
                    }
                    f.l_term.push_back(uint32_t(f.term_alpha.size()));
                }
                f.u_line.push_back(uint32_t(f.l_b1.size()));
            }
            f.c_unit.push_back(uint32_t(f.u_offset.size()));
        }
        f.g_t.push_back(uint32_t(f.t_lb.size()));
        f.g_c.push_back(uint32_t(f.c_lb.size()));
    }
    dmrgb200_plan_desc& d = f.desc;
    d.kind = DMRGB200_PLAN_HPSI;
    d.n_groups = uint32_t(sched.size());
    d.g_t = ptr(f.g_t);
    d.g_c = ptr(f.g_c);
    d.n_in_blocks = uint32_t(f.in_rows.size());
    d.in_rows = ptr(f.in_rows);
    d.in_cols = ptr(f.in_cols);
    d.in_off = ptr(f.in_off);
    d.in_size = in_size;
    d.n_out_blocks = uint32_t(f.out_rows.size());
    d.out_rows = ptr(f.out_rows);
    d.out_cols = ptr(f.out_cols);
    d.out_off = ptr(f.out_off);
    d.out_size = out_size;
    d.n_t = uint32_t(f.t_lb.size());
    d.t_lb = ptr(f.t_lb);
    d.t_col = ptr(f.t_col);
    d.t_ci = ptr(f.t_ci);
    d.t_trans = ptr(f.t_trans);
    d.t_nb = ptr(f.t_nb);
    d.t_brows = ptr(f.t_brows);
    d.t_bcols = ptr(f.t_bcols);
    d.t_width = nullptr;
    d.n_cohorts = uint32_t(f.c_lb.size());
    d.c_lb = ptr(f.c_lb);
    d.c_rb = ptr(f.c_rb);
    d.c_ls = ptr(f.c_ls);
    d.c_rs = ptr(f.c_rs);
    d.c_ci = ptr(f.c_ci);
    d.c_trans = ptr(f.c_trans);
    d.c_nsrows = ptr(f.c_nsrows);
    d.c_stripe = ptr(f.c_stripe);
    d.c_out_ci = ptr(f.c_out_ci);
    d.c_unit = ptr(f.c_unit);
    d.n_units = uint32_t(f.u_offset.size());
    d.u_offset = ptr(f.u_offset);
    d.u_ms = ptr(f.u_ms);
    d.u_line = ptr(f.u_line);
    d.n_lines = uint32_t(f.l_b1.size());
    d.l_b1 = ptr(f.l_b1);
    d.l_term = ptr(f.l_term);
    d.n_terms = uint32_t(f.term_alpha.size());
    d.term_alpha = ptr(f.term_alpha);
    d.term_t = ptr(f.term_t);
    d.term_col = ptr(f.term_col);
}

extern "C" RefFlat* ref_flat_new() { return new RefFlat; }
extern "C" void ref_flat_delete(RefFlat* f) { delete f; }
extern "C" const dmrgb200_plan_desc* ref_flat_desc(RefFlat* f) { return &f->desc; }
