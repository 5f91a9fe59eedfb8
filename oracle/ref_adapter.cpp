// ORACLE — test infrastructure only.  Drives the reference's own solver core
// (dmrg/framework/dmrg/solver/tasks.cpp, compiled from the read-only reference
// tree by oracle/build_ref.sh into oracle/_ref/) with a flat plan: the plan is
// replayed into ScheduleNew / MPSBlock / Cohort through their public API
// (tasks.h:50-348: Cohort(...), add_unit, push_back, add_line, finalize,
// MPSBlock::t_schedule) and executed by the reference's CPU kernels
// create_T / contract (super_hamil_mv.hpp:121-132), create_T_left / prop_l
// (move_boundary.hpp:260-276) and create_T / prop_r (move_boundary.hpp:385-401).
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "dmrg/solver/tasks.h"
#include "../include/dmrgb200.h"

using contraction::common::Cohort;
using contraction::common::MPSBlock;
using contraction::common::ScheduleNew;

namespace {

// cohort sizes of a boundary plus one Hermitian-complement entry per stored
// cohort (index n + ci) with swapped sizes, so that T tasks can name a virtual ci
BoundaryIndexRT make_rt(uint32_t n, const uint32_t* lsz, const uint32_t* rsz, const uint32_t* nb) {
    BoundaryIndexRT rt;
    for (uint32_t i = 0; i < n; ++i) {
        rt.lszs().push_back(lsz[i]);
        rt.rszs().push_back(rsz[i]);
        rt.nbs().push_back(nb[i]);
    }
    for (uint32_t i = 0; i < n; ++i) {
        rt.lszs().push_back(rsz[i]);
        rt.rszs().push_back(lsz[i]);
        rt.nbs().push_back(0);
    }
    return rt;
}

void fill_group(dmrgb200_plan_desc const& d, uint32_t g, uint32_t nbnd, MPSBlock<double>& mb, bool left, bool finalize,
                bool hpsi) {
    for (uint32_t t = d.g_t[g]; t < d.g_t[g + 1]; ++t) {
        unsigned ci = d.t_trans[t] ? nbnd + d.t_ci[t] : d.t_ci[t];
        mb.t_schedule.push_back(std::make_tuple(d.t_col[t], ci, d.t_ci[t], d.t_lb[t], size_t(0)));
    }
    for (uint32_t c = d.g_c[g]; c < d.g_c[g + 1]; ++c) {
        uint32_t nu = d.c_unit[c + 1] - d.c_unit[c];
        std::vector<std::size_t> phys(nu, 1);
        unsigned ci = 0, ci_eff = 0;
        if (hpsi) {
            ci_eff = d.c_ci[c];
            ci = d.c_trans[c] ? ci_eff + 1 + 1000000 : ci_eff;
        }
        // H psi: (lb_in, lb_out, ls_in, ls_out); left step: (rb_bra, rb_ket = group); right step:
        // (lb_ket = group, lb_bra) -- site_hamil_tasks.hpp:78, left_tasks.hpp:113, right_tasks.hpp:110
        Cohort<double> coh =
            hpsi ? Cohort<double>(phys, d.c_lb[c], d.c_rb[c], d.c_ls[c], d.c_rs[c], ci, ci_eff, d.c_nsrows[c], false)
            : left ? Cohort<double>(phys, d.c_lb[c], g, d.c_ls[c], d.c_rs[c], 0, 0, d.c_nsrows[c], true)
                   : Cohort<double>(phys, g, d.c_rb[c], d.c_ls[c], d.c_rs[c], 0, 0, d.c_nsrows[c], false);
        for (uint32_t u = d.c_unit[c]; u < d.c_unit[c + 1]; ++u) {
            unsigned s = u - d.c_unit[c];
            coh.add_unit(s, 1, d.u_ms[u], d.u_offset[u]);
        }
        for (uint32_t u = d.c_unit[c]; u < d.c_unit[c + 1]; ++u) {
            unsigned s = u - d.c_unit[c];
            for (uint32_t l = d.u_line[u]; l < d.u_line[u + 1]; ++l) {
                for (uint32_t k = d.l_term[l]; k < d.l_term[l + 1]; ++k)
                    coh.push_back(s, 0, d.term_alpha[k], d.term_t[k] - d.g_t[g], d.term_col[k]);
                coh.add_line(d.l_b1[l]);
            }
        }
        if (finalize) coh.finalize();
        mb.push_back(std::move(coh));
    }
}

std::vector<const double*> block_views(const double* base, const uint64_t* off, uint32_t n) {
    std::vector<const double*> v(n);
    for (uint32_t i = 0; i < n; ++i) v[i] = base + off[i];
    return v;
}

}  // namespace

extern "C" {

int ref_hpsi(const dmrgb200_plan_desc* dp, uint32_t nR, const uint32_t* R_lsz, const uint32_t* R_rsz,
             const uint32_t* R_nb, const double* const* L, uint32_t nL, const double* const* R, const double* x,
             double* y) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_HPSI) return 1;
    BoundaryIndexRT rrt = make_rt(nR, R_lsz, R_rsz, R_nb), lrt;
    std::vector<std::size_t> lr(d.in_rows, d.in_rows + d.n_in_blocks), mpsbs(d.n_in_blocks, 0);
    ScheduleNew<double> tasks(mpsbs, lr, lrt, rrt);
    for (uint32_t g = 0; g < d.n_groups; ++g) fill_group(d, g, nR, tasks[g], false, false, true);
    std::vector<const double*> lv(L, L + nL), rv(R, R + nR);
    auto xv = block_views(x, d.in_off, d.n_in_blocks);
    for (uint32_t b = 0; b < d.n_out_blocks; ++b)
        std::memset(y + d.out_off[b], 0, sizeof(double) * size_t(d.out_rows[b]) * d.out_cols[b]);
    std::vector<std::mutex> mutexes(d.n_out_blocks);
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < ng; ++g) {
        auto T = tasks[g].create_T(rv, xv);
        for (auto it = tasks[g].begin(); it != tasks[g].end(); ++it)
            it->contract(lv, T, y + d.out_off[it->get_rb()], mutexes[it->get_rb()]);
    }
    return 0;
}

// A ScheduleNew built once from a flat H psi plan and kept with its boundary
// views, as the reference builds one schedule per site problem and reuses it
// for every Davidson iteration (site_hamil_schedule.hpp:40-93,
// solver_interface.hpp:30-77); ref_hpsi_run then times only create_T and
// contract (super_hamil_mv.hpp:121-132).
struct RefFlat;
void ref_flatten_hpsi(ScheduleNew<double> const& sched, BoundaryIndexRT const& right_rt,
                      std::vector<uint32_t> const& in_rows, std::vector<uint32_t> const& in_cols,
                      std::vector<uint64_t> const& in_off, uint64_t in_size, std::vector<uint32_t> const& out_rows,
                      std::vector<uint32_t> const& out_cols, std::vector<uint64_t> const& out_off, uint64_t out_size,
                      RefFlat& f);
RefFlat* ref_flat_new();
void ref_flat_delete(RefFlat* f);
const dmrgb200_plan_desc* ref_flat_desc(RefFlat* f);

struct RefHpsi {
    std::vector<uint32_t> in_rows, in_cols;
    std::vector<uint64_t> in_off, out_off;
    std::vector<uint32_t> out_rows, out_cols;
    uint64_t in_size = 0, out_size = 0;
    RefFlat* flat = nullptr;
    BoundaryIndexRT rrt, lrt;
    std::unique_ptr<ScheduleNew<double>> tasks;
    std::vector<const double*> lv, rv;
    std::vector<std::mutex> mutexes;
};

void* ref_hpsi_create(const dmrgb200_plan_desc* dp, uint32_t nR, const uint32_t* R_lsz, const uint32_t* R_rsz,
                      const uint32_t* R_nb, const double* const* L, uint32_t nL, const double* const* R) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_HPSI) return nullptr;
    auto* h = new RefHpsi;
    h->in_off.assign(d.in_off, d.in_off + d.n_in_blocks);
    h->in_rows.assign(d.in_rows, d.in_rows + d.n_in_blocks);
    h->in_cols.assign(d.in_cols, d.in_cols + d.n_in_blocks);
    h->in_size = d.in_size;
    h->out_size = d.out_size;
    h->out_off.assign(d.out_off, d.out_off + d.n_out_blocks);
    h->out_rows.assign(d.out_rows, d.out_rows + d.n_out_blocks);
    h->out_cols.assign(d.out_cols, d.out_cols + d.n_out_blocks);
    h->rrt = make_rt(nR, R_lsz, R_rsz, R_nb);
    std::vector<std::size_t> lr(d.in_rows, d.in_rows + d.n_in_blocks), mpsbs(d.n_in_blocks, 0);
    h->tasks.reset(new ScheduleNew<double>(mpsbs, lr, h->lrt, h->rrt));
    for (uint32_t g = 0; g < d.n_groups; ++g) fill_group(d, g, nR, (*h->tasks)[g], false, false, true);
    h->lv.assign(L, L + nL);
    h->rv.assign(R, R + nR);
    h->mutexes = std::vector<std::mutex>(d.n_out_blocks);
    return h;
}

int ref_hpsi_run(void* handle, const double* x, double* y) {
    auto* h = static_cast<RefHpsi*>(handle);
    if (!h) return 1;
    auto xv = block_views(x, h->in_off.data(), uint32_t(h->in_off.size()));
    for (size_t b = 0; b < h->out_off.size(); ++b)
        std::memset(y + h->out_off[b], 0, sizeof(double) * size_t(h->out_rows[b]) * h->out_cols[b]);
    ScheduleNew<double>& tasks = *h->tasks;
    int ng = int(tasks.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < ng; ++g) {
        auto T = tasks[g].create_T(h->rv, xv);
        for (auto it = tasks[g].begin(); it != tasks[g].end(); ++it)
            it->contract(h->lv, T, y + h->out_off[it->get_rb()], h->mutexes[it->get_rb()]);
    }
    return 0;
}

void ref_hpsi_destroy(void* handle) {
    auto* h = static_cast<RefHpsi*>(handle);
    if (h) ref_flat_delete(h->flat);
    delete h;
}

// The handle's ScheduleNew flattened back into a plan description (ref_flatten.cpp);
// the arrays live until the handle is destroyed.
const dmrgb200_plan_desc* ref_hpsi_flatten(void* handle) {
    auto* h = static_cast<RefHpsi*>(handle);
    if (!h) return nullptr;
    if (!h->flat) h->flat = ref_flat_new();
    ref_flatten_hpsi(*h->tasks, h->rrt, h->in_rows, h->in_cols, h->in_off, h->in_size, h->out_rows, h->out_cols,
                     h->out_off, h->out_size, *h->flat);
    return ref_flat_desc(h->flat);
}

int ref_left_step(const dmrgb200_plan_desc* dp, uint32_t nL, const uint32_t* L_lsz, const uint32_t* L_rsz,
                  const uint32_t* L_nb, const double* const* L, const double* ket, const double* bra,
                  double* const* out) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_LEFT_STEP) return 1;
    BoundaryIndexRT lrt = make_rt(nL, L_lsz, L_rsz, L_nb);
    std::vector<std::size_t> widths(d.n_groups, 0), mpsbs(d.n_in_blocks, 0);
    for (uint32_t g = 0; g < d.n_groups; ++g) {
        if (d.g_t[g] < d.g_t[g + 1]) widths[g] = d.t_width[d.g_t[g]];
        else if (d.g_c[g] < d.g_c[g + 1]) widths[g] = d.c_rs[d.g_c[g]];
    }
    ScheduleNew<double> tasks(mpsbs, widths, lrt, lrt);
    for (uint32_t g = 0; g < d.n_groups; ++g) fill_group(d, g, nL, tasks[g], true, true, false);
    std::vector<const double*> lv(L, L + nL);
    auto kv = block_views(ket, d.in_off, d.n_in_blocks);
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < ng; ++g) {
        auto T = tasks[g].create_T_left(lv, kv);
        uint32_t c = d.g_c[g];
        for (auto it = tasks[g].begin(); it != tasks[g].end(); ++it, ++c)
            it->prop_l(bra + d.out_off[it->get_lb()], T, out[d.c_out_ci[c]]);
    }
    return 0;
}

int ref_right_step(const dmrgb200_plan_desc* dp, uint32_t nR, const uint32_t* R_lsz, const uint32_t* R_rsz,
                   const uint32_t* R_nb, const double* const* R, const double* ket, const double* bra,
                   double* const* out) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_RIGHT_STEP) return 1;
    BoundaryIndexRT rrt = make_rt(nR, R_lsz, R_rsz, R_nb);
    std::vector<std::size_t> lr(d.in_rows, d.in_rows + d.n_in_blocks), mpsbs(d.n_in_blocks, 0);
    ScheduleNew<double> tasks(mpsbs, lr, rrt, rrt);
    for (uint32_t g = 0; g < d.n_groups; ++g) fill_group(d, g, nR, tasks[g], false, true, false);
    std::vector<const double*> rv(R, R + nR);
    auto kv = block_views(ket, d.in_off, d.n_in_blocks);
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < ng; ++g) {
        auto T = tasks[g].create_T(rv, kv);
        uint32_t c = d.g_c[g];
        for (auto it = tasks[g].begin(); it != tasks[g].end(); ++it, ++c)
            it->prop_r(bra + d.out_off[it->get_rb()], T, out[d.c_out_ci[c]]);
    }
    return 0;
}

// The reference's perturbation terms on a step plan (bra = ket = the tensor viewed
// as one site): Cohort::lbtm / rbtm (tasks.cpp:346-380) of every cohort added into
// dm[lb] (left) or dm[rb] (right), as alpha_dm_direct / alpha_dm_direct_right do
// (move_boundary.hpp:38-143).  dm is not cleared.
int ref_alpha_dm(const dmrgb200_plan_desc* dp, uint32_t nB, const uint32_t* B_lsz, const uint32_t* B_rsz,
                 const uint32_t* B_nb, const double* const* B, const double* ket, double alpha, double* const* dm) {
    dmrgb200_plan_desc const& d = *dp;
    const bool left = d.kind == DMRGB200_PLAN_LEFT_STEP;
    if (!left && d.kind != DMRGB200_PLAN_RIGHT_STEP) return 1;
    BoundaryIndexRT rt = make_rt(nB, B_lsz, B_rsz, B_nb);
    std::vector<std::size_t> mpsbs(d.n_in_blocks, 0), sizes;
    if (left) {
        sizes.assign(d.n_groups, 0);
        for (uint32_t g = 0; g < d.n_groups; ++g) {
            if (d.g_t[g] < d.g_t[g + 1]) sizes[g] = d.t_width[d.g_t[g]];
            else if (d.g_c[g] < d.g_c[g + 1]) sizes[g] = d.c_rs[d.g_c[g]];
        }
    } else {
        sizes.assign(d.in_rows, d.in_rows + d.n_in_blocks);
    }
    ScheduleNew<double> tasks(mpsbs, sizes, rt, rt);
    for (uint32_t g = 0; g < d.n_groups; ++g) fill_group(d, g, nB, tasks[g], left, true, false);
    std::vector<const double*> bv(B, B + nB);
    auto kv = block_views(ket, d.in_off, d.n_in_blocks);
    std::vector<std::mutex> mutexes(d.n_out_blocks);
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < ng; ++g) {
        auto T = left ? tasks[g].create_T_left(bv, kv) : tasks[g].create_T(bv, kv);
        for (auto it = tasks[g].begin(); it != tasks[g].end(); ++it) {
            const unsigned b = left ? it->get_lb() : it->get_rb();
            std::lock_guard<std::mutex> lk(mutexes[b]);
            if (left)
                it->lbtm(T, dm[b], alpha);
            else
                it->rbtm(T, dm[b], alpha);
        }
    }
    return 0;
}

}  // extern "C"
