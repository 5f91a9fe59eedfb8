#include "plan.hpp"

#include <sstream>
#include <stdexcept>

namespace dmrgb200 {

uint64_t FlatPlan::flops() const {
    uint64_t f = 0;
    // stage 1: 2 * M * (cohort size) per T task (MPSBlock::n_flops, tasks.cpp:777-796)
    for (uint32_t t = 0; t < n_t(); ++t) {
        uint64_t csz = uint64_t(t_nb[t]) * t_brows[t] * t_bcols[t];
        uint64_t m = (kind == KIND_LEFT) ? t_width[t] : in_rows[t_lb[t]];
        f += 2 * m * csz;
    }
    // stages 2 and 3 (Cohort::n_flops, tasks.cpp:388-398)
    for (uint32_t c = 0; c < n_cohorts(); ++c) {
        f += 2ull * c_rs[c] * c_ls[c] * c_nsrows[c] * c_stripe[c];
        for (uint32_t u = c_unit[c]; u < c_unit[c + 1]; ++u) {
            uint64_t nterms = l_term[u_line[u + 1]] - l_term[u_line[u]];
            f += 2ull * c_ls[c] * u_ms[u] * nterms;
        }
    }
    return f;
}

void FlatPlan::stage_flops(uint64_t out[3]) const {
    out[0] = out[1] = out[2] = 0;
    for (uint32_t t = 0; t < n_t(); ++t) {
        uint64_t csz = uint64_t(t_nb[t]) * t_brows[t] * t_bcols[t];
        uint64_t m = (kind == KIND_LEFT) ? t_width[t] : in_rows[t_lb[t]];
        out[0] += 2 * m * csz;
    }
    for (uint32_t c = 0; c < n_cohorts(); ++c) {
        out[2] += 2ull * c_rs[c] * c_ls[c] * c_nsrows[c] * c_stripe[c];
        for (uint32_t u = c_unit[c]; u < c_unit[c + 1]; ++u)
            out[1] += 2ull * c_ls[c] * u_ms[u] * (l_term[u_line[u + 1]] - l_term[u_line[u]]);
    }
}

std::string FlatPlan::validate() const {
    std::ostringstream e;
    auto bad = [&](const char* what, uint64_t i) {
        e << what << " (entry " << i << ")";
        return e.str();
    };
    if (kind < KIND_HPSI || kind > KIND_RIGHT) return "unknown plan kind";
    if (in_rows.size() != in_cols.size() || in_rows.size() != in_off.size()) return "in-block arrays differ in length";
    if (out_rows.size() != out_cols.size() || out_rows.size() != out_off.size())
        return "out-block arrays differ in length";
    for (size_t b = 0; b < in_rows.size(); ++b)
        if (in_off[b] + uint64_t(in_rows[b]) * in_cols[b] > in_size) return bad("in block exceeds in_size", b);
    for (size_t b = 0; b < out_rows.size(); ++b)
        if (out_off[b] + uint64_t(out_rows[b]) * out_cols[b] > out_size) return bad("out block exceeds out_size", b);
    size_t nt = t_lb.size();
    if (t_col.size() != nt || t_ci.size() != nt || t_nb.size() != nt || t_brows.size() != nt ||
        t_bcols.size() != nt || t_trans.size() != nt || (kind == KIND_LEFT && t_width.size() != nt))
        return "T-task arrays differ in length";
    for (size_t t = 0; t < nt; ++t) {
        if (t_lb[t] >= in_rows.size()) return bad("T task block out of range", t);
        uint64_t width = (kind == KIND_LEFT) ? t_width[t] : t_brows[t];
        if (uint64_t(t_col[t]) + width > in_cols[t_lb[t]]) return bad("T task column slice exceeds block", t);
        if (kind == KIND_LEFT && t_bcols[t] != in_rows[t_lb[t]]) return bad("left T task inner size mismatch", t);
    }
    size_t nc = c_lb.size();
    if (c_rb.size() != nc || c_ls.size() != nc || c_rs.size() != nc || c_nsrows.size() != nc ||
        c_stripe.size() != nc || c_unit.size() != nc + 1 || c_trans.size() != nc || c_ci.size() != nc ||
        c_out_ci.size() != nc)
        return "cohort arrays differ in length";
    if (u_line.size() != u_offset.size() + 1 || u_ms.size() != u_offset.size()) return "unit arrays differ in length";
    if (l_term.size() != l_b1.size() + 1) return "line arrays differ in length";
    if (term_t.size() != term_alpha.size() || term_col.size() != term_alpha.size()) return "term arrays differ";
    if ((!term_src.empty() && term_src.size() != term_alpha.size()) || term_src.size() != term_dscale.size())
        return "term provenance arrays differ";
    if (!c_unit.empty() && c_unit.back() != u_offset.size()) return "cohort unit ranges do not cover the units";
    if (!u_line.empty() && u_line.back() != l_b1.size()) return "unit line ranges do not cover the lines";
    if (!l_term.empty() && l_term.back() != term_alpha.size()) return "line term ranges do not cover the terms";
    if (g_t.size() != g_c.size() || g_t.empty()) return "task-group arrays missing or differ in length";
    if (g_t.front() != 0 || g_c.front() != 0 || g_t.back() != nt || g_c.back() != nc)
        return "task groups do not cover the T tasks and cohorts";
    for (size_t g = 0; g + 1 < g_t.size(); ++g) {
        if (g_t[g] > g_t[g + 1] || g_c[g] > g_c[g + 1]) return bad("task-group range decreasing", g);
        for (uint32_t c = g_c[g]; c < g_c[g + 1]; ++c)
            for (uint32_t u = c_unit[c]; u < c_unit[c + 1] && u + 1 < u_line.size(); ++u)
                for (uint32_t l = u_line[u]; l < u_line[u + 1] && l + 1 < l_term.size(); ++l)
                    for (uint32_t k = l_term[l]; k < l_term[l + 1] && k < term_t.size(); ++k)
                        if (term_t[k] < g_t[g] || term_t[k] >= g_t[g + 1])
                            return bad("term references a T task of another group", k);
    }
    for (size_t c = 0; c < nc; ++c) {
        if (c_unit[c] > c_unit[c + 1]) return bad("cohort unit range decreasing", c);
        for (uint32_t u = c_unit[c]; u < c_unit[c + 1]; ++u) {
            if (u_line[u] > u_line[u + 1]) return bad("unit line range decreasing", u);
            if (uint64_t(u_offset[u]) + u_ms[u] > c_stripe[c]) return bad("unit exceeds stripe", u);
            for (uint32_t l = u_line[u]; l < u_line[u + 1]; ++l) {
                if (l_b1[l] >= c_nsrows[c]) return bad("line row block out of range", l);
                if (l_term[l] > l_term[l + 1]) return bad("line term range decreasing", l);
                for (uint32_t k = l_term[l]; k < l_term[l + 1]; ++k) {
                    uint32_t t = term_t[k];
                    if (t >= nt) return bad("term T index out of range", k);
                    if (kind == KIND_LEFT) {
                        // source block (ms x rs) at column col*rs of T_t
                        if (t_brows[t] != u_ms[u] || t_width[t] != c_rs[c]) return bad("left term shape mismatch", k);
                        if (uint64_t(term_col[k]) * c_rs[c] + uint64_t(u_ms[u]) * c_rs[c] > t_size(t))
                            return bad("left term reads past T", k);
                    } else {
                        if (t_rows(t) != c_ls[c]) return bad("term row count mismatch", k);
                        if (uint64_t(term_col[k]) + u_ms[u] > uint64_t(t_nb[t]) * t_bcols[t])
                            return bad("term reads past T columns", k);
                    }
                }
            }
        }
        if (kind == KIND_HPSI) {
            if (c_lb[c] >= in_rows.size() || c_rb[c] >= out_rows.size()) return bad("cohort block out of range", c);
            if (c_ls[c] != in_rows[c_lb[c]] || c_rs[c] != out_rows[c_rb[c]]) return bad("cohort sizes mismatch", c);
            if (c_stripe[c] != out_cols[c_rb[c]]) return bad("cohort stripe differs from output width", c);
        } else if (kind == KIND_RIGHT) {
            if (c_rb[c] >= out_rows.size()) return bad("right-step bra block out of range", c);
            if (c_rs[c] != out_rows[c_rb[c]] || c_stripe[c] != out_cols[c_rb[c]]) return bad("bra block shape", c);
        } else {
            if (c_lb[c] >= out_rows.size()) return bad("left-step bra block out of range", c);
            if (c_ls[c] != out_cols[c_lb[c]] || c_stripe[c] != out_rows[c_lb[c]]) return bad("bra block shape", c);
        }
    }
    return std::string();
}

FlatPlan merge_plans(std::vector<FlatPlan> const& plans, std::vector<uint32_t> const& left_ci_base,
                     std::vector<uint32_t> const& right_ci_base, std::vector<uint64_t>& in_base,
                     std::vector<uint64_t>& out_base) {
    FlatPlan m;
    m.kind = KIND_HPSI;
    m.g_t.push_back(0);
    m.g_c.push_back(0);
    m.c_unit.push_back(0);
    m.u_line.push_back(0);
    m.l_term.push_back(0);
    in_base.clear();
    out_base.clear();
    for (size_t i = 0; i < plans.size(); ++i) {
        FlatPlan const& p = plans[i];
        if (p.kind != KIND_HPSI) throw std::runtime_error("only H psi plans can be batched");
        const uint64_t ib = round_up(m.in_size, 128), ob = round_up(m.out_size, 128);
        in_base.push_back(ib);
        out_base.push_back(ob);
        const uint32_t nb_in = uint32_t(m.in_rows.size()), nb_out = uint32_t(m.out_rows.size());
        const uint32_t t0 = m.n_t(), c0 = m.n_cohorts(), u0 = m.n_units(), l0 = m.n_lines(), k0 = m.n_terms();
        for (size_t b = 0; b < p.in_rows.size(); ++b) {
            m.in_rows.push_back(p.in_rows[b]);
            m.in_cols.push_back(p.in_cols[b]);
            m.in_off.push_back(ib + p.in_off[b]);
        }
        for (size_t b = 0; b < p.out_rows.size(); ++b) {
            m.out_rows.push_back(p.out_rows[b]);
            m.out_cols.push_back(p.out_cols[b]);
            m.out_off.push_back(ob + p.out_off[b]);
        }
        m.in_size = ib + p.in_size;
        m.out_size = ob + p.out_size;
        for (uint32_t t = 0; t < p.n_t(); ++t) {
            m.t_lb.push_back(nb_in + p.t_lb[t]);
            m.t_col.push_back(p.t_col[t]);
            m.t_ci.push_back(right_ci_base[i] + p.t_ci[t]);
            m.t_trans.push_back(p.t_trans[t]);
            m.t_nb.push_back(p.t_nb[t]);
            m.t_brows.push_back(p.t_brows[t]);
            m.t_bcols.push_back(p.t_bcols[t]);
        }
        for (uint32_t c = 0; c < p.n_cohorts(); ++c) {
            m.c_lb.push_back(nb_in + p.c_lb[c]);
            m.c_rb.push_back(nb_out + p.c_rb[c]);
            m.c_ls.push_back(p.c_ls[c]);
            m.c_rs.push_back(p.c_rs[c]);
            m.c_ci.push_back(left_ci_base[i] + p.c_ci[c]);
            m.c_trans.push_back(p.c_trans[c]);
            m.c_nsrows.push_back(p.c_nsrows[c]);
            m.c_stripe.push_back(p.c_stripe[c]);
            m.c_out_ci.push_back(0);
            m.c_unit.push_back(u0 + p.c_unit[c + 1]);
        }
        for (uint32_t u = 0; u < p.n_units(); ++u) {
            m.u_offset.push_back(p.u_offset[u]);
            m.u_ms.push_back(p.u_ms[u]);
            m.u_line.push_back(l0 + p.u_line[u + 1]);
        }
        for (uint32_t l = 0; l < p.n_lines(); ++l) {
            m.l_b1.push_back(p.l_b1[l]);
            m.l_term.push_back(k0 + p.l_term[l + 1]);
        }
        for (uint32_t k = 0; k < p.n_terms(); ++k) {
            m.term_alpha.push_back(p.term_alpha[k]);
            m.term_t.push_back(t0 + p.term_t[k]);
            m.term_col.push_back(p.term_col[k]);
        }
        for (uint32_t g = 0; g < p.n_groups(); ++g) {
            m.g_t.push_back(t0 + p.g_t[g + 1]);
            m.g_c.push_back(c0 + p.g_c[g + 1]);
        }
    }
    return m;
}

TensorLayout right_paired_layout(Index const& phys, Index const& left, Index const& right) {
    TensorLayout t;
    for (unsigned lb = 0; lb < left.size(); ++lb) {
        uint64_t cols = 0;
        for (unsigned s = 0; s < phys.size(); ++s) {
            unsigned rb = right.position(fuse(left.charge(lb), phys.charge(s)));
            if (rb == right.size()) continue;
            cols += uint64_t(phys.block_size(s)) * right.block_size(rb);
        }
        t.rows.push_back(left.block_size(lb));
        t.cols.push_back(uint32_t(cols));
        t.off.push_back(t.total);
        t.total += round_up(uint64_t(left.block_size(lb)) * cols, 128);
    }
    return t;
}

TensorLayout left_paired_layout(Index const& phys, Index const& left, Index const& right) {
    TensorLayout t;
    for (unsigned rb = 0; rb < right.size(); ++rb) {
        uint64_t rows = 0;
        for (unsigned s = 0; s < phys.size(); ++s) {
            unsigned lb = left.position(fuse(right.charge(rb), neg(phys.charge(s))));
            if (lb == left.size()) continue;
            rows += uint64_t(phys.block_size(s)) * left.block_size(lb);
        }
        t.rows.push_back(uint32_t(rows));
        t.cols.push_back(right.block_size(rb));
        t.off.push_back(t.total);
        t.total += round_up(rows * right.block_size(rb), 128);
    }
    return t;
}

namespace {

void set_blocks(FlatPlan& p, TensorLayout const& in, TensorLayout const& out) {
    p.in_rows = in.rows;
    p.in_cols = in.cols;
    p.in_off = in.off;
    p.in_size = in.total;
    p.out_rows = out.rows;
    p.out_cols = out.cols;
    p.out_off = out.off;
    p.out_size = out.total;
}

// Append the T tasks and cohorts of every task group in order.
template <class TaskDims, class CohortExtra>
void append_groups(FlatPlan& p, Schedule const& s, TaskDims tdims, CohortExtra cextra) {
    p.c_unit.push_back(0);
    p.u_line.push_back(0);
    p.l_term.push_back(0);
    p.g_t.push_back(0);
    p.g_c.push_back(0);
    for (size_t g = 0; g < s.blocks.size(); ++g) {
        MPSBlock const& mb = s.blocks[g];
        uint32_t tbase = p.n_t();
        for (auto const& t : mb.t_schedule) tdims(p, g, t);
        for (auto const& c : mb.cohorts) {
            p.c_lb.push_back(c.lb);
            p.c_rb.push_back(c.rb);
            p.c_ls.push_back(c.ls);
            p.c_rs.push_back(c.rs);
            p.c_nsrows.push_back(c.nSrows);
            p.c_stripe.push_back(c.stripe_);
            cextra(p, g, c);
            for (auto const& u : c.suv_) {
                p.u_offset.push_back(u.offset);
                p.u_ms.push_back(u.ms);
                size_t seek = 0;
                for (size_t l = 0; l < u.b2s.size(); ++l) {
                    p.l_b1.push_back(u.b1[l]);
                    for (size_t ia = seek; ia < seek + u.b2s[l]; ++ia) {
                        p.term_alpha.push_back(u.alpha[ia]);
                        p.term_t.push_back(tbase + u.tidx[2 * ia]);
                        p.term_col.push_back(u.tidx[2 * ia + 1]);
                        p.term_src.push_back(u.src[ia]);
                        p.term_dscale.push_back(u.dscale[ia]);
                    }
                    seek += u.b2s[l];
                    p.l_term.push_back(uint32_t(p.term_alpha.size()));
                }
                p.u_line.push_back(uint32_t(p.l_b1.size()));
            }
            p.c_unit.push_back(uint32_t(p.u_offset.size()));
        }
        p.g_t.push_back(p.n_t());
        p.g_c.push_back(p.n_cohorts());
    }
}

}  // namespace

FlatPlan flatten_hpsi(Schedule const& s, TensorLayout const& psi, BoundaryIndex const& L, BoundaryIndex const& R) {
    FlatPlan p;
    p.kind = KIND_HPSI;
    set_blocks(p, psi, psi);
    append_groups(
        p, s,
        [&](FlatPlan& q, size_t, TTask const& t) {
            q.t_lb.push_back(t.lb_ket);
            q.t_col.push_back(t.mps_offset);
            q.t_ci.push_back(t.ci_eff);
            q.t_trans.push_back(t.ci != t.ci_eff);
            q.t_nb.push_back(uint32_t(R.n_blocks(t.ci_eff)));
            q.t_brows.push_back(uint32_t(R.left_size(t.ci)));
            q.t_bcols.push_back(uint32_t(R.right_size(t.ci)));
        },
        [&](FlatPlan& q, size_t, Cohort const& c) {
            q.c_ci.push_back(c.ci_eff);
            q.c_trans.push_back(c.ci != c.ci_eff);
            q.c_out_ci.push_back(0);
        });
    (void)L;
    return p;
}

FlatPlan flatten_left_step(Schedule const& s, TensorLayout const& ket_rp, TensorLayout const& bra_lp,
                           Index const& ket_right_i, BoundaryIndex const& L, BoundaryIndex const& out_index) {
    FlatPlan p;
    p.kind = KIND_LEFT;
    set_blocks(p, ket_rp, bra_lp);
    append_groups(
        p, s,
        [&](FlatPlan& q, size_t g, TTask const& t) {
            q.t_lb.push_back(t.lb_ket);
            q.t_col.push_back(t.mps_offset);
            q.t_ci.push_back(t.ci_eff);
            q.t_trans.push_back(t.ci != t.ci_eff);
            q.t_nb.push_back(uint32_t(L.n_blocks(t.ci_eff)));
            q.t_brows.push_back(uint32_t(L.left_size(t.ci)));
            q.t_bcols.push_back(uint32_t(L.right_size(t.ci)));
            q.t_width.push_back(ket_right_i.block_size(unsigned(g)));
        },
        [&](FlatPlan& q, size_t g, Cohort const& c) {
            q.c_ci.push_back(0);
            q.c_trans.push_back(0);
            q.c_out_ci.push_back(out_index.cohort_index(c.lb, unsigned(g)));
        });
    return p;
}

FlatPlan flatten_right_step(Schedule const& s, TensorLayout const& ket_rp, TensorLayout const& bra_rp,
                            BoundaryIndex const& R, BoundaryIndex const& out_index) {
    FlatPlan p;
    p.kind = KIND_RIGHT;
    set_blocks(p, ket_rp, bra_rp);
    append_groups(
        p, s,
        [&](FlatPlan& q, size_t, TTask const& t) {
            q.t_lb.push_back(t.lb_ket);
            q.t_col.push_back(t.mps_offset);
            q.t_ci.push_back(t.ci_eff);
            q.t_trans.push_back(t.ci != t.ci_eff);
            q.t_nb.push_back(uint32_t(R.n_blocks(t.ci_eff)));
            q.t_brows.push_back(uint32_t(R.left_size(t.ci)));
            q.t_bcols.push_back(uint32_t(R.right_size(t.ci)));
        },
        [&](FlatPlan& q, size_t g, Cohort const& c) {
            q.c_ci.push_back(0);
            q.c_trans.push_back(0);
            q.c_out_ci.push_back(out_index.cohort_index(unsigned(g), c.rb));
        });
    return p;
}

}  // namespace dmrgb200
