#include "schedule.hpp"

#include <map>
#include <stdexcept>
#include <tuple>

#include "coupling.hpp"

namespace dmrgb200 {

Cohort::Cohort(std::vector<unsigned> const& phys_sizes, unsigned lb_, unsigned rb_, unsigned ls_, unsigned rs_,
               unsigned ci_, unsigned ci_eff_, unsigned mpodim, bool left)
    : lb(lb_), rb(rb_), ls(ls_), rs(rs_), ci(ci_), ci_eff(ci_eff_), nSrows(mpodim), mpo_offsets_(mpodim, 0),
      sfold_(phys_sizes.size()) {
    unsigned sum = 0;
    for (size_t s = 0; s < phys_sizes.size(); ++s) {
        sfold_[s] = sum;
        sum += phys_sizes[s];
    }
    suv_.resize(sum);
    // the left-step S has the MPO index on the column side of each block
    sblock = left ? rs : ls;
}

void Cohort::finalize() {
    std::vector<long> remap = mpo_offsets_;
    unsigned n = 0;
    for (auto& v : remap)
        if (v) v = n++;
    nSrows = n;
    for (auto& u : suv_)
        for (auto& b : u.b1) b = static_cast<unsigned>(remap[b]);
    size_t bsz = size_t(ls) * rs;
    unsigned cnt = 0;
    for (auto& v : mpo_offsets_) v = v ? long(bsz * cnt++) : -1;
}

size_t Cohort::n_tasks() const {
    size_t n = 0;
    for (auto const& u : suv_) n += u.n_tasks();
    return n;
}

size_t Cohort::n_flops() const {
    // tasks.cpp:388-398
    size_t f = 2 * size_t(rs) * ls * nSrows * stripe_;
    for (auto const& u : suv_) f += 2 * size_t(ls) * u.ms * u.alpha.size();
    return f;
}

namespace {

std::vector<unsigned> phys_sizes_of(Index const& phys) { return phys.sz; }

// Expand one operator block into cohort pushes (op_iterate.hpp:37-69).  `from`
// is the MPO term the block belongs to; dcouplings (may be NULL) are the
// couplings with the term's scale set to one, so that e.coeff * dcouplings[c]
// is the derivative of the pushed alpha with respect to that scale.
void op_iterate(OpBlock const& blk, double const couplings[4], double const* dcouplings, unsigned from, Cohort& cg,
                unsigned s, unsigned m2_size, MPSBlock const& mpsb, unsigned mps_offset, unsigned ci,
                unsigned boundary_col) {
    for (auto const& e : blk.entries) {
        unsigned casenr = 0;
        if (e.row_spin == 2 && e.col_spin == 2)
            casenr = 3;
        else if (e.row_spin == 2)
            casenr = 1;
        else if (e.col_spin == 2)
            casenr = 2;
        double scale = e.coeff * couplings[casenr];
        double dsc = dcouplings ? e.coeff * dcouplings[casenr] : 0.0;
        unsigned ti = mpsb.get_ti(mps_offset + e.row * m2_size, ci);
        if (ti != 0xFFFFFFFFu) cg.push_back(s, e.col, scale, ti, boundary_col, from, dsc);
    }
}

// Couplings of the H psi / right-step builders.  The reference reads them from
// a per-(J, I, I') table indexed by a hash of (A, K, A') and multiplies by the
// scale afterwards (gsl_coupling.h:145-223); the same table slot is used here.
// `unit` (may be NULL) receives the couplings for scale one.
void w9j_couplings(Symm symm, Charge lc, Charge mc, Charge rc, int A, int K, int Ap, Charge jp, double scale,
                   double out[4], double* unit = nullptr) {
    if (!has_su2(symm)) {
        out[0] = out[1] = out[2] = out[3] = scale;
        if (unit) unit[0] = unit[1] = unit[2] = unit[3] = 1.0;
        return;
    }
    int J = spin_of(mc), I = spin_of(lc), Ip = spin_of(rc), Jp = spin_of(jp);
    int jpmin = (J - 2 < 0) ? 0 : J - 2, jpmax = J + 2;
    if (Jp < jpmin || Jp > jpmax) throw std::runtime_error("SU2 coupling requested outside the cached spin range");
    static const int Ktab[12] = {0, 1, 2, 0, 0, 1, 2, 1, 0, 1, 2, 0};
    static const int Aptab[12] = {0, 1, 2, 0, 1, 0, 1, 2, 2, 1, 0, 0};
    int slot = 4 * A + K + ((A == 1 && K == 1) ? Ap : 0);
    if (slot < 0 || slot >= 12) throw std::runtime_error("SU2 coupling: (A, K, A') outside the supported ranks");
    double base[4];
    set_coupling(J, std::abs(J - Jp), Jp, A, Ktab[slot], Aptab[slot], I, std::abs(I - Ip), Ip, 1.0, base);
    for (int c = 0; c < 4; ++c) out[c] = base[c] * scale;
    if (unit)
        for (int c = 0; c < 4; ++c) unit[c] = base[c];
}

void lshtm_couplings(Symm symm, Charge lc_ket, Charge rc_ket, int A, int K, int Ap, Charge lc_bra, Charge rc_bra,
                     double scale, double out[4]) {
    if (!has_su2(symm)) {
        out[0] = out[1] = out[2] = out[3] = scale;
        return;
    }
    set_coupling(spin_of(lc_ket), std::abs(spin_of(fuse(rc_ket, neg(lc_ket)))), spin_of(rc_ket), A, K, Ap,
                 spin_of(lc_bra), std::abs(spin_of(fuse(rc_bra, neg(lc_bra)))), spin_of(rc_bra), scale, out);
}

// stage-1 tasks of H psi and of the right step (right_tasks.hpp:39-78)
void rshtm_t_tasks(BoundaryIndex const& right, Index const& left_i, Index const& right_i, Index const& phys_i,
                   ProductBasis const& right_pb, unsigned lb_ket, MPSBlock& mpsb) {
    Charge lc_ket = left_i.charge(lb_ket);
    for (unsigned s = 0; s < phys_i.size(); ++s) {
        Charge phys_in = phys_i.charge(s);
        Charge rc_ket = fuse(lc_ket, phys_in);
        unsigned rb_ket = right_i.position(rc_ket);
        if (rb_ket == right_i.size()) continue;
        unsigned rs_ket = right_i.block_size(rb_ket);
        unsigned ket_offset = static_cast<unsigned>(right_pb(phys_in, rc_ket));
        for (unsigned rb_bra = 0; rb_bra < right_i.size(); ++rb_bra) {
            unsigned ci = right.cohort_index(rc_ket, right_i.charge(rb_bra));
            if (ci == right.n_cohorts()) continue;
            unsigned ci_eff = right.tr(ci) ? right.cohort_index(right_i.charge(rb_bra), rc_ket) : ci;
            for (unsigned ss = 0; ss < phys_i.block_size(s); ++ss)
                mpsb.push_t(TTask{ket_offset + ss * rs_ket, ci, ci_eff, lb_ket});
        }
    }
}

// H psi cohorts of one input block (site_hamil_tasks.hpp:41-137)
void shtm_tasks(Symm symm, MPOTensor const& mpo, BoundaryIndex const& left, BoundaryIndex const& right,
                Index const& left_i, Index const& right_i, Index const& phys_i, ProductBasis const& right_pb,
                unsigned lb_in, MPSBlock& mpsb) {
    auto phys_s = phys_sizes_of(phys_i);
    Charge lc_in = left_i.charge(lb_in);
    unsigned ls_in = left_i.block_size(lb_in);

    for (unsigned lb_out = 0; lb_out < left_i.size(); ++lb_out) {
        Charge lc_out = left_i.charge(lb_out);
        unsigned ls_out = left_i.block_size(lb_out);
        unsigned ci = left.cohort_index(lc_out, lc_in);
        if (ci == left.n_cohorts()) continue;
        unsigned ci_eff = left.tr(ci) ? left.cohort_index(lc_in, lc_out) : ci;

        Cohort cohort(phys_s, lb_in, lb_out, ls_in, ls_out, ci, ci_eff, static_cast<unsigned>(left.n_blocks(ci_eff)));

        for (unsigned s = 0; s < phys_i.size(); ++s) {
            Charge phys_out = phys_i.charge(s);
            Charge rc_out = fuse(lc_out, phys_out);
            unsigned rb_out = right_i.position(rc_out);
            if (rb_out == right_i.size()) continue;
            unsigned rs_out = right_i.block_size(rb_out);
            unsigned out_offset = static_cast<unsigned>(right_pb(phys_out, rc_out));
            cohort.add_unit(s, phys_i.block_size(s), rs_out, out_offset);

            for (unsigned b1 = 0; b1 < mpo.row_dim; ++b1) {
                if (!left.has_block(ci, b1)) continue;
                unsigned left_idx = static_cast<unsigned>(left.offset(ci, b1) / (long(ls_in) * ls_out));
                int A = mpo.lspin(b1);
                if (!triangle(symm, lc_in, A, lc_out)) continue;

                for (auto const& rowent : mpo.rows[b1]) {
                    unsigned b2 = rowent.other;
                    int Ap = mpo.rspin(b2);
                    for (auto const& tr : rowent.terms) {
                        SiteOp const& W = mpo.ops[tr.op];
                        int K = W.spin;
                        for (auto const& blk : W.blocks) {
                            if (phys_out != blk.right) continue;
                            Charge phys_in = blk.left;
                            Charge rc_in = fuse(lc_in, phys_in);
                            unsigned ci_right = right.cohort_index(rc_in, rc_out);
                            if (!right.has_block(ci_right, b2)) continue;
                            unsigned rb_in = right_i.position(rc_in);
                            if (rb_in == right_i.size()) continue;
                            unsigned rs_in = right_i.block_size(rb_in);
                            unsigned in_offset = static_cast<unsigned>(right_pb(phys_in, rc_in));
                            long right_offset = right.offset(ci_right, b2);

                            double couplings[4], unit[4], dcouplings[4];
                            double cscale = right.conjugate_scale(ci_right, b2) * left.conjugate_scale(ci, b1);
                            double scale = right.conjugate_scale(ci_right, b2) * tr.scale * left.conjugate_scale(ci, b1);
                            w9j_couplings(symm, lc_out, lc_in, rc_out, A, K, Ap, rc_in, scale, couplings, unit);
                            for (int c = 0; c < 4; ++c) dcouplings[c] = unit[c] * cscale;
                            op_iterate(blk, couplings, dcouplings, tr.id, cohort, s, rs_in, mpsb, in_offset, ci_right,
                                       static_cast<unsigned>(right_offset / rs_in));
                        }
                    }
                }
                cohort.add_line(left_idx);
            }
        }
        if (cohort.n_tasks()) mpsb.cohorts.push_back(std::move(cohort));
    }
}

// right-step cohorts of one ket block (right_tasks.hpp:80-167)
void rshtm_tasks(Symm symm, MPOTensor const& mpo, BoundaryIndex const& right, Index const& left_i,
                 Index const& right_i, Index const& phys_i, ProductBasis const& right_pb, unsigned lb_ket,
                 MPSBlock& mpsb, bool skip) {
    const int site_basis_max_diff = 2;
    auto phys_s = phys_sizes_of(phys_i);
    Charge lc_ket = left_i.charge(lb_ket);
    unsigned ls_ket = left_i.block_size(lb_ket);

    for (unsigned lb_bra = 0; lb_bra < left_i.size(); ++lb_bra) {
        Charge lc_bra = left_i.charge(lb_bra);
        if (std::abs(particle_number(symm, lc_ket) - particle_number(symm, lc_bra)) > site_basis_max_diff) continue;
        unsigned ls_bra = left_i.block_size(lb_bra);

        Cohort cohort(phys_s, lb_ket, lb_bra, ls_ket, ls_bra, 0, 0, mpo.row_dim);

        for (unsigned s = 0; s < phys_i.size(); ++s) {
            Charge phys_out = phys_i.charge(s);
            Charge rc_bra = fuse(lc_bra, phys_out);
            unsigned rb_bra = right_i.position(rc_bra);
            if (rb_bra == right_i.size()) continue;
            unsigned rs_bra = right_i.block_size(rb_bra);
            unsigned bra_offset = static_cast<unsigned>(right_pb(phys_out, rc_bra));
            cohort.add_unit(s, phys_i.block_size(s), rs_bra, bra_offset);

            for (unsigned b1 = 0; b1 < mpo.row_dim; ++b1) {
                if (skip && mpo.left_herm.skip(b1, lc_ket, lc_bra)) continue;
                int A = mpo.lspin(b1);
                if (!triangle(symm, lc_ket, A, lc_bra)) continue;

                for (auto const& rowent : mpo.rows[b1]) {
                    unsigned b2 = rowent.other;
                    int Ap = mpo.rspin(b2);
                    for (auto const& tr : rowent.terms) {
                        SiteOp const& W = mpo.ops[tr.op];
                        int K = W.spin;
                        for (auto const& blk : W.blocks) {
                            if (phys_out != blk.right) continue;
                            Charge phys_in = blk.left;
                            Charge rc_ket = fuse(lc_ket, phys_in);
                            unsigned ci = right.cohort_index(rc_ket, rc_bra);
                            if (!right.has_block(ci, b2)) continue;
                            unsigned rb_ket = right_i.position(rc_ket);
                            if (rb_ket == right_i.size()) continue;
                            unsigned rs_ket = right_i.block_size(rb_ket);
                            unsigned ket_offset = static_cast<unsigned>(right_pb(phys_in, rc_ket));
                            long right_offset = right.offset(ci, b2);

                            double couplings[4];
                            double scale = right.conjugate_scale(ci, b2) * tr.scale;
                            w9j_couplings(symm, lc_bra, lc_ket, rc_bra, A, K, Ap, rc_ket, scale, couplings);
                            op_iterate(blk, couplings, nullptr, tr.id, cohort, s, rs_ket, mpsb, ket_offset, ci,
                                       static_cast<unsigned>(right_offset / rs_ket));
                        }
                    }
                }
                cohort.add_line(b1);
            }
        }
        cohort.finalize();
        if (cohort.n_tasks()) mpsb.cohorts.push_back(std::move(cohort));
    }
}

// stage-1 tasks of the left step (left_tasks.hpp:38-76)
void lshtm_t_tasks(BoundaryIndex const& left, Index const& left_i, Index const& right_i, Index const& phys_i,
                   ProductBasis const& right_pb, unsigned rb_ket, MPSBlock& mpsb) {
    Charge rc_ket = right_i.charge(rb_ket);
    unsigned rs_ket = right_i.block_size(rb_ket);
    for (unsigned s = 0; s < phys_i.size(); ++s) {
        Charge phys_in = phys_i.charge(s);
        Charge lc_ket = fuse(rc_ket, neg(phys_in));
        unsigned lb_ket = left_i.position(lc_ket);
        if (lb_ket == left_i.size()) continue;
        unsigned ket_offset = static_cast<unsigned>(right_pb(phys_in, rc_ket));
        for (unsigned lb_bra = 0; lb_bra < left_i.size(); ++lb_bra) {
            unsigned ci = left.cohort_index(left_i.charge(lb_bra), lc_ket);
            if (ci == left.n_cohorts()) continue;
            unsigned ci_eff = left.tr(ci) ? left.cohort_index(lc_ket, left_i.charge(lb_bra)) : ci;
            for (unsigned ss = 0; ss < phys_i.block_size(s); ++ss)
                mpsb.push_t(TTask{ket_offset + ss * rs_ket, ci, ci_eff, lb_ket});
        }
    }
}

// left-step cohorts of one ket right block (left_tasks.hpp:78-172)
void lshtm_tasks(Symm symm, MPOTensor const& mpo, Index const& phys_i, Index const& bra_left_i,
                 Index const& bra_right_i, Index const& ket_left_i, Index const& ket_right_i,
                 BoundaryIndex const& left, ProductBasis const& bra_left_pb, ProductBasis const& ket_right_pb,
                 unsigned rb_ket, MPSBlock& mpsb, bool skip) {
    const int site_basis_max_diff = 2;
    auto phys_s = phys_sizes_of(phys_i);
    Charge rc_ket = ket_right_i.charge(rb_ket);
    unsigned rs_ket = ket_right_i.block_size(rb_ket);

    for (unsigned rb_bra = 0; rb_bra < bra_right_i.size(); ++rb_bra) {
        Charge rc_bra = bra_right_i.charge(rb_bra);
        if (std::abs(particle_number(symm, rc_bra) - particle_number(symm, rc_ket)) > site_basis_max_diff) continue;
        unsigned rs_bra = bra_right_i.block_size(rb_bra);

        Cohort cohort(phys_s, rb_bra, rb_ket, rs_bra, rs_ket, 0, 0, mpo.col_dim, true);

        for (unsigned s = 0; s < phys_i.size(); ++s) {
            Charge phys_out = phys_i.charge(s);
            Charge lc_bra = fuse(rc_bra, neg(phys_out));
            unsigned lb_bra = bra_left_i.position(lc_bra);
            if (lb_bra == bra_left_i.size()) continue;
            unsigned ls_bra = bra_left_i.block_size(lb_bra);
            unsigned bra_offset = static_cast<unsigned>(bra_left_pb(phys_out, lc_bra));
            cohort.add_unit(s, phys_i.block_size(s), ls_bra, bra_offset);

            for (unsigned b2 = 0; b2 < mpo.col_dim; ++b2) {
                if (skip && mpo.right_herm.skip(b2, rc_bra, rc_ket)) continue;
                int Ap = mpo.rspin(b2);
                if (!triangle(symm, rc_ket, Ap, rc_bra)) continue;

                for (auto const& colent : mpo.cols[b2]) {
                    unsigned b1 = colent.other;
                    int A = mpo.lspin(b1);
                    for (auto const& tr : colent.terms) {
                        SiteOp const& W = mpo.ops[tr.op];
                        int K = W.spin;
                        for (auto const& blk : W.blocks) {
                            if (phys_out != blk.right) continue;
                            Charge phys_in = blk.left;
                            Charge lc_ket = fuse(rc_ket, neg(phys_in));
                            unsigned lb_ket = ket_left_i.position(lc_ket);
                            if (lb_ket == ket_left_i.size()) continue;
                            unsigned ci = left.cohort_index(lc_bra, lc_ket);
                            if (!left.has_block(ci, b1)) continue;
                            unsigned ls_ket = ket_left_i.block_size(lb_ket);
                            unsigned ket_offset = static_cast<unsigned>(ket_right_pb(phys_in, rc_ket));
                            long left_offset = left.offset(ci, b1);

                            double couplings[4];
                            double scale = left.conjugate_scale(ci, b1) * tr.scale;
                            lshtm_couplings(symm, lc_ket, rc_ket, A, K, Ap, lc_bra, rc_bra, scale, couplings);
                            op_iterate(blk, couplings, nullptr, tr.id, cohort, s, rs_ket, mpsb, ket_offset, ci,
                                       static_cast<unsigned>(left_offset / ls_ket));
                        }
                    }
                }
                cohort.add_line(b2);
            }
        }
        cohort.finalize();
        if (cohort.n_tasks()) mpsb.cohorts.push_back(std::move(cohort));
    }
}

}  // namespace

Schedule create_contraction_schedule(Symm symm, Index const& phys_i, Index const& left_i, Index const& right_i,
                                     BoundaryIndex const& left, BoundaryIndex const& right, MPOTensor const& mpo) {
    ProductBasis out_right_pb = right_paired_basis(phys_i, right_i);
    Schedule sched;
    sched.blocks.resize(left_i.size());
    #pragma omp parallel for schedule(dynamic, 1)
    for (int mb = 0; mb < int(left_i.size()); ++mb) {
        rshtm_t_tasks(right, left_i, right_i, phys_i, out_right_pb, mb, sched.blocks[mb]);
        shtm_tasks(symm, mpo, left, right, left_i, right_i, phys_i, out_right_pb, mb, sched.blocks[mb]);
    }
    return sched;
}

Schedule left_step_schedule(Symm symm, Index const& phys_i, Index const& bra_left_i, Index const& bra_right_i,
                            Index const& ket_left_i, Index const& ket_right_i, BoundaryIndex const& left,
                            MPOTensor const& mpo, bool symmetric, BoundaryIndex& out_index) {
    ProductBasis bra_left_pb = left_paired_basis(phys_i, bra_left_i);
    ProductBasis ket_right_pb = right_paired_basis(phys_i, ket_right_i);
    Schedule sched;
    sched.blocks.resize(ket_right_i.size());
    #pragma omp parallel for schedule(dynamic, 1)
    for (int rb = 0; rb < int(ket_right_i.size()); ++rb) {
        lshtm_t_tasks(left, ket_left_i, ket_right_i, phys_i, ket_right_pb, rb, sched.blocks[rb]);
        lshtm_tasks(symm, mpo, phys_i, bra_left_i, bra_right_i, ket_left_i, ket_right_i, left, bra_left_pb,
                    ket_right_pb, rb, sched.blocks[rb], symmetric);
    }
    out_index = BoundaryIndex(symm, bra_right_i, ket_right_i);
    for (unsigned rb = 0; rb < ket_right_i.size(); ++rb)
        for (auto const& c : sched.blocks[rb].cohorts) out_index.add_cohort(c.lb, rb, c.mpo_offsets_);
    if (symmetric) out_index.complement_transpose(mpo.right_herm, true);
    return sched;
}

Schedule right_step_schedule(Symm symm, Index const& phys_i, Index const& bra_left_i, Index const& bra_right_i,
                             Index const& ket_left_i, BoundaryIndex const& right, MPOTensor const& mpo, bool symmetric,
                             BoundaryIndex& out_index) {
    ProductBasis bra_right_pb = right_paired_basis(phys_i, bra_right_i);
    Schedule sched;
    sched.blocks.resize(ket_left_i.size());
    #pragma omp parallel for schedule(dynamic, 1)
    for (int lb = 0; lb < int(ket_left_i.size()); ++lb) {
        rshtm_t_tasks(right, bra_left_i, bra_right_i, phys_i, bra_right_pb, lb, sched.blocks[lb]);
        rshtm_tasks(symm, mpo, right, bra_left_i, bra_right_i, phys_i, bra_right_pb, lb, sched.blocks[lb], symmetric);
    }
    out_index = BoundaryIndex(symm, ket_left_i, bra_left_i);
    for (unsigned lb = 0; lb < ket_left_i.size(); ++lb)
        for (auto const& c : sched.blocks[lb].cohorts) out_index.add_cohort(lb, c.rb, c.mpo_offsets_);
    out_index.complement_transpose(mpo.left_herm, false);
    return sched;
}

}  // namespace dmrgb200
