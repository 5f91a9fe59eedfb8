// Cohort-packed boundary index.
//
// A boundary is a set of cohorts, one per (bra charge, ket charge) pair.  A
// cohort stores n_blocks consecutive column-major blocks of
// left_size x right_size, one per MPO bond index b that is present
// (offset(ci, b) in elements, -1 if absent).  Hermitian-complement cohorts
// (tr(ci) = 1) own no storage: their blocks are transposes of the partner
// cohort's blocks at the conjugate bond index, scaled by conjugate_scale.
// Semantics follow dmrg/framework/dmrg/mp_tensors/boundary.h:76-234 and
// boundary_index_rt.hpp:37-86.
#pragma once

#include <limits>
#include <vector>

#include "coupling.hpp"
#include "mpo.hpp"
#include "symm.hpp"

namespace dmrgb200 {

class BoundaryIndex {
public:
    static constexpr unsigned NONE = std::numeric_limits<unsigned>::max();

    BoundaryIndex() = default;
    BoundaryIndex(Symm s, Index bra, Index ket)
        : symm_(s), bra_(std::move(bra)), ket_(std::move(ket)), lbrb_ci_(size_t(bra_.size()) * ket_.size(), NONE) {}

    Symm symm() const { return symm_; }
    Index const& bra() const { return bra_; }
    Index const& ket() const { return ket_; }

    unsigned n_cohorts() const { return static_cast<unsigned>(offsets_.size()); }
    long offset(unsigned ci, unsigned b) const { return offsets_[ci][b]; }
    bool has_block(unsigned ci, unsigned b) const { return ci < n_cohorts() && offsets_[ci][b] > -1; }
    double conjugate_scale(unsigned ci, unsigned b) const { return conj_scales_[ci][b]; }
    bool trans(unsigned ci, unsigned b) const { return transposes_[ci][b]; }
    bool tr(unsigned ci) const { return tr_[ci]; }
    size_t aux_dim() const { return n_cohorts() ? offsets_[0].size() : 0; }

    size_t left_size(unsigned ci) const { return lsz_[ci]; }
    size_t right_size(unsigned ci) const { return rsz_[ci]; }
    size_t n_blocks(unsigned ci) const { return nbs_[ci]; }
    size_t block_size(unsigned ci) const { return lsz_[ci] * rsz_[ci]; }
    size_t cohort_size(unsigned ci) const { return nbs_[ci] * block_size(ci); }

    unsigned cohort_index(unsigned lb, unsigned rb) const {
        if (lb < bra_.size() && rb < ket_.size() && lbrb_ci_[size_t(lb) * ket_.size() + rb] != NONE)
            return lbrb_ci_[size_t(lb) * ket_.size() + rb];
        return n_cohorts();
    }
    unsigned cohort_index(Charge lc, Charge rc) const { return cohort_index(bra_.position(lc), ket_.position(rc)); }

    unsigned add_cohort(unsigned lb, unsigned rb, std::vector<long> const& off) {
        unsigned ci = n_cohorts();
        lbrb_ci_[size_t(lb) * ket_.size() + rb] = ci;
        offsets_.push_back(off);
        conj_scales_.push_back(std::vector<double>(off.size(), 1.0));
        transposes_.push_back(std::vector<char>(off.size(), 0));
        tr_.push_back(0);
        lsz_.push_back(bra_.block_size(lb));
        rsz_.push_back(ket_.block_size(rb));
        unsigned nb = 0;
        for (long o : off) nb += (o > -1);
        nbs_.push_back(nb);
        return ci;
    }

    // Fill the blocks skipped by a symmetric boundary step with references to the
    // transposed partner blocks (boundary.h:161-191).
    void complement_transpose(Hermitian const& herm, bool forward) {
        for (unsigned rb = 0; rb < ket_.size(); ++rb)
            for (unsigned lb = 0; lb < bra_.size(); ++lb) {
                if (lbrb_ci_[size_t(lb) * ket_.size() + rb] == NONE) continue;
                unsigned ci_A = lbrb_ci_[size_t(lb) * ket_.size() + rb];
                unsigned ci_B = cohort_index(ket_.charge(rb), bra_.charge(lb));
                if (ci_B == n_cohorts()) {
                    // bra and ket indices coincide for the symmetric boundaries this is used on
                    ci_B = add_cohort(rb, lb, std::vector<long>(herm.size(), -1));
                    tr_[ci_B] = 1;
                }
                for (unsigned b = 0; b < herm.size(); ++b) {
                    if (herm.skip(b, ket_.charge(rb), bra_.charge(lb))) {
                        offsets_[ci_B][b] = offsets_[ci_A][herm.conj(b)];
                        double cc = has_su2(symm_) ? conjugate_correction_su2(spin_of(ket_.charge(rb)),
                                                                              spin_of(bra_.charge(lb)))
                                                   : 1.0;
                        conj_scales_[ci_B][b] = cc * double(herm.phase(forward ? b : herm.conj(b)));
                        transposes_[ci_B][b] = 1;
                    }
                }
            }
    }

private:
    Symm symm_ = Symm::U1;
    Index bra_, ket_;
    std::vector<unsigned> lbrb_ci_;
    std::vector<std::vector<long>> offsets_;
    std::vector<std::vector<double>> conj_scales_;
    std::vector<std::vector<char>> transposes_;
    std::vector<char> tr_;
    std::vector<size_t> lsz_, rsz_;
    std::vector<unsigned> nbs_;
};

}  // namespace dmrgb200
