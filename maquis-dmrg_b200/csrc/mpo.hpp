// MPO tensor as consumed by the schedule builders.
//
// Mirrors the parts of the reference's MPOTensor that the hot path reads
// (dmrg/framework/dmrg/mp_tensors/mpotensor.h:45-135, mpotensor_detail.h:48-239):
//  * row(b1) iteration over b2 in increasing order and column(b2) over b1,
//  * at(b1, b2) -> list of (operator, scale),
//  * left/right bond spins (SU2 only) and the Hermitian pairing of bond indices
//    (Herm[b], Phase[b], skip(b, l, r) = l < r && Herm[b] defined).
// Site operators are block-sparse over physical charges; each block
// (left = phys_in, right = phys_out) carries its non-zero entries in row-major
// order with row/column spins (block_matrix/sparse_operator.h:35-235).
#pragma once

#include <cstdint>
#include <limits>
#include <vector>

#include "symm.hpp"

namespace dmrgb200 {

struct SparseEntry {
    unsigned row, col;
    int row_spin, col_spin;
    double coeff;
};

struct OpBlock {
    Charge left, right;  // left = input physical charge, right = output physical charge
    std::vector<SparseEntry> entries;
};

struct SiteOp {
    int spin = 0;  // SU2 rank K (2x spin)
    std::vector<OpBlock> blocks;
};

class Hermitian {
public:
    static constexpr unsigned NONE = std::numeric_limits<unsigned>::max();
    Hermitian() = default;
    explicit Hermitian(unsigned d) : herm_(d, NONE), phase_(d, 1) {}
    Hermitian(std::vector<unsigned> h, std::vector<int> p) : herm_(std::move(h)), phase_(std::move(p)) {}

    // b-index complete cohorts: skip when l < r and b has a registered partner
    bool skip(unsigned b, Charge l, Charge r) const { return (l < r) && herm_[b] != NONE; }
    unsigned conj(unsigned b) const { return herm_[b]; }
    int phase(unsigned b) const { return phase_[b]; }
    size_t size() const { return herm_.size(); }

private:
    std::vector<unsigned> herm_;
    std::vector<int> phase_;
};

struct TermRef {
    unsigned op;
    double scale;
    unsigned id = 0;  // position of the term in the MPO description (term provenance of the schedule)
};

struct MPOEntry {
    unsigned other;  // b2 for a row list, b1 for a column list
    std::vector<TermRef> terms;
};

struct MPOTensor {
    unsigned row_dim = 0, col_dim = 0;
    std::vector<int> left_spin, right_spin;
    Hermitian left_herm, right_herm;
    std::vector<std::vector<MPOEntry>> rows;  // rows[b1]: sorted by b2
    std::vector<std::vector<MPOEntry>> cols;  // cols[b2]: sorted by b1
    std::vector<SiteOp> ops;

    int lspin(unsigned b) const { return left_spin.empty() ? 0 : left_spin[b]; }
    int rspin(unsigned b) const { return right_spin.empty() ? 0 : right_spin[b]; }
};

}  // namespace dmrgb200
