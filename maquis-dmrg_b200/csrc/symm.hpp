// Symmetry-group charges, Index and ProductBasis for the host-side schedule builder.
//
// Charges follow the reference's symmetry groups:
//   U1     one integer, fuse = addition, particleNumber = the charge
//          (dmrg/framework/dmrg/block_matrix/symmetry/u1.h:39-56)
//   TwoU1  two integers, component-wise addition, particleNumber = sum,
//          lexicographic order (symmetry/nu1_tpl.h:215-230, :266-296)
//   SU2U1  (N, 2S) with component-wise addition, particleNumber = N, spin = 2S
//          (symmetry/su2u1.h:37-71)
// Index is an ordered list of (charge, size) sectors; ProductBasis assigns the
// offset of each (a, b) pair inside the fused sector, a-major then b
// (block_matrix/indexing_stable.hpp:310-345).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <utility>
#include <vector>

namespace dmrgb200 {

enum class Symm : int { U1 = 1, TwoU1 = 2, SU2U1 = 3 };

inline bool has_su2(Symm s) { return s == Symm::SU2U1; }

struct Charge {
    int q[2] = {0, 0};
    Charge() = default;
    Charge(int a, int b) { q[0] = a; q[1] = b; }
};

inline bool operator==(Charge a, Charge b) { return a.q[0] == b.q[0] && a.q[1] == b.q[1]; }
inline bool operator!=(Charge a, Charge b) { return !(a == b); }
inline bool operator<(Charge a, Charge b) {
    return a.q[0] < b.q[0] || (a.q[0] == b.q[0] && a.q[1] < b.q[1]);
}
inline Charge fuse(Charge a, Charge b) { return Charge(a.q[0] + b.q[0], a.q[1] + b.q[1]); }
inline Charge neg(Charge a) { return Charge(-a.q[0], -a.q[1]); }

inline int particle_number(Symm s, Charge c) {
    switch (s) {
        case Symm::U1: return c.q[0];
        case Symm::TwoU1: return c.q[0] + c.q[1];
        case Symm::SU2U1: return c.q[0];
    }
    return 0;
}
inline int spin_of(Charge c) { return c.q[1]; }

// SU2 triangle condition on (a, b, c) with b an MPO-bond spin; always true
// without SU2 (block_matrix/symmetry/gsl_coupling.h:49-70).
inline bool triangle_int(int a, int b, int c) { return std::abs(a - b) <= c && c <= a + b; }
inline bool triangle(Symm s, Charge a, int b, Charge c) {
    if (!has_su2(s)) return true;
    return triangle_int(spin_of(a), b, spin_of(c));
}

struct Index {
    std::vector<Charge> ch;
    std::vector<unsigned> sz;
    std::map<std::pair<int, int>, unsigned> pos;

    void push(Charge c, unsigned s) {
        pos[{c.q[0], c.q[1]}] = static_cast<unsigned>(ch.size());
        ch.push_back(c);
        sz.push_back(s);
    }
    unsigned size() const { return static_cast<unsigned>(ch.size()); }
    // position of a charge, size() if absent (reference Index::position semantics)
    unsigned position(Charge c) const {
        auto it = pos.find({c.q[0], c.q[1]});
        return it == pos.end() ? size() : it->second;
    }
    Charge charge(unsigned i) const { return ch[i]; }
    unsigned block_size(unsigned i) const { return sz[i]; }
};

// Offsets of (a_i, b_j) inside the fused sector f(a_i, b_j), a-major.
class ProductBasis {
public:
    template <class F>
    ProductBasis(Index const& a, Index const& b, F f) {
        for (unsigned i = 0; i < a.size(); ++i)
            for (unsigned j = 0; j < b.size(); ++j) {
                Charge pc = f(a.charge(i), b.charge(j));
                auto key = std::make_pair(pc.q[0], pc.q[1]);
                size_t& acc = sizes_[key];
                offs_[{i, j}] = acc;
                acc += size_t(a.block_size(i)) * b.block_size(j);
            }
        a_ = a;
        b_ = b;
    }
    size_t operator()(Charge ca, Charge cb) const {
        unsigned i = a_.position(ca), j = b_.position(cb);
        auto it = offs_.find({i, j});
        if (it == offs_.end()) throw std::runtime_error("ProductBasis: pair not in basis");
        return it->second;
    }

private:
    Index a_, b_;
    std::map<std::pair<unsigned, unsigned>, size_t> offs_;
    std::map<std::pair<int, int>, size_t> sizes_;
};

// right-paired column basis: fused charge = -sigma + rc  (site_hamil_schedule.hpp:61-63)
inline ProductBasis right_paired_basis(Index const& phys, Index const& right) {
    return ProductBasis(phys, right, [](Charge s, Charge r) { return fuse(neg(s), r); });
}
// left-paired row basis: fused charge = sigma + lc  (move_boundary.hpp:186)
inline ProductBasis left_paired_basis(Index const& phys, Index const& left) {
    return ProductBasis(phys, left, [](Charge s, Charge l) { return fuse(s, l); });
}

}  // namespace dmrgb200
