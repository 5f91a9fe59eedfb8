// ORACLE shim (test infrastructure): the one boost::lambda facility the
// reference's solver core uses (sort_invert in dmrg/utils/utils.hpp).
#pragma once
#include <utility>
namespace boost { namespace lambda {
template <class T> struct constructor {
    template <class... A> T operator()(A&&... a) const { return T(std::forward<A>(a)...); }
};
}}
