#include "coupling.hpp"

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <stdexcept>
#include <tuple>

namespace dmrgb200 {

namespace {

// log-factorials in long double; arguments stay well below 400 for any bond spin here
struct LogFact {
    std::vector<long double> v;
    LogFact() : v(512) {
        v[0] = 0.0L;
        for (size_t n = 1; n < v.size(); ++n) v[n] = v[n - 1] + std::log((long double)n);
    }
    long double operator()(int n) const { return v.at(static_cast<size_t>(n)); }
};
const LogFact& lf() {
    static LogFact t;
    return t;
}

bool tri2(int a, int b, int c) {  // triangle + integer-perimeter test on doubled spins
    return a >= 0 && b >= 0 && c >= 0 && std::abs(a - b) <= c && c <= a + b && ((a + b + c) % 2 == 0);
}

// log of the triangle coefficient Delta(abc) on doubled spins
long double log_delta(int a, int b, int c) {
    const LogFact& F = lf();
    return 0.5L * (F((a + b - c) / 2) + F((a - b + c) / 2) + F((-a + b + c) / 2) - F((a + b + c) / 2 + 1));
}

}  // namespace

double wigner6j(int j1, int j2, int j3, int j4, int j5, int j6) {
    // {j1 j2 j3; j4 j5 j6}: triangles (j1 j2 j3), (j1 j5 j6), (j4 j2 j6), (j4 j5 j3)
    if (!tri2(j1, j2, j3) || !tri2(j1, j5, j6) || !tri2(j4, j2, j6) || !tri2(j4, j5, j3)) return 0.0;
    const LogFact& F = lf();
    int a1 = (j1 + j2 + j3) / 2, a2 = (j1 + j5 + j6) / 2, a3 = (j4 + j2 + j6) / 2, a4 = (j4 + j5 + j3) / 2;
    int b1 = (j1 + j2 + j4 + j5) / 2, b2 = (j2 + j3 + j5 + j6) / 2, b3 = (j3 + j1 + j6 + j4) / 2;
    int tmin = std::max(std::max(a1, a2), std::max(a3, a4));
    int tmax = std::min(b1, std::min(b2, b3));
    long double pre = log_delta(j1, j2, j3) + log_delta(j1, j5, j6) + log_delta(j4, j2, j6) + log_delta(j4, j5, j3);
    long double sum = 0.0L;
    for (int t = tmin; t <= tmax; ++t) {
        long double lg = F(t + 1) - F(t - a1) - F(t - a2) - F(t - a3) - F(t - a4) - F(b1 - t) - F(b2 - t) - F(b3 - t);
        long double term = std::exp(lg + pre);
        sum += (t % 2 ? -term : term);
    }
    return static_cast<double>(sum);
}

double wigner9j(int j1, int j2, int j3, int j4, int j5, int j6, int j7, int j8, int j9) {
    // sum_x (-1)^(2x) (2x+1) {j1 j4 j7; j8 j9 x} {j2 j5 j8; j4 x j6} {j3 j6 j9; x j1 j2}
    if (!tri2(j1, j2, j3) || !tri2(j4, j5, j6) || !tri2(j7, j8, j9) || !tri2(j1, j4, j7) || !tri2(j2, j5, j8) ||
        !tri2(j3, j6, j9))
        return 0.0;
    int xmin = std::max(std::max(std::abs(j1 - j9), std::abs(j4 - j8)), std::abs(j2 - j6));
    int xmax = std::min(std::min(j1 + j9, j4 + j8), j2 + j6);
    long double sum = 0.0L;
    for (int x = xmin; x <= xmax; x += 2) {
        long double w = (long double)(x + 1) * wigner6j(j1, j4, j7, j8, j9, x) * wigner6j(j2, j5, j8, j4, x, j6) *
                        wigner6j(j3, j6, j9, x, j1, j2);
        sum += (x % 2 ? -w : w);  // (-1)^(2x) with x doubled: odd doubled value -> half-integer x
    }
    return static_cast<double>(sum);
}

double mod_coupling(int a, int b, int c, int d, int e, int f, int g, int h, int i) {
    using Key = std::tuple<int, int, int, int, int, int, int, int, int>;
    static std::map<Key, double> cache;
    static std::mutex mu;
    Key k{a, b, c, d, e, f, g, h, i};
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(k);
        if (it != cache.end()) return it->second;
    }
    double v = std::sqrt((g + 1.0) * (h + 1.0) * (c + 1.0) * (f + 1.0)) * wigner9j(a, b, c, d, e, f, g, h, i);
    std::lock_guard<std::mutex> lk(mu);
    cache[k] = v;
    return v;
}

static bool tri(int a, int b, int c) { return std::abs(a - b) <= c && c <= a + b; }

void set_coupling(int a, int b, int c, int d, int e, int f, int g, int h, int i, double init, double couplings[4]) {
    couplings[0] = couplings[1] = couplings[2] = couplings[3] = 0.0;
    double pre = std::sqrt((i + 1.0) * (a + 1.0) / ((g + 1.0) * (c + 1.0))) * init;
    if (tri(a, b, c)) {
        couplings[0] = pre * mod_coupling(a, b, c, d, e, f, g, h, i);
        couplings[2] = pre * mod_coupling(a, b, c, d, e, f, g, 2, i);
    }
    if (tri(a, 2, c)) {
        couplings[1] = pre * mod_coupling(a, 2, c, d, e, f, g, h, i);
        couplings[3] = pre * mod_coupling(a, 2, c, d, e, f, g, 2, i);
    }
}

double conjugate_correction_su2(int lspin, int rspin) {
    int S = std::min(lspin, rspin);
    int diff = rspin - lspin;
    switch (diff) {
        case 0: return 1.0;
        case 1: return -std::sqrt((S + 1.0) / (S + 2.0));
        case -1: return std::sqrt((S + 2.0) / (S + 1.0));
        case 2: return -std::sqrt((S + 1.0) / (S + 3.0));
        case -2: return -std::sqrt((S + 3.0) / (S + 1.0));
        default: throw std::runtime_error("conjugate correction defined only up to rank-1 spin differences");
    }
}

}  // namespace dmrgb200
