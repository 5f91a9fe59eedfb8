// ORACLE — test infrastructure only.  Nothing in the product imports, links or
// executes this file; tests, __graft_entry__.smoke() and bench.py's CPU
// baseline use it as the checker.
//
// CPU restatement of the reference's execution of a contraction schedule, in
// FP64 with OpenMP over task groups and BLAS dgemm/daxpy, on the flat plan
// description of include/dmrgb200.h:
//   hpsi        super_hamil_mv CPU branch    solver/super_hamil_mv.hpp:121-132
//     create_T                               solver/tasks.cpp:650-705
//     create_s_r                             solver/tasks.cpp:466-494
//     contract (tr_tile_v for virtual L)     solver/tasks.cpp:49-62, 286-313
//   left step   move_boundary.hpp:260-276
//     create_T_left                          solver/tasks.cpp:545-601
//     create_s                               solver/tasks.cpp:425-454
//     prop_l                                 solver/tasks.cpp:198-209
//   right step  move_boundary.hpp:385-401
//     create_T, create_s_r                   (as above)
//     prop_r                                 solver/tasks.cpp:243-260
//   alpha_dm    prediction.hpp:41-69, move_boundary.hpp:38-143
//     lbtm, rbtm                             solver/tasks.cpp:346-380
// Output accumulation of H psi is serialised per output block with a mutex,
// as in the reference (tasks.cpp:310-312).
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include <omp.h>

#include "../include/dmrgb200.h"

extern "C" {
void scipy_dgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k, const double* alpha,
                  const double* a, const int* lda, const double* b, const int* ldb, const double* beta, double* c,
                  const int* ldc);
void scipy_daxpy_(const int* n, const double* a, const double* x, const int* incx, double* y, const int* incy);
void scipy_openblas_set_num_threads(int n);
}

namespace {

void gemm(char ta, char tb, int m, int n, int k, double alpha, const double* a, int lda, const double* b, int ldb,
          double beta, double* c, int ldc) {
    if (m == 0 || n == 0) return;
    if (k == 0) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < m; ++i) c[i + size_t(j) * ldc] = beta == 0.0 ? 0.0 : beta * c[i + size_t(j) * ldc];
        return;
    }
    scipy_dgemm_(&ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
}

void axpy(size_t n, double a, const double* x, double* y) {
    int nn = int(n), one = 1;
    if (n) scipy_daxpy_(&nn, &a, x, &one, y, &one);
}

// transpose each of cnt (nrows x ncols) blocks into (ncols x nrows) (tasks.cpp:49-62)
void tr_tile_v(unsigned nrows, unsigned ncols, size_t cnt, const double* in, double* out) {
    for (size_t b = 0; b < cnt; ++b) {
        size_t off = b * nrows * ncols;
        for (unsigned i = 0; i < nrows; ++i)
            for (unsigned j = 0; j < ncols; ++j) out[off + size_t(ncols) * i + j] = in[off + size_t(nrows) * j + i];
    }
}

// stage 1 of H psi / right step: T_t = x-slice * R (per block, transposed when virtual)
std::vector<double> create_T(dmrgb200_plan_desc const& d, uint32_t t, const double* const* R, const double* x) {
    int M = int(d.in_rows[d.t_lb[t]]);
    int K = int(d.t_brows[t]);
    int N = int(d.t_bcols[t]);
    const double* mps = x + d.in_off[d.t_lb[t]] + size_t(M) * d.t_col[t];
    std::vector<double> T(size_t(M) * N * d.t_nb[t]);
    for (uint32_t b = 0; b < d.t_nb[t]; ++b) {
        const double* rb = R[d.t_ci[t]] + size_t(b) * K * N;
        double* out = T.data() + size_t(b) * M * N;
        if (d.t_trans[t])
            gemm('N', 'T', M, N, K, 1.0, mps, M, rb, N, 0.0, out, M);
        else
            gemm('N', 'N', M, N, K, 1.0, mps, M, rb, K, 0.0, out, M);
    }
    return T;
}

// stage 1 of the left step: T_t[b] = L_b (^T) * ket-slice
std::vector<double> create_T_left(dmrgb200_plan_desc const& d, uint32_t t, const double* const* Lb, const double* ket) {
    int M = int(d.t_brows[t]);
    int K = int(d.t_bcols[t]);
    int N = int(d.t_width[t]);
    const double* mps = ket + d.in_off[d.t_lb[t]] + size_t(K) * d.t_col[t];
    std::vector<double> T(size_t(M) * N * d.t_nb[t]);
    for (uint32_t b = 0; b < d.t_nb[t]; ++b) {
        const double* lb = Lb[d.t_ci[t]] + size_t(b) * M * K;
        double* out = T.data() + size_t(b) * M * N;
        if (d.t_trans[t])
            gemm('T', 'N', M, N, K, 1.0, lb, K, mps, K, 0.0, out, M);
        else
            gemm('N', 'N', M, N, K, 1.0, lb, M, mps, K, 0.0, out, M);
    }
    return T;
}

// S of H psi / right step: (nSrows*ls) x stripe, row block b1 per line
std::vector<double> create_s_r(dmrgb200_plan_desc const& d, uint32_t c, std::vector<std::vector<double>> const& T,
                               uint32_t tbase) {
    size_t ls = d.c_ls[c], ns = d.c_nsrows[c], stripe = d.c_stripe[c];
    std::vector<double> S(ns * ls * stripe, 0.0);
    for (uint32_t u = d.c_unit[c]; u < d.c_unit[c + 1]; ++u) {
        size_t ms = d.u_ms[u];
        std::vector<double> buf(ls * ms);
        for (uint32_t l = d.u_line[u]; l < d.u_line[u + 1]; ++l) {
            std::fill(buf.begin(), buf.end(), 0.0);
            for (uint32_t k = d.l_term[l]; k < d.l_term[l + 1]; ++k)
                axpy(ms * ls, d.term_alpha[k], T[d.term_t[k] - tbase].data() + size_t(d.term_col[k]) * ls, buf.data());
            size_t bb = d.l_b1[l];
            for (size_t col = 0; col < ms; ++col)
                std::memcpy(&S[ns * ls * (d.u_offset[u] + col) + bb * ls], &buf[col * ls], ls * sizeof(double));
        }
    }
    return S;
}

// S of the left step: stripe x (nSrows*rs), column block b per line
std::vector<double> create_s(dmrgb200_plan_desc const& d, uint32_t c, std::vector<std::vector<double>> const& T,
                             uint32_t tbase) {
    size_t rs = d.c_rs[c], ns = d.c_nsrows[c], stripe = d.c_stripe[c];
    std::vector<double> S(ns * rs * stripe, 0.0);
    for (uint32_t u = d.c_unit[c]; u < d.c_unit[c + 1]; ++u) {
        size_t ms = d.u_ms[u];
        std::vector<double> buf(ms * rs);
        for (uint32_t l = d.u_line[u]; l < d.u_line[u + 1]; ++l) {
            std::fill(buf.begin(), buf.end(), 0.0);
            for (uint32_t k = d.l_term[l]; k < d.l_term[l + 1]; ++k)
                axpy(ms * rs, d.term_alpha[k], T[d.term_t[k] - tbase].data() + size_t(d.term_col[k]) * rs, buf.data());
            size_t bb = d.l_b1[l];
            for (size_t col = 0; col < rs; ++col)
                std::memcpy(&S[stripe * (bb * rs + col) + d.u_offset[u]], &buf[col * ms], ms * sizeof(double));
        }
    }
    return S;
}

}  // namespace

extern "C" {

int oracle_set_threads(int n) {
    omp_set_num_threads(n);
    scipy_openblas_set_num_threads(1);
    return 0;
}

// y = H x on the plan; L and R are per-cohort host pointers; y's blocks are overwritten.
int oracle_hpsi(const dmrgb200_plan_desc* dp, const double* const* L, const double* const* R, const double* x,
                double* y) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_HPSI) return 1;
    for (uint32_t b = 0; b < d.n_out_blocks; ++b)
        std::memset(y + d.out_off[b], 0, sizeof(double) * size_t(d.out_rows[b]) * d.out_cols[b]);
    std::vector<std::mutex> mutexes(d.n_out_blocks);
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int gi = 0; gi < ng; ++gi) {
        std::vector<std::vector<double>> T;
        for (uint32_t t = d.g_t[gi]; t < d.g_t[gi + 1]; ++t) T.push_back(create_T(d, t, R, x));
        for (uint32_t c = d.g_c[gi]; c < d.g_c[gi + 1]; ++c) {
            std::vector<double> S = create_s_r(d, c, T, d.g_t[gi]);
            int M = int(d.c_rs[c]), N = int(d.c_stripe[c]), K = int(d.c_nsrows[c] * d.c_ls[c]);
            const double* luse = L[d.c_ci[c]];
            std::vector<double> lbuf;
            if (d.c_trans[c]) {
                lbuf.resize(size_t(M) * K);
                tr_tile_v(d.c_ls[c], d.c_rs[c], d.c_nsrows[c], L[d.c_ci[c]], lbuf.data());
                luse = lbuf.data();
            }
            std::vector<double> buf(size_t(M) * N);
            gemm('N', 'N', M, N, K, 1.0, luse, M, S.data(), K, 0.0, buf.data(), M);
            std::lock_guard<std::mutex> lk(mutexes[d.c_rb[c]]);
            axpy(size_t(M) * N, 1.0, buf.data(), y + d.out_off[d.c_rb[c]]);
        }
    }
    return 0;
}

// Left step: out[c_out_ci] = bra^T * S per cohort.
int oracle_left_step(const dmrgb200_plan_desc* dp, const double* const* L, const double* ket, const double* bra,
                     double* const* out) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_LEFT_STEP) return 1;
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int gi = 0; gi < ng; ++gi) {
        std::vector<std::vector<double>> T;
        for (uint32_t t = d.g_t[gi]; t < d.g_t[gi + 1]; ++t) T.push_back(create_T_left(d, t, L, ket));
        for (uint32_t c = d.g_c[gi]; c < d.g_c[gi + 1]; ++c) {
            std::vector<double> S = create_s(d, c, T, d.g_t[gi]);
            int M = int(d.c_ls[c]), N = int(d.c_nsrows[c] * d.c_rs[c]), K = int(d.c_stripe[c]);
            gemm('T', 'N', M, N, K, 1.0, bra + d.out_off[d.c_lb[c]], K, S.data(), K, 0.0, out[d.c_out_ci[c]], M);
        }
    }
    return 0;
}

// Right step: out[c_out_ci] block b = S rows b * bra^T per cohort.
int oracle_right_step(const dmrgb200_plan_desc* dp, const double* const* R, const double* ket, const double* bra,
                      double* const* out) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_RIGHT_STEP) return 1;
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int gi = 0; gi < ng; ++gi) {
        std::vector<std::vector<double>> T;
        for (uint32_t t = d.g_t[gi]; t < d.g_t[gi + 1]; ++t) T.push_back(create_T(d, t, R, ket));
        for (uint32_t c = d.g_c[gi]; c < d.g_c[gi + 1]; ++c) {
            std::vector<double> S = create_s_r(d, c, T, d.g_t[gi]);
            int ls = int(d.c_ls[c]), rs = int(d.c_rs[c]), ns = int(d.c_nsrows[c]);
            int M = ns * ls, N = rs, K = int(d.c_stripe[c]);
            std::vector<double> buf(size_t(M) * N);
            gemm('N', 'T', M, N, K, 1.0, S.data(), M, bra + d.out_off[d.c_rb[c]], rs, 0.0, buf.data(), M);
            double* o = out[d.c_out_ci[c]];
            for (int b = 0; b < ns; ++b)
                for (int col = 0; col < rs; ++col)
                    std::memcpy(o + (size_t(b) * rs + col) * ls, &buf[size_t(ls) * b + size_t(col) * M],
                                ls * sizeof(double));
        }
    }
    return 0;
}

// Density matrix of a two-site split with the perturbation (state prediction) of the
// reference, on a step plan whose ket and bra are the same tensor Theta (the two-site
// tensor viewed as one site; prediction.hpp:41-69 alpha_dm / alpha_dm_right):
//   left step:  dm_b = Theta_b Theta_b^T + alpha sum_{c: c_lb = b} S_c S_c^T
//               (Theta_b the left-paired bra block b, S_c = create_s; Cohort::lbtm,
//                tasks.cpp:346-362, driven by alpha_dm_direct, move_boundary.hpp:38-91)
//   right step: dm_b = Theta_b^T Theta_b + alpha sum_{c: c_rb = b} S_c^T S_c
//               (Theta_b the right-paired bra block b, S_c = create_s_r; Cohort::rbtm,
//                tasks.cpp:364-380, driven by alpha_dm_direct_right, :93-143)
// dm[b] is stripe_b x stripe_b; with_theta = 0 leaves the Theta term out (the
// reference's alpha_dm_direct alone, accumulated into dm, which is not cleared then).
int oracle_alpha_dm(const dmrgb200_plan_desc* dp, const double* const* B, const double* ket, const double* bra,
                    double alpha, int with_theta, double* const* dm) {
    dmrgb200_plan_desc const& d = *dp;
    const bool left = d.kind == DMRGB200_PLAN_LEFT_STEP;
    if (!left && d.kind != DMRGB200_PLAN_RIGHT_STEP) return 1;
    if (with_theta)
        for (uint32_t b = 0; b < d.n_out_blocks; ++b) {
            const int r = int(d.out_rows[b]), c = int(d.out_cols[b]);
            const double* th = bra + d.out_off[b];
            if (left)
                gemm('N', 'T', r, r, c, 1.0, th, r, th, r, 0.0, dm[b], r);
            else
                gemm('T', 'N', c, c, r, 1.0, th, r, th, r, 0.0, dm[b], c);
        }
    std::vector<std::mutex> mutexes(d.n_out_blocks);
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int gi = 0; gi < ng; ++gi) {
        std::vector<std::vector<double>> T;
        for (uint32_t t = d.g_t[gi]; t < d.g_t[gi + 1]; ++t)
            T.push_back(left ? create_T_left(d, t, B, ket) : create_T(d, t, B, ket));
        for (uint32_t c = d.g_c[gi]; c < d.g_c[gi + 1]; ++c) {
            const int M = int(d.c_stripe[c]);
            std::vector<double> tmp(size_t(M) * M, 0.0);
            uint32_t b;
            if (left) {
                std::vector<double> S = create_s(d, c, T, d.g_t[gi]);
                const int K = int(S.size() / size_t(M));
                gemm('N', 'T', M, M, K, alpha, S.data(), M, S.data(), M, 1.0, tmp.data(), M);
                b = d.c_lb[c];
            } else {
                std::vector<double> S = create_s_r(d, c, T, d.g_t[gi]);
                const int K = int(d.c_nsrows[c] * d.c_ls[c]);
                gemm('T', 'N', M, M, K, alpha, S.data(), K, S.data(), K, 1.0, tmp.data(), M);
                b = d.c_rb[c];
            }
            std::lock_guard<std::mutex> lk(mutexes[b]);
            axpy(size_t(M) * M, 1.0, tmp.data(), dm[b]);
        }
    }
    return 0;
}

// Adjoint of H psi on the plan (the reference has no derivative code; this is
// the transpose of the three stages above, run per task group):
//   G_c = L_c^T w[rb]  (transpose of contract, tasks.cpp:286-313)
//   galpha[k] = <G cell(k), T cell(k)>, gT cell(k) += alpha_k G cell(k)
//                      (transpose of create_s_r, tasks.cpp:466-494)
//   gx slice += gT_t R_t^T  (transpose of create_T, tasks.cpp:650-705)
// gx (whole in_size range) is overwritten; galpha has n_terms entries.  Either
// output may be NULL.  A task group owns its input block, so gx needs no lock.
int oracle_hpsi_adjoint(const dmrgb200_plan_desc* dp, const double* const* L, const double* const* R,
                        const double* w, const double* x, double* gx, double* galpha) {
    dmrgb200_plan_desc const& d = *dp;
    if (d.kind != DMRGB200_PLAN_HPSI) return 1;
    if (gx) std::memset(gx, 0, sizeof(double) * d.in_size);
    int ng = int(d.n_groups);
#pragma omp parallel for schedule(dynamic, 1)
    for (int gi = 0; gi < ng; ++gi) {
        const uint32_t t0 = d.g_t[gi], t1 = d.g_t[gi + 1];
        std::vector<std::vector<double>> T, gT;
        for (uint32_t t = t0; t < t1; ++t) {
            if (galpha) T.push_back(create_T(d, t, R, x));
            gT.emplace_back(size_t(d.in_rows[d.t_lb[t]]) * d.t_bcols[t] * d.t_nb[t], 0.0);
        }
        for (uint32_t c = d.g_c[gi]; c < d.g_c[gi + 1]; ++c) {
            int M = int(d.c_rs[c]), N = int(d.c_stripe[c]), K = int(d.c_nsrows[c] * d.c_ls[c]);
            const double* luse = L[d.c_ci[c]];
            std::vector<double> lbuf;
            if (d.c_trans[c]) {
                lbuf.resize(size_t(M) * K);
                tr_tile_v(d.c_ls[c], d.c_rs[c], d.c_nsrows[c], L[d.c_ci[c]], lbuf.data());
                luse = lbuf.data();
            }
            std::vector<double> G(size_t(K) * N);
            gemm('T', 'N', K, N, M, 1.0, luse, M, w + d.out_off[d.c_rb[c]], M, 0.0, G.data(), K);
            size_t ls = d.c_ls[c];
            for (uint32_t u = d.c_unit[c]; u < d.c_unit[c + 1]; ++u) {
                size_t ms = d.u_ms[u];
                for (uint32_t l = d.u_line[u]; l < d.u_line[u + 1]; ++l) {
                    const double* gcell = G.data() + size_t(d.l_b1[l]) * ls + size_t(d.u_offset[u]) * K;
                    for (uint32_t k = d.l_term[l]; k < d.l_term[l + 1]; ++k) {
                        size_t toff = size_t(d.term_col[k]) * ls;
                        if (galpha) {
                            const double* tc = T[d.term_t[k] - t0].data() + toff;
                            double s = 0.0;
                            for (size_t j = 0; j < ms; ++j)
                                for (size_t r = 0; r < ls; ++r) s += gcell[r + j * K] * tc[r + j * ls];
                            galpha[k] = s;
                        }
                        double* gc = gT[d.term_t[k] - t0].data() + toff;
                        for (size_t j = 0; j < ms; ++j)
                            for (size_t r = 0; r < ls; ++r) gc[r + j * ls] += d.term_alpha[k] * gcell[r + j * K];
                    }
                }
            }
        }
        if (!gx) continue;
        for (uint32_t t = t0; t < t1; ++t) {
            int M = int(d.in_rows[d.t_lb[t]]), K = int(d.t_brows[t]), N = int(d.t_bcols[t]);
            double* out = gx + d.in_off[d.t_lb[t]] + size_t(M) * d.t_col[t];
            for (uint32_t b = 0; b < d.t_nb[t]; ++b) {
                const double* rb = R[d.t_ci[t]] + size_t(b) * K * N;
                const double* g = gT[t - t0].data() + size_t(b) * M * N;
                if (d.t_trans[t])
                    gemm('N', 'N', M, K, N, 1.0, g, M, rb, N, 1.0, out, M);
                else
                    gemm('N', 'T', M, K, N, 1.0, g, M, rb, K, 1.0, out, M);
            }
        }
    }
    return 0;
}

}  // extern "C"
