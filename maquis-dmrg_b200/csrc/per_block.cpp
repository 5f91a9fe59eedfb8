// H·psi with one library GEMM launch per block product: the launch pattern of the
// reference's GPU path, kept as the comparison arm of the grouped kernels.
//
// The reference stages every T task as its own cuBLAS DGEMM
// (MPSBlock::create_T_gpu, dmrg/framework/dmrg/solver/tasks.cpp:707-752) and
// every cohort's contraction as its own DGEMM into the output block
// (Cohort::contract_gpu, tasks.cpp:315-344), transposing Hermitian-complement
// boundary blocks before use (tr_tile_v, tasks.cpp:49-62).  Here, on one stream:
//   stage 1: one cublasDgemm per T task (per stored block when the task reads a
//            transposed cohort);
//   stage 2: the library's S build (one launch: it is not a GEMM);
//   stage 3: one cublasDgemm per cohort, accumulating into its output block (per
//            block with the operand transposed for Hermitian-complement cohorts).
// The sums are those of the grouped path up to the order of the floating-point
// additions inside the library GEMMs.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"

namespace dmrgb200 {
dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);
// plan internals (capi.cpp)
FlatPlan const& plan_flat(dmrgb200_plan_t plan);
DeviceProgram const& plan_program(dmrgb200_plan_t plan);
std::vector<uint64_t> const& plan_stage1_bnd(dmrgb200_plan_t plan);
std::vector<uint64_t> const& plan_stage3_bnd(dmrgb200_plan_t plan);
double* plan_T(dmrgb200_plan_t plan);
double* plan_S(dmrgb200_plan_t plan);
void*& plan_blas_handle(dmrgb200_plan_t plan);
}  // namespace dmrgb200

using namespace dmrgb200;

extern "C" dmrgb200_status dmrgb200_hpsi_per_block(dmrgb200_plan_t plan, const double* x, double* y,
                                                   void* cuda_stream, uint64_t* launches) {
    if (!plan || !x || !y) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    FlatPlan const& p = plan_flat(plan);
    if (p.kind != KIND_HPSI || !plan_T(plan)) return noalloc_fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    void*& hv = plan_blas_handle(plan);
    if (!hv) {
        cublasHandle_t h = nullptr;
        if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return noalloc_fail(DMRGB200_DEVICE_ERROR, "cublasCreate");
        hv = h;
    }
    cublasHandle_t h = static_cast<cublasHandle_t>(hv);
    if (cublasSetStream(h, st) != CUBLAS_STATUS_SUCCESS) return noalloc_fail(DMRGB200_DEVICE_ERROR, "cublasSetStream");
    std::vector<uint64_t> const& rb = plan_stage1_bnd(plan);
    std::vector<uint64_t> const& lb = plan_stage3_bnd(plan);
    double* T = plan_T(plan);
    double* S = plan_S(plan);
    const std::vector<uint64_t> t_off = t_offsets(p, nullptr);
    const std::vector<uint64_t> s_off = s_offsets(p, nullptr);
    const double one = 1.0, zero = 0.0;
    uint64_t n = 0;
    auto gemm = [&](cublasOperation_t ta, cublasOperation_t tb, int M, int N, int K, const double* A, int lda,
                    const double* B, int ldb, double beta, double* C, int ldc) -> bool {
        ++n;
        return cublasDgemm(h, ta, tb, M, N, K, &one, A, lda, B, ldb, &beta, C, ldc) == CUBLAS_STATUS_SUCCESS;
    };
    // stage 1: T_t = psi slice (ls_in x brows) * R cohort
    for (uint32_t t = 0; t < p.n_t(); ++t) {
        const uint32_t M = p.in_rows[p.t_lb[t]], K = p.t_brows[t], N = p.t_bcols[t], nb = p.t_nb[t];
        if (!M || !K || !N || !nb) continue;
        const double* A = x + p.in_off[p.t_lb[t]] + uint64_t(p.t_col[t]) * M;
        const double* R = reinterpret_cast<const double*>(rb[p.t_ci[t]]);
        double* C = T + t_off[t];
        if (!p.t_trans[t]) {
            if (!gemm(CUBLAS_OP_N, CUBLAS_OP_N, M, int(N * nb), K, A, M, R, K, zero, C, M))
                return noalloc_fail(DMRGB200_DEVICE_ERROR, "per-block stage 1 GEMM");
        } else {
            for (uint32_t b = 0; b < nb; ++b)
                if (!gemm(CUBLAS_OP_N, CUBLAS_OP_T, M, N, K, A, M, R + uint64_t(b) * N * K, N, zero,
                          C + uint64_t(b) * M * N, M))
                    return noalloc_fail(DMRGB200_DEVICE_ERROR, "per-block stage 1 GEMM");
        }
    }
    // stage 2: the S build
    cudaError_t e = run_sbuild(plan_program(plan), T, S, st);
    if (e != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("S build: ") + cudaGetErrorString(e));
    // stage 3: y[lb_out] = sum over cohorts of L (ls_out x nsrows ls_in) * S (nsrows ls_in x stripe)
    for (uint32_t b = 0; b < p.out_rows.size(); ++b) {
        const uint64_t cnt = uint64_t(p.out_rows[b]) * p.out_cols[b];
        if (cnt && (e = cudaMemsetAsync(y + p.out_off[b], 0, cnt * sizeof(double), st)) != cudaSuccess)
            return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("output clear: ") + cudaGetErrorString(e));
    }
    for (uint32_t c = 0; c < p.n_cohorts(); ++c) {
        const uint32_t M = p.c_rs[c], ls = p.c_ls[c], nsr = p.c_nsrows[c], N = p.c_stripe[c];
        if (!M || !ls || !nsr || !N) continue;
        const double* Lc = reinterpret_cast<const double*>(lb[p.c_ci[c]]);
        const double* Sc = S + s_off[c];
        double* Y = y + p.out_off[p.c_rb[c]];
        const int ldy = int(p.out_rows[p.c_rb[c]]);
        if (!p.c_trans[c]) {
            if (!gemm(CUBLAS_OP_N, CUBLAS_OP_N, M, N, int(nsr * ls), Lc, M, Sc, int(nsr * ls), one, Y, ldy))
                return noalloc_fail(DMRGB200_DEVICE_ERROR, "per-block stage 3 GEMM");
        } else {
            // stored blocks are ls x M: one GEMM per block with the operand transposed
            for (uint32_t k = 0; k < nsr; ++k)
                if (!gemm(CUBLAS_OP_T, CUBLAS_OP_N, M, N, ls, Lc + uint64_t(k) * ls * M, ls, Sc + uint64_t(k) * ls,
                          int(nsr * ls), one, Y, ldy))
                    return noalloc_fail(DMRGB200_DEVICE_ERROR, "per-block stage 3 GEMM");
        }
    }
    if (launches) *launches = n + 1;
    return DMRGB200_OK;
}

namespace dmrgb200 {
void blas_handle_free(void* h) {
    if (h) cublasDestroy(static_cast<cublasHandle_t>(h));
}
}  // namespace dmrgb200
