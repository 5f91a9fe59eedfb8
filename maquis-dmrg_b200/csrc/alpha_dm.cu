// Density matrix of a two-site split with the reference's state prediction
// (perturbation), on a boundary-step plan whose ket and bra are the two-site tensor
// viewed as one site (prediction.hpp:41-69 alpha_dm / alpha_dm_right,
// move_boundary.hpp:38-143 alpha_dm_direct, Cohort::lbtm / rbtm tasks.cpp:346-380):
//
//   left step  (left-to-right split): dm_b = Theta_b Theta_b^T + alpha sum_{c: lb(c) = b} S_c S_c^T
//   right step (right-to-left split): dm_b = Theta_b^T Theta_b + alpha sum_{c: rb(c) = b} S_c^T S_c
//
// with S_c the cohort's S of the step (stages 1 and 2 of the step program) and
// Theta_b the bra block b.  After the S build, S is scaled by sqrt(alpha) in place;
// every dm block is then one problem of the grouped FP64 GEMM whose K segments are
// Theta_b and the S of each cohort that adds to it, in cohort order, so each block
// has one owner per output tile and is written once, without atomics (the
// reference adds its cohorts under a critical section in thread order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "device.hpp"

namespace dmrgb200 {

namespace {
__global__ void __launch_bounds__(256) scale_kernel(double* __restrict__ x, uint64_t n, double a) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        x[i] *= a;
}
}  // namespace

cudaError_t scale_buffer(double* x, uint64_t n, double a, cudaStream_t st) {
    if (!n) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, uint64_t(device_sm_count()) * 8);
    scale_kernel<<<uint32_t(blocks), 256, 0, st>>>(x, n, a);
    return cudaGetLastError();
}

void build_alpha_dm(FlatPlan const& p, std::vector<uint64_t> const& dm, GemmList& gl) {
    gl = GemmList();
    const bool left = p.kind == KIND_LEFT;
    const uint32_t nb = uint32_t(p.out_rows.size());
    std::vector<uint64_t> s_off = s_offsets(p, nullptr);
    std::vector<std::vector<uint32_t>> by_block(nb);
    for (uint32_t c = 0; c < p.n_cohorts(); ++c) by_block[left ? p.c_lb[c] : p.c_rb[c]].push_back(c);
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t r = p.out_rows[b], cols = p.out_cols[b];
        const uint32_t stripe = left ? r : cols;  // dm_b is stripe x stripe
        DevProb pr;
        pr.M = stripe;
        pr.N = stripe;
        pr.C = dev_op(BUF_ABS, dm[b] / 8, std::max<uint32_t>(stripe, 1), false);
        pr.seg_begin = uint32_t(gl.segs.size());
        DevSeg th{};
        if (left) {  // Theta_b (stripe x cols) times its transpose
            th.A = dev_op(BUF_OUT, p.out_off[b], std::max<uint32_t>(r, 1), false);
            th.B = dev_op(BUF_OUT, p.out_off[b], std::max<uint32_t>(r, 1), true);
            th.K = cols;
        } else {  // Theta_b^T Theta_b, Theta_b is r x stripe
            th.A = dev_op(BUF_OUT, p.out_off[b], std::max<uint32_t>(r, 1), true);
            th.B = dev_op(BUF_OUT, p.out_off[b], std::max<uint32_t>(r, 1), false);
            th.K = r;
        }
        gl.segs.push_back(th);
        for (uint32_t c : by_block[b]) {
            DevSeg sg{};
            if (left) {  // S_c: stripe x (nSrows rs), leading dimension stripe
                sg.A = dev_op(BUF_S, s_off[c], p.c_stripe[c], false);
                sg.B = dev_op(BUF_S, s_off[c], p.c_stripe[c], true);
                sg.K = p.c_nsrows[c] * p.c_rs[c];
            } else {  // S_c: (nSrows ls) x stripe
                const uint32_t K = p.c_nsrows[c] * p.c_ls[c];
                sg.A = dev_op(BUF_S, s_off[c], std::max<uint32_t>(K, 1), true);
                sg.B = dev_op(BUF_S, s_off[c], std::max<uint32_t>(K, 1), false);
                sg.K = K;
            }
            gl.segs.push_back(sg);
        }
        pr.seg_end = uint32_t(gl.segs.size());
        gl.probs.push_back(pr);
        gemm_add_tiles(gl, uint32_t(gl.probs.size() - 1), 1);
    }
    gemm_sort_tiles(gl);
}

}  // namespace dmrgb200
