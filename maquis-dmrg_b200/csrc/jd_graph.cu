// Jacobi-Davidson as one CUDA graph: every scalar of the iteration lives on the
// device, one iteration is the body of a conditional WHILE node, and the body's
// last reduction decides whether it runs again.  The steps are those of the
// stepwise solver in jd.cu (ietl/jacobi.h:386-474, ietl_jacobi_davidson.h:35-76):
// MGS with one refinement pass below kappa = 0.25, projection of the
// orthogonal vectors, Rayleigh-Ritz (cyclic Jacobi on the k x k projected
// matrix, here by one warp), convergence |r| <= tol |theta| or |r| < tol, and
// the correction t = -r + (r.u / u.u) u.
//
// Reductions: every vector kernel runs on a fixed grid; each block reduces its
// slice in a fixed order and the last block to arrive sums the block partials
// in block order, so a solve is bitwise reproducible.  Each body sets the WHILE
// condition to 0 first and only the residual kernel sets it back to 1, after
// incrementing the iteration count, so the loop ends after at most max_iter
// bodies whatever the data.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"

namespace dmrgb200 {

dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);
cudaError_t plan_hpsi_launch(dmrgb200_plan_t plan, const double* x, double* y, cudaStream_t stream);
cudaError_t plan_ensure_tuned(dmrgb200_plan_t plan, const double* x, double* y, cudaStream_t stream);

namespace {

constexpr int JT = 256;        // threads per block of the vector kernels
constexpr int MAXK = 32;       // max_iter bound
constexpr int MAXO = 8;        // orthogonal vectors bound

struct JdState {
    unsigned counter;
    int iter, done, status, converged, refine;
    double tau, tn, theta, rnorm, corr;
    double c[2][MAXK];     // MGS coefficients, per pass
    double pc[MAXO];       // projection coefficients of the current target
    double oo[MAXO];       // <o_i, o_i>
    double M[MAXK * MAXK]; // projected matrix, column-major, leading dimension MAXK
    double s[MAXK];        // Ritz vector coefficients
};

struct JdArgs {
    double* vec;          // vector slots, n doubles each
    uint64_t n;
    uint64_t chunk;       // elements per block
    int max_iter, n_ortho;
    double tol;
    JdState* st;
    double* partial;      // per-block partial sums: MAXK + 2 rows of gridDim
    cudaGraphConditionalHandle cond;
};

// slots: V(0..max_iter), VA(0..max_iter), u, uA, t, y, O(0..n_ortho)
__device__ __forceinline__ double* V(JdArgs const& a, int i) { return a.vec + a.n * uint64_t(i); }
__device__ __forceinline__ double* VA(JdArgs const& a, int i) { return a.vec + a.n * uint64_t(a.max_iter + i); }
__device__ __forceinline__ double* U(JdArgs const& a) { return a.vec + a.n * uint64_t(2 * a.max_iter); }
__device__ __forceinline__ double* UA(JdArgs const& a) { return a.vec + a.n * uint64_t(2 * a.max_iter + 1); }
__device__ __forceinline__ double* Tv(JdArgs const& a) { return a.vec + a.n * uint64_t(2 * a.max_iter + 2); }
__device__ __forceinline__ double* Yv(JdArgs const& a) { return a.vec + a.n * uint64_t(2 * a.max_iter + 3); }
__device__ __forceinline__ double* Ov(JdArgs const& a, int i) { return a.vec + a.n * uint64_t(2 * a.max_iter + 4 + i); }

__device__ __forceinline__ uint64_t lo(JdArgs const& a) { return blockIdx.x * a.chunk; }
__device__ __forceinline__ uint64_t hi(JdArgs const& a) {
    uint64_t h = (blockIdx.x + 1) * a.chunk;
    return h < a.n ? h : a.n;
}

// block sum in a fixed order; the result is valid in thread 0
__device__ double block_sum(double v) {
    __shared__ double red[JT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < JT / 32; ++w) s += red[w];
    return s;
}

// publish this block's partials and report whether it is the last block to arrive
__device__ bool arrive(JdState* st) {
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&st->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    return last;
}

// sum of row r of the partial table over all blocks, by the whole (last) block:
// every thread sums a fixed subset in order, then the fixed block tree; the
// result is valid in thread 0
__device__ double gather(JdArgs const& a, int r) {
    double s = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += JT) s += __ldcg(a.partial + uint64_t(r) * gridDim.x + b);
    return block_sum(s);
}

__device__ void finish(JdArgs const& a) {
    if (threadIdx.x == 0) a.st->counter = 0;
}

// dot of two slices
__device__ double slice_dot(JdArgs const& a, const double* x, const double* y) {
    double s = 0.0;
    for (uint64_t i = lo(a) + threadIdx.x; i < hi(a); i += JT) s += x[i] * y[i];
    return block_sum(s);
}

__global__ void __launch_bounds__(JT) jd_init(JdArgs a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        JdState* st = a.st;
        st->counter = 0;
        st->iter = st->done = st->status = st->converged = st->refine = 0;
        st->tau = st->tn = st->theta = st->rnorm = st->corr = 0.0;
    }
}

// <O(i), O(i)> into oo[i]
__global__ void __launch_bounds__(JT) jd_oo(JdArgs a, int i) {
    double p = slice_dot(a, Ov(a, i), Ov(a, i));
    if (threadIdx.x == 0) a.partial[blockIdx.x] = p;
    if (arrive(a.st)) {
        const double g = gather(a, 0);
        if (threadIdx.x == 0) a.st->oo[i] = g;
        finish(a);
    }
}

// target -= pc[i-1] O(i-1) (i > 0), then pc[i] = <O(i), target> / oo[i].
// target: 0 = t, 1 = uA, 2 + j = O(j)
__device__ double* target_of(JdArgs const& a, int target) {
    return target == 0 ? Tv(a) : target == 1 ? UA(a) : Ov(a, target - 2);
}
__global__ void __launch_bounds__(JT) jd_proj(JdArgs a, int i, int target) {
    double* x = target_of(a, target);
    if (i > 0) {
        const double c = a.st->pc[i - 1];
        const double* o = Ov(a, i - 1);
        for (uint64_t k = lo(a) + threadIdx.x; k < hi(a); k += JT) x[k] -= c * o[k];
    }
    double p = slice_dot(a, Ov(a, i), x);
    if (threadIdx.x == 0) a.partial[blockIdx.x] = p;
    if (arrive(a.st)) {
        const double g = gather(a, 0);
        if (threadIdx.x == 0) a.st->pc[i] = g / a.st->oo[i];
        finish(a);
    }
}
__global__ void __launch_bounds__(JT) jd_proj_close(JdArgs a, int last, int target) {
    double* x = target_of(a, target);
    const double c = a.st->pc[last];
    const double* o = Ov(a, last);
    for (uint64_t k = lo(a) + threadIdx.x; k < hi(a); k += JT) x[k] -= c * o[k];
}

// first kernel of an iteration: stop unless the residual kernel says otherwise; tau = |t|
__global__ void __launch_bounds__(JT) jd_tau(JdArgs a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
    double p = slice_dot(a, Tv(a), Tv(a));
    if (threadIdx.x == 0) a.partial[blockIdx.x] = p;
    if (arrive(a.st)) {
        const double g = gather(a, 0);
        if (threadIdx.x == 0) a.st->tau = sqrt(g);
        finish(a);
    }
}

// MGS step j of a pass: t -= c[pass][j-1] V(j-1), then c[pass][j] = <V(j), t>
__global__ void __launch_bounds__(JT) jd_mgs(JdArgs a, int j, int pass) {
    JdState* st = a.st;
    if (j >= st->iter || (pass == 1 && !st->refine)) return;
    double* t = Tv(a);
    if (j > 0) {
        const double c = st->c[pass][j - 1];
        const double* v = V(a, j - 1);
        for (uint64_t k = lo(a) + threadIdx.x; k < hi(a); k += JT) t[k] -= c * v[k];
    }
    double p = slice_dot(a, V(a, j), t);
    if (threadIdx.x == 0) a.partial[blockIdx.x] = p;
    if (arrive(st)) {
        const double g = gather(a, 0);
        if (threadIdx.x == 0) st->c[pass][j] = g;
        finish(a);
    }
}

// end of an MGS pass: apply the last coefficient; after pass 0 decide on refinement
__global__ void __launch_bounds__(JT) jd_mgs_close(JdArgs a, int pass) {
    JdState* st = a.st;
    const int it = st->iter;
    double* t = Tv(a);
    const bool active = it > 0 && (pass == 0 || st->refine);
    if (active) {
        const double c = st->c[pass][it - 1];
        const double* v = V(a, it - 1);
        for (uint64_t k = lo(a) + threadIdx.x; k < hi(a); k += JT) t[k] -= c * v[k];
    }
    if (pass != 0) return;
    double p = slice_dot(a, t, t);
    if (threadIdx.x == 0) a.partial[blockIdx.x] = p;
    if (arrive(st)) {
        const double g = gather(a, 0);
        if (threadIdx.x == 0) {
            st->tn = sqrt(g);
            st->refine = (it > 0 && st->tn < 0.25 * st->tau) ? 1 : 0;
        }
        finish(a);
    }
}

// |t| after orthogonalisation; a vanished direction ends the solve
__global__ void __launch_bounds__(JT) jd_tnorm(JdArgs a) {
    double p = slice_dot(a, Tv(a), Tv(a));
    if (threadIdx.x == 0) a.partial[blockIdx.x] = p;
    if (arrive(a.st)) {
        const double g = gather(a, 0);
        if (threadIdx.x == 0) {
            JdState* st = a.st;
            st->tn = sqrt(g);
            if (!(st->tn > 0.0)) {
                st->status = 1;
                st->done = 1;
            }
        }
        finish(a);
    }
}

// t /= |t|; V(iter) = t
__global__ void __launch_bounds__(JT) jd_store(JdArgs a) {
    JdState* st = a.st;
    const double inv = st->status ? 0.0 : 1.0 / st->tn;
    double* t = Tv(a);
    double* v = V(a, st->iter);
    for (uint64_t k = lo(a) + threadIdx.x; k < hi(a); k += JT) {
        double x = t[k] * inv;
        t[k] = x;
        v[k] = x;
    }
}

// VA(iter) = y; M(j, iter) = <V(j), y> for j <= iter
__global__ void __launch_bounds__(JT) jd_mcol(JdArgs a) {
    JdState* st = a.st;
    const int it = st->iter;
    const double* y = Yv(a);
    double* va = VA(a, it);
    for (uint64_t k = lo(a) + threadIdx.x; k < hi(a); k += JT) va[k] = y[k];
    for (int j = 0; j <= it; ++j) {
        double p = slice_dot(a, V(a, j), y);
        if (threadIdx.x == 0) a.partial[uint64_t(j) * gridDim.x + blockIdx.x] = p;
    }
    if (arrive(st)) {
        for (int j = 0; j <= it; ++j) {
            const double g = gather(a, j);
            if (threadIdx.x == 0) st->M[j + it * MAXK] = g;
        }
        finish(a);
    }
}

// smallest eigenpair of the leading k x k block of M (cyclic Jacobi, one warp;
// lane r owns row/column r of the rotation updates)
__global__ void __launch_bounds__(32) jd_ritz(JdArgs a) {
    __shared__ double A[MAXK][MAXK + 1];
    __shared__ double Vm[MAXK][MAXK + 1];
    JdState* st = a.st;
    const int k = st->iter + 1, r = threadIdx.x;
    for (int j = 0; j < k; ++j)
        if (r < k) {
            A[r][j] = r <= j ? st->M[r + j * MAXK] : st->M[j + r * MAXK];
            Vm[r][j] = r == j ? 1.0 : 0.0;
        }
    __syncwarp();
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        if (r < k)
            for (int j = 0; j < k; ++j) {
                double v = A[r][j] * A[r][j];
                tot += v;
                if (j != r) off += v;
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        off = __shfl_sync(0xffffffffu, off, 0);  // one decision for the whole warp
        tot = __shfl_sync(0xffffffffu, tot, 0);
        if (off <= 1e-34 * tot || off == 0.0) break;
        for (int p = 0; p < k; ++p)
            for (int q = p + 1; q < k; ++q) {
                const double apq = A[p][q];
                if (apq == 0.0) continue;
                const double app = A[p][p], aqq = A[q][q];
                // negligible against both diagonal entries: drop it (as in jd.cu)
                if (fabs(app) + 100.0 * fabs(apq) == fabs(app) && fabs(aqq) + 100.0 * fabs(apq) == fabs(aqq)) {
                    __syncwarp();
                    if (r == 0) A[p][q] = A[q][p] = 0.0;
                    __syncwarp();
                    continue;
                }
                const double tau = (aqq - app) / (2.0 * apq);
                const double tt = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double c = 1.0 / sqrt(1.0 + tt * tt), sn = tt * c;
                __syncwarp();
                if (r < k) {  // A <- A J
                    double arp = A[r][p], arq = A[r][q];
                    A[r][p] = c * arp - sn * arq;
                    A[r][q] = sn * arp + c * arq;
                }
                __syncwarp();
                if (r < k) {  // A <- J^T A
                    double apr = A[p][r], aqr = A[q][r];
                    A[p][r] = c * apr - sn * aqr;
                    A[q][r] = sn * apr + c * aqr;
                }
                if (r < k) {
                    double vrp = Vm[r][p], vrq = Vm[r][q];
                    Vm[r][p] = c * vrp - sn * vrq;
                    Vm[r][q] = sn * vrp + c * vrq;
                }
                __syncwarp();
            }
    }
    __syncwarp();
    int best = 0;
    for (int i = 1; i < k; ++i)
        if (A[i][i] < A[best][best]) best = i;
    if (r == 0) st->theta = A[best][best];
    if (r < k) st->s[r] = Vm[r][best];
}

// u = sum_j s_j V(j), uA = sum_j s_j VA(j)
__global__ void __launch_bounds__(JT) jd_lincomb(JdArgs a) {
    JdState* st = a.st;
    const int k = st->iter + 1;
    double* u = U(a);
    double* ua = UA(a);
    for (uint64_t i = lo(a) + threadIdx.x; i < hi(a); i += JT) {
        double x = V(a, 0)[i] * st->s[0], y = VA(a, 0)[i] * st->s[0];
        for (int j = 1; j < k; ++j) {
            x += V(a, j)[i] * st->s[j];
            y += VA(a, j)[i] * st->s[j];
        }
        u[i] = x;
        ua[i] = y;
    }
}

// r = uA - theta u; convergence test; next iteration or stop
__global__ void __launch_bounds__(JT) jd_residual(JdArgs a) {
    JdState* st = a.st;
    const double theta = st->theta;
    double* ua = UA(a);
    const double* u = U(a);
    double rr = 0.0, ru = 0.0, uu = 0.0;
    for (uint64_t i = lo(a) + threadIdx.x; i < hi(a); i += JT) {
        double r = ua[i] - theta * u[i];
        ua[i] = r;
        rr += r * r;
        ru += r * u[i];
        uu += u[i] * u[i];
    }
    rr = block_sum(rr);
    ru = block_sum(ru);
    uu = block_sum(uu);
    if (threadIdx.x == 0) {
        a.partial[blockIdx.x] = rr;
        a.partial[gridDim.x + blockIdx.x] = ru;
        a.partial[2 * gridDim.x + blockIdx.x] = uu;
    }
    if (arrive(st)) {
        const double rrs = gather(a, 0), rus = gather(a, 1), uus = gather(a, 2);
        if (threadIdx.x == 0) {
            st->rnorm = sqrt(rrs);
            st->corr = rus / uus;
            st->iter += 1;
            const bool conv = st->rnorm <= a.tol * fabs(theta) || st->rnorm < a.tol;
            st->converged = conv ? 1 : 0;
            if (conv || st->iter >= a.max_iter) st->done = 1;
            cudaGraphSetConditional(a.cond, st->done ? 0u : 1u);
        }
        finish(a);
    }
}

// t = -r + corr u for the next iteration
__global__ void __launch_bounds__(JT) jd_correction(JdArgs a) {
    JdState* st = a.st;
    if (st->done) return;
    const double c = st->corr;
    const double* r = UA(a);
    const double* u = U(a);
    double* t = Tv(a);
    for (uint64_t i = lo(a) + threadIdx.x; i < hi(a); i += JT) t[i] = -r[i] + c * u[i];
}

}  // namespace

// Per-plan solver graph, rebuilt when the sizes, tolerance or stream change.
struct JdGraph {
    uint64_t n = 0;
    uint32_t max_iter = 0, n_ortho = 0;
    double tol = 0.0;
    double* vec = nullptr;
    JdState* st = nullptr;
    double* partial = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~JdGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(vec);
        cudaFree(st);
        cudaFree(partial);
    }
};

void jd_graph_free(void* g) { delete static_cast<JdGraph*>(g); }

namespace {

cudaError_t build_graph(JdGraph& g, dmrgb200_plan_t plan, cudaStream_t s) {
    // s: a private non-blocking stream (the legacy default stream cannot capture)
    cudaError_t e;
    const uint64_t n = g.n;
    const int nslots = int(2 * g.max_iter + 4 + g.n_ortho);
    const int nb = 2 * device_sm_count();
    if ((e = cudaMalloc(&g.vec, sizeof(double) * n * nslots)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&g.st, sizeof(JdState))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&g.partial, sizeof(double) * nb * (MAXK + 2))) != cudaSuccess) return e;
    // H psi writes only block elements: the padding of every slot stays zero
    if ((e = cudaMemset(g.vec, 0, sizeof(double) * n * nslots)) != cudaSuccess) return e;
    if ((e = cudaMemset(g.st, 0, sizeof(JdState))) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&g.e0)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&g.e1)) != cudaSuccess) return e;

    JdArgs a{};
    a.vec = g.vec;
    a.n = n;
    a.chunk = (n + nb - 1) / nb;
    a.max_iter = int(g.max_iter);
    a.n_ortho = int(g.n_ortho);
    a.tol = g.tol;
    a.st = g.st;
    a.partial = g.partial;

    // the grouped GEMMs are tuned before capture (on the zeroed t and y slots)
    if ((e = plan_ensure_tuned(plan, g.vec + n * (2 * g.max_iter + 2), g.vec + n * (2 * g.max_iter + 3), s)) !=
        cudaSuccess)
        return e;
    if ((e = cudaGraphCreate(&g.graph, 0)) != cudaSuccess) return e;
    if ((e = cudaGraphConditionalHandleCreate(&a.cond, g.graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
        return e;

    // prologue: state, orthogonal vectors among themselves (ietl_jacobi_davidson.h:44-48),
    // projection of the start vector (t holds x0)
    if ((e = cudaStreamBeginCaptureToGraph(s, g.graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
        cudaSuccess)
        return e;
    jd_init<<<1, 32, 0, s>>>(a);
    const int no = int(g.n_ortho);
    for (int i = 0; i < no; ++i) {
        if (i > 0) {
            for (int b = 0; b < i; ++b) jd_proj<<<nb, JT, 0, s>>>(a, b, 2 + i);
            jd_proj_close<<<nb, JT, 0, s>>>(a, i - 1, 2 + i);
        }
        jd_oo<<<nb, JT, 0, s>>>(a, i);
    }
    if (no > 0) {
        for (int i = 0; i < no; ++i) jd_proj<<<nb, JT, 0, s>>>(a, i, 0);
        jd_proj_close<<<nb, JT, 0, s>>>(a, no - 1, 0);
    }
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(s, &captured);
    if (e != cudaSuccess) return e;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;

    // the WHILE node after the prologue
    std::vector<cudaGraphNode_t> leaves;
    size_t nn = 0;
    if ((e = cudaGraphGetNodes(g.graph, nullptr, &nn)) != cudaSuccess) return e;
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn && (e = cudaGraphGetNodes(g.graph, nodes.data(), &nn)) != cudaSuccess) return e;
    for (auto nd : nodes) {
        size_t ndep = 0;
        if ((e = cudaGraphNodeGetDependentNodes(nd, nullptr, &ndep)) != cudaSuccess) return e;
        if (ndep == 0) leaves.push_back(nd);
    }
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = a.cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    if ((e = cudaGraphAddNode(&wnode, g.graph, leaves.data(), leaves.size(), &cp)) != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];

    // one iteration (jacobi.h:386-474)
    if ((e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
        cudaSuccess)
        return e;
    jd_tau<<<nb, JT, 0, s>>>(a);
    for (int pass = 0; pass < 2; ++pass) {
        for (int j = 0; j + 1 < int(g.max_iter); ++j) jd_mgs<<<nb, JT, 0, s>>>(a, j, pass);
        jd_mgs_close<<<nb, JT, 0, s>>>(a, pass);
    }
    if (no > 0) {
        for (int i = 0; i < no; ++i) jd_proj<<<nb, JT, 0, s>>>(a, i, 0);
        jd_proj_close<<<nb, JT, 0, s>>>(a, no - 1, 0);
    }
    jd_tnorm<<<nb, JT, 0, s>>>(a);
    jd_store<<<nb, JT, 0, s>>>(a);
    cudaError_t he = plan_hpsi_launch(plan, g.vec + n * (2 * g.max_iter + 2), g.vec + n * (2 * g.max_iter + 3), s);
    jd_mcol<<<nb, JT, 0, s>>>(a);
    jd_ritz<<<1, 32, 0, s>>>(a);
    jd_lincomb<<<nb, JT, 0, s>>>(a);
    if (no > 0) {
        for (int i = 0; i < no; ++i) jd_proj<<<nb, JT, 0, s>>>(a, i, 1);
        jd_proj_close<<<nb, JT, 0, s>>>(a, no - 1, 1);
    }
    jd_residual<<<nb, JT, 0, s>>>(a);
    jd_correction<<<nb, JT, 0, s>>>(a);
    cudaGraph_t body_out = nullptr;
    e = cudaStreamEndCapture(s, &body_out);
    if (e != cudaSuccess) return e;
    if (he != cudaSuccess) return he;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaGraphInstantiate(&g.exec, g.graph, 0);
}

}  // namespace

dmrgb200_status solve_graph(dmrgb200_plan_t plan, void** cache, uint64_t n, const double* x0,
                            const double* const* ortho, uint32_t n_ortho, double tol, uint32_t max_iter,
                            double* energy, double* x_out, dmrgb200_solve_stats* stats, cudaStream_t s) {
    JdGraph* g = static_cast<JdGraph*>(*cache);
    if (!g || g->n != n || g->max_iter != max_iter || g->n_ortho != n_ortho || g->tol != tol) {
        delete g;
        *cache = nullptr;
        g = new JdGraph;
        g->n = n;
        g->max_iter = max_iter;
        g->n_ortho = n_ortho;
        g->tol = tol;
        cudaStream_t cs = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // inputs of earlier work on s are complete
        if (e == cudaSuccess) e = build_graph(*g, plan, cs);
        if (cs) {
            cudaStreamCaptureStatus st;
            if (cudaStreamIsCapturing(cs, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
                cudaGraph_t junk = nullptr;
                cudaStreamEndCapture(cs, &junk);
                if (junk) cudaGraphDestroy(junk);
            }
            cudaStreamDestroy(cs);
        }
        if (e != cudaSuccess) {
            delete g;
            cudaGetLastError();
            return noalloc_fail(e == cudaErrorMemoryAllocation ? DMRGB200_OUT_OF_MEMORY : DMRGB200_DEVICE_ERROR,
                                std::string("solver graph: ") + cudaGetErrorString(e));
        }
        *cache = g;
    }
    const uint64_t T = n * (2 * max_iter + 2);
    cudaError_t e;
#define CK(x)                                                                                                \
    do {                                                                                                     \
        if ((e = (x)) != cudaSuccess)                                                                        \
            return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("solver: ") + cudaGetErrorString(e));     \
    } while (0)
    CK(cudaMemcpyAsync(g->vec + T, x0, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    for (uint32_t i = 0; i < n_ortho; ++i)
        CK(cudaMemcpyAsync(g->vec + n * (2 * max_iter + 4 + i), ortho[i], n * sizeof(double), cudaMemcpyDeviceToDevice,
                           s));
    CK(cudaEventRecord(g->e0, s));
    CK(cudaGraphLaunch(g->exec, s));
    CK(cudaEventRecord(g->e1, s));
    CK(cudaMemcpyAsync(x_out, g->vec + n * (2 * max_iter), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    JdState hs;
    CK(cudaMemcpyAsync(&hs, g->st, sizeof(JdState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
#undef CK
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->e0, g->e1);
    if (hs.status) return noalloc_fail(DMRGB200_NUMERIC, "Davidson direction vanished");
    *energy = hs.theta;
    if (stats) {
        stats->iterations = uint32_t(hs.iter);
        stats->converged = hs.converged;
        stats->residual = hs.rnorm;
        stats->hpsi_ms = 0.0;
        stats->solve_ms = ms;
    }
    return DMRGB200_OK;
}

}  // namespace dmrgb200
