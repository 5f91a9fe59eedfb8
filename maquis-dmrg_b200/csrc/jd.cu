// Jacobi-Davidson eigensolver for the lowest eigenpair of H_eff, FP64.
//
// Restates the reference's solver step by step (solve_ietl_jcd,
// dmrg/framework/dmrg/solver/ietl_jacobi_davidson.h:35-76, and
// jacobi_davidson::calculate_eigenvalue, dmrg/framework/ietl/jacobi.h:386-474):
//   * the orthogonal vectors are Gram-Schmidt'ed among themselves and projected
//     out of every new direction (DavidsonVS::project, ietl_interface_dv.h:93-98),
//   * modified Gram-Schmidt against the basis with one refinement pass when the
//     norm drops below kappa = 0.25 of its starting value,
//   * Rayleigh-Ritz on the projected matrix M(i, k) = <V_i, H V_k>, smallest
//     eigenpair (the reference calls LAPACK dsyevx, jacobi.h:476-516; here a
//     cyclic Jacobi rotation solver on the k x k matrix, k <= max_iter),
//   * convergence |r| <= tol |theta| or |r| < tol (ietl/iteration.h:56-58),
//   * correction t = -r + (r.u / u.u) u (jcd_gmres_solver with 0 GMRES steps,
//     jacobi.h:141-157).
// All vectors stay on the device; reductions are two-pass with a fixed block
// count and fixed summation order, so a solve is bitwise reproducible.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"

namespace dmrgb200 {

dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);  // error recording (capi.cpp)
cudaError_t plan_hpsi_launch(dmrgb200_plan_t plan, const double* x, double* y, cudaStream_t stream);
int plan_solver_mode(dmrgb200_plan_t plan);
void** plan_jd_cache(dmrgb200_plan_t plan);
dmrgb200_status solve_graph(dmrgb200_plan_t plan, void** cache, uint64_t n, const double* x0,
                            const double* const* ortho, uint32_t n_ortho, double tol, uint32_t max_iter,
                            double* energy, double* x_out, dmrgb200_solve_stats* stats, cudaStream_t s);

namespace {

constexpr int RED_BLOCKS = 512, RED_THREADS = 256;

// partial[b * nvec + v] = sum over block b's slice of X_v . y
__global__ void __launch_bounds__(RED_THREADS) dot_partials(const double* const* __restrict__ X, int nvec,
                                                            const double* __restrict__ y, uint64_t n,
                                                            double* __restrict__ partial) {
    __shared__ double red[RED_THREADS];
    for (int v = 0; v < nvec; ++v) {
        const double* x = X[v];
        double s = 0.0;
        for (uint64_t i = blockIdx.x * uint64_t(RED_THREADS) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * RED_THREADS)
            s += x[i] * y[i];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[blockIdx.x * nvec + v] = red[0];
        __syncthreads();
    }
}

// out[v] = sum over blocks of partial[b * nvec + v]; one block per vector: every
// thread sums a fixed subset of the blocks in order, then a fixed tree
__global__ void __launch_bounds__(RED_THREADS) dot_finish(const double* __restrict__ partial, int nvec, int nblocks,
                                                          double* __restrict__ out) {
    __shared__ double red[RED_THREADS];
    const int v = blockIdx.x;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += RED_THREADS) s += partial[b * nvec + v];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[v] = red[0];
}

// y += a * x with a = sign * num / den read from device memory (den == nullptr: a = sign * num)
__global__ void axpy_dev(double* __restrict__ y, const double* __restrict__ x, uint64_t n, const double* num,
                         const double* den, double sign) {
    double a = sign * (*num) / (den ? *den : 1.0);
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        y[i] += a * x[i];
}

__global__ void scal_host(double* __restrict__ y, uint64_t n, double a) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        y[i] *= a;
}

struct Coeffs {
    double c[64];
};

// out = sum_j c_j X_j, in the reference's order u = V0 s0; u += Vj sj
__global__ void lincomb(double* __restrict__ out, const double* const* __restrict__ X, int k, Coeffs cf, uint64_t n) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        double s = X[0][i] * cf.c[0];
        for (int j = 1; j < k; ++j) s += X[j][i] * cf.c[j];
        out[i] = s;
    }
}

// r = uA - theta u  (in place in uA)
__global__ void residual(double* __restrict__ uA, const double* __restrict__ u, double theta, uint64_t n) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        uA[i] -= theta * u[i];
}

// t = -r + a u with a = num/den from device memory
__global__ void correction(double* __restrict__ t, const double* __restrict__ r, const double* __restrict__ u,
                           uint64_t n, const double* num, const double* den) {
    double a = (*num) / (*den);
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        t[i] = -r[i] + a * u[i];
}

// smallest eigenpair of a symmetric k x k matrix (column-major, upper triangle used)
void smallest_eigenpair(std::vector<double> A, int k, double& theta, std::vector<double>& s) {
    for (int j = 0; j < k; ++j)
        for (int i = j + 1; i < k; ++i) A[i + j * k] = A[j + i * k];
    std::vector<double> Vm(size_t(k) * k, 0.0);
    for (int i = 0; i < k; ++i) Vm[i + i * k] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < k; ++j)
            for (int i = 0; i < k; ++i) {
                tot += A[i + j * k] * A[i + j * k];
                if (i != j) off += A[i + j * k] * A[i + j * k];
            }
        if (off <= 1e-34 * tot || off == 0.0) break;
        for (int p = 0; p < k; ++p)
            for (int q = p + 1; q < k; ++q) {
                double apq = A[p + q * k];
                if (apq == 0.0) continue;
                double app = A[p + p * k], aqq = A[q + q * k];
                // negligible against both diagonal entries: drop it (the sweep then ends
                // with an exactly diagonal matrix instead of running out of sweeps)
                if (std::fabs(app) + 100.0 * std::fabs(apq) == std::fabs(app) &&
                    std::fabs(aqq) + 100.0 * std::fabs(apq) == std::fabs(aqq)) {
                    A[p + q * k] = A[q + p * k] = 0.0;
                    continue;
                }
                double tau = (aqq - app) / (2.0 * apq);
                double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
                double c = 1.0 / std::sqrt(1.0 + t * t), sn = t * c;
                for (int r = 0; r < k; ++r) {  // A <- A J
                    double arp = A[r + p * k], arq = A[r + q * k];
                    A[r + p * k] = c * arp - sn * arq;
                    A[r + q * k] = sn * arp + c * arq;
                }
                for (int r = 0; r < k; ++r) {  // A <- J^T A
                    double apr = A[p + r * k], aqr = A[q + r * k];
                    A[p + r * k] = c * apr - sn * aqr;
                    A[q + r * k] = sn * apr + c * aqr;
                }
                for (int r = 0; r < k; ++r) {
                    double vrp = Vm[r + p * k], vrq = Vm[r + q * k];
                    Vm[r + p * k] = c * vrp - sn * vrq;
                    Vm[r + q * k] = sn * vrp + c * vrq;
                }
            }
    }
    int best = 0;
    for (int i = 1; i < k; ++i)
        if (A[i + i * k] < A[best + best * k]) best = i;
    theta = A[best + best * k];
    s.assign(k, 0.0);
    for (int i = 0; i < k; ++i) s[i] = Vm[i + best * k];
}

struct Workspace {
    double* vec = nullptr;       // (2 * max_iter + 2 + n_ortho) vectors
    double* partial = nullptr;   // RED_BLOCKS * 64
    double* scal = nullptr;      // 64 device scalars
    const double** ptrs = nullptr;  // device pointer table
    ~Workspace() {
        cudaFree(vec);
        cudaFree(partial);
        cudaFree(scal);
        cudaFree(ptrs);
    }
};

}  // namespace

}  // namespace dmrgb200

using namespace dmrgb200;

namespace dmrgb200 {
dmrgb200_status solve_stepwise(dmrgb200_plan_t plan, uint64_t n, const double* x0, const double* const* ortho,
                               uint32_t n_ortho, double tol, uint32_t max_iter, double* energy, double* x_out,
                               dmrgb200_solve_stats* stats, void* cuda_stream);
int plan_error_words(dmrgb200_plan_t plan);
cudaError_t plan_refresh_constants(dmrgb200_plan_t plan, const double* x, double* y, cudaStream_t stream);
}  // namespace dmrgb200

// Both solver forms end synchronised; a kernel whose bounded wait ran out during
// the solve (grouped S build, emulated stages) turns the result into
// DMRGB200_TIMEOUT.
extern "C" dmrgb200_status dmrgb200_solve(dmrgb200_plan_t plan, uint64_t n, const double* x0,
                                          const double* const* ortho, uint32_t n_ortho, double tol, uint32_t max_iter,
                                          double* energy, double* x_out, dmrgb200_solve_stats* stats,
                                          void* cuda_stream) {
    if (plan && x0 && x_out) {
        cudaError_t e = dmrgb200::plan_refresh_constants(plan, x0, x_out, static_cast<cudaStream_t>(cuda_stream));
        if (e != cudaSuccess)
            return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("emulated boundary digit planes: ") +
                                                           cudaGetErrorString(e));
    }
    dmrgb200_status s =
        dmrgb200::solve_stepwise(plan, n, x0, ortho, n_ortho, tol, max_iter, energy, x_out, stats, cuda_stream);
    // a wait that ran out is the cause of whatever else went wrong in the solve (garbage H psi
    // products can stop the iteration with a numeric error): it is reported first
    const int bits = plan ? dmrgb200::plan_error_words(plan) : 0;
    if (bits)
        return noalloc_fail(DMRGB200_TIMEOUT, (bits & 1) ? "S build: a bulk-copy wait timed out"
                                                         : "emulated H psi: a pipeline wait timed out");
    return s;
}

dmrgb200_status dmrgb200::solve_stepwise(dmrgb200_plan_t plan, uint64_t n, const double* x0,
                                         const double* const* ortho, uint32_t n_ortho, double tol,
                                         uint32_t max_iter, double* energy, double* x_out,
                                         dmrgb200_solve_stats* stats, void* cuda_stream) {
    if (!plan || !x0 || !x_out || !energy || n == 0) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (max_iter < 1 || max_iter > 32) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "max_iter must be in 1..32");
    if (n_ortho > 8) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "at most 8 orthogonal vectors");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    if (plan_solver_mode(plan) == DMRGB200_SOLVER_GRAPH)
        return solve_graph(plan, plan_jd_cache(plan), n, x0, ortho, n_ortho, tol, max_iter, energy, x_out, stats, st);
    const int nv = int(2 * max_iter + 2 + n_ortho);
    Workspace w;
    cudaError_t e;
    if ((e = cudaMalloc(&w.vec, sizeof(double) * n * nv)) != cudaSuccess ||
        (e = cudaMalloc(&w.partial, sizeof(double) * RED_BLOCKS * 64)) != cudaSuccess ||
        (e = cudaMalloc(&w.scal, sizeof(double) * 64)) != cudaSuccess ||
        (e = cudaMalloc(&w.ptrs, sizeof(double*) * 64)) != cudaSuccess)
        return noalloc_fail(e == cudaErrorMemoryAllocation ? DMRGB200_OUT_OF_MEMORY : DMRGB200_DEVICE_ERROR,
                            std::string("solver workspace: ") + cudaGetErrorString(e));
    // H psi writes only block elements: the padding of every work vector must stay zero
    if ((e = cudaMemsetAsync(w.vec, 0, sizeof(double) * n * nv, st)) != cudaSuccess)
        return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("solver workspace: ") + cudaGetErrorString(e));
    auto V = [&](int i) { return w.vec + n * size_t(i); };
    auto VA = [&](int i) { return w.vec + n * size_t(max_iter + i); };
    double* u = w.vec + n * size_t(2 * max_iter);
    double* uA = w.vec + n * size_t(2 * max_iter + 1);
    auto O = [&](int i) { return w.vec + n * size_t(2 * max_iter + 2 + i); };
    const int EB = 4 * device_sm_count(), ET = 256;

    std::vector<const double*> ptr_host(64);
    // dots of y against the vectors xs (<= 64), result in w.scal[0..k)
    auto dots = [&](std::vector<const double*> const& xs, const double* y) -> cudaError_t {
        for (size_t i = 0; i < xs.size(); ++i) ptr_host[i] = xs[i];
        cudaError_t r = cudaMemcpyAsync(w.ptrs, ptr_host.data(), xs.size() * sizeof(double*), cudaMemcpyHostToDevice, st);
        if (r != cudaSuccess) return r;
        dot_partials<<<RED_BLOCKS, RED_THREADS, 0, st>>>(w.ptrs, int(xs.size()), y, n, w.partial);
        dot_finish<<<int(xs.size()), RED_THREADS, 0, st>>>(w.partial, int(xs.size()), RED_BLOCKS, w.scal);
        return cudaGetLastError();
    };
    auto fetch = [&](int k, double* out) -> cudaError_t {
        cudaError_t r = cudaMemcpyAsync(out, w.scal, k * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (r != cudaSuccess) return r;
        return cudaStreamSynchronize(st);
    };
    auto norm = [&](const double* x, double& out) -> cudaError_t {
        cudaError_t r = dots({x}, x);
        if (r != cudaSuccess) return r;
        double v;
        r = fetch(1, &v);
        out = std::sqrt(v);
        return r;
    };
    // t -= <x, t> x  (coefficient stays on the device)
    auto mgs_step = [&](double* t, const double* x) -> cudaError_t {
        cudaError_t r = dots({x}, t);
        if (r != cudaSuccess) return r;
        axpy_dev<<<EB, ET, 0, st>>>(t, x, n, w.scal, nullptr, -1.0);
        return cudaGetLastError();
    };
    // project out the orthogonal vectors: t -= <o, t>/<o, o> o
    auto project = [&](double* t) -> cudaError_t {
        for (uint32_t i = 0; i < n_ortho; ++i) {
            cudaError_t r = dots({O(i)}, t);
            if (r != cudaSuccess) return r;
            r = cudaMemcpyAsync(w.scal + 8, w.scal, sizeof(double), cudaMemcpyDeviceToDevice, st);
            if (r != cudaSuccess) return r;
            r = dots({O(i)}, O(i));
            if (r != cudaSuccess) return r;
            axpy_dev<<<EB, ET, 0, st>>>(t, O(i), n, w.scal + 8, w.scal, -1.0);
        }
        return cudaGetLastError();
    };
#define CK(x)                                                                                           \
    do {                                                                                                \
        cudaError_t _e = (x);                                                                           \
        if (_e != cudaSuccess)                                                                          \
            return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("solver: ") + cudaGetErrorString(_e)); \
    } while (0)

    // orthogonal vectors, Gram-Schmidt'ed among themselves (ietl_jacobi_davidson.h:44-48)
    for (uint32_t i = 0; i < n_ortho; ++i) CK(cudaMemcpyAsync(O(i), ortho[i], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    for (uint32_t a = 1; a < n_ortho; ++a)
        for (uint32_t b = 0; b < a; ++b) {
            CK(dots({O(b)}, O(a)));
            CK(cudaMemcpyAsync(w.scal + 8, w.scal, sizeof(double), cudaMemcpyDeviceToDevice, st));
            CK(dots({O(b)}, O(b)));
            axpy_dev<<<EB, ET, 0, st>>>(O(a), O(b), n, w.scal + 8, w.scal, -1.0);
        }

    std::vector<double> M(size_t(max_iter) * max_iter, 0.0), s;
    const double kappa = 0.25;
    double theta = 0.0, rnorm = 0.0;
    uint32_t iter = 0;
    bool converged = false;
    float hpsi_ms = 0.f;
    cudaEvent_t e0, e1, s0, s1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&s0);
    cudaEventCreate(&s1);
    cudaEventRecord(s0, st);

    CK(cudaMemcpyAsync(V(0), x0, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CK(project(V(0)));
    while (true) {
        double* t = V(int(iter));
        double tau;
        CK(norm(t, tau));
        for (uint32_t i = 1; i <= iter; ++i) CK(mgs_step(t, V(int(i - 1))));
        double tn;
        CK(norm(t, tn));
        if (tn < kappa * tau)
            for (uint32_t i = 1; i <= iter; ++i) CK(mgs_step(t, V(int(i - 1))));
        CK(project(t));
        CK(norm(t, tn));
        if (!(tn > 0.0)) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            cudaEventDestroy(s0);
            cudaEventDestroy(s1);
            return noalloc_fail(DMRGB200_NUMERIC, "Davidson direction vanished");
        }
        scal_host<<<EB, ET, 0, st>>>(t, n, 1.0 / tn);
        cudaEventRecord(e0, st);
        CK(plan_hpsi_launch(plan, t, VA(int(iter)), st));
        cudaEventRecord(e1, st);
        std::vector<const double*> basis;
        for (uint32_t i = 0; i <= iter; ++i) basis.push_back(V(int(i)));
        CK(dots(basis, VA(int(iter))));
        std::vector<double> col(iter + 1);
        CK(fetch(int(iter + 1), col.data()));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        hpsi_ms += ms;
        for (uint32_t i = 0; i <= iter; ++i) M[i + size_t(iter) * max_iter] = col[i];
        // Rayleigh-Ritz on the leading (iter+1) x (iter+1) block
        int k = int(iter + 1);
        std::vector<double> Mk(size_t(k) * k);
        for (int j = 0; j < k; ++j)
            for (int i = 0; i <= j; ++i) Mk[i + j * k] = M[i + size_t(j) * max_iter];
        smallest_eigenpair(Mk, k, theta, s);
        Coeffs cf{};
        for (int j = 0; j < k; ++j) cf.c[j] = s[j];
        CK(cudaMemcpyAsync(w.ptrs, basis.data(), k * sizeof(double*), cudaMemcpyHostToDevice, st));
        lincomb<<<EB, ET, 0, st>>>(u, w.ptrs, k, cf, n);
        std::vector<const double*> abasis;
        for (int i = 0; i < k; ++i) abasis.push_back(VA(i));
        CK(cudaMemcpyAsync(w.ptrs + 32, abasis.data(), k * sizeof(double*), cudaMemcpyHostToDevice, st));
        lincomb<<<EB, ET, 0, st>>>(uA, w.ptrs + 32, k, cf, n);
        CK(project(uA));
        residual<<<EB, ET, 0, st>>>(uA, u, theta, n);
        CK(norm(uA, rnorm));
        ++iter;
        if (rnorm <= tol * std::fabs(theta) || rnorm < tol) {
            converged = true;
            break;
        }
        if (iter >= max_iter) break;
        // correction t = -r + (r.u / u.u) u into V[iter]
        CK(dots({u}, uA));
        CK(cudaMemcpyAsync(w.scal + 8, w.scal, sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(dots({u}, u));
        correction<<<EB, ET, 0, st>>>(V(int(iter)), uA, u, n, w.scal + 8, w.scal);
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(x_out, u, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    cudaEventRecord(s1, st);
    CK(cudaStreamSynchronize(st));
    float solve_ms = 0.f;
    cudaEventElapsedTime(&solve_ms, s0, s1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(s0);
    cudaEventDestroy(s1);
    *energy = theta;
    if (stats) {
        stats->iterations = iter;
        stats->converged = converged ? 1 : 0;
        stats->residual = rnorm;
        stats->hpsi_ms = hpsi_ms;
        stats->solve_ms = solve_ms;
    }
#undef CK
    return DMRGB200_OK;
}
