// Block-wise thin SVD and block copies for the two-site split on the device.
//
// The reference splits a two-site tensor by a thin SVD of every symmetry block
// of the matrix Theta (rows (l, s1), columns (s2, r) of one middle charge),
// keeps the largest singular values over all blocks and writes U and S V^T (or
// U S and V^T) back as site tensors (svd: block_matrix/block_matrix_algorithms.h:
// 95-113; svd_truncate: :185-298; TwoSiteTensor::split_mps_l2r / r2l:
// mp_tensors/twositetensor.hpp:153-200).
//
// block_svd_jacobi: one CTA of 16 warps per block, one-sided (Hestenes) Jacobi.  The block is
// taken as m x n columns with n = min(rows, cols) (the transpose when rows < cols).
// Column pairs are orthogonalised in round-robin order, n/2 disjoint pairs per
// round spread over the warps; a pair rotates when |g_p . g_q| > tol |g_p| |g_q|
// (tol = sqrt(m) eps), on the block scaled exactly by a power of two to a
// largest element in [1, 2).  Sweeps repeat until one makes no rotation (at most
// SVD_MAX_SWEEPS; exhausting them sets the error flag).  Then sigma_j = |g_j|,
// U = G / sigma, V is the accumulated rotation, all sorted by descending sigma.
// The columns and V live in shared memory when they fit, else in a global
// scratch (L2-resident at these sizes).  There is no spin-wait: every loop is
// bounded.
//
// copy_blocks: dst block = src block (column-major, own leading dimensions),
// optionally scaled per row or per column; it gathers Theta from the two-site
// tensor and scatters U / V^T into the new site tensors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"

namespace dmrgb200 {

dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);

namespace {

constexpr int SVD_THREADS = 512, SVD_WARPS = SVD_THREADS / 32, SVD_MAX_SWEEPS = 60;
constexpr int SVD_REG = 8;  // register path for columns of up to 32 * SVD_REG elements
constexpr size_t SVD_SMEM_LIMIT = 200 * 1024;

struct SvdBlock {
    const double* a;  // rows x cols, ld = rows
    double* u;        // rows x k, ld = rows
    double* s;        // k
    double* vt;       // k x cols, ld = k
    double* work;     // null: shared memory
    uint32_t rows, cols;
};

// work elements of one block: G (m x n), V (n x n), sigma (n), rank table (n ints in n doubles)
__host__ __device__ inline size_t svd_work_elems(uint32_t rows, uint32_t cols) {
    const size_t m = rows > cols ? rows : cols, n = rows < cols ? rows : cols;
    return m * n + n * n + 2 * n;
}

__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Rutishauser's rotation of columns p, q from their squared norms al, be and
// inner product ga: t the smaller root of t^2 + 2 zeta t - 1 = 0.  Returns false
// when the pair is already orthogonal to tol.
__device__ inline bool jacobi_cs(double al, double be, double ga, double tol, double& c, double& s) {
    if (ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) return false;
    const double zeta = (be - al) / (2.0 * ga);
    const double az = fabs(zeta);
    const double t = (az > 1e150) ? 0.5 / zeta : copysign(1.0, zeta) / (az + sqrt(1.0 + zeta * zeta));
    c = 1.0 / sqrt(1.0 + t * t);
    s = c * t;
    return true;
}

// One pair, columns of up to 32 * SVD_REG elements: every lane loads its
// elements of both columns in one unrolled batch (one memory latency instead of
// one per element), and the same for V when the pair rotates.
__device__ inline bool pair_rotate_regs(double* gp, double* gq, uint32_t m, double* vp, double* vq, uint32_t n,
                                        double tol) {
    const uint32_t lane = threadIdx.x & 31u;
    double x[SVD_REG], y[SVD_REG];
#pragma unroll
    for (int r = 0; r < SVD_REG; ++r) {
        const uint32_t i = lane + 32u * r;
        x[r] = i < m ? gp[i] : 0.0;
        y[r] = i < m ? gq[i] : 0.0;
    }
    double al = 0.0, be = 0.0, ga = 0.0;
#pragma unroll
    for (int r = 0; r < SVD_REG; ++r) {
        al = fma(x[r], x[r], al);
        be = fma(y[r], y[r], be);
        ga = fma(x[r], y[r], ga);
    }
    al = warp_sum(al);
    be = warp_sum(be);
    ga = warp_sum(ga);
    double c, s;
    if (!jacobi_cs(al, be, ga, tol, c, s)) return false;
#pragma unroll
    for (int r = 0; r < SVD_REG; ++r) {
        const uint32_t i = lane + 32u * r;
        if (i < m) {
            gp[i] = c * x[r] - s * y[r];
            gq[i] = s * x[r] + c * y[r];
        }
    }
#pragma unroll
    for (int r = 0; r < SVD_REG; ++r) {
        const uint32_t i = lane + 32u * r;
        x[r] = i < n ? vp[i] : 0.0;
        y[r] = i < n ? vq[i] : 0.0;
    }
#pragma unroll
    for (int r = 0; r < SVD_REG; ++r) {
        const uint32_t i = lane + 32u * r;
        if (i < n) {
            vp[i] = c * x[r] - s * y[r];
            vq[i] = s * x[r] + c * y[r];
        }
    }
    return true;
}

// The same for longer columns, element by element.
__device__ inline bool pair_rotate_loop(double* gp, double* gq, uint32_t m, double* vp, double* vq, uint32_t n,
                                        double tol) {
    const uint32_t lane = threadIdx.x & 31u;
    double al = 0.0, be = 0.0, ga = 0.0;
    for (uint32_t i = lane; i < m; i += 32) {
        const double x = gp[i], y = gq[i];
        al = fma(x, x, al);
        be = fma(y, y, be);
        ga = fma(x, y, ga);
    }
    al = warp_sum(al);
    be = warp_sum(be);
    ga = warp_sum(ga);
    double c, s;
    if (!jacobi_cs(al, be, ga, tol, c, s)) return false;
    for (uint32_t i = lane; i < m; i += 32) {
        const double x = gp[i], y = gq[i];
        gp[i] = c * x - s * y;
        gq[i] = s * x + c * y;
    }
    for (uint32_t i = lane; i < n; i += 32) {
        const double x = vp[i], y = vq[i];
        vp[i] = c * x - s * y;
        vq[i] = s * x + c * y;
    }
    return true;
}

__global__ void __launch_bounds__(SVD_THREADS) block_svd_jacobi(const SvdBlock* blocks, int* err) {
    extern __shared__ double smem[];
    const SvdBlock b = blocks[blockIdx.x];
    const bool tr = b.rows < b.cols;
    const uint32_t m = tr ? b.cols : b.rows, n = tr ? b.rows : b.cols;
    if (n == 0) return;
    double* G = b.work ? b.work : smem;
    double* V = G + size_t(m) * n;
    double* sig = V + size_t(n) * n;
    int* rank_col = reinterpret_cast<int*>(sig + n);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    __shared__ double red[SVD_WARPS];
    double amax = 0.0;
    for (size_t e = threadIdx.x; e < size_t(m) * n; e += blockDim.x) {
        const uint32_t j = uint32_t(e / m), i = uint32_t(e % m);
        const double v = tr ? b.a[j + size_t(i) * b.rows] : b.a[i + size_t(j) * b.rows];
        G[e] = v;
        amax = fmax(amax, fabs(v));
    }
    for (size_t e = threadIdx.x; e < size_t(n) * n; e += blockDim.x) V[e] = (e / n == e % n) ? 1.0 : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if (lane == 0) red[warp] = amax;
    __syncthreads();
    for (int w = 0; w < SVD_WARPS; ++w) amax = fmax(amax, red[w]);
    // exact power-of-two scaling to a largest element in [1, 2): the squared
    // norms neither underflow nor overflow; sigma is scaled back at the end
    const int ex = amax > 0.0 ? ilogb(amax) : 0;
    if (ex != 0) {
        for (size_t e = threadIdx.x; e < size_t(m) * n; e += blockDim.x) G[e] = ldexp(G[e], -ex);
    }
    __syncthreads();

    const double tol = sqrt(double(m)) * 2.220446049250313e-16;
    const uint32_t n2 = n + (n & 1u);  // even player count; index n is the bye when n is odd
    bool converged = n < 2;
    for (int sweep = 0; sweep < SVD_MAX_SWEEPS && !converged; ++sweep) {
        int rotated = 0;
        for (uint32_t r = 0; r + 1 < n2; ++r) {
            // circle method: player n2-1 meets r, player (r+k) meets (r-k) (mod n2-1)
            for (uint32_t k = warp; k < n2 / 2; k += SVD_WARPS) {
                uint32_t p, q;
                if (k == 0) {
                    p = n2 - 1;
                    q = r;
                } else {
                    p = (r + k) % (n2 - 1);
                    q = (r + (n2 - 1) - k) % (n2 - 1);
                }
                if (p >= n || q >= n) continue;
                if (p > q) {
                    const uint32_t t = p;
                    p = q;
                    q = t;
                }
                double* gp = G + size_t(p) * m;
                double* gq = G + size_t(q) * m;
                double* vp = V + size_t(p) * n;
                double* vq = V + size_t(q) * n;
                const bool rot = (m <= 32u * SVD_REG) ? pair_rotate_regs(gp, gq, m, vp, vq, n, tol)
                                                     : pair_rotate_loop(gp, gq, m, vp, vq, n, tol);
                if (rot) rotated = 1;
            }
            __syncthreads();
        }
        converged = __syncthreads_or(rotated) == 0;
    }
    if (!converged && threadIdx.x == 0) atomicOr(err, 1);

    for (uint32_t j = warp; j < n; j += SVD_WARPS) {
        const double* g = G + size_t(j) * m;
        double ss = 0.0;
        for (uint32_t i = lane; i < m; i += 32) ss = fma(g[i], g[i], ss);
        ss = warp_sum(ss);
        if (lane == 0) sig[j] = sqrt(ss);
    }
    __syncthreads();
    // descending order, ties by column index
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
        const double sj = sig[j];
        uint32_t rk = 0;
        for (uint32_t i = 0; i < n; ++i) rk += (sig[i] > sj || (sig[i] == sj && i < j)) ? 1u : 0u;
        rank_col[rk] = int(j);
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < n; r += blockDim.x) b.s[r] = ldexp(sig[rank_col[r]], ex);
    // U (rows x n) and V^T (n x cols)
    for (size_t e = threadIdx.x; e < size_t(b.rows) * n; e += blockDim.x) {
        const uint32_t r = uint32_t(e / b.rows), i = uint32_t(e % b.rows);
        const uint32_t j = uint32_t(rank_col[r]);
        double v;
        if (tr) {
            v = V[size_t(j) * n + i];
        } else {
            const double sj = sig[j];
            v = sj > 0.0 ? G[size_t(j) * m + i] / sj : 0.0;
        }
        b.u[e] = v;
    }
    for (size_t e = threadIdx.x; e < size_t(n) * b.cols; e += blockDim.x) {
        const uint32_t c = uint32_t(e / n), r = uint32_t(e % n);
        const uint32_t j = uint32_t(rank_col[r]);
        double v;
        if (tr) {
            const double sj = sig[j];
            v = sj > 0.0 ? G[size_t(j) * m + c] / sj : 0.0;
        } else {
            v = V[size_t(j) * n + c];
        }
        b.vt[e] = v;
    }
}

__global__ void copy_blocks(const dmrgb200_block_copy* cp, uint32_t n, const double* src, double* dst,
                            const double* scale) {
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const dmrgb200_block_copy c = cp[k];
        const size_t total = size_t(c.rows) * c.cols;
        for (size_t e = threadIdx.x; e < total; e += blockDim.x) {
            const uint32_t j = uint32_t(e / c.rows), i = uint32_t(e % c.rows);
            double v = src[c.src_off + i + size_t(j) * c.src_ld];
            if (c.scale_mode == DMRGB200_SCALE_ROWS) v *= scale[c.scale_off + i];
            else if (c.scale_mode == DMRGB200_SCALE_COLS) v *= scale[c.scale_off + j];
            dst[c.dst_off + i + size_t(j) * c.dst_ld] = v;
        }
    }
}

}  // namespace
}  // namespace dmrgb200

using namespace dmrgb200;

extern "C" dmrgb200_status dmrgb200_block_svd(uint32_t n_blocks, const uint32_t* rows, const uint32_t* cols,
                                              const double* const* a, double* const* u, double* const* s,
                                              double* const* vt, void* cuda_stream) {
    if (n_blocks && (!rows || !cols || !a || !u || !s || !vt))
        return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "block SVD: null argument");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    std::vector<SvdBlock> bl;
    std::vector<size_t> work_off;  // per block: offset in the global scratch, or SIZE_MAX for shared memory
    size_t work = 0, smem = 0;
    for (uint32_t i = 0; i < n_blocks; ++i) {
        if (!rows[i] || !cols[i]) continue;
        if (!a[i] || !u[i] || !s[i] || !vt[i]) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "block SVD: null block");
        bl.push_back(SvdBlock{a[i], u[i], s[i], vt[i], nullptr, rows[i], cols[i]});
        const size_t w = svd_work_elems(rows[i], cols[i]);
        if (w * sizeof(double) <= SVD_SMEM_LIMIT) {
            smem = std::max(smem, w * sizeof(double));
            work_off.push_back(SIZE_MAX);
        } else {
            work_off.push_back(work);
            work += w;
        }
    }
    if (bl.empty()) return DMRGB200_OK;
    const size_t tab = (bl.size() * sizeof(SvdBlock) + 255) / 256 * 256;
    unsigned char* mem = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&mem), tab + 256 + work * sizeof(double), st);
    if (e != cudaSuccess) return noalloc_fail(DMRGB200_OUT_OF_MEMORY, std::string("block SVD: ") + cudaGetErrorString(e));
    int* d_err = reinterpret_cast<int*>(mem + tab);
    double* scratch = reinterpret_cast<double*>(mem + tab + 256);
    for (size_t i = 0; i < bl.size(); ++i)
        if (work_off[i] != SIZE_MAX) bl[i].work = scratch + work_off[i];
    e = ensure_smem_limit(reinterpret_cast<const void*>(block_svd_jacobi), int(SVD_SMEM_LIMIT));
    if (e != cudaSuccess) {
        cudaFreeAsync(mem, st);
        return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("block SVD shared memory: ") + cudaGetErrorString(e));
    }
    cudaMemcpyAsync(mem, bl.data(), bl.size() * sizeof(SvdBlock), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_err, 0, sizeof(int), st);
    block_svd_jacobi<<<uint32_t(bl.size()), SVD_THREADS, smem, st>>>(reinterpret_cast<const SvdBlock*>(mem), d_err);
    e = cudaGetLastError();
    int h_err = 0;
    cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    cudaFreeAsync(mem, st);
    if (e != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("block SVD launch: ") + cudaGetErrorString(e));
    if (e2 != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("block SVD: ") + cudaGetErrorString(e2));
    if (h_err) return noalloc_fail(DMRGB200_NUMERIC, "block SVD: Jacobi sweeps did not converge");
    return DMRGB200_OK;
}

extern "C" dmrgb200_status dmrgb200_copy_blocks(uint32_t n, const dmrgb200_block_copy* copies, const double* src,
                                                double* dst, const double* scale, void* cuda_stream) {
    if (!n) return DMRGB200_OK;
    if (!copies || !src || !dst) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "block copy: null argument");
    for (uint32_t k = 0; k < n; ++k) {
        dmrgb200_block_copy const& c = copies[k];
        if (c.scale_mode > DMRGB200_SCALE_COLS) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "block copy: scale mode");
        if (c.scale_mode != DMRGB200_SCALE_NONE && !scale)
            return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "block copy: scaling without factors");
        if (c.cols > 1 && (c.src_ld < c.rows || c.dst_ld < c.rows))
            return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "block copy: leading dimension below the row count");
    }
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    void* d = nullptr;
    cudaError_t e = cudaMallocAsync(&d, size_t(n) * sizeof(dmrgb200_block_copy), st);
    if (e != cudaSuccess) return noalloc_fail(DMRGB200_OUT_OF_MEMORY, std::string("block copy: ") + cudaGetErrorString(e));
    // upload from a pageable copy: a pageable source is staged before cudaMemcpyAsync
    // returns, so the caller's array (pinned or not) may be released on return
    std::vector<dmrgb200_block_copy> staged(copies, copies + n);
    cudaMemcpyAsync(d, staged.data(), size_t(n) * sizeof(dmrgb200_block_copy), cudaMemcpyHostToDevice, st);
    copy_blocks<<<std::min<uint32_t>(n, 148u * 8u), 256, 0, st>>>(static_cast<const dmrgb200_block_copy*>(d), n, src,
                                                                   dst, scale);
    e = cudaGetLastError();
    cudaFreeAsync(d, st);
    if (e != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("block copy: ") + cudaGetErrorString(e));
    return DMRGB200_OK;
}
