// FP64 matrix products emulated on the INT8 tensor cores (tcgen05, sm_100a).
//
// Split-precision scheme (Ozaki, Ogita, Oishi, Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication", Numer. Algorithms 59 (2012); integer variant of Ootomo,
// Ozaki, Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 2024):
//   * every row i of A is scaled by 2^-e_i so that |A_ij 2^-e_i| < 1 and cut into
//     s signed 7-bit digits a_p (p = 0..s-1): A_ij 2^-e_i = sum_p a_p 2^-7(p+1) + r,
//     |r| < 2^-7s; every column j of B likewise with 2^-f_j;
//   * products of digit matrices are exact in INT32 (|a b| <= 127^2, K <= 2^17/s);
//     digit pairs with p + q = g share one accumulator D_g, pairs with p + q >= s
//     are dropped (their weight is below the truncation error);
//   * C_ij = 2^(e_i + f_j) sum_g 2^-7(g+2) D_g[i][j], combined in FP64 from the
//     smallest group up.
// The MMA kernel keeps s INT32 accumulators of a 128 x 64 output tile in TMEM
// (tcgen05.alloc), stages the digit tiles of a 64-byte K slab with bulk copies
// completing on an mbarrier, issues tcgen05.mma.kind::i8 from one thread and
// reads the accumulators back with tcgen05.ld for the FP64 epilogue.  Every
// wait is bounded in time; on timeout the kernel records an error, releases
// its TMEM and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "../../include/dmrgb200.h"
#include "device.hpp"

namespace dmrgb200 {

dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);

namespace {

constexpr int OZ_BM = 128, OZ_BN = 64, OZ_BK = 64;        // tile rows, tile columns, K bytes per slab
constexpr int A_TILE = OZ_BM * OZ_BK, B_TILE = OZ_BN * OZ_BK;
constexpr int OZ_THREADS = 128, OZ_STAGES = 2, OZ_MAX_SLICES = 8;
constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// byte offset of element (r, k) of a (rows x 64-byte) K-major tile in the
// canonical no-swizzle layout: 8x16-byte core matrices, LBO = 128 B along K,
// SBO = 512 B between 8-row groups
__device__ __forceinline__ uint32_t tile_off(uint32_t r, uint32_t k) {
    return (r >> 3) * 512u + (k >> 4) * 128u + (r & 7u) * 16u + (k & 15u);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFFu);
    d |= uint64_t((128u >> 4) & 0x3FFFu) << 16;  // leading (K) byte offset
    d |= uint64_t((512u >> 4) & 0x3FFFu) << 32;  // stride (row-group) byte offset
    d |= uint64_t(1) << 46;                       // descriptor version (sm_100)
    return d;                                      // base offset 0, no swizzle
}

__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4)                       // D: S32
           | (1u << 7) | (1u << 10)        // A, B: signed 8-bit
           | (uint32_t(N >> 3) << 17)      // N / 8
           | (uint32_t(M >> 4) << 24);     // M / 16   (both operands K-major, no negation)
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; false (and *err set) when the phase does not complete in time
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
    unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity)) {
        if (*reinterpret_cast<volatile int*>(err)) return false;
        if (global_ns() - t0 > WAIT_LIMIT_NS) {
            atomicExch(err, 1);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void bulk_load(void* smem, const void* gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem)),
                 "l"(gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---- digit extraction --------------------------------------------------------------

// per-row (A) or per-column (B) power-of-two exponent: |x 2^-e| < 1 for the whole row
__global__ void row_exponents(const double* __restrict__ X, uint64_t ld, uint32_t rows, uint32_t cols,
                              int along_rows, int* __restrict__ e) {
    // along_rows = 1: row r spans X[r + c*ld] (A rows); 0: column r spans X[c + r*ld] (B columns)
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= rows) return;
    double m = 0.0;
    for (uint32_t c = lane; c < cols; c += 32) {
        double v = along_rows ? X[warp + c * ld] : X[c + uint64_t(warp) * ld];
        m = fmax(m, fabs(v));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) e[warp] = (m > 0.0) ? ilogb(m) + 1 : 0;
}

// digits of A (rows x K, element (r, k) at X[r + k*ld] when along_rows, else
// X[k + r*ld] for B^T) into s tiled digit planes of shape (RT*128 or NT*64) x (KT*64)
template <int TR>
__global__ void split_digits(const double* __restrict__ X, uint64_t ld, uint32_t rows, uint32_t K, int along_rows,
                             const int* __restrict__ e, int s, int8_t* __restrict__ out, uint32_t row_tiles,
                             uint32_t k_tiles) {
    const uint64_t plane = uint64_t(row_tiles) * k_tiles * TR * OZ_BK;
    const uint64_t total = uint64_t(row_tiles) * TR * k_tiles * OZ_BK;
    for (uint64_t idx = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; idx < total;
         idx += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t r, k;
        if (along_rows) {  // consecutive threads walk rows (contiguous in A)
            r = uint32_t(idx % (uint64_t(row_tiles) * TR));
            k = uint32_t(idx / (uint64_t(row_tiles) * TR));
        } else {           // consecutive threads walk K (contiguous in B)
            k = uint32_t(idx % (uint64_t(k_tiles) * OZ_BK));
            r = uint32_t(idx / (uint64_t(k_tiles) * OZ_BK));
        }
        double x = 0.0;
        if (r < rows && k < K) x = along_rows ? X[r + uint64_t(k) * ld] : X[k + uint64_t(r) * ld];
        if (r < rows) x = ldexp(x, -e[r]);
        uint64_t tile = uint64_t(r / TR) * k_tiles + (k / OZ_BK);
        uint64_t off = tile * (TR * OZ_BK) + tile_off(r % TR, k % OZ_BK);
        for (int p = 0; p < s; ++p) {
            double t = x * 128.0;       // exact
            double d = trunc(t);        // |d| <= 127
            x = t - d;                  // exact
            out[p * plane + off] = static_cast<int8_t>(d);
        }
    }
}

// ---- MMA kernel ------------------------------------------------------------------------

struct OzArgs {
    const int8_t* A8;  // s planes of MT x KT tiles (8 KB each)
    const int8_t* B8;  // s planes of NT x KT tiles (4 KB each)
    const int* e;      // row exponents of A (M)
    const int* f;      // column exponents of B (N)
    double* C;
    uint64_t ldc;
    uint32_t M, N, MT, NT, KT;
    int s;
    int beta;          // 0: C = A B, 1: C += A B
    int* err;
};

__global__ void __launch_bounds__(OZ_THREADS, 1) ozaki_mma(OzArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int s = a.s;
    const uint32_t stage_bytes = uint32_t(s) * (A_TILE + B_TILE);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + OZ_STAGES * stage_bytes);
    uint64_t* empty = full + OZ_STAGES;
    uint64_t* done = empty + OZ_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ncols = (s * OZ_BN <= 256) ? ((s * OZ_BN <= 128) ? 128u : 256u) : 512u;
    const uint64_t a_plane = uint64_t(a.MT) * a.KT * A_TILE, b_plane = uint64_t(a.NT) * a.KT * B_TILE;
    const uint32_t idesc = idesc_i8(OZ_BM, OZ_BN);
    volatile int* verr = a.err;

    if (threadIdx.x == 0) {
        for (int i = 0; i < OZ_STAGES; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // running slab / tile counters: every arrival on every barrier is waited for exactly once, in order
    uint32_t slab0 = 0, tiles = 0, issued = 0, consumed = 0;
    bool failed = false;
    for (uint32_t tile = blockIdx.x; tile < a.MT * a.NT && !failed; tile += gridDim.x) {
        const uint32_t mt = tile % a.MT, nt = tile / a.MT;
        if (threadIdx.x == 0) {
            auto load = [&](uint32_t kt) -> bool {
                const uint32_t gs = slab0 + kt, st = gs % OZ_STAGES;
                if (gs >= OZ_STAGES && !mbar_wait(&empty[st], ((gs - OZ_STAGES) / OZ_STAGES) & 1u, a.err)) return false;
                unsigned char* base = smem + st * stage_bytes;
                mbar_expect_tx(&full[st], stage_bytes);
                for (int p = 0; p < s; ++p) {
                    bulk_load(base + p * A_TILE, a.A8 + p * a_plane + (uint64_t(mt) * a.KT + kt) * A_TILE, A_TILE,
                              &full[st]);
                    bulk_load(base + s * A_TILE + p * B_TILE,
                              a.B8 + p * b_plane + (uint64_t(nt) * a.KT + kt) * B_TILE, B_TILE, &full[st]);
                }
                ++issued;
                return true;
            };
            bool ok = true;
            for (uint32_t kt = 0; kt < a.KT && kt < OZ_STAGES && ok; ++kt) ok = load(kt);
            for (uint32_t kt = 0; kt < a.KT && ok; ++kt) {
                const uint32_t gs = slab0 + kt, st = gs % OZ_STAGES;
                ok = mbar_wait(&full[st], (gs / OZ_STAGES) & 1u, a.err);
                if (!ok) break;
                ++consumed;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t abase = smem_u32(smem + st * stage_bytes);
                const uint32_t bbase = abase + s * A_TILE;
                for (int ks = 0; ks < OZ_BK / 32; ++ks)
                    for (int g = 0; g < s; ++g)
                        for (int p = 0; p <= g; ++p) {
                            const uint64_t da = umma_desc(abase + p * A_TILE + ks * 256);
                            const uint64_t db = umma_desc(bbase + (g - p) * B_TILE + ks * 256);
                            const uint32_t accum = (kt > 0 || ks > 0 || p > 0) ? 1u : 0u;
                            umma_i8(tmem + uint32_t(g * OZ_BN), da, db, idesc, accum);
                        }
                umma_commit(&empty[st]);
                if (kt + OZ_STAGES < a.KT) ok = load(kt + OZ_STAGES);
            }
            if (!ok) atomicExch(a.err, 1);
            umma_commit(done);  // arrives once every MMA issued so far has completed
        }
        slab0 += a.KT;
        __syncwarp();
        const bool ready = mbar_wait(done, tiles & 1u, a.err);
        ++tiles;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const bool go = __all_sync(0xffffffffu, ready && *verr == 0);
        if (go) {
            const uint32_t row = mt * OZ_BM + warp * 32 + lane;
            const double escale = (row < a.M) ? ldexp(1.0, a.e[row]) : 0.0;
            for (int c0 = 0; c0 < OZ_BN; c0 += 16) {
                double acc[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[j] = 0.0;
                for (int g = s - 1; g >= 0; --g) {
                    int32_t v[16];
                    tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(g * OZ_BN + c0), v);
                    const double w = ldexp(1.0, -7 * (g + 2));
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[j] += double(v[j]) * w;
                }
                if (row < a.M) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const uint32_t col = nt * OZ_BN + c0 + j;
                        if (col < a.N) {
                            double val = acc[j] * escale * ldexp(1.0, a.f[col]);
                            double* dst = a.C + row + uint64_t(col) * a.ldc;
                            *dst = a.beta ? *dst + val : val;
                        }
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        failed = (*verr != 0);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // after a timeout: let the bulk copies still in flight land before the CTA leaves (bounded);
        // slabs are issued and consumed in global order, so `consumed` is the next slab's index
        for (; consumed < issued; ++consumed) {
            unsigned long long t0 = global_ns();
            while (!mbar_try(&full[consumed % OZ_STAGES], (consumed / OZ_STAGES) & 1u) &&
                   global_ns() - t0 < WAIT_LIMIT_NS) {
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

}  // namespace

size_t ozaki_smem_bytes(int s) { return size_t(OZ_STAGES) * s * (A_TILE + B_TILE) + 8 * (2 * OZ_STAGES + 1) + 16; }

// C (M x N, ldc) = A (M x K, lda) * B (K x N, ldb), all column-major FP64, on the stream.
// Scratch digit planes are allocated stream-ordered.
cudaError_t ozaki_dgemm(uint32_t M, uint32_t N, uint32_t K, const double* A, uint64_t lda, const double* B,
                        uint64_t ldb, double* C, uint64_t ldc, int s, int beta, cudaStream_t st, int* err_flag) {
    const uint32_t MT = (M + OZ_BM - 1) / OZ_BM, NT = (N + OZ_BN - 1) / OZ_BN, KT = (K + OZ_BK - 1) / OZ_BK;
    if (!M || !N) return cudaSuccess;
    const uint64_t a_bytes = uint64_t(s) * MT * KT * A_TILE, b_bytes = uint64_t(s) * NT * KT * B_TILE;
    int8_t *A8 = nullptr, *B8 = nullptr;
    int *e = nullptr, *f = nullptr;
    cudaError_t r;
    if ((r = cudaMallocAsync(&A8, a_bytes, st)) != cudaSuccess) return r;
    if ((r = cudaMallocAsync(&B8, b_bytes, st)) != cudaSuccess) return r;
    if ((r = cudaMallocAsync(&e, sizeof(int) * MT * OZ_BM, st)) != cudaSuccess) return r;
    if ((r = cudaMallocAsync(&f, sizeof(int) * NT * OZ_BN, st)) != cudaSuccess) return r;
    cudaMemsetAsync(e, 0, sizeof(int) * MT * OZ_BM, st);
    cudaMemsetAsync(f, 0, sizeof(int) * NT * OZ_BN, st);
    const int sms = device_sm_count();
    row_exponents<<<(M * 32 + 255) / 256, 256, 0, st>>>(A, lda, M, K, 1, e);
    row_exponents<<<(N * 32 + 255) / 256, 256, 0, st>>>(B, ldb, N, K, 0, f);
    split_digits<OZ_BM><<<sms * 8, 256, 0, st>>>(A, lda, M, K, 1, e, s, A8, MT, KT);
    split_digits<OZ_BN><<<sms * 8, 256, 0, st>>>(B, ldb, N, K, 0, f, s, B8, NT, KT);
    OzArgs args{A8, B8, e, f, C, ldc, M, N, MT, NT, KT, s, beta, err_flag};
    const size_t smem = ozaki_smem_bytes(s);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(ozaki_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ozaki_smem_bytes(OZ_MAX_SLICES)));
        attr = true;
    }
    ozaki_mma<<<std::min<uint32_t>(MT * NT, uint32_t(sms)), OZ_THREADS, smem, st>>>(args);
    r = cudaGetLastError();
    cudaFreeAsync(A8, st);
    cudaFreeAsync(B8, st);
    cudaFreeAsync(e, st);
    cudaFreeAsync(f, st);
    return r;
}

}  // namespace dmrgb200

using namespace dmrgb200;

extern "C" dmrgb200_status dmrgb200_dgemm_emulated(uint32_t M, uint32_t N, uint32_t K, const double* A, uint64_t lda,
                                                   const double* B, uint64_t ldb, double* C, uint64_t ldc,
                                                   int slices, void* cuda_stream) {
    if (!A || !B || !C) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (slices < 2 || slices > OZ_MAX_SLICES) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "slices must be 2..8");
    if (uint64_t(K) * uint64_t(slices) > (1ull << 17))
        return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "K * slices exceeds the exact INT32 accumulation range");
    if (lda < M || ldb < K || ldc < M) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "leading dimension too small");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    int* err = nullptr;
    cudaError_t r = cudaMallocAsync(&err, sizeof(int), st);
    if (r != cudaSuccess) return noalloc_fail(DMRGB200_OUT_OF_MEMORY, cudaGetErrorString(r));
    cudaMemsetAsync(err, 0, sizeof(int), st);
    r = ozaki_dgemm(M, N, K, A, lda, B, ldb, C, ldc, slices, 0, st, err);
    int h_err = 0;
    cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t r2 = cudaStreamSynchronize(st);
    cudaFree(err);
    if (r != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("emulated GEMM: ") + cudaGetErrorString(r));
    if (r2 != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("emulated GEMM: ") + cudaGetErrorString(r2));
    if (h_err) return noalloc_fail(DMRGB200_TIMEOUT, "emulated GEMM: a pipeline wait timed out");
    return DMRGB200_OK;
}
