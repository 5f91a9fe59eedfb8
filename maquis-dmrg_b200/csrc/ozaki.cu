// FP64 matrix products emulated on the INT8 tensor cores (tcgen05, sm_100a).
//
// Split-precision scheme (Ozaki, Ogita, Oishi, Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication", Numer. Algorithms 59 (2012); integer variant of Ootomo,
// Ozaki, Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 2024):
//   * every row i of A is scaled by 2^-e_i so that |A_ij 2^-e_i| < 1 and cut into
//     s signed 7-bit digits a_p (p = 0..s-1): A_ij 2^-e_i = sum_p a_p 2^-7(p+1) + r,
//     |r| < 2^-7s; every column j of B likewise with 2^-f_j;
//   * products of digit matrices are exact in INT32 (|a b| <= 127^2) over up to
//     2^17/s K elements; longer contractions accumulate in chunks of that length,
//     each chunk's partial product added into C in FP64; digit pairs with p + q = g share one accumulator D_g, pairs with p + q >= s
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
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"
#include "async_copy.cuh"

namespace dmrgb200 {

dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);

namespace {

constexpr int OZ_BM = 128, OZ_BN = 64, OZ_BK = 64;        // tile rows, tile columns, K bytes per slab
constexpr int A_TILE = OZ_BM * OZ_BK, B_TILE = OZ_BN * OZ_BK;
constexpr int OZ_THREADS = 128, OZ_STAGES = 2, OZ_MAX_SLICES = 8;
using namespace async;

// K slabs per exact INT32 accumulation: accumulator D_g sums (g + 1) <= s digit
// products of |a b| <= 127^2 per K element, and 127^2 * 2^17 < 2^31
constexpr uint32_t oz_chunk_slabs(int s) { return std::max<uint32_t>(1u, (1u << 17) / uint32_t(s * OZ_BK)); }

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

// One operand of one segment to be cut into digit planes.  For an A operand the
// digit matrix is A itself (row r, column k); for a B operand it is B^T (row n,
// column k), both stored K-major in 8 KB (A, 128 rows) or 4 KB (B, 64 rows)
// tiles: tile (rt, ks) at out_base + (rt * KS + ks) * tile_bytes.
struct OzSplit {
    DevOp op;           // batch already folded into op.off
    uint32_t rows, K;   // logical rows (M or N) and K of the segment
    uint32_t RT, KS;    // row tiles, K slabs
    uint64_t out_base;  // byte offset inside a digit plane
    uint64_t e_off;     // exponent array offset of row 0
    uint32_t is_b;      // 0: A operand, 1: B operand (read transposed)
    uint32_t is_const;  // the operand and its exponents are constant between calls
    uint32_t rowtab;    // A of a row-table problem: row r at rowtab[rowtab + r]; DevProb::NO_ROWS otherwise
    uint32_t pad;
};

__device__ __forceinline__ double op_elem(Bases const& bs, OzSplit const& j, uint32_t r, uint32_t k,
                                          const DevRow* __restrict__ rowtab) {
    if (!j.is_b && j.rowtab != DevProb::NO_ROWS) {
        const DevRow rw = rowtab[j.rowtab + r];
        return reinterpret_cast<const double*>(base_of(bs, j.op.buf))[rw.a_off + uint64_t(k) * rw.ld];
    }
    const double* base = reinterpret_cast<const double*>(base_of(bs, j.op.buf) + 8ull * j.op.off);
    const uint64_t ld = j.op.ld;
    if (!j.is_b) return j.op.trans ? base[k + uint64_t(r) * ld] : base[r + uint64_t(k) * ld];
    // B(k, r): non-transposed B[k + r * ld], transposed B[r + k * ld]
    return j.op.trans ? base[r + uint64_t(k) * ld] : base[k + uint64_t(r) * ld];
}

__global__ void fill_int(int* __restrict__ p, uint64_t n, int v) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        p[i] = v;
}

// exponent of every row of every job (max over segments by atomicMax):
// |x 2^-e| < 1 for the whole row of the output matrix.  blockIdx.y walks the
// jobs, blockIdx.x and the warps the rows, the lanes K.
__global__ void __launch_bounds__(256) oz_exponents(const OzSplit* __restrict__ jobs, uint32_t njobs, Bases bs,
                                                    int* __restrict__ e, const DevRow* __restrict__ rowtab) {
    const uint32_t lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (uint32_t j = blockIdx.y; j < njobs; j += gridDim.y) {
        const OzSplit job = jobs[j];
        for (uint32_t r = blockIdx.x * warps + (threadIdx.x >> 5); r < job.rows; r += gridDim.x * warps) {
            double m = 0.0;
            for (uint32_t k = lane; k < job.K; k += 32) m = fmax(m, fabs(op_elem(bs, job, r, k, rowtab)));
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0 && m > 0.0) atomicMax(&e[job.e_off + r], ilogb(m) + 1);
        }
    }
}

// Digit planes: every thread cuts four consecutive K elements of one row and
// stores each plane's four digits as one 32-bit word (K-contiguous bytes of the
// tile layout).  Rows outside the operand and K beyond it give zero digits.
__global__ void __launch_bounds__(256) oz_split(const OzSplit* __restrict__ jobs, uint32_t njobs, Bases bs,
                                                const int* __restrict__ e, int s, uint64_t a_plane,
                                                int8_t* __restrict__ A8, uint64_t b_plane, int8_t* __restrict__ B8,
                                                const DevRow* __restrict__ rowtab) {
    for (uint32_t j = blockIdx.y; j < njobs; j += gridDim.y) {
        const OzSplit job = jobs[j];
        int8_t* out = job.is_b ? B8 : A8;
        const uint64_t plane = job.is_b ? b_plane : a_plane;
        const uint32_t TR = job.is_b ? uint32_t(OZ_BN) : uint32_t(OZ_BM);
        const uint32_t tile_bytes = TR * OZ_BK;
        const uint32_t nrows = job.RT * TR, ngroups = job.KS * (OZ_BK / 4);
        const uint32_t total = nrows * ngroups;
        // column-major A: rows are contiguous (row-table rows are separate slices: K-major order)
        const bool rows_fast = !job.is_b && !job.op.trans && job.rowtab == DevProb::NO_ROWS;
        for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
            const uint32_t r = rows_fast ? idx % nrows : idx / ngroups;
            const uint32_t k0 = 4 * (rows_fast ? idx / nrows : idx % ngroups);
            double x[4];
            const int ex = r < job.rows ? e[job.e_off + r] : 0;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                x[u] = (r < job.rows && k0 + u < job.K) ? ldexp(op_elem(bs, job, r, k0 + u, rowtab), -ex) : 0.0;
            const uint64_t off = job.out_base + (uint64_t(r / TR) * job.KS + k0 / OZ_BK) * tile_bytes +
                                 tile_off(r % TR, k0 % OZ_BK);
            for (int p = 0; p < s; ++p) {
                uint32_t word = 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const double t = x[u] * 128.0;  // exact
                    const double d = trunc(t);      // |d| <= 127
                    x[u] = t - d;                   // exact
                    word |= (uint32_t(uint8_t(int8_t(d)))) << (8 * u);
                }
                *reinterpret_cast<uint32_t*>(out + p * plane + off) = word;
            }
        }
    }
}

// ---- MMA kernel ------------------------------------------------------------------------

struct OzPB {  // one output matrix (a GEMM problem of one batch index)
    uint32_t M, N, MT, NT;
    uint32_t slab_begin, slab_end;  // K slabs (over all segments) in OzSlab
    uint64_t e_off, f_off;          // exponents of its rows / columns
    DevOp C;                        // destination (batch folded into C.off)
    uint32_t beta, pad;
    uint32_t rowtab, batch;         // row-table problems: C row r at rowtab[rowtab + r] (batch `batch`)
};
struct OzSlab {  // K slab: A tile of row tile mt at a_off + mt * a_ts, B tile of nt at b_off + nt * b_ts
    uint64_t a_off, b_off;
    uint32_t a_ts, b_ts;
};
struct OzTile {
    uint32_t pb, mt, nt, pad;
};

struct OzArgs {
    const int8_t* A8;
    const int8_t* B8;
    uint64_t a_plane, b_plane;  // bytes per digit plane
    const int* e;
    const OzPB* pbs;
    const OzSlab* slabs;
    const OzTile* tiles;
    uint32_t n_tiles;
    uint32_t chunk;  // K slabs accumulated in TMEM before a partial epilogue (>= 1)
    int s;
    Bases bases;
    int* err;
    const DevRow* rowtab;
    unsigned long long wait_ns;  // limit of the waits for operand slabs
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

    // running slab / round counters: every arrival on every barrier is waited for exactly once, in order.
    // A tile's slabs are accumulated in chunks of a.chunk slabs (the exact INT32 range); each chunk
    // ends with one epilogue round that adds its partial product into C.
    uint32_t slab0 = 0, rounds = 0, issued = 0, consumed = 0;
    bool failed = false;
    for (uint32_t tile = blockIdx.x; tile < a.n_tiles && !failed; tile += gridDim.x) {
        const OzTile tl = a.tiles[tile];
        const OzPB pb = a.pbs[tl.pb];
        const uint32_t mt = tl.mt, nt = tl.nt;
        const uint32_t KT = pb.slab_end - pb.slab_begin;
        const uint32_t nch = KT ? (KT + a.chunk - 1) / a.chunk : 1;
        bool ok = true;  // thread 0's pipeline state over the tile's chunks
        auto load = [&](uint32_t kt) -> bool {
            const uint32_t gs = slab0 + kt, st = gs % OZ_STAGES;
            if (gs >= OZ_STAGES && !mbar_wait(&empty[st], ((gs - OZ_STAGES) / OZ_STAGES) & 1u, a.err, a.wait_ns))
                return false;
            const OzSlab sl = a.slabs[pb.slab_begin + kt];
            unsigned char* base = smem + st * stage_bytes;
            mbar_expect_tx(&full[st], stage_bytes);
            for (int p = 0; p < s; ++p) {
                bulk_load(base + p * A_TILE, a.A8 + p * a.a_plane + sl.a_off + uint64_t(mt) * sl.a_ts, A_TILE,
                          &full[st]);
                bulk_load(base + s * A_TILE + p * B_TILE, a.B8 + p * a.b_plane + sl.b_off + uint64_t(nt) * sl.b_ts,
                          B_TILE, &full[st]);
            }
            ++issued;
            return true;
        };
        for (uint32_t ch = 0; ch < nch && !failed; ++ch) {
            const uint32_t k_begin = ch * a.chunk, k_end = min(KT, k_begin + a.chunk);
            if (threadIdx.x == 0) {
                if (ch == 0)
                    for (uint32_t kt = 0; kt < KT && kt < OZ_STAGES && ok; ++kt) ok = load(kt);
                for (uint32_t kt = k_begin; kt < k_end && ok; ++kt) {
                    const uint32_t gs = slab0 + kt, st = gs % OZ_STAGES;
                    ok = mbar_wait(&full[st], (gs / OZ_STAGES) & 1u, a.err, a.wait_ns);
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
                                const uint32_t accum = (kt > k_begin || ks > 0 || p > 0) ? 1u : 0u;
                                umma_i8(tmem + uint32_t(g * OZ_BN), da, db, idesc, accum);
                            }
                    umma_commit(&empty[st]);
                    if (kt + OZ_STAGES < KT) ok = load(kt + OZ_STAGES);
                }
                if (!ok) atomicExch(a.err, 1);
                umma_commit(done);  // arrives once every MMA issued so far has completed
            }
            __syncwarp();
            // the MMAs issued so far always complete: their wait keeps the fixed limit even when
            // the error word is set, so TMEM is never released under a running MMA
            bool ready = true;
            {
                const unsigned long long t0 = global_ns();
                while (!mbar_try(done, rounds & 1u))
                    if (global_ns() - t0 > WAIT_LIMIT_NS) {
                        atomicExch(a.err, 1);
                        ready = false;
                        break;
                    }
            }
            ++rounds;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const bool go = __all_sync(0xffffffffu, ready && *verr == 0);
            if (go) {
                const uint32_t row = mt * OZ_BM + warp * 32 + lane;
                const int erow = (row < pb.M) ? a.e[pb.e_off + row] : 0;
                const bool add = pb.beta || ch > 0;
                double* Cb = reinterpret_cast<double*>(base_of(a.bases, pb.C.buf) + 8ull * pb.C.off);
                for (int c0 = 0; c0 < OZ_BN; c0 += 16) {
                    double acc[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[j] = 0.0;
                    for (int g = s - 1; g >= 0 && KT > 0; --g) {
                        int32_t v[16];
                        tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(g * OZ_BN + c0), v);
                        const double w = ldexp(1.0, -7 * (g + 2));
#pragma unroll
                        for (int j = 0; j < 16; ++j) acc[j] += double(v[j]) * w;
                    }
                    if (row < pb.M) {
                        // the row's start and leading dimension: from the row table or the plain operand
                        double* crow = Cb + row;
                        uint64_t ldc = pb.C.ld;
                        if (pb.rowtab != DevProb::NO_ROWS) {
                            const DevRow rw = a.rowtab[pb.rowtab + row];
                            crow = reinterpret_cast<double*>(base_of(a.bases, pb.C.buf)) + rw.c_off +
                                   uint64_t(pb.batch) * rw.cbs;
                            ldc = rw.ld;
                        }
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const uint32_t col = nt * OZ_BN + c0 + j;
                            if (col < pb.N) {
                                const double val = ldexp(acc[j], erow + a.e[pb.f_off + col]);
                                double* dst = crow + uint64_t(col) * ldc;
                                *dst = add ? *dst + val : val;
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
        slab0 += KT;
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

// Operands held in boundary memory (BUF_ABS) do not change between calls of a
// plan: their digit planes and exponents are computed on the first run and kept
// in the program's scratch; later runs split only the other operands.  The
// exponents of constant operands occupy [0, n_exp_c) of the exponent array.
struct OzProgram {
    std::vector<OzSplit> jobs;      // every operand (constant ones first)
    uint32_t n_const_jobs = 0;
    std::vector<OzPB> pbs;
    std::vector<OzSlab> slabs;
    std::vector<OzTile> tiles;
    uint64_t a_plane = 0, b_plane = 0, n_exp = 0, n_exp_c = 0;
    bool const_ready = false;       // constant digit planes present in the scratch
    std::vector<DevRow> rowtab;     // rows of row-table problems (the GEMM list's table)
    OzSplit* d_jobs = nullptr;
    OzPB* d_pbs = nullptr;
    OzSlab* d_slabs = nullptr;
    OzTile* d_tiles = nullptr;
    DevRow* d_rowtab = nullptr;
};

OzProgram* oz_build(GemmList const& gl) {
    auto* oz = new OzProgram;
    std::vector<uint32_t> nbatch(gl.probs.size(), 0);
    for (auto const& t : gl.tiles) nbatch[t.prob] = std::max(nbatch[t.prob], t.batch + 1);
    // exponent offsets: constant operands count in n_exp_c, the others in n_exp
    // (shifted behind the constant region below); var_e / var_f mark the latter
    std::vector<uint8_t> var_e, var_f;
    for (uint32_t p = 0; p < gl.probs.size(); ++p) {
        DevProb const& pr = gl.probs[p];
        bool a_const = true, b_const = true;
        for (uint32_t sgi = pr.seg_begin; sgi < pr.seg_end; ++sgi) {
            a_const = a_const && gl.segs[sgi].A.buf == BUF_ABS;
            b_const = b_const && gl.segs[sgi].B.buf == BUF_ABS;
        }
        for (uint32_t b = 0; b < nbatch[p]; ++b) {
            OzPB pb{};
            pb.M = pr.M;
            pb.N = pr.N;
            pb.MT = std::max<uint32_t>(1, (pr.M + OZ_BM - 1) / OZ_BM);
            pb.NT = std::max<uint32_t>(1, (pr.N + OZ_BN - 1) / OZ_BN);
            uint64_t& ce = a_const ? oz->n_exp_c : oz->n_exp;
            pb.e_off = ce;
            ce += uint64_t(pb.MT) * OZ_BM;
            uint64_t& cf = b_const ? oz->n_exp_c : oz->n_exp;
            pb.f_off = cf;
            cf += uint64_t(pb.NT) * OZ_BN;
            var_e.push_back(!a_const);
            var_f.push_back(!b_const);
            pb.C = pr.C;
            pb.C.off += uint64_t(b) * pr.C.bstride;
            pb.beta = 0;
            pb.rowtab = pr.rows;
            pb.batch = b;
            pb.slab_begin = uint32_t(oz->slabs.size());
            for (uint32_t sgi = pr.seg_begin; sgi < pr.seg_end; ++sgi) {
                DevSeg const& sg = gl.segs[sgi];
                if (!sg.K) continue;
                const uint32_t KS = (sg.K + OZ_BK - 1) / OZ_BK;
                OzSplit ja{}, jb{};
                ja.op = sg.A;
                ja.op.off += uint64_t(b) * sg.A.bstride;
                ja.rows = pr.M;
                ja.K = sg.K;
                ja.RT = pb.MT;
                ja.KS = KS;
                ja.out_base = oz->a_plane;
                ja.e_off = pb.e_off;
                ja.is_b = 0;
                ja.is_const = a_const ? 1 : 0;
                ja.rowtab = pr.rows;
                oz->a_plane += uint64_t(pb.MT) * KS * A_TILE;
                jb.op = sg.B;
                jb.op.off += uint64_t(b) * sg.B.bstride;
                jb.rows = pr.N;
                jb.K = sg.K;
                jb.RT = pb.NT;
                jb.KS = KS;
                jb.out_base = oz->b_plane;
                jb.e_off = pb.f_off;
                jb.is_b = 1;
                jb.is_const = b_const ? 1 : 0;
                jb.rowtab = DevProb::NO_ROWS;
                oz->b_plane += uint64_t(pb.NT) * KS * B_TILE;
                for (uint32_t ks = 0; ks < KS; ++ks)
                    oz->slabs.push_back(OzSlab{ja.out_base + uint64_t(ks) * A_TILE, jb.out_base + uint64_t(ks) * B_TILE,
                                               KS * uint32_t(A_TILE), KS * uint32_t(B_TILE)});
                oz->jobs.push_back(ja);
                oz->jobs.push_back(jb);
            }
            pb.slab_end = uint32_t(oz->slabs.size());
            uint32_t pbi = uint32_t(oz->pbs.size());
            oz->pbs.push_back(pb);
            for (uint32_t mt = 0; mt < pb.MT; ++mt)
                for (uint32_t nt = 0; nt < pb.NT; ++nt) oz->tiles.push_back(OzTile{pbi, mt, nt, 0});
        }
    }
    for (size_t i = 0; i < oz->pbs.size(); ++i) {
        if (var_e[i]) oz->pbs[i].e_off += oz->n_exp_c;
        if (var_f[i]) oz->pbs[i].f_off += oz->n_exp_c;
    }
    for (auto& j : oz->jobs)
        if (!j.is_const) j.e_off += oz->n_exp_c;
    oz->n_exp += oz->n_exp_c;
    std::stable_partition(oz->jobs.begin(), oz->jobs.end(), [](OzSplit const& j) { return j.is_const != 0; });
    oz->n_const_jobs =
        uint32_t(std::count_if(oz->jobs.begin(), oz->jobs.end(), [](OzSplit const& j) { return j.is_const != 0; }));
    // longest K first for the static round-robin over the persistent grid
    std::stable_sort(oz->tiles.begin(), oz->tiles.end(), [&](OzTile const& x, OzTile const& y) {
        auto kx = oz->pbs[x.pb].slab_end - oz->pbs[x.pb].slab_begin;
        auto ky = oz->pbs[y.pb].slab_end - oz->pbs[y.pb].slab_begin;
        return kx > ky;
    });
    auto up = [](auto const& v, auto** d) -> cudaError_t {
        *d = nullptr;
        if (v.empty()) return cudaSuccess;
        cudaError_t e = cudaMalloc(d, v.size() * sizeof(v[0]));
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice);
    };
    oz->rowtab = gl.rowtab;
    if (up(oz->jobs, &oz->d_jobs) != cudaSuccess || up(oz->pbs, &oz->d_pbs) != cudaSuccess ||
        up(oz->slabs, &oz->d_slabs) != cudaSuccess || up(oz->tiles, &oz->d_tiles) != cudaSuccess ||
        up(oz->rowtab, &oz->d_rowtab) != cudaSuccess) {
        oz_free(oz);
        return nullptr;
    }
    return oz;
}

void oz_invalidate(OzProgram* oz) {
    if (oz) oz->const_ready = false;
}

void oz_free(OzProgram* oz) {
    if (!oz) return;
    cudaFree(oz->d_jobs);
    cudaFree(oz->d_pbs);
    cudaFree(oz->d_slabs);
    cudaFree(oz->d_tiles);
    cudaFree(oz->d_rowtab);
    delete oz;
}

namespace {
struct OzScratch {
    int8_t* A8;
    int8_t* B8;
    int* e;
};
OzScratch carve(OzProgram const* oz, int s, void* scratch) {
    auto* p = static_cast<unsigned char*>(scratch);
    OzScratch c;
    c.A8 = reinterpret_cast<int8_t*>(p);
    p += round_up(uint64_t(s) * oz->a_plane, 256);
    c.B8 = reinterpret_cast<int8_t*>(p);
    p += round_up(uint64_t(s) * oz->b_plane, 256);
    c.e = reinterpret_cast<int*>(p);
    return c;
}
}  // namespace

uint64_t oz_scratch_bytes(OzProgram const* oz, int s) {
    return round_up(uint64_t(s) * oz->a_plane, 256) + round_up(uint64_t(s) * oz->b_plane, 256) +
           round_up(oz->n_exp * sizeof(int), 256);
}

cudaError_t oz_run(OzProgram* oz, Bases const& bs, int s, void* scratch, int* err, cudaStream_t st) {
    if (s < 2 || s > OZ_MAX_SLICES) return cudaErrorInvalidValue;
    OzScratch c = carve(oz, s, scratch);
    const int sms = device_sm_count();
    // the error word is not cleared here: it collects timeouts until the caller reads it
    // first run: every operand; later runs: only the operands that change between calls
    const uint64_t e0 = oz->const_ready ? oz->n_exp_c : 0;
    const uint32_t j0 = oz->const_ready ? oz->n_const_jobs : 0;
    if (oz->n_exp > e0)
        fill_int<<<std::min<uint64_t>((oz->n_exp - e0 + 255) / 256, 4096), 256, 0, st>>>(c.e + e0, oz->n_exp - e0,
                                                                                        -100000);
    const uint32_t nj = uint32_t(oz->jobs.size()) - j0;
    if (nj) {
        oz_exponents<<<dim3(8, std::min<uint32_t>(nj, 65535u)), 256, 0, st>>>(oz->d_jobs + j0, nj, bs, c.e,
                                                                             oz->d_rowtab);
        dim3 grid(16, std::min<uint32_t>(nj, 65535u));
        oz_split<<<grid, 256, 0, st>>>(oz->d_jobs + j0, nj, bs, c.e, s, oz->a_plane, c.A8, oz->b_plane, c.B8,
                                       oz->d_rowtab);
    }
    oz->const_ready = true;
    if (!oz->tiles.empty()) {
        cudaError_t ea = ensure_smem_limit(reinterpret_cast<const void*>(ozaki_mma), int(ozaki_smem_bytes(OZ_MAX_SLICES)));
        if (ea != cudaSuccess) return ea;
        OzArgs args{c.A8, c.B8, oz->a_plane, oz->b_plane, c.e, oz->d_pbs, oz->d_slabs, oz->d_tiles,
                    uint32_t(oz->tiles.size()), oz_chunk_slabs(s), s, bs, err, oz->d_rowtab, wait_limit_ns()};
        ozaki_mma<<<std::min<uint32_t>(uint32_t(oz->tiles.size()), uint32_t(sms)), OZ_THREADS, ozaki_smem_bytes(s),
                    st>>>(args);
    }
    return cudaGetLastError();
}

bool oz_constants_ready(OzProgram const* oz) { return oz && oz->const_ready; }

namespace {
// out[0] = sum (a - b)^2, out[1] = sum b^2 (one block, FP64)
__global__ void __launch_bounds__(256) diff_norms_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                                         uint64_t n, double* __restrict__ out) {
    __shared__ double sd[256], sb[256];
    double d = 0.0, q = 0.0;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = a[i] - b[i];
        d += x * x;
        q += b[i] * b[i];
    }
    sd[threadIdx.x] = d;
    sb[threadIdx.x] = q;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sd[threadIdx.x] += sd[threadIdx.x + o];
            sb[threadIdx.x] += sb[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sd[0];
        out[1] = sb[0];
    }
}
}  // namespace

cudaError_t diff_norms(const double* a, const double* b, uint64_t n, double* out, cudaStream_t st) {
    diff_norms_kernel<<<1, 256, 0, st>>>(a, b, n, out);
    return cudaGetLastError();
}

}  // namespace dmrgb200

using namespace dmrgb200;

extern "C" dmrgb200_status dmrgb200_dgemm_emulated(uint32_t M, uint32_t N, uint32_t K, const double* A, uint64_t lda,
                                                   const double* B, uint64_t ldb, double* C, uint64_t ldc,
                                                   int slices, void* cuda_stream) {
    if (!A || !B || !C) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (slices < 2 || slices > OZ_MAX_SLICES) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "slices must be 2..8");
    if (lda < M || ldb < K || ldc < M) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "leading dimension too small");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    GemmList gl;
    DevProb pr{};
    pr.M = M;
    pr.N = N;
    pr.C = DevOp{reinterpret_cast<uint64_t>(C) / 8, 0, uint32_t(ldc), uint16_t(BUF_ABS), 0};
    pr.seg_begin = 0;
    pr.seg_end = 1;
    DevSeg sg{};
    sg.A = DevOp{reinterpret_cast<uint64_t>(A) / 8, 0, uint32_t(lda), uint16_t(BUF_ABS), 0};
    sg.B = DevOp{reinterpret_cast<uint64_t>(B) / 8, 0, uint32_t(ldb), uint16_t(BUF_ABS), 0};
    sg.K = K;
    gl.probs.push_back(pr);
    gl.segs.push_back(sg);
    gl.tiles.push_back(DevTile{0, 0, 0, 0});
    OzProgram* oz = oz_build(gl);
    if (!oz) return noalloc_fail(DMRGB200_OUT_OF_MEMORY, "emulated GEMM tables");
    void* scratch = nullptr;
    const uint64_t sbytes = oz_scratch_bytes(oz, slices);
    cudaError_t r = cudaMallocAsync(&scratch, sbytes + 256, st);
    if (r != cudaSuccess) {
        oz_free(oz);
        return noalloc_fail(DMRGB200_OUT_OF_MEMORY, cudaGetErrorString(r));
    }
    int* err = reinterpret_cast<int*>(static_cast<unsigned char*>(scratch) + sbytes);
    Bases bs{};
    int to = 0;
    cudaMemsetAsync(err, 0, sizeof(int), st);
    r = oz_run(oz, bs, slices, scratch, err, st);
    cudaMemcpyAsync(&to, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t r2 = cudaStreamSynchronize(st);
    cudaFreeAsync(scratch, st);
    cudaStreamSynchronize(st);
    oz_free(oz);
    if (r != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("emulated GEMM: ") + cudaGetErrorString(r));
    if (r2 != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("emulated GEMM: ") + cudaGetErrorString(r2));
    if (to) return noalloc_fail(DMRGB200_TIMEOUT, "emulated GEMM: a pipeline wait timed out");
    return DMRGB200_OK;
}
