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
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"
#include "async_copy.cuh"

namespace dmrgb200 {

dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);

namespace {

// Output tiles are 128 rows by BN = 64 or 128 columns (chosen per program, oz_build).
// TMEM holds 512 int32 columns: 512 / BN accumulators at a time, so with BN = 128 the
// digit groups g = 0 .. s-1 of a tile run as passes of up to 4 groups over its K slabs
// (BN = 64: one pass for s <= 8).
constexpr int OZ_BM = 128, OZ_BK = 32;  // tile rows, K bytes per slab
constexpr int A_TILE = OZ_BM * OZ_BK;
constexpr int OZ_MAX_SLICES = 8, OZ_MAX_STAGES = 8;
__host__ __device__ constexpr int oz_pass_groups(int bn) { return 512 / bn; }
__host__ __device__ constexpr int oz_passes(int s, int bn) { return (s + oz_pass_groups(bn) - 1) / oz_pass_groups(bn); }
// warps 0-7 drain the accumulators (TMEM lane quarter = warp % 4, column half = warp / 4),
// warp 8 loads the slabs, warp 9 issues the MMAs
constexpr int OZ_EPI_WARPS = 8, OZ_LOAD_WARP = 8, OZ_MMA_WARP = 9, OZ_THREADS = 32 * 10;
constexpr uint32_t OZ_SMEM_CAP = 227u * 1024u;  // dynamic shared memory of one CTA
constexpr uint32_t OZ_BAR_BYTES = 256;          // barriers and slots behind the stages
// pipeline depth for s digit planes: as many stages of s (A + B) tiles as fit
__host__ __device__ constexpr uint32_t oz_stages(int s, int bn) {
    return (OZ_SMEM_CAP - OZ_BAR_BYTES) / (uint32_t(s) * uint32_t(A_TILE + bn * OZ_BK)) < uint32_t(OZ_MAX_STAGES)
               ? (OZ_SMEM_CAP - OZ_BAR_BYTES) / (uint32_t(s) * uint32_t(A_TILE + bn * OZ_BK))
               : uint32_t(OZ_MAX_STAGES);
}
using namespace async;

// K slabs per exact INT32 accumulation: accumulator D_g sums (g + 1) <= s digit
// products of |a b| <= 127^2 per K element, and 127^2 * 2^17 < 2^31
constexpr uint32_t oz_chunk_slabs(int s) { return std::max<uint32_t>(1u, (1u << 17) / uint32_t(s * OZ_BK)); }

// byte offset of element (r, k) of a (rows x 32-byte) K-major tile in the
// canonical no-swizzle layout: 8x16-byte core matrices, LBO = 128 B along K,
// SBO = 256 B between 8-row groups
__device__ __forceinline__ uint32_t tile_off(uint32_t r, uint32_t k) {
    return (r >> 3) * 256u + (k >> 4) * 128u + (r & 7u) * 16u + (k & 15u);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFFu);
    d |= uint64_t((128u >> 4) & 0x3FFFu) << 16;  // leading (K) byte offset
    d |= uint64_t((256u >> 4) & 0x3FFFu) << 32;  // stride (row-group) byte offset
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
// 16 consecutive TMEM columns of this warp's 32 lanes; the values are valid after tmem_wait_ld
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- digit extraction --------------------------------------------------------------

// One operand of one segment to be cut into digit planes.  For an A operand the
// digit matrix is A itself (row r, column k); for a B operand it is B^T (row n,
// column k), both stored K-major in 4 KB (A, 128 rows) or 2 KB (B, 64 rows) tiles.
// Tile (rt, ks) has the index t = out_base / tile_bytes + rt * KS + ks, and its s
// digit planes lie side by side: plane p at (t * s + p) * tile_bytes, so that one
// bulk copy moves every plane of a slab.  Offsets and sizes that count one plane
// (out_base, a_plane, the slab offsets) are scaled by s where memory is addressed.
struct OzSplit {
    DevOp op;           // batch already folded into op.off
    uint32_t rows, K;   // logical rows (M or N) and K of the segment
    uint32_t RT, KS;    // row tiles, K slabs
    uint64_t out_base;  // byte offset inside a digit plane
    uint64_t e_off;     // exponent array offset of row 0
    uint32_t is_b;      // 0: A operand, 1: B operand (read transposed)
    uint32_t is_const;  // the operand and its exponents are constant between calls
    uint32_t rowtab;    // A of a row-table problem: row r at rowtab[rowtab + r]; DevProb::NO_ROWS otherwise
    uint32_t tr;        // rows of a digit tile: OZ_BM (A) or the program's BN (B)
};

__global__ void fill_int(int* __restrict__ p, uint64_t n, int v) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        p[i] = v;
}

// Addressing of a split job: element (r, k) of a plain operand is base[r * sr + k * sk];
// a row-table A row r starts at rowtab[rowtab + r].a_off with K stride rowtab[..].ld.
struct OzAddr {
    const double* base;
    uint64_t sr, sk;
};
__device__ __forceinline__ OzAddr oz_addr(Bases const& bs, OzSplit const& j) {
    OzAddr a;
    a.base = reinterpret_cast<const double*>(base_of(bs, j.op.buf) + 8ull * j.op.off);
    const uint64_t ld = j.op.ld;
    const bool rows_contig = j.is_b ? (j.op.trans != 0) : (j.op.trans == 0);
    a.sr = rows_contig ? 1 : ld;
    a.sk = rows_contig ? ld : 1;
    return a;
}
// k-major jobs (K contiguous for a row, no row table): a warp walks one row
__host__ __device__ __forceinline__ bool oz_kmajor(OzSplit const& j) {
    const bool rows_contig = j.is_b ? (j.op.trans != 0) : (j.op.trans == 0);
    return !rows_contig && (j.is_b || j.rowtab == DevProb::NO_ROWS);
}
constexpr uint32_t OZ_EXP_KCH = 1024;  // K elements of a k-major exponent item (one warp)
constexpr uint32_t OZ_EXP_RCH = 256;   // K elements of a row-major exponent item (32 rows, one per lane)

// Warp items of the exponent pass:
//   k-major:   (row, K chunk of OZ_EXP_KCH): the lanes read the chunk contiguously
//   row-major: (32 consecutive rows, K chunk of OZ_EXP_RCH): one row per lane, the
//              lanes read consecutive rows of one K column (contiguous)
__host__ __device__ __forceinline__ uint64_t oz_exp_items(OzSplit const& j) {
    if (oz_kmajor(j)) return uint64_t(j.rows) * ((j.K + OZ_EXP_KCH - 1) / OZ_EXP_KCH);
    return uint64_t((j.rows + 31) / 32) * ((j.K + OZ_EXP_RCH - 1) / OZ_EXP_RCH);
}
// Warp items of the split pass (every padded row and K slab of the digit tiles):
//   k-major:   (16-row group, 32-element slab): lane t takes row (t & 15) and the 16
//              K elements (t >> 4) * 16 .. + 15, so the warp writes two contiguous
//              256-byte core-matrix groups (512 bytes) per digit plane
//   row-major: (32 consecutive rows, 16-element K group): one row per lane, the lanes
//              read one K column of 32 rows at a time and write 16 bytes each
__host__ __device__ __forceinline__ uint64_t oz_split_items(OzSplit const& j, uint32_t TR) {
    if (oz_kmajor(j)) return uint64_t(j.RT) * (TR / 16) * j.KS;
    return uint64_t(j.RT) * (TR / 32) * j.KS * (OZ_BK / 16);
}

// job of a warp item: the job j with first[j] <= it < first[j + 1] (jobs without items
// have first[j] == first[j + 1] and are never chosen)
__device__ __forceinline__ uint32_t oz_job_of(const uint64_t* __restrict__ first, uint32_t njobs, uint64_t it) {
    uint32_t lo = 0, hi = njobs;  // first[lo] <= it < first[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (first[mid] <= it) lo = mid;
        else hi = mid;
    }
    return lo;
}

// exponent of every row of every job (max over segments and chunks by atomicMax):
// |x 2^-e| < 1 for the whole row of the output matrix.  `first` holds the first warp
// item of every job and the end (njobs + 1 entries; the items of the launched jobs are
// first[0] .. first[njobs] - 1).
__global__ void __launch_bounds__(256) oz_exponents(const OzSplit* __restrict__ jobs, const uint64_t* __restrict__ first,
                                                    uint32_t njobs, Bases bs, int* __restrict__ e,
                                                    const DevRow* __restrict__ rowtab) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t total = first[njobs];
    const uint64_t nwarps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t it = first[0] + uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); it < total;
         it += nwarps) {
        const uint32_t jn = oz_job_of(first, njobs, it);
        const OzSplit job = jobs[jn];
        const uint64_t local = it - first[jn];
        if (oz_kmajor(job)) {
            const uint32_t nch = (job.K + OZ_EXP_KCH - 1) / OZ_EXP_KCH;
            const uint32_t r = uint32_t(local / nch), k0 = uint32_t(local % nch) * OZ_EXP_KCH;
            const OzAddr a = oz_addr(bs, job);
            const double* row = a.base + uint64_t(r) * a.sr;
            const uint32_t k1 = min(job.K, k0 + OZ_EXP_KCH);
            double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
            uint32_t k = k0 + lane;
            for (; k + 96 < k1; k += 128) {
                m0 = fmax(m0, fabs(row[k]));
                m1 = fmax(m1, fabs(row[k + 32]));
                m2 = fmax(m2, fabs(row[k + 64]));
                m3 = fmax(m3, fabs(row[k + 96]));
            }
            for (; k < k1; k += 32) m0 = fmax(m0, fabs(row[k]));
            double m = fmax(fmax(m0, m1), fmax(m2, m3));
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0 && m > 0.0) atomicMax(&e[job.e_off + r], ilogb(m) + 1);
        } else {
            const uint32_t nch = (job.K + OZ_EXP_RCH - 1) / OZ_EXP_RCH;
            const uint32_t r = uint32_t(local / nch) * 32 + lane, k0 = uint32_t(local % nch) * OZ_EXP_RCH;
            if (r >= job.rows) continue;
            const double* row;
            uint64_t sk;
            if (!job.is_b && job.rowtab != DevProb::NO_ROWS) {
                const DevRow rw = rowtab[job.rowtab + r];
                row = reinterpret_cast<const double*>(base_of(bs, job.op.buf)) + rw.a_off;
                sk = rw.ld;
            } else {
                const OzAddr a = oz_addr(bs, job);
                row = a.base + r;  // rows contiguous: sr = 1
                sk = a.sk;
            }
            const uint32_t k1 = min(job.K, k0 + OZ_EXP_RCH);
            double m0 = 0.0, m1 = 0.0;
            uint32_t k = k0;
            for (; k + 1 < k1; k += 2) {
                m0 = fmax(m0, fabs(row[uint64_t(k) * sk]));
                m1 = fmax(m1, fabs(row[uint64_t(k + 1) * sk]));
            }
            if (k < k1) m0 = fmax(m0, fabs(row[uint64_t(k) * sk]));
            const double m = fmax(m0, m1);
            if (m > 0.0) atomicMax(&e[job.e_off + r], ilogb(m) + 1);
        }
    }
}

// The digits of y = x 2^-ex (|y| < 1) are those of the repeated step d = trunc(128 y),
// y <- 128 y - d: digit p is sign(x) times bits 49 - 7p .. 55 - 7p of the integer
// trunc(|x| 2^(56 - ex)), p = 0 .. 7.  That integer is formed from the bits of x
// alone (mantissa shifted by the exponent difference; exact, no rounding), so the
// split needs no floating-point conversions.
__device__ __forceinline__ uint64_t oz_fixed(double x, int ex, uint32_t& neg) {
    const uint64_t b = static_cast<uint64_t>(__double_as_longlong(x));
    neg = uint32_t(b >> 63);
    int E = int((b >> 52) & 0x7ffu);
    uint64_t m = b & ((1ull << 52) - 1ull);
    if (E) m |= 1ull << 52;  // normal: implicit bit
    else E = 1;              // subnormal: m units of 2^-1074
    const int sh = E - 1075 + 56 - ex;  // |x| 2^(56 - ex) = m 2^sh < 2^56 when |y| < 1
    if (sh >= 0) return sh < 64 ? (m << sh) : 0ull;
    return sh > -64 ? (m >> -sh) : 0ull;
}
// 0xFF in byte j of the word of four elements where element j is negative
__device__ __forceinline__ uint32_t oz_sign_bytes(uint32_t const* neg) {
    return ((0u - neg[0]) & 0xFFu) | (((0u - neg[1]) & 0xFFu) << 8) | (((0u - neg[2]) & 0xFFu) << 16) |
           ((0u - neg[3]) << 24);
}
// digit p of four fixed-point values as one word of bytes (two's complement): the four
// 7-bit magnitudes packed by byte permutes, then negated per byte where the sign byte is
// 0xFF ((d ^ 0xFF) - 0xFF = -d mod 256, no borrow between bytes).  p is a constant in the
// unrolled plane loops, so the shifts are immediate.
__device__ __forceinline__ uint32_t oz_digits4(uint64_t const* X, uint32_t sign, int p) {
    const int sh = 49 - 7 * p;
    const uint32_t d0 = uint32_t(X[0] >> sh) & 127u, d1 = uint32_t(X[1] >> sh) & 127u;
    const uint32_t d2 = uint32_t(X[2] >> sh) & 127u, d3 = uint32_t(X[3] >> sh) & 127u;
    const uint32_t w = __byte_perm(__byte_perm(d0, d1, 0x0040), __byte_perm(d2, d3, 0x0040), 0x5410);
    return __vsub4(w ^ sign, sign);
}

// Digit planes of every job: the s signed 7-bit digits of every element scaled by its
// row's exponent, in the K-major core-matrix layout of the MMA tiles (rows beyond the
// operand and K beyond it give zero digits).  `first` as for oz_exponents.
__global__ void __launch_bounds__(256) oz_split(const OzSplit* __restrict__ jobs, const uint64_t* __restrict__ first,
                                                uint32_t njobs, Bases bs, const int* __restrict__ e, int s,
                                                int8_t* __restrict__ A8, int8_t* __restrict__ B8,
                                                const DevRow* __restrict__ rowtab) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t total = first[njobs];
    const uint64_t nwarps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t it = first[0] + uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); it < total;
         it += nwarps) {
        const uint32_t jn = oz_job_of(first, njobs, it);
        const OzSplit job = jobs[jn];
        const uint64_t local = it - first[jn];
        int8_t* out = job.is_b ? B8 : A8;
        const uint32_t TR = job.tr;
        const uint32_t tile_bytes = TR * OZ_BK;
        if (oz_kmajor(job)) {
            // item = (16-row group g, slab ks); lane: row g * 16 + (lane & 15), K 16 (lane >> 4) .. + 15
            const uint32_t ks = uint32_t(local % job.KS);
            const uint32_t g = uint32_t(local / job.KS);
            const uint32_t r = g * 16 + (lane & 15);
            const uint32_t kk = (lane >> 4) * 16;  // within the slab
            const uint32_t k0 = ks * OZ_BK + kk;
            const bool live = r < job.rows;
            const int ex = live ? e[job.e_off + r] : 0;
            const OzAddr a = oz_addr(bs, job);
            const double* row = a.base + uint64_t(r) * a.sr;
            uint64_t X[16];
            uint32_t neg[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) X[u] = oz_fixed((live && k0 + u < job.K) ? row[k0 + u] : 0.0, ex, neg[u]);
            const uint64_t off = (job.out_base + (uint64_t(r / TR) * job.KS + ks) * tile_bytes) * s + tile_off(r % TR, kk);
            uint32_t sign[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) sign[q] = oz_sign_bytes(neg + 4 * q);
#pragma unroll
            for (int p = 0; p < OZ_MAX_SLICES; ++p) {
                if (p >= s) break;
                uint32_t w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) w[q] = oz_digits4(X + 4 * q, sign[q], p);
                *reinterpret_cast<uint4*>(out + off + p * tile_bytes) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        } else {
            // item = (32-row group, 16-element K group); lane: one row
            const uint32_t ngroups = job.KS * (OZ_BK / 16);
            const uint32_t r = uint32_t(local / ngroups) * 32 + lane;
            const uint32_t k0 = 16 * uint32_t(local % ngroups);
            const bool live = r < job.rows;
            const int ex = live ? e[job.e_off + r] : 0;
            const double* row = nullptr;
            uint64_t sk = 0;
            if (live) {
                if (!job.is_b && job.rowtab != DevProb::NO_ROWS) {
                    const DevRow rw = rowtab[job.rowtab + r];
                    row = reinterpret_cast<const double*>(base_of(bs, job.op.buf)) + rw.a_off;
                    sk = rw.ld;
                } else {
                    const OzAddr a = oz_addr(bs, job);
                    row = a.base + r;  // rows contiguous: sr = 1
                    sk = a.sk;
                }
            }
            uint64_t X[16];
            uint32_t neg[16];
#pragma unroll
            for (int u = 0; u < 16; ++u)
                X[u] = oz_fixed((live && k0 + u < job.K) ? row[uint64_t(k0 + u) * sk] : 0.0, ex, neg[u]);
            const uint64_t off = (job.out_base + (uint64_t(r / TR) * job.KS + k0 / OZ_BK) * tile_bytes) * s +
                                 tile_off(r % TR, k0 % OZ_BK);
            uint32_t sign[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) sign[q] = oz_sign_bytes(neg + 4 * q);
#pragma unroll
            for (int p = 0; p < OZ_MAX_SLICES; ++p) {
                if (p >= s) break;
                uint32_t w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) w[q] = oz_digits4(X + 4 * q, sign[q], p);
                *reinterpret_cast<uint4*>(out + off + p * tile_bytes) = make_uint4(w[0], w[1], w[2], w[3]);
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
    const int* e;
    const OzPB* pbs;
    const OzSlab* slabs;
    const OzTile* tiles;
    uint32_t n_tiles;
    uint32_t chunk;   // K slabs accumulated in TMEM before a partial epilogue (>= 1)
    uint32_t stages;  // pipeline stages of s (A + B) tiles
    int s;
    Bases bases;
    int* err;
    const DevRow* rowtab;
    unsigned long long wait_ns;  // limit of the waits for operand slabs
};

// exact int32 -> double on the integer and FP64 pipes: the bit pattern of 2^52 + 2^51
// plus v is the double 2^52 + 2^51 + v (unit spacing there, |v| < 2^51)
__device__ __forceinline__ double i2d_exact(int32_t v) {
    return __longlong_as_double(0x4338000000000000ll + static_cast<long long>(v)) - 6755399441055744.0;
}
// 2^e for -1022 <= e <= 1023
__device__ __forceinline__ double pow2_normal(int e) { return __longlong_as_double(static_cast<long long>(e + 1023) << 52); }

// bounded wait that ignores the error word: for events that always happen once work is
// in flight (issued MMAs completing, issued copies landing before the CTA leaves)
__device__ __forceinline__ void oz_settle(uint64_t* bar, uint32_t parity, int* err) {
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > WAIT_LIMIT_NS) {
            atomicExch(err, 1);
            return;
        }
}

// Persistent grouped INT8 GEMM over the digit planes, one 128 x OZ_BN output tile at a
// time.  The digit groups g = p + q < s of a tile run as passes of up to 512 / OZ_BN
// groups (the accumulators of one pass fill at most the 512 TMEM columns), smallest
// weights first; a pass needs the digit planes 0 .. (its last group).  Warp roles:
//   load warp (lane 0): per (tile, pass, K slab) one bulk copy of the pass's A planes
//     and one of its B planes into a ring of `stages` stages (full barriers), refilling
//     a stage once the MMAs that read it have completed (empty barriers, MMA commits);
//   MMA warp (lane 0): for each slab, the digit products of the pass's groups into
//     accumulator g - g0 (TMEM columns (g - g0) * OZ_BN ..), one 128 x OZ_BN x 32
//     tcgen05.mma each; after a chunk of slabs it commits to `tfull`;
//   epilogue warps 0-3: wait `tfull`, read their 32 TMEM lanes of the pass's
//     accumulators 32 columns at a time, sum them scaled by 2^-7(g+2) in FP64
//     (smallest weight first), add 2^(e_row + e_col) times the sum into C, and release
//     the accumulators (`tempty`, which the MMA warp waits for before the next chunk).
// The load warp runs ahead across passes and tiles, so copies overlap the epilogue.
// Every wait is bounded; on a timeout or a set error word each role stops, the issued
// MMAs and copies are waited for (fixed limit), TMEM is released and the CTA returns.
template <int OZ_BN>
__global__ void __launch_bounds__(OZ_THREADS, 1) ozaki_mma(OzArgs a) {
    constexpr int B_TILE = OZ_BN * OZ_BK, OZ_PASS_GROUPS = oz_pass_groups(OZ_BN);
    extern __shared__ __align__(1024) unsigned char smem[];
    const int s = a.s;
    const int npass = oz_passes(s, OZ_BN);
    const uint32_t nst = a.stages;
    const uint32_t a_room = uint32_t(s) * A_TILE, stage_bytes = uint32_t(s) * (A_TILE + B_TILE);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + nst * stage_bytes);
    uint64_t* empty = full + nst;
    uint64_t* tfull = empty + nst;
    // accumulator releases: one per group of the pass with 64-column tiles (the MMA warp
    // reuses a group as soon as the epilogue has read it), one for the pass otherwise
    constexpr int NREL = OZ_BN == 64 ? OZ_PASS_GROUPS : 1;
    uint64_t* tempty = tfull + 1;
    uint64_t* fin = tempty + NREL;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);
    uint32_t* consumed_slot = tmem_slot + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ncols = min(s, OZ_PASS_GROUPS) * OZ_BN <= 128 ? 128u : (min(s, OZ_PASS_GROUPS) * OZ_BN <= 256 ? 256u : 512u);
    // groups [g0, g1) of pass q (passes run q = npass - 1 .. 0) and the planes it reads
    auto pass_groups = [&](int q, int& g0, int& g1) {
        g0 = q * OZ_PASS_GROUPS;
        g1 = min(s, g0 + OZ_PASS_GROUPS);
    };

    if (threadIdx.x == 0) {
        for (uint32_t i = 0; i < nst; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(tfull, 1);
        for (int i = 0; i < NREL; ++i) mbar_init(&tempty[i], OZ_EPI_WARPS);
        mbar_init(fin, 1);
        *consumed_slot = 0;
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
    uint32_t issued = 0;  // load warp lane 0: slabs whose copies were issued

    if (warp == OZ_LOAD_WARP) {
        if (lane == 0) {
            uint32_t gs = 0;
            bool ok = true;
            for (uint32_t tile = blockIdx.x; tile < a.n_tiles && ok; tile += gridDim.x) {
                const OzTile tl = a.tiles[tile];
                const OzPB pb = a.pbs[tl.pb];
                for (int q = npass - 1; q >= 0 && ok; --q) {
                    int g0, g1;
                    pass_groups(q, g0, g1);
                    const uint32_t planes = uint32_t(g1);  // planes 0 .. g1 - 1
                    for (uint32_t kt = pb.slab_begin; kt < pb.slab_end; ++kt, ++gs) {
                        const uint32_t st = gs % nst;
                        if (gs >= nst && !mbar_wait(&empty[st], ((gs / nst) - 1) & 1u, a.err, a.wait_ns)) {
                            ok = false;
                            break;
                        }
                        const OzSlab sl = a.slabs[kt];
                        unsigned char* base = smem + st * stage_bytes;
                        mbar_expect_tx(&full[st], planes * (A_TILE + B_TILE));
                        bulk_load(base, a.A8 + (sl.a_off + uint64_t(tl.mt) * sl.a_ts) * s, planes * A_TILE,
                                  &full[st]);
                        bulk_load(base + a_room, a.B8 + (sl.b_off + uint64_t(tl.nt) * sl.b_ts) * s, planes * B_TILE,
                                  &full[st]);
                    }
                }
            }
            issued = gs;
        }
        __syncwarp();
    } else if (warp == OZ_MMA_WARP) {
        if (lane == 0) {
            const uint32_t idesc = idesc_i8(OZ_BM, OZ_BN);
            uint32_t gs = 0, rounds = 0;
            bool ok = true;
            for (uint32_t tile = blockIdx.x; tile < a.n_tiles && ok; tile += gridDim.x) {
                const OzPB pb = a.pbs[a.tiles[tile].pb];
                const uint32_t KT = pb.slab_end - pb.slab_begin;
                const uint32_t nch = KT ? (KT + a.chunk - 1) / a.chunk : 1;
                for (int q = npass - 1; q >= 0 && ok; --q) {
                    int g0, g1;
                    pass_groups(q, g0, g1);
                    for (uint32_t ch = 0; ch < nch && ok; ++ch) {
                        // the accumulators are free once the epilogue of the previous round has
                        // read them: the whole pass (128-column tiles) before the chunk, each group
                        // (64-column tiles) before its first product, largest g first as the
                        // epilogue releases them
                        if (NREL == 1 && rounds > 0 && !mbar_wait_suspend(tempty, (rounds - 1) & 1u, a.err)) {
                            ok = false;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint32_t k_begin = ch * a.chunk, k_end = min(KT, k_begin + a.chunk);
                        for (uint32_t kt = k_begin; kt < k_end && ok; ++kt, ++gs) {
                            const uint32_t st = gs % nst;
                            if (!mbar_wait(&full[st], (gs / nst) & 1u, a.err, a.wait_ns)) {
                                ok = false;
                                break;
                            }
                            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                            const uint32_t abase = smem_u32(smem + st * stage_bytes);
                            const uint32_t bbase = abase + a_room;
                            for (int g = g1 - 1; g >= g0; --g) {
                                if (NREL > 1 && kt == k_begin && rounds > 0) {
                                    if (!mbar_wait_suspend(&tempty[g - g0], (rounds - 1) & 1u, a.err)) {
                                        ok = false;
                                        break;
                                    }
                                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                                }
                                for (int pl = 0; pl <= g; ++pl)
                                    umma_i8(tmem + uint32_t((g - g0) * OZ_BN), umma_desc(abase + pl * A_TILE),
                                            umma_desc(bbase + (g - pl) * B_TILE), idesc,
                                            (kt > k_begin || pl > 0) ? 1u : 0u);
                            }
                            umma_commit(&empty[st]);  // the stage is free once these MMAs complete
                        }
                        if (!ok) break;
                        umma_commit(tfull);  // the chunk's sums are complete once every MMA issued so far is
                        ++rounds;
                    }
                }
            }
            *consumed_slot = gs;
            umma_commit(fin);  // every MMA this thread issued
        }
        __syncwarp();
    } else {
        // epilogue warps: TMEM lanes (warp % 4) * 32 .. + 31 are rows (warp % 4) * 32 .. of the
        // tile; the warp drains the columns half * OZ_BN / 2 .. of them
        const int quarter = warp & 3, half = warp >> 2;
        constexpr int HALF = OZ_BN / 2;
        uint32_t rounds = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; tile < a.n_tiles && ok; tile += gridDim.x) {
            const OzTile tl = a.tiles[tile];
            const OzPB pb = a.pbs[tl.pb];
            const uint32_t KT = pb.slab_end - pb.slab_begin;
            const uint32_t nch = KT ? (KT + a.chunk - 1) / a.chunk : 1;
            const uint32_t row = tl.mt * OZ_BM + quarter * 32 + lane;
            const int erow = (row < pb.M) ? a.e[pb.e_off + row] : 0;
            double* crow = nullptr;
            uint64_t ldc = pb.C.ld;
            if (row < pb.M) {
                // the row's start and leading dimension: from the row table or the plain operand
                if (pb.rowtab != DevProb::NO_ROWS) {
                    const DevRow rw = a.rowtab[pb.rowtab + row];
                    crow = reinterpret_cast<double*>(base_of(a.bases, pb.C.buf)) + rw.c_off +
                           uint64_t(pb.batch) * rw.cbs;
                    ldc = rw.ld;
                } else {
                    crow = reinterpret_cast<double*>(base_of(a.bases, pb.C.buf) + 8ull * pb.C.off) + row;
                }
            }
            bool first = true;  // the tile's first round writes C (adds when the problem has beta)
            for (int q = npass - 1; q >= 0 && ok; --q) {
                int g0, g1;
                pass_groups(q, g0, g1);
                for (uint32_t ch = 0; ch < nch; ++ch) {
                    if (!mbar_wait_suspend(tfull, rounds & 1u, a.err)) {
                        ok = false;
                        break;
                    }
                    ++rounds;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const bool add = pb.beta || !first;
                    first = false;
                    if constexpr (OZ_BN == 64) {
                        // read the groups largest g first, releasing each as soon as all eight
                        // warps have read it, then scale and store the warp's 32 sums
                        double acc[HALF];
#pragma unroll
                        for (int j = 0; j < HALF; ++j) acc[j] = 0.0;
                        for (int g = g1 - 1; g >= g0; --g) {
                            if (KT > 0) {
                                const double w = pow2_normal(-7 * (g + 2));
                                const uint32_t taddr =
                                    tmem + (uint32_t(quarter * 32) << 16) + uint32_t((g - g0) * OZ_BN + half * HALF);
                                int32_t v[32];
                                tmem_ld16(taddr, v);
                                tmem_ld16(taddr + 16, v + 16);
                                tmem_wait_ld();
#pragma unroll
                                for (int j = 0; j < 32; ++j) acc[j] += i2d_exact(v[j]) * w;
                            }
                            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                            __syncwarp();
                            if (lane == 0) mbar_arrive(&tempty[g - g0]);
                        }
                        if (crow) {
#pragma unroll
                            for (int j = 0; j < HALF; ++j) {
                                const uint32_t col = tl.nt * OZ_BN + half * HALF + j;
                                if (col < pb.N) {
                                    // x 2^(e_row + e_col): one multiplication by the exact power
                                    // where it is normal (the value ldexp gives), ldexp otherwise
                                    const int ex = erow + a.e[pb.f_off + col];
                                    const double val =
                                        (ex >= -1022 && ex <= 1023) ? acc[j] * pow2_normal(ex) : ldexp(acc[j], ex);
                                    double* dst = crow + uint64_t(col) * ldc;
                                    *dst = add ? *dst + val : val;
                                }
                            }
                        }
                    } else {
                    for (int c0 = half * HALF; c0 < (half + 1) * HALF; c0 += 32) {
                        double acc[32];
#pragma unroll
                        for (int j = 0; j < 32; ++j) acc[j] = 0.0;
                        for (int g = g1 - 1; g >= g0 && KT > 0; --g) {
                            const double w = pow2_normal(-7 * (g + 2));
                            int32_t v[32];
                            const uint32_t taddr = tmem + (uint32_t(quarter * 32) << 16) + uint32_t((g - g0) * OZ_BN + c0);
                            tmem_ld16(taddr, v);
                            tmem_ld16(taddr + 16, v + 16);
                            tmem_wait_ld();
#pragma unroll
                            for (int j = 0; j < 32; ++j) acc[j] += i2d_exact(v[j]) * w;
                        }
                        if (crow) {
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                const uint32_t col = tl.nt * OZ_BN + c0 + j;
                                if (col < pb.N) {
                                    // x 2^(e_row + e_col): one multiplication by the exact power
                                    // where it is normal (the value ldexp gives), ldexp otherwise
                                    const int ex = erow + a.e[pb.f_off + col];
                                    const double val =
                                        (ex >= -1022 && ex <= 1023) ? acc[j] * pow2_normal(ex) : ldexp(acc[j], ex);
                                    double* dst = crow + uint64_t(col) * ldc;
                                    *dst = add ? *dst + val : val;
                                }
                            }
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(tempty);
                    }
                }
            }
        }
    }
    __syncthreads();
    if (warp == OZ_MMA_WARP && lane == 0) oz_settle(fin, 0, a.err);
    if (warp == OZ_LOAD_WARP && lane == 0) {
        // copies still in flight after a stop land before the CTA leaves; slabs are issued
        // and consumed in order, so they are the slabs consumed .. issued - 1
        for (uint32_t g = *consumed_slot; g < issued; ++g) oz_settle(&full[g % nst], (g / nst) & 1u, a.err);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

}  // namespace

size_t ozaki_smem_bytes(int s, int bn) {
    return size_t(oz_stages(s, bn)) * s * (A_TILE + bn * OZ_BK) + OZ_BAR_BYTES;
}

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
    int bn = 64;                    // output tile columns (64 or 128)
    bool const_ready = false;       // constant digit planes present in the scratch
    std::vector<DevRow> rowtab;     // rows of row-table problems (the GEMM list's table)
    // first warp item of every job in the exponent and split passes (jobs + 1 entries)
    std::vector<uint64_t> exp_first, split_first;
    OzSplit* d_jobs = nullptr;
    uint64_t* d_exp_first = nullptr;
    uint64_t* d_split_first = nullptr;
    OzPB* d_pbs = nullptr;
    OzSlab* d_slabs = nullptr;
    OzTile* d_tiles = nullptr;
    DevRow* d_rowtab = nullptr;
};

OzProgram* oz_build(GemmList const& gl) {
    auto* oz = new OzProgram;
    std::vector<uint32_t> nbatch(gl.probs.size(), 0);
    for (auto const& t : gl.tiles) nbatch[t.prob] = std::max(nbatch[t.prob], t.batch + 1);
    // Tile width: 128-column tiles run the tensor pipe at twice the rate of 64-column
    // ones but need two passes over K for more than 4 digit groups (reading the digit
    // planes 11/7 times as often at s = 7) and twice the epilogue per tile; they pay where
    // the tiles' K walks are long (>= 32 slabs on average) and the columns fill them
    {
        uint64_t tiles64 = 0, tiles128 = 0, slabs64 = 0, area64 = 0, area128 = 0;
        for (uint32_t p = 0; p < gl.probs.size(); ++p) {
            DevProb const& pr = gl.probs[p];
            uint64_t kt = 0;
            for (uint32_t sgi = pr.seg_begin; sgi < pr.seg_end; ++sgi) kt += (gl.segs[sgi].K + OZ_BK - 1) / OZ_BK;
            const uint64_t mt = std::max<uint32_t>(1, (pr.M + OZ_BM - 1) / OZ_BM) * uint64_t(nbatch[p]);
            const uint64_t n64 = std::max<uint32_t>(1, (pr.N + 63) / 64), n128 = std::max<uint32_t>(1, (pr.N + 127) / 128);
            tiles64 += mt * n64;
            tiles128 += mt * n128;
            slabs64 += mt * n64 * kt;
            area64 += mt * n64 * 64 * kt;
            area128 += mt * n128 * 128 * kt;
        }
        // ... and where the wider tiles still give every SM two of them
        oz->bn = (tiles64 && slabs64 >= 32 * tiles64 && area128 * 100 <= area64 * 115 &&
                  tiles128 >= 2 * uint64_t(device_sm_count()))
                     ? 128
                     : 64;
        // DMRGB200_OZ_BN=64 or 128 forces the width for programs built while it is set
        if (const char* v = std::getenv("DMRGB200_OZ_BN")) {
            if (!std::strcmp(v, "64")) oz->bn = 64;
            if (!std::strcmp(v, "128")) oz->bn = 128;
        }
    }
    const uint32_t OZ_BN = uint32_t(oz->bn), B_TILE = OZ_BN * OZ_BK;
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
                ja.tr = OZ_BM;
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
                jb.tr = OZ_BN;
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
            // the tiles that share the larger operand's digit tile next to each other: CTAs that
            // start together read the same tile of it, so it comes from DRAM once and from L2 for
            // the others (the smaller operand is re-read, from L2)
            if (pb.N > pb.M) {
                for (uint32_t nt = 0; nt < pb.NT; ++nt)
                    for (uint32_t mt = 0; mt < pb.MT; ++mt) oz->tiles.push_back(OzTile{pbi, mt, nt, 0});
            } else {
                for (uint32_t mt = 0; mt < pb.MT; ++mt)
                    for (uint32_t nt = 0; nt < pb.NT; ++nt) oz->tiles.push_back(OzTile{pbi, mt, nt, 0});
            }
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
    oz->exp_first.assign(1, 0);
    oz->split_first.assign(1, 0);
    for (auto const& j : oz->jobs) {
        oz->exp_first.push_back(oz->exp_first.back() + oz_exp_items(j));
        oz->split_first.push_back(oz->split_first.back() + oz_split_items(j, j.tr));
    }
    if (up(oz->jobs, &oz->d_jobs) != cudaSuccess || up(oz->exp_first, &oz->d_exp_first) != cudaSuccess ||
        up(oz->split_first, &oz->d_split_first) != cudaSuccess || up(oz->pbs, &oz->d_pbs) != cudaSuccess ||
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
    cudaFree(oz->d_exp_first);
    cudaFree(oz->d_split_first);
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
        // 8 warps a block; at most 8 blocks an SM, the warps stride over the items
        auto blocks = [&](std::vector<uint64_t> const& first) {
            const uint64_t items = first[j0 + nj] - first[j0];
            return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>((items + 7) / 8, uint64_t(sms) * 8)));
        };
        oz_exponents<<<blocks(oz->exp_first), 256, 0, st>>>(oz->d_jobs + j0, oz->d_exp_first + j0, nj, bs, c.e,
                                                            oz->d_rowtab);
        oz_split<<<blocks(oz->split_first), 256, 0, st>>>(oz->d_jobs + j0, oz->d_split_first + j0, nj, bs, c.e, s,
                                                          c.A8, c.B8, oz->d_rowtab);
    }
    oz->const_ready = true;
    if (!oz->tiles.empty()) {
        // the kernel of the program's tile width, its shared-memory limit raised once for all slice counts
        auto launch = [&](auto kernel, int bn) -> cudaError_t {
            size_t smem_max = 0;
            for (int sl = 2; sl <= OZ_MAX_SLICES; ++sl) smem_max = std::max(smem_max, ozaki_smem_bytes(sl, bn));
            cudaError_t ea = ensure_smem_limit(reinterpret_cast<const void*>(kernel), int(smem_max));
            if (ea != cudaSuccess) return ea;
            OzArgs args{c.A8, c.B8, c.e, oz->d_pbs, oz->d_slabs, oz->d_tiles, uint32_t(oz->tiles.size()),
                        oz_chunk_slabs(s), oz_stages(s, bn), s, bs, err, oz->d_rowtab, wait_limit_ns()};
            kernel<<<std::min<uint32_t>(uint32_t(oz->tiles.size()), uint32_t(sms)), OZ_THREADS, ozaki_smem_bytes(s, bn),
                     st>>>(args);
            return cudaSuccess;
        };
        cudaError_t el = oz->bn == 128 ? launch(ozaki_mma<128>, 128) : launch(ozaki_mma<64>, 64);
        if (el != cudaSuccess) return el;
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
