// Native-FP64 execution of a lowered plan on sm_100a.
//
// Stage 1 (T tasks) and stage 3 (cohort contractions) run as grouped,
// persistent GEMM launches over precomputed tile lists; every output tile is
// owned by exactly one CTA, which loops over the tile's K segments (for H psi:
// every cohort that writes the output block), so the result is written once,
// without atomics, and is bitwise reproducible.  Stage 2 (S build) gathers
// alpha-weighted T columns (Cohort::create_s_r / create_s, tasks.cpp:425-494).
//
// The FP64 inner product uses the FP64 tensor-core instruction
// mma.sync.m8n8k4.f64 (DMMA) on 64x64x16 CTA tiles, 4 warps of 32x32.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <tuple>
#include <string>
#include <unordered_map>

#include "../../include/dmrgb200.h"
#include "device.hpp"
#include "async_copy.cuh"

namespace dmrgb200 {

namespace {

// shared-memory row pitch of a tile of ROWS (m or n) columns: 8 words mod 32,
// which makes the fragment loads conflict-free
template <int ROWS>
__host__ __device__ constexpr int pitch() {
    return ROWS + 4;
}

__device__ __forceinline__ const double* op_base(Bases const& bs, DevOp const& op, uint32_t batch) {
    return reinterpret_cast<const double*>(base_of(bs, op.buf) + 8ull * (op.off + uint64_t(batch) * op.bstride));
}

// Kernels launched with programmatic stream serialisation (launch_pdl) may be
// scheduled while the previous kernel of the stream drains; each starts with this
// wait, so none touches memory before its predecessor has completed and its
// writes are visible.
__device__ __forceinline__ void wait_for_predecessor() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// 8-byte asynchronous global->shared copy; src_bytes = 0 writes a zero (out-of-range element).
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
    unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Shared-memory column swizzle of the operand tiles: row k stores column c at
// c ^ ((k >> 2) & 3).  With row pitches of 8 words mod 32, copies in which
// consecutive threads take consecutive k (the coalesced order for K-contiguous
// operands) then hit distinct banks, and the fragment loads of one 4-deep K
// step (one XOR constant) stay conflict-free.
__device__ __forceinline__ int swz(int k) { return (k >> 2) & 3; }

// One thread's copies of one operand tile over the K steps of a segment.  The
// operand tile is ROWS (m or n) x BK_ (k), stored in shared memory as
// [k][ROWS + pad]; a thread issues NC = ROWS * BK_ / NTHREADS 8-byte copies per
// K step.  When the operand's contiguous global dimension is m or n
// ("row-major copies": A not transposed or read through the row table, B
// transposed), the thread's copies share one row r = tid % ROWS and take
// k = kt + j * (NTHREADS / ROWS); otherwise they share k = kt = tid % BK_ and
// take rows r + j * (NTHREADS / BK_).  Copy j reads base + j * jstride; every
// K step advances base by kstep.  All byte strides, fixed per segment.
struct CopyStream {
    const char* base;
    const char* safe;  // a readable address for copies that fetch nothing
    uint64_t jstride, kstep;
    uint32_t mask;  // bit j: copy j's row lies inside the problem
    uint32_t r, kt;
    bool rowmajor;
};

template <int ROWS, int BK_, int NTHREADS, int LD>
__device__ __forceinline__ void issue_copies(double* tile, CopyStream& cs, uint32_t krem) {
    constexpr int NC = ROWS * BK_ / NTHREADS;
    if (cs.rowmajor) {
        constexpr int KJ = NTHREADS / ROWS;
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            const uint32_t k = cs.kt + j * KJ;
            const bool ok = ((cs.mask >> j) & 1u) && k < krem;
            cp_async8(&tile[k * LD + (cs.r ^ swz(k))],
                      reinterpret_cast<const double*>(ok ? cs.base + j * cs.jstride : cs.safe), ok);
        }
    } else {
        constexpr int RJ = NTHREADS / BK_;
        const bool kok = cs.kt < krem;
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            const bool ok = kok && ((cs.mask >> j) & 1u);
            cp_async8(&tile[cs.kt * LD + ((cs.r + j * RJ) ^ swz(cs.kt))],
                      reinterpret_cast<const double*>(ok ? cs.base + j * cs.jstride : cs.safe), ok);
        }
    }
    cs.base += cs.kstep;
}

// Copy stream of an operand whose element (row, k) sits at elem + row * rs + k * ks
// (element strides; rows from row0, nrows of them inside the problem).
template <int ROWS, int BK_, int NTHREADS>
__device__ __forceinline__ void setup_copies(CopyStream& cs, const double* elem, uint64_t rs, uint64_t ks,
                                             uint32_t row0, uint32_t nrows, int tid) {
    constexpr int NC = ROWS * BK_ / NTHREADS;
    cs.safe = reinterpret_cast<const char*>(elem);
    cs.rowmajor = rs == 1;
    if (cs.rowmajor) {
        constexpr int KJ = NTHREADS / ROWS;
        cs.r = tid % ROWS;
        cs.kt = tid / ROWS;
        cs.base = reinterpret_cast<const char*>(elem + (row0 + cs.r) + cs.kt * ks);
        cs.jstride = 8ull * KJ * ks;
        cs.kstep = 8ull * BK_ * ks;
        cs.mask = row0 + cs.r < nrows ? (1u << NC) - 1u : 0u;
    } else {
        constexpr int RJ = NTHREADS / BK_;
        cs.kt = tid % BK_;
        cs.r = tid / BK_;
        cs.base = reinterpret_cast<const char*>(elem + (row0 + cs.r) * rs + cs.kt * ks);
        cs.jstride = 8ull * RJ * rs;
        cs.kstep = 8ull * BK_ * ks;
        cs.mask = 0;
#pragma unroll
        for (int j = 0; j < NC; ++j)
            if (row0 + cs.r + j * RJ < nrows) cs.mask |= 1u << j;
    }
}

// Grouped, persistent FP64 GEMM over a tile list.  Each CTA owns whole output
// tiles (BM_ x 64) and walks every K step (BK_ deep) of every segment of its
// problem; the CTA's K steps over all its tiles form one stream, so the
// cp.async pipeline (STAGES deep) keeps loading the next tile's operands while
// the current tile finishes and stores.  Warps: 2 x 2 of (BM_/2) x 32 (BM_ = 32,
// 64), or for BM_ = 16 a row of 16 x (64 / warps), DMMA m8n8k4.  A tile whose segments are all
// empty (one step, no copies) stores zeros.
struct LoadCursor {
    uint32_t ti, seg, seg_end, krem;
    bool valid;
};

template <int BM_, int BN_, int BK_, int STAGES, int MINB, int NTHREADS, int WARPS_M>
__global__ void __launch_bounds__(NTHREADS, MINB) gemm_f64_grouped(const DevProb* __restrict__ probs,
                                                                   const DevSeg* __restrict__ segs,
                                                                   const DevTile* __restrict__ tiles, uint32_t n_tiles,
                                                                   const DevRow* __restrict__ rowtab, Bases bases) {
    // warps: WARPS_M x (warps / WARPS_M), warp tiles WM x WN of 8 x 8 DMMA tiles
    constexpr int WM = BM_ / WARPS_M;
    constexpr int WN = BN_ / (NTHREADS / 32 / WARPS_M), NJ = WN / 8;
    constexpr int MI = WM / 8;  // 8 x 8 accumulator tiles (m8n8k4)
    constexpr int NCA = BM_ * BK_ / NTHREADS;
    static_assert(MI >= 1 && NJ >= 1 && NTHREADS % BM_ == 0 && NTHREADS % BN_ == 0 && NTHREADS % BK_ == 0,
                  "tile shape");
    __shared__ __align__(16) double As[STAGES][BK_][pitch<BM_>()];
    __shared__ __align__(16) double Bs[STAGES][BK_][pitch<BN_>()];
    wait_for_predecessor();

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int wm = (warp % WARPS_M) * WM, wn = (warp / WARPS_M) * WN;
    const int g = lane >> 2, q = lane & 3;

    // ---- producer: walks (tile, segment, K step) and issues one K step per call;
    // the copy streams are set up once per segment ----
    LoadCursor L{blockIdx.x, 0, 0, 0, false};
    CopyStream ca, cb;
    auto enter_segment = [&]() {
        while (L.seg < L.seg_end && segs[L.seg].K == 0) ++L.seg;
        if (L.seg >= L.seg_end) return;
        const DevTile tl = tiles[L.ti];
        const DevProb& pr = probs[tl.prob];
        const DevSeg sg = segs[L.seg];
        L.krem = sg.K;
        const double* A = op_base(bases, sg.A, tl.batch);
        const double* B = op_base(bases, sg.B, tl.batch);
        if (pr.rows != DevProb::NO_ROWS) {
            // row-table A: this thread's row (tid % BM_ in every copy) has its own start and stride
            const uint32_t gm = tl.m0 + uint32_t(tid % BM_);
            ca.safe = reinterpret_cast<const char*>(B);
            ca.rowmajor = true;
            ca.r = tid % BM_;
            ca.kt = tid / BM_;
            ca.mask = 0;
            ca.base = ca.safe;
            ca.jstride = ca.kstep = 0;
            if (gm < pr.M) {
                const DevRow rw = rowtab[pr.rows + gm];
                ca.base = reinterpret_cast<const char*>(base_of(bases, sg.A.buf) + 8ull * (rw.a_off + uint64_t(ca.kt) * rw.ld));
                ca.jstride = 8ull * (NTHREADS / BM_) * rw.ld;
                ca.kstep = 8ull * BK_ * rw.ld;
                ca.mask = (1u << NCA) - 1u;
            }
        } else if (!sg.A.trans) {
            setup_copies<BM_, BK_, NTHREADS>(ca, A, 1, sg.A.ld, tl.m0, pr.M, tid);
        } else {
            setup_copies<BM_, BK_, NTHREADS>(ca, A, sg.A.ld, 1, tl.m0, pr.M, tid);
        }
        if (!sg.B.trans)
            setup_copies<BN_, BK_, NTHREADS>(cb, B, sg.B.ld, 1, tl.n0, pr.N, tid);
        else
            setup_copies<BN_, BK_, NTHREADS>(cb, B, 1, sg.B.ld, tl.n0, pr.N, tid);
    };
    auto enter_tile = [&]() {
        L.valid = L.ti < n_tiles;
        if (!L.valid) return;
        const DevProb& pr = probs[tiles[L.ti].prob];
        L.seg = pr.seg_begin;
        L.seg_end = pr.seg_end;
        enter_segment();
    };
    auto issue = [&](int slot) {
        if (!L.valid) return;
        if (L.seg < L.seg_end) {  // an empty tile issues no copies
            issue_copies<BM_, BK_, NTHREADS, pitch<BM_>()>(&As[slot][0][0], ca, L.krem);
            issue_copies<BN_, BK_, NTHREADS, pitch<BN_>()>(&Bs[slot][0][0], cb, L.krem);
            if (L.krem > uint32_t(BK_)) {
                L.krem -= BK_;
                return;
            }
            ++L.seg;
            enter_segment();
            if (L.seg < L.seg_end) return;
        }
        L.ti += gridDim.x;
        enter_tile();
    };

    enter_tile();
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        issue(s);
        cp_async_commit();
    }

    double acc[MI][NJ][2];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    // ---- consumer: tiles in the same order, nsteps K steps each ----
    int slot = 0;
    for (uint32_t ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const uint32_t nsteps = tiles[ti].nsteps;
        for (uint32_t st = 0; st < nsteps; ++st) {
            issue((slot + STAGES - 1) % STAGES);
            cp_async_commit();
            cp_async_wait<STAGES - 1>();
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < BK_; kk += 4) {
                double a[MI], b[NJ];
#pragma unroll
                for (int i = 0; i < MI; ++i) a[i] = As[slot][kk + q][(wm + i * 8 + g) ^ (kk >> 2)];
#pragma unroll
                for (int j = 0; j < NJ; ++j) b[j] = Bs[slot][kk + q][(wn + j * 8 + g) ^ (kk >> 2)];
#pragma unroll
                for (int i = 0; i < MI; ++i)
#pragma unroll
                    for (int j = 0; j < NJ; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
            }
            __syncthreads();
            slot = (slot + 1) % STAGES;
        }
        // epilogue (the next tile's first steps are already in flight); an empty
        // tile's single step multiplied zero-filled or stale shared memory, so its
        // accumulators are cleared instead of stored
        const DevTile tl = tiles[ti];
        const DevProb pr = probs[tl.prob];
        bool empty = true;
        for (uint32_t sg = pr.seg_begin; sg < pr.seg_end; ++sg) empty = empty && segs[sg].K == 0;
        const bool rowmode = pr.rows != DevProb::NO_ROWS;
        double* C = const_cast<double*>(op_base(bases, pr.C, tl.batch));
        const uint64_t ldc = pr.C.ld;
#pragma unroll
        for (int i = 0; i < MI; ++i) {
            const uint32_t r = tl.m0 + wm + i * 8 + g;
            // the row's start and leading dimension: from the row table or the plain operand
            double* crow = C + r;
            uint64_t ld = ldc;
            if (rowmode && r < pr.M) {
                const DevRow rw = rowtab[pr.rows + r];
                crow = reinterpret_cast<double*>(base_of(bases, pr.C.buf) + 8ull * (rw.c_off + tl.batch * rw.cbs));
                ld = rw.ld;
            }
#pragma unroll
            for (int j = 0; j < NJ; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    uint32_t c = tl.n0 + wn + j * 8 + q * 2 + e;
                    if (r < pr.M && c < pr.N) crow[c * ld] = empty ? 0.0 : acc[i][j][e];
                    acc[i][j][e] = 0.0;
                }
        }
    }
    cp_async_wait<0>();
}

// S build: S is tiled by cells (one per unit and MPO row block); a cell with a
// line writes the alpha-weighted sum of its T sources (summed in term order like
// the reference's axpy sequence), a cell without one writes zeros, so S needs
// no separate clearing.  One warp per work item (a line and a chunk of SB_CHUNK
// consecutive elements of its column-major walk): every lane owns SB_EPT elements
// (lane + 32 u); the line's terms are read 32 at a time, one per lane, and handed
// round by shuffles, so no block barrier is needed and the warps of a CTA, on
// neighbouring chunks of one line, share its term list through L1.
constexpr int SB_EPT = 4, SB_CHUNK = 32 * SB_EPT;
__global__ void __launch_bounds__(256) sbuild_lines(const DevSLine* __restrict__ lines,
                                                    const DevSTerm* __restrict__ terms,
                                                    const DevSItem* __restrict__ items, uint32_t n_items,
                                                    double* __restrict__ S, const double* __restrict__ T) {
    wait_for_predecessor();
    const uint32_t lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (uint32_t it = blockIdx.x * wpb + (threadIdx.x >> 5); it < n_items; it += gridDim.x * wpb) {
        const DevSItem I = items[it];
        const DevSLine L = lines[I.group];
        const uint32_t n = L.rows * L.cols;
        uint64_t toff[SB_EPT], soff[SB_EPT];
        bool in[SB_EPT];
        double v[SB_EPT];
#pragma unroll
        for (int u = 0; u < SB_EPT; ++u) {
            const uint32_t e = I.e0 + lane + 32u * u;
            in[u] = e < n;
            const uint32_t c = in[u] ? e / L.rows : 0, i = in[u] ? e - c * L.rows : 0;
            toff[u] = i + uint64_t(c) * L.ld_t;
            soff[u] = L.s_base + i + uint64_t(c) * L.ld_s;
            v[u] = 0.0;
        }
        for (uint32_t t0 = L.term_begin; t0 < L.term_end; t0 += 32) {
            const uint32_t nt = min(32u, L.term_end - t0);
            double my_a = 0.0;
            uint64_t my_b = 0;
            if (lane < nt) {
                const DevSTerm tm = terms[t0 + lane];
                my_a = tm.alpha;
                my_b = tm.t_base;
            }
            for (uint32_t t = 0; t < nt; ++t) {
                const double a = __shfl_sync(0xffffffffu, my_a, t);
                const uint64_t b = __shfl_sync(0xffffffffu, my_b, t);
#pragma unroll
                for (int u = 0; u < SB_EPT; ++u)
                    if (in[u]) v[u] += a * T[b + toff[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < SB_EPT; ++u)
            if (in[u]) S[soff[u]] = v[u];
    }
}

// S build of line groups (DevSGroup): one warp per work item (a group and a
// chunk of SG_CHUNK consecutive elements of its lines).  The chunk of every line is
// one product (elements x sources) * (sources x lines) on the FP64 tensor cores
// (DMMA m8n8k4: 8 elements x 8 lines x 4 sources per instruction, the warp holding
// SG_CHUNK x lines accumulators), so each source cell is read once for all lines of
// the group and one warp instruction does 256 multiply-adds.  The sources stream
// through the warp's own shared-memory ring with bulk copies (TMA engine, no
// multicast): a stage holds SGB_NC source rows of the chunk and their alpha
// columns; lanes 0 .. SGB_NC - 1 each copy one row and lane SGB_NC the alphas,
// every lane expecting its own bytes on the stage's mbarrier before lane 0
// arrives, SGB_STAGES - 1 stages ahead of the multiply-adds.  The copies bypass
// the L1 miss path, so a warp keeps kilobytes in flight without registers.  A
// bulk copy starts on a 16-byte boundary, so a row whose first element is odd is
// copied from one element earlier and read with that shift.  Every wait is
// bounded (2 s; the thread is suspended while it waits): on a timeout the warp
// records it in *err, lets its copies land (bounded) and stops.  Each line sums
// its sources in the group's entry order, four per DMMA.  The row pitch of a stage
// (SG_CHUNK + 4 doubles, 4 mod 16) puts the four sources of a K step in different
// banks for the fragment loads.
// Groups of up to 8 lines run as one launch (8 accumulated lines), larger groups as
// another (SG_LINES lines); both with 2 stages and 3 CTAs (12 warps) per SM, which caps
// the wide launch (its 128 x 16 accumulators included) at 168 registers.
constexpr int SGB_WARPS = 4, SGB_NC = 8, SGB_ROW = SG_CHUNK + 4;
template <int STAGES>
struct alignas(16) SgbRing {
    double rows[STAGES][SGB_NC][SGB_ROW];
    double alpha[STAGES][SGB_NC][SG_LINES];
    uint64_t full[STAGES];
    uint32_t shift[STAGES][SGB_NC];
};
static_assert(sizeof(double) * SGB_ROW % 16 == 0 && sizeof(SgbRing<2>) % 16 == 0 && sizeof(SgbRing<3>) % 16 == 0,
              "bulk copy alignment");
static_assert(SGB_NC < 32 && SGB_NC % 4 == 0, "one lane per row plus one for the alphas; whole DMMA K steps");
template <int NL>
struct SgbShape;
template <>
struct SgbShape<8> {
    static constexpr int STAGES = 2, MINB = 3;
};
template <>
struct SgbShape<SG_LINES> {
    static constexpr int STAGES = 2, MINB = 3;
};
template <int NL>
constexpr size_t sgb_smem() {
    return sizeof(SgbRing<SgbShape<NL>::STAGES>) * SGB_WARPS;
}

// One work item of the grouped S build with NL accumulated lines (NL = 8 for groups of
// at most 8 lines, SG_LINES otherwise; the alpha columns always hold SG_LINES entries).
// Returns false when a wait failed (the warp then stops).
template <int NL, int SGB_STAGES>
__device__ __forceinline__ bool sgb_item(SgbRing<SGB_STAGES>& R, DevSGroup const& G, uint32_t e0,
                                         const uint64_t* __restrict__ ent_t,
                                         const double* __restrict__ ent_a, double* __restrict__ S,
                                         const double* __restrict__ T, int* err, unsigned long long wait_ns,
                                         uint32_t lane, uint32_t& issued, uint32_t& consumed) {
    using namespace async;
    const uint32_t n = G.rows * G.cols, cnt = min(uint32_t(SG_CHUNK), n - e0);
    const uint32_t k0 = G.ent_begin, k1 = G.ent_end;
    constexpr int MT = SG_CHUNK / 8, NT = NL / 8;  // m8n8k4 tiles: elements x lines
    const uint32_t g = lane >> 2, q = lane & 3;
    double acc[MT][NT][2];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    // every lane: the stage of sources kb .. kb + SGB_NC - 1 (those below k1)
    auto fill = [&](uint32_t kb) {
        const uint32_t slot = issued % SGB_STAGES, nc = min(uint32_t(SGB_NC), k1 - kb);
        if (lane < nc) {
            const uint64_t tb = ent_t[kb + lane];
            const uint32_t sh = uint32_t((tb + e0) & 1u), sz = ((cnt + sh) * 8u + 15u) & ~15u;
            R.shift[slot][lane] = sh;
            mbar_expect_tx_only(&R.full[slot], sz);
            bulk_load(R.rows[slot][lane], T + tb + e0 - sh, sz, &R.full[slot]);
        } else if (lane == uint32_t(SGB_NC)) {
            const uint32_t sz = nc * SG_LINES * uint32_t(sizeof(double));
            mbar_expect_tx_only(&R.full[slot], sz);
            bulk_load(R.alpha[slot], ent_a + uint64_t(kb) * SG_LINES, sz, &R.full[slot]);
        }
        __syncwarp();  // every expected byte count is in before the phase can complete
        if (lane == 0) mbar_arrive(&R.full[slot]);
        ++issued;
    };
    const uint32_t nst = (k1 - k0 + SGB_NC - 1) / SGB_NC;
    for (uint32_t st = 0; st < min(nst, uint32_t(SGB_STAGES - 1)); ++st) fill(k0 + st * SGB_NC);
    for (uint32_t st = 0; st < nst; ++st) {
        const uint32_t slot = consumed % SGB_STAGES, kb = k0 + st * SGB_NC;
        // the stage SGB_STAGES - 1 ahead goes into the slot freed in the previous step
        if (st + SGB_STAGES - 1 < nst) {
            fence_proxy_async_smem();
            fill(k0 + (st + SGB_STAGES - 1) * SGB_NC);
        }
        const bool ok = mbar_wait_suspend(&R.full[slot], (consumed / SGB_STAGES) & 1u, err, wait_ns);
        if (__any_sync(0xffffffffu, !ok)) return false;
        const uint32_t nc = min(uint32_t(SGB_NC), k1 - kb);
        // D (elements x lines) += T (elements x 4 sources) * alpha (4 sources x lines) per
        // K step of four sources (a group's sources are padded to a multiple of four, so a
        // stage holds one or two whole steps); the alphas of both steps are read first
        double b[SGB_NC / 4][NT];
#pragma unroll
        for (int ks = 0; ks < SGB_NC / 4; ++ks) {
            const uint32_t c = uint32_t(ks * 4) + q;
#pragma unroll
            for (int j = 0; j < NT; ++j) b[ks][j] = c < nc ? R.alpha[slot][c][j * 8 + g] : 0.0;
        }
#pragma unroll
        for (int ks = 0; ks < SGB_NC / 4; ++ks) {
            if (uint32_t(ks * 4) >= nc) break;
            const uint32_t c = uint32_t(ks * 4) + q;
            const bool live = c < nc;
            const double* row = R.rows[slot][c] + R.shift[slot][c] + g;
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const double a = live ? row[i * 8] : 0.0;
#pragma unroll
                for (int j = 0; j < NT; ++j) dmma(acc[i][j][0], acc[i][j][1], a, b[ks][j]);
            }
        }
        ++consumed;
        __syncwarp();  // every lane's reads of this slot are done before it is refilled
    }
#pragma unroll
    for (int i = 0; i < MT; ++i) {
        const uint32_t e = e0 + uint32_t(i * 8) + g;
        if (e >= n) continue;
        const uint32_t col = e / G.rows, r = e - col * G.rows;
        double* dst = S + G.s_base + r + uint64_t(col) * G.ld_s;
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t line = uint32_t(j * 8) + 2u * q + uint32_t(h);
                if (line < G.nlines)
                    dst[uint64_t(line) * G.line_stride] = ((G.mask >> line) & 1u) ? acc[i][j][h] : 0.0;
            }
    }
    return true;
}

template <int NL>
__global__ void __launch_bounds__(32 * SGB_WARPS, SgbShape<NL>::MINB)
    sbuild_groups(const DevSGroup* __restrict__ groups, const DevSItem* __restrict__ items, uint32_t n_items,
                  const uint64_t* __restrict__ ent_t, const double* __restrict__ ent_a, double* __restrict__ S,
                  const double* __restrict__ T, int* err, unsigned long long wait_ns) {
    using namespace async;
    constexpr int SGB_STAGES = SgbShape<NL>::STAGES;
    extern __shared__ __align__(16) unsigned char sgb_smem_raw[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    SgbRing<SGB_STAGES>& R = reinterpret_cast<SgbRing<SGB_STAGES>*>(sgb_smem_raw)[warp];
    wait_for_predecessor();
    if (lane == 0) {
        for (int i = 0; i < SGB_STAGES; ++i) mbar_init(&R.full[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t issued = 0, consumed = 0;  // stage fills of this warp, in order (the same in every lane)
    bool failed = false;
    for (uint32_t it = blockIdx.x * SGB_WARPS + warp; it < n_items && !failed; it += gridDim.x * SGB_WARPS) {
        const DevSItem I = items[it];
        failed = !sgb_item<NL, SGB_STAGES>(R, groups[I.group], I.e0, ent_t, ent_a, S, T, err, wait_ns, lane, issued,
                                           consumed);
    }
    if (failed && lane == 0) {
        // let the copies still in flight land before the warp's shared memory is released (bounded)
        for (; consumed < issued; ++consumed) {
            const unsigned long long t0 = global_ns();
            while (!mbar_try(&R.full[consumed % SGB_STAGES], (consumed / SGB_STAGES) & 1u) &&
                   global_ns() - t0 < WAIT_LIMIT_NS) {
            }
        }
    }
}

// Register-resident DMMA loop for the FP64 tensor-core rate (calibration).
__global__ void __launch_bounds__(128) dmma_rate_loop(int iters, double* sink) {
    double acc[8][2];
    double a = 1.0 + threadIdx.x * 1e-9, b = 1.0 - threadIdx.x * 1e-9;
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) dmma(acc[i][0], acc[i][1], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1];
    if (s == 1.2345) sink[threadIdx.x] = s;
}

// --- host-side lowering ---------------------------------------------------------

// tile classes (rows x columns, K step): 0 = 32 x 64 / 16, 1 = 16 x 64 / 8,
// 2 = 64 x 64 / 16, 3 = 16 x 64 / 16 (two warps), 4 = 128 x 32 / 16, 5 = 64 x 32 / 8
constexpr int CLASS_BM[N_TILE_CLASSES] = {32, 16, 64, 16, 128, 64};
constexpr int CLASS_BN[N_TILE_CLASSES] = {64, 64, 64, 64, 32, 32};
constexpr int CLASS_BK[N_TILE_CLASSES] = {16, 8, 16, 16, 16, 8};

void add_tiles(GemmList& gl, uint32_t prob, uint32_t nbatch) {
    DevProb const& p = gl.probs[prob];
    for (int c = 0; c < N_TILE_CLASSES; ++c) {
        const uint32_t bm = CLASS_BM[c], bn = CLASS_BN[c], bk = CLASS_BK[c];
        uint32_t nsteps = 0;
        for (uint32_t s = p.seg_begin; s < p.seg_end; ++s) nsteps += (gl.segs[s].K + bk - 1) / bk;
        nsteps = std::max<uint32_t>(nsteps, 1);  // an empty problem: one step that issues no copies
        auto& out = c == 0 ? gl.tiles : gl.tiles_cls[c];
        for (uint32_t b = 0; b < nbatch; ++b)
            for (uint32_t m0 = 0; m0 < std::max<uint32_t>(p.M, 1); m0 += bm)
                for (uint32_t n0 = 0; n0 < std::max<uint32_t>(p.N, 1); n0 += bn)
                    out.push_back(DevTile{prob, b, m0, n0, nsteps});
    }
}

// Order tiles by decreasing K work so that the static round-robin of the
// persistent grid starts with the longest tiles (LPT-style balance).
void sort_tiles(GemmList& gl) {
    std::vector<uint64_t> kwork(gl.probs.size(), 0);
    for (size_t p = 0; p < gl.probs.size(); ++p)
        for (uint32_t s = gl.probs[p].seg_begin; s < gl.probs[p].seg_end; ++s) kwork[p] += gl.segs[s].K;
    for (int c = 0; c < N_TILE_CLASSES; ++c) {
        auto& tl = c == 0 ? gl.tiles : gl.tiles_cls[c];
        std::stable_sort(tl.begin(), tl.end(),
                         [&](DevTile const& a, DevTile const& b) { return kwork[a.prob] > kwork[b.prob]; });
    }
}

DevOp op(uint16_t buf, uint64_t off, uint32_t ld, bool trans, uint64_t bstride = 0) {
    DevOp o;
    o.off = off;
    o.bstride = bstride;
    o.ld = ld;
    o.buf = buf;
    o.trans = trans ? 1 : 0;
    return o;
}

}  // namespace

DevOp dev_op(uint16_t buf, uint64_t off, uint32_t ld, bool trans, uint64_t bstride) {
    return op(buf, off, ld, trans, bstride);
}
void gemm_add_tiles(GemmList& gl, uint32_t prob, uint32_t nbatch) { add_tiles(gl, prob, nbatch); }
void gemm_sort_tiles(GemmList& gl) { sort_tiles(gl); }

std::vector<uint64_t> t_offsets(FlatPlan const& p, uint64_t* total) {
    std::vector<uint64_t> off(p.n_t());
    uint64_t sum = 0;
    for (uint32_t t = 0; t < p.n_t(); ++t) {
        off[t] = sum;
        sum += round_up(p.t_size(t), 32);
    }
    if (total) *total = sum;
    return off;
}

std::vector<uint64_t> s_offsets(FlatPlan const& p, uint64_t* total) {
    std::vector<uint64_t> off(p.n_cohorts());
    uint64_t sum = 0;
    for (uint32_t c = 0; c < p.n_cohorts(); ++c) {
        off[c] = sum;
        sum += round_up(uint64_t(p.c_nsrows[c]) * p.c_stripe[c] * (p.kind == KIND_LEFT ? p.c_rs[c] : p.c_ls[c]), 32);
    }
    if (total) *total = sum;
    return off;
}

namespace {
// Stage 1 of H psi / right step with the rows of all T tasks that share a
// boundary cohort (same cohort, transposition and shape) stacked into one
// row-table problem: A row r is row r' of task t's psi slice, C row r is row r'
// of T_t (leading dimension = the task's row count), so one tile covers several
// small psi blocks instead of padding each to a full tile.
void stack_stage1(FlatPlan const& p, std::vector<uint64_t> const& stage1_bnd, std::vector<uint64_t> const& t_off,
                  GemmList& g1, std::vector<char> const* keep = nullptr) {
    g1 = GemmList();
    std::map<std::tuple<uint32_t, uint8_t, uint32_t, uint32_t, uint32_t>, std::vector<uint32_t>> groups;
    for (uint32_t t = 0; t < p.n_t(); ++t)
        if (!keep || (*keep)[t]) groups[{p.t_ci[t], p.t_trans[t], p.t_brows[t], p.t_bcols[t], p.t_nb[t]}].push_back(t);
    for (auto const& kv : groups) {
        const uint32_t t0 = kv.second.front();
        const uint32_t K = p.t_brows[t0], Nf = p.t_bcols[t0], nb = p.t_nb[t0];
        const bool tr = p.t_trans[t0] != 0;
        const uint64_t bnd = stage1_bnd.at(p.t_ci[t0]) / 8;
        DevProb pr;
        pr.rows = uint32_t(g1.rowtab.size());
        uint32_t M = 0;
        for (uint32_t t : kv.second) {
            const uint32_t Mt = p.in_rows[p.t_lb[t]];
            for (uint32_t r = 0; r < Mt; ++r)
                g1.rowtab.push_back(DevRow{p.in_off[p.t_lb[t]] + uint64_t(p.t_col[t]) * Mt + r, t_off[t] + r,
                                           tr ? uint64_t(Mt) * Nf : 0, Mt, 0});
            M += Mt;
        }
        pr.M = M;
        pr.C = op(BUF_T, 0, 0, false);
        DevSeg sg{};
        sg.A = op(BUF_IN, 0, 0, false);
        sg.K = K;
        uint32_t nbatch = 1;
        if (!tr) {
            // the nb stored blocks are adjacent K x Nf column blocks: one product of width nb * Nf
            pr.N = Nf * nb;
            sg.B = op(BUF_ABS, bnd, K, false, 0);
        } else {
            pr.N = Nf;
            sg.B = op(BUF_ABS, bnd, Nf, true, uint64_t(K) * Nf);
            nbatch = nb;
        }
        pr.seg_begin = uint32_t(g1.segs.size());
        g1.segs.push_back(sg);
        pr.seg_end = uint32_t(g1.segs.size());
        g1.probs.push_back(pr);
        add_tiles(g1, uint32_t(g1.probs.size() - 1), nbatch);
    }
    sort_tiles(g1);
}
}  // namespace

namespace {
// S build of one unit as line groups: groups of `width` (8 or SG_LINES) consecutive
// MPO row blocks, each with the union of its lines' source cells in address order
// and the summed alphas per (cell, line) (SG_LINES alpha slots per entry either
// way).  Returns the multiply-adds per element this issues (entries x the lines the
// kernel accumulates); `terms` receives the per-line walk's count.
struct UnitGroups {
    std::vector<DevSGroup> groups;
    std::vector<uint64_t> ent_t;
    std::vector<double> ent_a;
    std::vector<uint32_t> term_k, term_slot;  // plan term -> entry * SG_LINES + line
};
uint64_t group_unit(FlatPlan const& p, uint32_t c, uint32_t u, std::vector<int64_t> const& line_of,
                    std::vector<uint64_t> const& t_off, std::vector<uint64_t> const& s_off, UnitGroups& out,
                    uint64_t* terms, uint32_t width) {
    const bool left = p.kind == KIND_LEFT;
    const uint32_t ns = p.c_nsrows[c], ls = p.c_ls[c], rs = p.c_rs[c];
    std::unordered_map<uint64_t, uint32_t> slot;
    uint64_t fmas = 0;
    *terms = 0;
    for (uint32_t g0 = 0; g0 < ns; g0 += width) {
        DevSGroup G{};
        G.nlines = std::min<uint32_t>(width, ns - g0);
        if (left) {
            G.rows = p.u_ms[u];
            G.cols = rs;
            G.ld_s = p.c_stripe[c];
            G.line_stride = rs * p.c_stripe[c];
            G.s_base = s_off[c] + p.u_offset[u] + uint64_t(g0) * rs * p.c_stripe[c];
        } else {
            G.rows = ls;
            G.cols = p.u_ms[u];
            G.ld_s = ns * ls;
            G.line_stride = ls;
            G.s_base = s_off[c] + uint64_t(g0) * ls + uint64_t(p.u_offset[u]) * G.ld_s;
        }
        G.ent_begin = uint32_t(out.ent_t.size());
        slot.clear();
        const size_t map0 = out.term_k.size();
        for (uint32_t j = 0; j < G.nlines; ++j) {
            const int64_t l = line_of[g0 + j];
            if (l < 0) continue;
            for (uint32_t k = p.l_term[l]; k < p.l_term[l + 1]; ++k) {
                const uint64_t src = t_off[p.term_t[k]] + uint64_t(p.term_col[k]) * (left ? rs : ls);
                auto it = slot.find(src);
                uint32_t e;
                if (it == slot.end()) {
                    e = uint32_t(out.ent_t.size());
                    slot.emplace(src, e);
                    out.ent_t.push_back(src);
                    out.ent_a.insert(out.ent_a.end(), SG_LINES, 0.0);
                } else {
                    e = it->second;
                }
                out.ent_a[uint64_t(e) * SG_LINES + j] += p.term_alpha[k];
                out.term_k.push_back(k);
                out.term_slot.push_back((e - G.ent_begin) * SG_LINES + j);  // group-local until sorted
                G.mask |= 1u << j;
                ++*terms;
            }
        }
        G.ent_end = uint32_t(out.ent_t.size());
        // sources in address order: the warps on the groups of one unit then sweep
        // the shared T slices together (L1 / L2 reuse)
        {
            const uint32_t n = G.ent_end - G.ent_begin;
            std::vector<uint32_t> ord(n);
            std::iota(ord.begin(), ord.end(), 0u);
            std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
                return out.ent_t[G.ent_begin + a] < out.ent_t[G.ent_begin + b];
            });
            std::vector<uint64_t> t(n);
            std::vector<double> al(uint64_t(n) * SG_LINES);
            for (uint32_t x = 0; x < n; ++x) {
                t[x] = out.ent_t[G.ent_begin + ord[x]];
                std::copy_n(&out.ent_a[uint64_t(G.ent_begin + ord[x]) * SG_LINES], SG_LINES, &al[uint64_t(x) * SG_LINES]);
            }
            std::copy(t.begin(), t.end(), out.ent_t.begin() + G.ent_begin);
            std::copy(al.begin(), al.end(), out.ent_a.begin() + uint64_t(G.ent_begin) * SG_LINES);
            // the terms' slots follow their entries to the sorted positions
            std::vector<uint32_t> pos(n);
            for (uint32_t x = 0; x < n; ++x) pos[ord[x]] = x;
            for (size_t q = map0; q < out.term_slot.size(); ++q) {
                const uint32_t le = out.term_slot[q] / SG_LINES, j = out.term_slot[q] % SG_LINES;
                out.term_slot[q] = (G.ent_begin + pos[le]) * SG_LINES + j;
            }
        }
        // the kernel accumulates 8 lines for groups of up to 8, SG_LINES otherwise
        fmas += uint64_t(G.ent_end - G.ent_begin) * (G.nlines <= 8 ? 8u : uint32_t(SG_LINES));
        // the kernel walks sources SG_UNROLL at a time: pad with zero-alpha copies of the
        // group's first source.  A padded source is multiplied by zero, so it must read
        // written T elements: T blocks are padded to 32 elements and stage 1 never writes
        // the gaps, which may hold non-finite leftovers (0 * NaN = NaN in every line)
        while ((out.ent_t.size() - G.ent_begin) % SG_UNROLL) {
            const uint64_t first = out.ent_t[G.ent_begin];
            out.ent_t.push_back(first);
            out.ent_a.insert(out.ent_a.end(), SG_LINES, 0.0);
        }
        G.ent_end = uint32_t(out.ent_t.size());
        out.groups.push_back(G);
    }
    return fmas;
}

// DMRGB200_SBUILD: "lines" or "groups" forces one S-build form; anything else chooses per unit
int sbuild_mode() {
    const char* v = std::getenv("DMRGB200_SBUILD");
    if (!v) return 0;
    if (!std::strcmp(v, "lines")) return 1;
    if (!std::strcmp(v, "groups")) return 2;
    return 0;
}
}  // namespace

namespace {
// Stage 3 of H psi: one problem per output block (every cohort writing the block is
// a K segment of it); keep (optional) selects output blocks.
void build_stage3_hpsi(FlatPlan const& p, std::vector<uint64_t> const& stage3_bnd, std::vector<uint64_t> const& s_off,
                       GemmList& g3, std::vector<char> const* keep) {
    const uint32_t nc = p.n_cohorts();
    std::vector<std::vector<uint32_t>> by_out(p.out_rows.size());
    for (uint32_t c = 0; c < nc; ++c) by_out[p.c_rb[c]].push_back(c);
    for (uint32_t ob = 0; ob < p.out_rows.size(); ++ob) {
        if (keep && !(*keep)[ob]) continue;
        DevProb pr;
        pr.M = p.out_rows[ob];
        pr.N = p.out_cols[ob];
        pr.C = op(BUF_OUT, p.out_off[ob], pr.M, false, 0);
        pr.seg_begin = uint32_t(g3.segs.size());
        for (uint32_t c : by_out[ob]) {
            uint32_t ls = p.c_ls[c], rs = p.c_rs[c], ns = p.c_nsrows[c];
            uint64_t lbase = stage3_bnd.at(p.c_ci[c]) / 8;
            if (!p.c_trans[c]) {
                DevSeg sg{};
                sg.A = op(BUF_ABS, lbase, rs, false);
                sg.B = op(BUF_S, s_off[c], ns * ls, false);
                sg.K = ns * ls;
                g3.segs.push_back(sg);
            } else {
                // each stored block (ls x rs) is read transposed: one segment per MPO row block
                for (uint32_t b = 0; b < ns; ++b) {
                    DevSeg sg{};
                    sg.A = op(BUF_ABS, lbase + uint64_t(b) * ls * rs, ls, true);
                    sg.B = op(BUF_S, s_off[c] + uint64_t(b) * ls, ns * ls, false);
                    sg.K = ls;
                    g3.segs.push_back(sg);
                }
            }
        }
        pr.seg_end = uint32_t(g3.segs.size());
        g3.probs.push_back(pr);
        add_tiles(g3, uint32_t(g3.probs.size() - 1), 1);
    }
}
}  // namespace

void compile_program(FlatPlan const& p, std::vector<uint64_t> const& stage3_bnd,
                     std::vector<uint64_t> const& stage1_bnd, std::vector<uint64_t> const& outptr,
                     DeviceProgram& prog, bool stack_rows, bool group_lines) {
    prog = DeviceProgram();
    const uint32_t nt = p.n_t(), nc = p.n_cohorts();
    std::vector<uint64_t> t_off = t_offsets(p, &prog.t_elems);
    // slack after the last T block: the grouped S build's bulk copies may read one
    // element past a source row
    prog.t_elems += 32;

    // ---- stage 1 ----
    GemmList& g1 = prog.stage1;
    for (uint32_t t = 0; t < nt; ++t) {
        DevProb pr;
        DevSeg sg{};
        uint64_t bnd = stage1_bnd.at(p.t_ci[t]) / 8;
        if (p.kind == KIND_LEFT) {
            uint32_t M = p.t_brows[t], N = p.t_width[t], K = p.t_bcols[t];
            sg.A = op(BUF_ABS, bnd, p.t_trans[t] ? K : M, p.t_trans[t], uint64_t(M) * K);
            sg.B = op(BUF_IN, p.in_off[p.t_lb[t]] + uint64_t(p.t_col[t]) * K, K, false, 0);
            sg.K = K;
            pr.C = op(BUF_T, t_off[t], M, false, uint64_t(M) * N);
            pr.M = M;
            pr.N = N;
        } else {
            uint32_t M = p.in_rows[p.t_lb[t]], N = p.t_bcols[t], K = p.t_brows[t];
            sg.A = op(BUF_IN, p.in_off[p.t_lb[t]] + uint64_t(p.t_col[t]) * M, M, false, 0);
            sg.B = op(BUF_ABS, bnd, p.t_trans[t] ? N : K, p.t_trans[t], uint64_t(K) * N);
            sg.K = K;
            pr.C = op(BUF_T, t_off[t], M, false, uint64_t(M) * N);
            pr.M = M;
            pr.N = N;
            if (!p.t_trans[t]) {
                // the nb stored blocks are adjacent K x N column blocks: one GEMM of width nb * N
                pr.N = N * p.t_nb[t];
                pr.seg_begin = uint32_t(g1.segs.size());
                g1.segs.push_back(sg);
                pr.seg_end = uint32_t(g1.segs.size());
                g1.probs.push_back(pr);
                add_tiles(g1, uint32_t(g1.probs.size() - 1), 1);
                continue;
            }
        }
        pr.seg_begin = uint32_t(g1.segs.size());
        g1.segs.push_back(sg);
        pr.seg_end = uint32_t(g1.segs.size());
        g1.probs.push_back(pr);
        add_tiles(g1, uint32_t(g1.probs.size() - 1), p.t_nb[t]);
    }
    sort_tiles(g1);
    if (stack_rows && p.kind != KIND_LEFT && p.n_t()) {
        prog.stage1_tasks = std::move(prog.stage1);
        stack_stage1(p, stage1_bnd, t_off, prog.stage1);
    }

    // ---- stage 2 (S lines) ----
    std::vector<uint64_t> s_off = s_offsets(p, &prog.s_elems);
    // units tile the S columns (rows for the left step) and b1 its row blocks, so
    // the cells (unit, b1) cover S exactly once
    const int mode = group_lines ? sbuild_mode() : 1;
    UnitGroups ug;
    std::vector<std::pair<uint32_t, uint32_t>> ug_units;  // group range of every grouped unit
    for (uint32_t c = 0; c < nc; ++c) {
        for (uint32_t u = p.c_unit[c]; u < p.c_unit[c + 1]; ++u) {
            std::vector<int64_t> line_of(p.c_nsrows[c], -1);
            for (uint32_t l = p.u_line[u]; l < p.u_line[u + 1]; ++l) line_of[p.l_b1[l]] = l;
            const uint64_t w = uint64_t(p.u_ms[u]) * (p.kind == KIND_LEFT ? p.c_rs[c] : p.c_ls[c]);
            // the group construction is tried only where lines average 4 or more terms: sparser
            // units (Heisenberg, Hubbard: about two terms per line) keep the line walk without
            // paying for the trial, which would cost more host time than it could save
            const uint64_t unit_terms = p.l_term[p.u_line[u + 1]] - p.l_term[p.u_line[u]];
            const bool dense_enough = unit_terms >= 4ull * (p.u_line[u + 1] - p.u_line[u]);
            if (mode != 1 && w && (mode == 2 || dense_enough)) {
                // line groups when they issue at most twice the per-line walk's multiply-adds
                // (a unit without terms is zero-filled by the line walk)
                // wide groups read each shared source once for more lines; narrow ones waste
                // fewer multiply-adds on lines that do not read a source
                const size_t g0 = ug.groups.size(), e0 = ug.ent_t.size(), m0 = ug.term_k.size();
                bool grouped = false;
                for (uint32_t width : {uint32_t(SG_LINES), 8u}) {
                    uint64_t nterms = 0;
                    const uint64_t fmas = group_unit(p, c, u, line_of, t_off, s_off, ug, &nterms, width);
                    if (mode == 2 || (nterms && fmas <= 2 * nterms)) {
                        ug_units.emplace_back(uint32_t(g0), uint32_t(ug.groups.size()));
                        grouped = true;
                        break;
                    }
                    ug.groups.resize(g0);
                    ug.ent_t.resize(e0);
                    ug.ent_a.resize(e0 * SG_LINES);
                    ug.term_k.resize(m0);
                    ug.term_slot.resize(m0);
                }
                if (grouped) continue;
            }
            for (uint32_t b1 = 0; b1 < p.c_nsrows[c]; ++b1) {
                DevSLine L;
                L.term_begin = uint32_t(prog.terms.size());
                int64_t l = line_of[b1];
                if (p.kind == KIND_LEFT) {
                    L.ld_s = p.c_stripe[c];
                    L.rows = p.u_ms[u];
                    L.cols = p.c_rs[c];
                    L.ld_t = p.u_ms[u];
                    L.s_base = s_off[c] + p.u_offset[u] + uint64_t(b1) * p.c_rs[c] * p.c_stripe[c];
                    if (l >= 0)
                        for (uint32_t k = p.l_term[l]; k < p.l_term[l + 1]; ++k)
                            prog.terms.push_back(
                                DevSTerm{p.term_alpha[k], t_off[p.term_t[k]] + uint64_t(p.term_col[k]) * p.c_rs[c]});
                } else {
                    uint32_t ls = p.c_ls[c];
                    L.ld_s = p.c_nsrows[c] * ls;
                    L.rows = ls;
                    L.cols = p.u_ms[u];
                    L.ld_t = ls;
                    L.s_base = s_off[c] + uint64_t(b1) * ls + uint64_t(p.u_offset[u]) * L.ld_s;
                    if (l >= 0)
                        for (uint32_t k = p.l_term[l]; k < p.l_term[l + 1]; ++k)
                            prog.terms.push_back(
                                DevSTerm{p.term_alpha[k], t_off[p.term_t[k]] + uint64_t(p.term_col[k]) * ls});
                }
                L.term_end = uint32_t(prog.terms.size());
                if (uint64_t(L.rows) * L.cols) prog.lines.push_back(L);
            }
        }
    }
    // warp items of the lines: every line in chunks of SB_CHUNK elements, in line order
    for (uint32_t li = 0; li < prog.lines.size(); ++li) {
        const uint64_t n = uint64_t(prog.lines[li].rows) * prog.lines[li].cols;
        for (uint64_t e0 = 0; e0 < n; e0 += SB_CHUNK) prog.litems.push_back(DevSItem{li, uint32_t(e0)});
    }
    // warp items of the line groups: units by decreasing work, then group by
    // group, each group's element chunks consecutive (the warps of a CTA share the
    // group's source list and read its T slices in long contiguous runs; the
    // groups of a unit follow each other and reuse the unit's slices from L2)
    prog.groups = std::move(ug.groups);
    prog.gent_t = std::move(ug.ent_t);
    prog.gent_a = std::move(ug.ent_a);
    prog.gterm_k = std::move(ug.term_k);
    prog.gterm_slot = std::move(ug.term_slot);
    {
        std::vector<uint64_t> work(ug_units.size(), 0);
        for (size_t x = 0; x < ug_units.size(); ++x)
            for (uint32_t gi = ug_units[x].first; gi < ug_units[x].second; ++gi) {
                DevSGroup const& G = prog.groups[gi];
                work[x] += uint64_t(G.ent_end - G.ent_begin + 1) * G.rows * G.cols;
            }
        std::vector<uint32_t> order(ug_units.size());
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return work[a] > work[b]; });
        // groups of up to 8 lines first (their own launch), then the wide ones
        for (int wide = 0; wide < 2; ++wide) {
            for (uint32_t x : order) {
                const uint32_t g0 = ug_units[x].first, g1 = ug_units[x].second;
                if (g0 == g1) continue;
                const uint64_t n = uint64_t(prog.groups[g0].rows) * prog.groups[g0].cols;
                for (uint32_t gi = g0; gi < g1; ++gi) {
                    if ((prog.groups[gi].nlines > 8) != (wide == 1)) continue;
                    for (uint64_t e0 = 0; e0 < n; e0 += SG_CHUNK) prog.gitems.push_back(DevSItem{gi, uint32_t(e0)});
                }
            }
            if (!wide) prog.n_gitems8 = uint32_t(prog.gitems.size());
        }
    }

    // ---- stage 3 ----
    GemmList& g3 = prog.stage3;
    if (p.kind == KIND_HPSI) {
        build_stage3_hpsi(p, stage3_bnd, s_off, g3, nullptr);
    } else if (p.kind == KIND_RIGHT) {
        for (uint32_t c = 0; c < nc; ++c) {
            uint32_t ls = p.c_ls[c], rs = p.c_rs[c], ns = p.c_nsrows[c];
            DevProb pr;
            pr.M = ls;
            pr.N = rs;
            pr.C = op(BUF_ABS, outptr.at(p.c_out_ci[c]) / 8, ls, false, uint64_t(ls) * rs);
            DevSeg sg{};
            sg.A = op(BUF_S, s_off[c], ns * ls, false, ls);
            sg.B = op(BUF_OUT, p.out_off[p.c_rb[c]], rs, true, 0);
            sg.K = p.c_stripe[c];
            pr.seg_begin = uint32_t(g3.segs.size());
            g3.segs.push_back(sg);
            pr.seg_end = uint32_t(g3.segs.size());
            g3.probs.push_back(pr);
            add_tiles(g3, uint32_t(g3.probs.size() - 1), ns);
        }
    } else {
        for (uint32_t c = 0; c < nc; ++c) {
            uint32_t ls = p.c_ls[c], rs = p.c_rs[c], ns = p.c_nsrows[c], stripe = p.c_stripe[c];
            DevProb pr;
            pr.M = ls;
            pr.N = ns * rs;
            pr.C = op(BUF_ABS, outptr.at(p.c_out_ci[c]) / 8, ls, false, 0);
            DevSeg sg{};
            sg.A = op(BUF_OUT, p.out_off[p.c_lb[c]], stripe, true, 0);
            sg.B = op(BUF_S, s_off[c], stripe, false, 0);
            sg.K = stripe;
            pr.seg_begin = uint32_t(g3.segs.size());
            g3.segs.push_back(sg);
            pr.seg_end = uint32_t(g3.segs.size());
            g3.probs.push_back(pr);
            add_tiles(g3, uint32_t(g3.probs.size() - 1), 1);
        }
    }
    sort_tiles(g3);
}

namespace {
template <class T>
cudaError_t up(std::vector<T> const& v, T** d) {
    *d = nullptr;
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(d, v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}
}  // namespace

namespace {
// All tables of a program in one device allocation: packed into one host buffer
// (each table 256-byte aligned), copied with one transfer, freed with one call.
struct TablePacker {
    std::vector<unsigned char> host;
    static constexpr size_t NONE = ~size_t(0);
    template <class T>
    size_t add(std::vector<T> const& v) {
        if (v.empty()) return NONE;
        const size_t off = (host.size() + 255) / 256 * 256;
        host.resize(off + v.size() * sizeof(T));
        std::memcpy(host.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
    size_t zeros(size_t bytes) {
        const size_t off = (host.size() + 255) / 256 * 256;
        host.resize(off + bytes, 0);
        return off;
    }
};
template <class T>
T* at(unsigned char* base, size_t off) {
    return off == TablePacker::NONE ? nullptr : reinterpret_cast<T*>(base + off);
}
}  // namespace

cudaError_t upload_program(DeviceProgram& prog) {
    TablePacker pk;
    const size_t o_p1 = pk.add(prog.stage1.probs), o_s1 = pk.add(prog.stage1.segs), o_t1 = pk.add(prog.stage1.tiles);
    const size_t o_p3 = pk.add(prog.stage3.probs), o_s3 = pk.add(prog.stage3.segs), o_t3 = pk.add(prog.stage3.tiles);
    const size_t o_r1 = pk.add(prog.stage1.rowtab);
    size_t o_x1[N_TILE_CLASSES], o_x3[N_TILE_CLASSES];
    for (int c = 1; c < N_TILE_CLASSES; ++c) {
        o_x1[c] = pk.add(prog.stage1.tiles_cls[c]);
        o_x3[c] = pk.add(prog.stage3.tiles_cls[c]);
    }
    const size_t o_l = pk.add(prog.lines), o_k = pk.add(prog.terms), o_li = pk.add(prog.litems);
    const size_t o_g = pk.add(prog.groups), o_gt = pk.add(prog.gent_t), o_ga = pk.add(prog.gent_a);
    const size_t o_gi = pk.add(prog.gitems);
    const size_t o_err = prog.gitems.empty() ? TablePacker::NONE : pk.zeros(sizeof(int));
    prog.d_arena = nullptr;
    if (!pk.host.empty()) {
        cudaError_t e = cudaMalloc(&prog.d_arena, pk.host.size());
        if (e != cudaSuccess) return e;
        if ((e = cudaMemcpy(prog.d_arena, pk.host.data(), pk.host.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
    }
    unsigned char* b = prog.d_arena;
    prog.d_p1 = at<DevProb>(b, o_p1);
    prog.d_s1 = at<DevSeg>(b, o_s1);
    prog.d_t1 = at<DevTile>(b, o_t1);
    prog.d_p3 = at<DevProb>(b, o_p3);
    prog.d_s3 = at<DevSeg>(b, o_s3);
    prog.d_t3 = at<DevTile>(b, o_t3);
    prog.d_r1 = at<DevRow>(b, o_r1);
    for (int c = 1; c < N_TILE_CLASSES; ++c) {
        prog.x1.t[c] = at<DevTile>(b, o_x1[c]);
        prog.x3.t[c] = at<DevTile>(b, o_x3[c]);
        prog.x1.n[c] = uint32_t(prog.stage1.tiles_cls[c].size());
        prog.x3.n[c] = uint32_t(prog.stage3.tiles_cls[c].size());
    }
    prog.d_lines = at<DevSLine>(b, o_l);
    prog.d_terms = at<DevSTerm>(b, o_k);
    prog.d_litems = at<DevSItem>(b, o_li);
    prog.d_groups = at<DevSGroup>(b, o_g);
    prog.d_gent_t = at<uint64_t>(b, o_gt);
    prog.d_gent_a = at<double>(b, o_ga);
    prog.d_gitems = at<DevSItem>(b, o_gi);
    prog.d_err = at<int>(b, o_err);
    prog.n_t1 = uint32_t(prog.stage1.tiles.size());
    prog.n_t3 = uint32_t(prog.stage3.tiles.size());
    prog.n_lines = uint32_t(prog.lines.size());
    prog.n_litems = uint32_t(prog.litems.size());
    prog.n_gitems = uint32_t(prog.gitems.size());
    return cudaSuccess;
}

void free_program(DeviceProgram& prog) {
    cudaFree(prog.d_arena);
    prog.d_arena = nullptr;
    prog.d_p1 = nullptr;
    prog.d_s1 = nullptr;
    prog.d_t1 = nullptr;
    prog.d_p3 = nullptr;
    prog.d_s3 = nullptr;
    prog.d_t3 = nullptr;
    prog.d_r1 = nullptr;
    prog.x1 = TileLists();
    prog.x3 = TileLists();
    prog.d_lines = nullptr;
    prog.d_terms = nullptr;
    prog.d_litems = nullptr;
    prog.d_groups = nullptr;
    prog.d_gent_t = nullptr;
    prog.d_gent_a = nullptr;
    prog.d_gitems = nullptr;
    prog.d_err = nullptr;
}

namespace {
// cut points at block boundaries near equal shares of [0, total)
std::vector<uint64_t> cut_ranges(std::vector<uint64_t> const& block_off, uint64_t total, uint32_t nparts) {
    std::vector<uint64_t> starts(block_off);
    std::sort(starts.begin(), starts.end());
    std::vector<uint64_t> cut{0};
    for (uint32_t q = 1; q < nparts; ++q) {
        const uint64_t want = total * q / nparts;
        auto it = std::lower_bound(starts.begin(), starts.end(), want);
        uint64_t c = it == starts.end() ? total : *it;
        cut.push_back(std::max(c, cut.back()));
    }
    cut.push_back(total);
    return cut;
}
}  // namespace

cudaError_t compile_pipeline(FlatPlan const& p, std::vector<uint64_t> const& stage3_bnd,
                             std::vector<uint64_t> const& stage1_bnd, uint32_t nparts, PipelineProgram& pp) {
    pp = PipelineProgram();
    pp.nparts = nparts;
    std::vector<uint64_t> in_off(p.in_off.begin(), p.in_off.end()), out_off(p.out_off.begin(), p.out_off.end());
    pp.in_cut = cut_ranges(in_off, p.in_size, nparts);
    pp.out_cut = cut_ranges(out_off, p.out_size, nparts);
    const std::vector<uint64_t> t_off = t_offsets(p, nullptr), s_off = s_offsets(p, nullptr);
    pp.s1.resize(nparts);
    pp.s3.resize(nparts);
    for (uint32_t q = 0; q < nparts; ++q) {
        std::vector<char> keep_t(p.n_t()), keep_o(p.out_rows.size());
        for (uint32_t t = 0; t < p.n_t(); ++t) {
            const uint64_t o = p.in_off[p.t_lb[t]];
            keep_t[t] = o >= pp.in_cut[q] && o < pp.in_cut[q + 1];
        }
        for (uint32_t ob = 0; ob < p.out_rows.size(); ++ob)
            keep_o[ob] = p.out_off[ob] >= pp.out_cut[q] && p.out_off[ob] < pp.out_cut[q + 1];
        GemmList g1, g3;
        stack_stage1(p, stage1_bnd, t_off, g1, &keep_t);
        build_stage3_hpsi(p, stage3_bnd, s_off, g3, &keep_o);
        sort_tiles(g3);
        cudaError_t e;
        if ((e = upload_gemm(g1, pp.s1[q])) != cudaSuccess) return e;
        if ((e = upload_gemm(g3, pp.s3[q])) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void free_pipeline(PipelineProgram& pp) {
    for (auto& g : pp.s1) free_gemm(g);
    for (auto& g : pp.s3) free_gemm(g);
    pp = PipelineProgram();
}

cudaError_t run_pipeline(DeviceProgram const& prog, PipelineProgram const& pp, const double* x_host, double* y_host,
                         double* xd, double* yd, double* T, double* S, cudaStream_t s, cudaStream_t c,
                         cudaEvent_t const* ev) {
    const uint32_t np = pp.nparts;
    Bases bs{};
    bs.b[BUF_IN] = reinterpret_cast<uint64_t>(xd);
    bs.b[BUF_OUT] = reinterpret_cast<uint64_t>(yd);
    bs.b[BUF_T] = reinterpret_cast<uint64_t>(T);
    bs.b[BUF_S] = reinterpret_cast<uint64_t>(S);
    cudaError_t e;
    // the copies start after the work already queued on the caller's stream
    if ((e = cudaEventRecord(ev[0], s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(c, ev[0], 0)) != cudaSuccess) return e;
    for (uint32_t q = 0; q < np; ++q) {
        const uint64_t n = pp.in_cut[q + 1] - pp.in_cut[q];
        if (n && (e = cudaMemcpyAsync(xd + pp.in_cut[q], x_host + pp.in_cut[q], n * sizeof(double),
                                      cudaMemcpyHostToDevice, c)) != cudaSuccess)
            return e;
        if ((e = cudaEventRecord(ev[1 + q], c)) != cudaSuccess) return e;
    }
    for (uint32_t q = 0; q < np; ++q) {
        if ((e = cudaStreamWaitEvent(s, ev[1 + q], 0)) != cudaSuccess) return e;
        GemmDev g = pp.s1[q];
        g.var = prog.var1;
        if ((e = launch_gemm(g, bs, s)) != cudaSuccess) return e;
    }
    if ((e = run_sbuild(prog, T, S, s)) != cudaSuccess) return e;
    for (uint32_t q = 0; q < np; ++q) {
        GemmDev g = pp.s3[q];
        g.var = prog.var3;
        if ((e = launch_gemm(g, bs, s)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(ev[1 + np + q], s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(c, ev[1 + np + q], 0)) != cudaSuccess) return e;
        const uint64_t n = pp.out_cut[q + 1] - pp.out_cut[q];
        if (n && (e = cudaMemcpyAsync(y_host + pp.out_cut[q], yd + pp.out_cut[q], n * sizeof(double),
                                      cudaMemcpyDeviceToHost, c)) != cudaSuccess)
            return e;
    }
    if ((e = cudaEventRecord(ev[1 + 2 * np], c)) != cudaSuccess) return e;
    return cudaStreamWaitEvent(s, ev[1 + 2 * np], 0);
}

double calibrate_fp64_tflops() {
    const int sms = device_sm_count();
    double* sink = nullptr;
    cudaMalloc(&sink, 128 * sizeof(double));
    const int iters = 20000, blocks = sms * 8;
    dmma_rate_loop<<<blocks, 128>>>(1000, sink);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    dmma_rate_loop<<<blocks, 128>>>(iters, sink);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    // one m8n8k4 DMMA = 8*8*4 FMA = 512 flops per warp instruction
    double flops = double(blocks) * 4 /*warps*/ * iters * 8 * 512.0;
    return ms > 0 ? flops / (ms * 1e-3) / 1e12 : 0.0;
}

cudaError_t upload_gemm(GemmList const& gl, GemmDev& d) {
    cudaError_t e;
    if ((e = up(gl.probs, &d.p)) != cudaSuccess) return e;
    if ((e = up(gl.segs, &d.s)) != cudaSuccess) return e;
    if ((e = up(gl.tiles, &d.t)) != cudaSuccess) return e;
    if ((e = up(gl.rowtab, &d.r)) != cudaSuccess) return e;
    for (int c = 1; c < N_TILE_CLASSES; ++c) {
        if ((e = up(gl.tiles_cls[c], &d.x.t[c])) != cudaSuccess) return e;
        d.x.n[c] = uint32_t(gl.tiles_cls[c].size());
    }
    d.n = uint32_t(gl.tiles.size());

    return cudaSuccess;
}

void free_gemm(GemmDev& d) {
    cudaFree(d.p);
    cudaFree(d.s);
    cudaFree(d.t);
    for (int c = 1; c < N_TILE_CLASSES; ++c) cudaFree(d.x.t[c]);
    cudaFree(d.r);
    d = GemmDev();
}

namespace {
using GemmKernel = void (*)(const DevProb*, const DevSeg*, const DevTile*, uint32_t, const DevRow*, Bases);

// pipeline depth x CTAs per SM of the grouped GEMM, chosen per stage by the autotuner
struct GemmVariant {
    GemmKernel fn;
    const char* name;
    int tile_class;  // which tile list it runs on
    int threads;     // CTA size
};
const GemmVariant kVariants[N_GEMM_VARIANTS] = {
    {gemm_f64_grouped<32, 64, 16, 2, 4, 128, 2>, "tile32x64_k16_stages2_ctas4", 0, 128},
    {gemm_f64_grouped<32, 64, 16, 3, 4, 128, 2>, "tile32x64_k16_stages3_ctas4", 0, 128},
    {gemm_f64_grouped<32, 64, 16, 2, 5, 128, 2>, "tile32x64_k16_stages2_ctas5", 0, 128},
    {gemm_f64_grouped<32, 64, 16, 3, 5, 128, 2>, "tile32x64_k16_stages3_ctas5", 0, 128},
    {gemm_f64_grouped<16, 64, 8, 3, 6, 128, 1>, "tile16x64_k8_stages3_ctas6", 1, 128},
    {gemm_f64_grouped<16, 64, 8, 4, 8, 128, 1>, "tile16x64_k8_stages4_ctas8", 1, 128},
    {gemm_f64_grouped<64, 64, 16, 2, 3, 128, 2>, "tile64x64_k16_stages2_ctas3", 2, 128},
    {gemm_f64_grouped<64, 64, 16, 2, 2, 128, 2>, "tile64x64_k16_stages2_ctas2", 2, 128},
    {gemm_f64_grouped<16, 64, 16, 2, 8, 64, 1>, "tile16x64_k16_warps2_stages2_ctas8", 3, 64},
    {gemm_f64_grouped<16, 64, 16, 3, 8, 64, 1>, "tile16x64_k16_warps2_stages3_ctas8", 3, 64},
    {gemm_f64_grouped<16, 64, 16, 2, 10, 64, 1>, "tile16x64_k16_warps2_stages2_ctas10", 3, 64},
    {gemm_f64_grouped<16, 64, 16, 3, 10, 64, 1>, "tile16x64_k16_warps2_stages3_ctas10", 3, 64},
    {gemm_f64_grouped<128, 32, 16, 2, 2, 128, 4>, "tile128x32_k16_stages2_ctas2", 4, 128},
    {gemm_f64_grouped<128, 32, 16, 2, 3, 128, 4>, "tile128x32_k16_stages2_ctas3", 4, 128},
    {gemm_f64_grouped<64, 32, 8, 3, 4, 128, 2>, "tile64x32_k8_stages3_ctas4", 5, 128},
    {gemm_f64_grouped<64, 32, 8, 4, 5, 128, 2>, "tile64x32_k8_stages4_ctas5", 5, 128},
};

int variant_occupancy(int v) {
    static int occ[N_GEMM_VARIANTS] = {0};
    if (!occ[v]) {
        int o = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kVariants[v].fn, kVariants[v].threads, 0);
        occ[v] = o > 0 ? o : 1;
    }
    return occ[v];
}

// t / n: the tile list of class 0; x: the other classes (a variant whose list is
// absent falls back to variant 0)
// Launch with programmatic stream serialisation (the kernel must begin with
// wait_for_predecessor): its CTAs can be scheduled while the previous kernel's last
// CTAs finish, which hides most of the launch gap between the H·psi stages.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), uint32_t grid, uint32_t block, size_t smem, cudaStream_t stream,
                       Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

cudaError_t launch_variant(int v, const DevProb* p, const DevSeg* sg, const DevTile* t, uint32_t n,
                           TileLists const& x, const DevRow* rows, Bases const& bs, cudaStream_t stream) {
    if (!n) return cudaSuccess;
    if (v < 0 || v >= N_GEMM_VARIANTS) v = 0;
    const int c = kVariants[v].tile_class;
    if (c > 0 && !x.t[c]) v = 0;
    if (kVariants[v].tile_class > 0) {
        t = x.t[c];
        n = x.n[c];
    }
    uint32_t grid = std::min<uint32_t>(n, uint32_t(device_sm_count()) * variant_occupancy(v));
    return launch_pdl(kVariants[v].fn, grid, uint32_t(kVariants[v].threads), 0, stream, p, sg, t, n, rows, bs);
}
}  // namespace

const char* gemm_variant_name(int v) { return (v >= 0 && v < N_GEMM_VARIANTS) ? kVariants[v].name : "?"; }

cudaError_t launch_gemm(GemmDev const& d, Bases const& bs, cudaStream_t stream) {
    return launch_variant(d.var, d.p, d.s, d.t, d.n, d.x, d.r, bs, stream);
}

cudaError_t tune_program(DeviceProgram& prog, uint64_t in, uint64_t out, double* T, double* S, cudaStream_t stream) {
    Bases bs{};
    bs.b[BUF_IN] = in;
    bs.b[BUF_OUT] = out;
    bs.b[BUF_T] = reinterpret_cast<uint64_t>(T);
    bs.b[BUF_S] = reinterpret_cast<uint64_t>(S);
    cudaEvent_t e0, e1;
    cudaError_t e;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
        cudaEventDestroy(e0);
        return e;
    }
    struct Stage {
        const DevProb* p;
        const DevSeg* s;
        const DevTile* t;
        uint32_t n;
        TileLists x;
        const DevRow* r;
        int* var;
    } stages[2] = {{prog.d_p1, prog.d_s1, prog.d_t1, prog.n_t1, prog.x1, prog.d_r1, &prog.var1},
                   {prog.d_p3, prog.d_s3, prog.d_t3, prog.n_t3, prog.x3, nullptr, &prog.var3}};
    // stage 1 writes T, read by nothing else here; stage 3 reads S: both are timed on the
    // plan's current scratch contents (the kernels' speed does not depend on the values)
    // the clocks settle on a short run of the default variant first; then every
    // variant is timed once per round, round-robin, and keeps its best round, so a
    // clock ramp or a stray slow launch favours no variant; a variant must beat the
    // default by 1.5% to replace it (at QC L=24 m=2000 the 64x64 stage-3 variants run 4%
    // faster than the default inside H psi, which a 3% margin missed in some runs)
    constexpr int ROUNDS = 4;
    for (auto& st : stages) {
        if (!st.n) continue;
        for (int w = 0; w < 8 && e == cudaSuccess; ++w) e = launch_variant(0, st.p, st.s, st.t, st.n, st.x, st.r, bs, stream);
        float best_v[N_GEMM_VARIANTS];
        for (int v = 0; v < N_GEMM_VARIANTS; ++v) best_v[v] = 1e30f;
        for (int round = 0; round < ROUNDS && e == cudaSuccess; ++round)
            for (int v = 0; v < N_GEMM_VARIANTS && e == cudaSuccess; ++v) {
                cudaEventRecord(e0, stream);
                e = launch_variant(v, st.p, st.s, st.t, st.n, st.x, st.r, bs, stream);
                cudaEventRecord(e1, stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (round > 0 || v > 0) best_v[v] = std::min(best_v[v], ms);  // round 0 of v 0 is a warm-up
            }
        int bv = 0;
        for (int v = 1; v < N_GEMM_VARIANTS; ++v)
            if (best_v[v] < best_v[bv] * (bv == 0 ? 0.985f : 1.0f)) bv = v;
        *st.var = bv;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    prog.tuned = e == cudaSuccess;
    return e;
}

cudaError_t run_sbuild(DeviceProgram const& prog, double* T, double* S, cudaStream_t stream) {
    const uint32_t sms = uint32_t(device_sm_count());
    if (prog.n_litems) {
        // 8 warps per CTA, up to 8 CTAs per SM resident
        uint32_t grid = std::min<uint32_t>((prog.n_litems + 7) / 8, sms * 8);
        cudaError_t e = launch_pdl(sbuild_lines, grid, 256, 0, stream, static_cast<const DevSLine*>(prog.d_lines),
                                   static_cast<const DevSTerm*>(prog.d_terms),
                                   static_cast<const DevSItem*>(prog.d_litems), prog.n_litems, S,
                                   static_cast<const double*>(T));
        if (e != cudaSuccess) return e;
    }
    // the items of groups of up to 8 lines come first (prog.n_gitems8 of them)
    auto groups_launch = [&](auto kernel, size_t smem, int minb, const DevSItem* items, uint32_t n) -> cudaError_t {
        if (!n) return cudaSuccess;
        cudaError_t ea = ensure_smem_limit(reinterpret_cast<const void*>(kernel), int(smem));
        if (ea != cudaSuccess) return ea;
        // SGB_WARPS warps per CTA, minb CTAs per SM resident
        const uint32_t grid = std::min<uint32_t>((n + SGB_WARPS - 1) / SGB_WARPS, sms * uint32_t(minb));
        return launch_pdl(kernel, grid, 32 * SGB_WARPS, smem, stream, static_cast<const DevSGroup*>(prog.d_groups),
                          items, n, static_cast<const uint64_t*>(prog.d_gent_t),
                          static_cast<const double*>(prog.d_gent_a), S, static_cast<const double*>(T), prog.d_err,
                          wait_limit_ns());
    };
    if (prog.n_gitems) {
        const DevSItem* items = static_cast<const DevSItem*>(prog.d_gitems);
        cudaError_t e = groups_launch(sbuild_groups<8>, sgb_smem<8>(), SgbShape<8>::MINB, items, prog.n_gitems8);
        if (e != cudaSuccess) return e;
        e = groups_launch(sbuild_groups<SG_LINES>, sgb_smem<SG_LINES>(), SgbShape<SG_LINES>::MINB,
                          items + prog.n_gitems8, prog.n_gitems - prog.n_gitems8);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

bool sbuild_timed_out(DeviceProgram const& prog) {
    if (!prog.d_err) return false;
    int v = 0;
    if (cudaMemcpy(&v, prog.d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    if (v) cudaMemset(prog.d_err, 0, sizeof(int));
    return v != 0;
}

int device_sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

cudaError_t run_stages12(DeviceProgram const& prog, uint64_t in, uint64_t out, double* T, double* S,
                         cudaStream_t stream) {
    Bases bs{};
    bs.b[BUF_IN] = in;
    bs.b[BUF_OUT] = out;
    bs.b[BUF_T] = reinterpret_cast<uint64_t>(T);
    bs.b[BUF_S] = reinterpret_cast<uint64_t>(S);
    bs.b[BUF_ABS] = 0;
    launch_variant(prog.var1, prog.d_p1, prog.d_s1, prog.d_t1, prog.n_t1, prog.x1, prog.d_r1, bs, stream);
    cudaError_t e = run_sbuild(prog, T, S, stream);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t run_program(DeviceProgram const& prog, uint64_t in, uint64_t out, double* T, double* S,
                        cudaStream_t stream, cudaEvent_t const* ev) {
    Bases bs{};
    bs.b[BUF_IN] = in;
    bs.b[BUF_OUT] = out;
    bs.b[BUF_T] = reinterpret_cast<uint64_t>(T);
    bs.b[BUF_S] = reinterpret_cast<uint64_t>(S);
    bs.b[BUF_ABS] = 0;
    if (ev) cudaEventRecord(ev[0], stream);
    launch_variant(prog.var1, prog.d_p1, prog.d_s1, prog.d_t1, prog.n_t1, prog.x1, prog.d_r1, bs, stream);
    if (ev) cudaEventRecord(ev[1], stream);
    cudaError_t e = run_sbuild(prog, T, S, stream);
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[2], stream);
    launch_variant(prog.var3, prog.d_p3, prog.d_s3, prog.d_t3, prog.n_t3, prog.x3, nullptr, bs, stream);
    if (ev) cudaEventRecord(ev[3], stream);
    return cudaGetLastError();
}

}  // namespace dmrgb200

using namespace dmrgb200;

namespace dmrgb200 {
dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);
}

extern "C" dmrgb200_status dmrgb200_dgemm_f64(uint32_t M, uint32_t N, uint32_t K, const double* A, uint64_t lda,
                                              const double* B, uint64_t ldb, double* C, uint64_t ldc, int variant,
                                              void* cuda_stream) {
    if (!A || !B || !C) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (lda < M || ldb < K || ldc < M) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "leading dimension too small");
    if (variant < 0 || variant >= N_GEMM_VARIANTS) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "unknown variant");
    if (lda > UINT32_MAX || ldb > UINT32_MAX || ldc > UINT32_MAX)
        return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "leading dimension above 2^32");
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
    add_tiles(gl, 0, 1);
    GemmDev d;
    cudaError_t e = upload_gemm(gl, d);
    if (e == cudaSuccess) {
        d.var = variant;
        e = launch_gemm(d, Bases{}, st);
    }
    cudaError_t e2 = cudaStreamSynchronize(st);
    free_gemm(d);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess)
        return noalloc_fail(e == cudaErrorMemoryAllocation ? DMRGB200_OUT_OF_MEMORY : DMRGB200_DEVICE_ERROR,
                            std::string("FP64 GEMM: ") + cudaGetErrorString(e));
    return DMRGB200_OK;
}
