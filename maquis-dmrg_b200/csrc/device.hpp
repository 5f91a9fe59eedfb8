// Device program: a flat plan lowered to grouped-GEMM tile lists and S-build
// line lists, plus the launch entry points.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "plan.hpp"

namespace dmrgb200 {

// Operand of a grouped GEMM: element (r, c) of batch b lives at
//   base[buf] + off + b * bstride + (trans ? c + r * ld : r + c * ld)
// (row r = M/K index of A / B, column c = K/N index).
struct DevOp {
    uint64_t off;
    uint64_t bstride;
    uint32_t ld;
    uint16_t buf;
    uint16_t trans;
};

struct DevProb {
    DevOp C;
    uint32_t M, N;
    uint32_t seg_begin, seg_end;
    // row-table problems: row r of A and C is described by rowtab[rows + r] (the
    // A operand of every segment is then read through the table, not through A.off
    // and A.ld); NO_ROWS for plain problems
    uint32_t rows = NO_ROWS;
    static constexpr uint32_t NO_ROWS = 0xFFFFFFFFu;
};

// one row of a row-table problem: A(r, k) = base(A.buf)[a_off + k * ld] and
// C(r, c) of batch b = base(C.buf)[c_off + b * cbs + c * ld]
struct DevRow {
    uint64_t a_off, c_off, cbs;
    uint32_t ld, pad;
};

struct DevSeg {
    DevOp A, B;
    uint32_t K;
    uint32_t pad;
};

struct DevTile {
    uint32_t prob, batch, m0, n0;
    uint32_t nsteps;  // K steps of the tile over all its segments (at least 1)
};

struct DevSLine {
    uint64_t s_base;
    uint32_t ld_s, rows, cols, ld_t;
    uint32_t term_begin, term_end;
};

struct DevSTerm {
    double alpha;
    uint64_t t_base;
};

// S build of a unit in line groups: up to SG_LINES lines of consecutive MPO row
// blocks b1 share one list of source cells (the union of their terms' T
// slices), each with a column of SG_LINES alphas (zero where a line does not
// read the cell, duplicate sources of a line summed).  Line j of the group
// starts at s_base + j * line_stride; element (i, c) of a line sits at
// i + c * ld_s, its source at t_base + i + c * rows.
constexpr int SG_LINES = 16, SG_UNROLL = 4, SG_EPT = 4, SG_CHUNK = 32 * SG_EPT;
// cells of an adjoint T group (DevTGroup)
constexpr int TG_CELLS = 8;
struct DevSGroup {
    uint64_t s_base;
    uint32_t line_stride, ld_s, rows, cols;
    uint32_t ent_begin, ent_end;
    uint32_t mask;  // bit j: line j has terms (the others are written as zeros)
    uint32_t nlines;
};
// one warp's work in the S build: elements e0 .. e0 + 127 of a group (or of a line)
struct DevSItem {
    uint32_t group, e0;
};

enum BufId : uint16_t { BUF_IN = 0, BUF_OUT = 1, BUF_T = 2, BUF_S = 3, BUF_ABS = 4, BUF_W = 5, NBUF = 8 };

struct Bases {
    uint64_t b[NBUF];
};

#ifdef __CUDACC__
// device address of buffer `buf`: a select chain keeps the kernel-parameter
// array out of local memory
__device__ __forceinline__ uint64_t base_of(Bases const& bs, uint32_t buf) {
    uint64_t b = bs.b[0];
    b = buf == 1 ? bs.b[1] : b;
    b = buf == 2 ? bs.b[2] : b;
    b = buf == 3 ? bs.b[3] : b;
    b = buf == 4 ? bs.b[4] : b;
    b = buf == 5 ? bs.b[5] : b;
    return b;
}
#endif

template <class T>
struct DevArray {
    T* ptr = nullptr;
    size_t n = 0;
};

// tile classes of the grouped GEMM: 0 = 32 x 64 tiles with 16-deep K steps,
// 1 = 16 x 64 with 8-deep steps, 2 = 64 x 64 with 16-deep steps, 3 = 16 x 64
// with 16-deep steps
constexpr int N_TILE_CLASSES = 6;

struct GemmList {
    std::vector<DevProb> probs;
    std::vector<DevSeg> segs;
    std::vector<DevTile> tiles;                        // class 0
    std::vector<DevTile> tiles_cls[N_TILE_CLASSES];    // classes 1.. (entry 0 unused)
    std::vector<DevRow> rowtab;                        // rows of row-table problems
};

// device tile lists of the classes above 0
struct TileLists {
    DevTile* t[N_TILE_CLASSES] = {};
    uint32_t n[N_TILE_CLASSES] = {};
};

struct DeviceProgram {
    GemmList stage1, stage3;
    std::vector<DevSLine> lines;
    std::vector<DevSTerm> terms;
    // units whose lines share sources run as line groups (see DevSGroup)
    std::vector<DevSGroup> groups;
    std::vector<uint64_t> gent_t;  // per group entry: source offset in T
    std::vector<double> gent_a;    // per group entry: SG_LINES alphas
    std::vector<DevSItem> gitems;  // warp items of the groups
    std::vector<DevSItem> litems;  // warp items of the lines (DevSItem.group = line index)
    // host only: the plan terms of grouped units and their slot (entry * SG_LINES + line)
    // in the groups' entry tables (the adjoint reads <G line, T source> from there)
    std::vector<uint32_t> gterm_k, gterm_slot;
    uint64_t t_elems = 0, s_elems = 0;

    // device copies
    DevProb* d_p1 = nullptr;
    DevSeg* d_s1 = nullptr;
    DevTile* d_t1 = nullptr;
    DevProb* d_p3 = nullptr;
    DevSeg* d_s3 = nullptr;
    DevTile* d_t3 = nullptr;
    DevSLine* d_lines = nullptr;
    DevSTerm* d_terms = nullptr;
    DevSGroup* d_groups = nullptr;
    uint64_t* d_gent_t = nullptr;
    double* d_gent_a = nullptr;
    DevSItem* d_gitems = nullptr;
    DevSItem* d_litems = nullptr;
    int* d_err = nullptr;  // set by a grouped S build whose bulk-copy wait timed out
    unsigned char* d_arena = nullptr;  // the one allocation holding every table above
    uint32_t n_t1 = 0, n_t3 = 0, n_lines = 0, n_litems = 0, n_gitems = 0;
    uint32_t n_gitems8 = 0;  // gitems[0, n_gitems8): groups of up to 8 lines (the narrow launch)
    TileLists x1, x3;  // tile lists of the other classes
    DevRow* d_r1 = nullptr;  // stage-1 row table (stacked T tasks)
    GemmList stage1_tasks;   // stage 1 as one problem per T task (when stage1 is stacked)
    // grouped-GEMM variant per stage (autotuned by tune_program)
    int var1 = 0, var3 = 0;
    bool tuned = false;
};

// Lower a flat plan.  lptr/rptr: device address of each cohort's storage of the
// boundary read by stage 3 (H psi: L) and by stage 1 (H psi, right step: R;
// left step: L).  outptr: device address of each output boundary cohort (steps).
// stack_rows: stage 1 of H psi / right step as one row-table problem per set of
// T tasks that share their boundary cohort (rows of all those tasks stacked);
// the per-task list is kept in prog.stage1_tasks.
// group_lines: a unit whose lines share enough sources runs its S build as line
// groups (DevSGroup) when that issues at most twice the multiply-adds of the
// per-line walk; DMRGB200_SBUILD=lines / groups in the environment forces one
// form for every unit.
void compile_program(FlatPlan const& p, std::vector<uint64_t> const& stage3_bnd, std::vector<uint64_t> const& stage1_bnd,
                     std::vector<uint64_t> const& outptr, DeviceProgram& prog, bool stack_rows = false,
                     bool group_lines = false);
cudaError_t upload_program(DeviceProgram& prog);
void free_program(DeviceProgram& prog);

// Launch the three stages on a stream; T and S are the scratch buffers.
// ev (optional): four events recorded before stage 1 and after stages 1, 2, 3.
cudaError_t run_program(DeviceProgram const& prog, uint64_t in, uint64_t out, double* T, double* S,
                        cudaStream_t stream, cudaEvent_t const* ev = nullptr);

int device_sm_count();
// stages 1 and 2 only (T and the S build), as run_program launches them
cudaError_t run_stages12(DeviceProgram const& prog, uint64_t in, uint64_t out, double* T, double* S,
                         cudaStream_t stream);

// ---- density matrix of a split with the perturbation (alpha_dm.cu) ----
// One grouped-GEMM problem per bra block b of a step plan, written at dm[b]
// (stripe x stripe, column-major): Theta_b Theta_b^T + sum_c S_c S_c^T (left step) or
// Theta_b^T Theta_b + sum_c S_c^T S_c (right step), over the cohorts c of block b with
// S as the step's S build leaves it (scaled by sqrt(alpha) beforehand) and Theta the bra.
void build_alpha_dm(FlatPlan const& p, std::vector<uint64_t> const& dm, GemmList& gl);
cudaError_t scale_buffer(double* x, uint64_t n, double a, cudaStream_t st);

// ---- lowering helpers shared by the forward and adjoint programs ----
DevOp dev_op(uint16_t buf, uint64_t off, uint32_t ld, bool trans, uint64_t bstride = 0);
void gemm_add_tiles(GemmList& gl, uint32_t prob, uint32_t nbatch);
void gemm_sort_tiles(GemmList& gl);
// element offsets of the plan's T matrices / S matrices in the scratch buffers
std::vector<uint64_t> t_offsets(FlatPlan const& p, uint64_t* total);
std::vector<uint64_t> s_offsets(FlatPlan const& p, uint64_t* total);

struct GemmDev {
    DevProb* p = nullptr;
    DevSeg* s = nullptr;
    DevTile* t = nullptr;
    uint32_t n = 0;
    TileLists x;  // tile lists of the other classes
    DevRow* r = nullptr;  // row table
    int var = 0;  // grouped-GEMM variant
};
// grouped-GEMM variants (tile shape x pipeline depth x CTAs per SM); all sum in the
// same order, so the choice never changes a result bit
constexpr int N_GEMM_VARIANTS = 16;
const char* gemm_variant_name(int v);
// Time every variant on the program's stage-1 and stage-3 tile lists (on the given
// buffers, whose contents are overwritten as by an H psi) and keep the fastest per
// stage.  Must not run during stream capture.
cudaError_t tune_program(DeviceProgram& prog, uint64_t in, uint64_t out, double* T, double* S, cudaStream_t stream);
cudaError_t upload_gemm(GemmList const& gl, GemmDev& d);
void free_gemm(GemmDev& d);
// one persistent grouped-GEMM launch over the tile list
cudaError_t launch_gemm(GemmDev const& d, Bases const& bs, cudaStream_t stream);

// H psi with host buffers: stage 1 split by ranges of the input (the T tasks whose
// psi block lies in a range, stacked per range) and stage 3 by ranges of the output,
// so the host-device copies of one range overlap the products of another.  Every T
// element and output element is computed by the same tile walk as in the whole-plan
// program, so the results are bitwise the same.
struct PipelineProgram {
    uint32_t nparts = 0;
    std::vector<uint64_t> in_cut, out_cut;  // nparts + 1 element offsets each
    std::vector<GemmDev> s1, s3;            // device tile lists per range
};
cudaError_t compile_pipeline(FlatPlan const& p, std::vector<uint64_t> const& stage3_bnd,
                             std::vector<uint64_t> const& stage1_bnd, uint32_t nparts, PipelineProgram& pp);
void free_pipeline(PipelineProgram& pp);
// ev: 2 * nparts + 2 events; c: a second stream for the copies
cudaError_t run_pipeline(DeviceProgram const& prog, PipelineProgram const& pp, const double* x_host, double* y_host,
                         double* xd, double* yd, double* T, double* S, cudaStream_t s, cudaStream_t c,
                         cudaEvent_t const* ev);

// ---- adjoint of H psi (adjoint.cu) ----
// galpha term: <G cell, T cell> for plan term k
struct DevATerm {
    uint64_t g_base, t_base;
    uint32_t rows, cols, ld_g, ld_t;
    uint32_t k, pad;
};
// adjoint gT of up to TG_CELLS consecutive T blocks (cells) of one T task over the union
// of their G lines: cell c is rows x cols at out_base + c * rows * cols
struct DevTGroup {
    uint64_t out_base;
    uint32_t rows, cols, ncells;
    uint32_t ent_begin, ent_end;
    uint32_t mask;  // bit c: cell c has sources (the others are written as zeros)
};
// gT source: alpha * G cell at g_base with leading dimension ld
struct DevGTerm {
    double alpha;
    uint64_t g_base;
    uint32_t ld, pad;
};
struct AdjointProgram {
    GemmList g3;                    // G = L^T w per cohort (into the S scratch)
    GemmList g1;                    // gx slice = sum over its T tasks of gT * R^T
    std::vector<DevATerm> aterms;       // one per plan term
    std::vector<DevATerm> aterms_walk;  // the terms of ungrouped units (galpha term by term)
    std::vector<DevSLine> tlines;       // one per T block: gT cell = sum of its sources
    std::vector<DevGTerm> gterms;
    std::vector<DevSItem> tl_items;     // warp items of the T blocks: (block, 128-element chunk)
    // galpha of grouped units: Gram blocks per (group, entry batch), then one slot per term
    std::vector<DevSItem> gram_items;
    std::vector<uint32_t> gram_k, gram_slot;
    uint64_t gram_elems = 0;
    // gT of T blocks in cell groups: groups, warp items, and per entry the G line
    // (start, leading dimension) with SG_LINES alphas
    std::vector<DevTGroup> tgroups;
    std::vector<DevSItem> tg_items;
    std::vector<uint64_t> tg_g;
    std::vector<uint32_t> tg_ld;
    std::vector<double> tg_a;
    GemmDev d3, d1;
    DevATerm* d_aterms = nullptr;
    DevSLine* d_tlines = nullptr;
    DevGTerm* d_gterms = nullptr;
    DevSItem* d_tl_items = nullptr;
    DevSItem* d_gram_items = nullptr;
    uint32_t* d_gram_k = nullptr;
    uint32_t* d_gram_slot = nullptr;
    double* d_gram = nullptr;
    DevTGroup* d_tgroups = nullptr;
    DevSItem* d_tg_items = nullptr;
    uint64_t* d_tg_g = nullptr;
    uint32_t* d_tg_ld = nullptr;
    double* d_tg_a = nullptr;
    uint32_t n_aterms = 0, n_tlines = 0, n_tl_items = 0, n_gram_items = 0, n_gram_terms = 0, n_tg_items = 0;
};
// Lower the adjoint of an H psi plan; returns an empty string, or why the plan
// has none (overlapping T slices, a term that is not one whole T block).
std::string compile_adjoint(FlatPlan const& p, std::vector<uint64_t> const& stage3_bnd,
                            std::vector<uint64_t> const& stage1_bnd, DeviceProgram const& fwd, AdjointProgram& a);
cudaError_t upload_adjoint(AdjointProgram& a);
void free_adjoint(AdjointProgram& a);
// gx = H^T w (NULL: skipped), galpha[k] = <w|H_k x> (NULL: skipped)
cudaError_t run_adjoint(DeviceProgram const& fwd, AdjointProgram const& a, uint64_t w, uint64_t x, double* gx,
                        uint64_t gx_elems, double* galpha, double* T, double* S, cudaStream_t stream);
// stage 2 only (S build), for the emulated path
cudaError_t run_sbuild(DeviceProgram const& prog, double* T, double* S, cudaStream_t stream);
// after the stream is synchronised: whether a grouped S build timed out since the
// last call (the flag is cleared)
bool sbuild_timed_out(DeviceProgram const& prog);
// largest K of any output matrix of a GEMM list (emulation needs K * slices <= 2^17)

// ---- FP64 emulated on the INT8 tensor cores (ozaki.cu) ----
struct OzProgram;  // lowered grouped problem list
OzProgram* oz_build(GemmList const& gl);
void oz_free(OzProgram* oz);
// forget the cached digit planes of constant operands (their scratch was replaced)
void oz_invalidate(OzProgram* oz);
// device bytes the program needs for s digit planes (digits, exponents, error flag)
uint64_t oz_scratch_bytes(OzProgram const* oz, int s);
// run on the stream with scratch of oz_scratch_bytes(oz, s); `err` is a device word that
// records pipeline-wait timeouts (not cleared by oz_run; the reader clears it); returns a
// CUDA error
cudaError_t oz_run(OzProgram* oz, Bases const& bs, int s, void* scratch, int* err, cudaStream_t st);
// the digit planes of the constant (boundary) operands are in the scratch
bool oz_constants_ready(OzProgram const* oz);
// out[0] = sum (a - b)^2, out[1] = sum b^2 over n elements (device scalars)
cudaError_t diff_norms(const double* a, const double* b, uint64_t n, double* out, cudaStream_t st);
double calibrate_fp64_tflops();
// solver graph cache of a plan (jd_graph.cu)
void jd_graph_free(void* g);
// cuBLAS handle of the per-block comparison path (per_block.cpp)
void blas_handle_free(void* h);

// Limit of the bounded waits for pipeline data (grouped S build, emulated stages), in
// nanoseconds, read at every launch (dmrgb200_set_wait_limit).
inline std::atomic<unsigned long long> g_wait_limit_ns{2000000000ull};
inline unsigned long long wait_limit_ns() { return g_wait_limit_ns.load(std::memory_order_relaxed); }

// Raise a kernel's dynamic shared-memory limit once per (device, kernel): the
// attribute belongs to the kernel on the current device, so a process-wide flag
// would skip it on a second device.  Thread-safe.
inline cudaError_t ensure_smem_limit(const void* kernel, int bytes) {
    static std::mutex mu;
    static std::set<std::pair<int, const void*>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({dev, kernel})) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.insert({dev, kernel});
    return e;
}

}  // namespace dmrgb200
