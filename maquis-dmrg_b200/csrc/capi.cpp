// C ABI of libdmrgb200 (declarations in include/dmrgb200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"
#include "plan.hpp"
#include "schedule.hpp"
#include "coupling.hpp"

using namespace dmrgb200;

struct dmrgb200_context_s {
    int device = 0;
};

struct dmrgb200_mpo_s {
    MPOTensor mpo;
    Symm symm = Symm::U1;
};

struct dmrgb200_bindex_s {
    BoundaryIndex idx;
    std::vector<uint64_t> coh_off;  // storage offset per cohort, UINT64_MAX without storage
    uint64_t n_elems = 0;

    // 32-double aligned storage of every cohort that owns data
    void layout() {
        coh_off.assign(idx.n_cohorts(), std::numeric_limits<uint64_t>::max());
        n_elems = 0;
        for (unsigned ci = 0; ci < idx.n_cohorts(); ++ci) {
            uint64_t sz = idx.cohort_size(ci);
            if (!sz) continue;
            coh_off[ci] = n_elems;
            n_elems += round_up(sz, 32);
        }
    }
};

struct dmrgb200_schedule_s {
    FlatPlan flat;
};

struct dmrgb200_plan_s {
    FlatPlan flat;
    DeviceProgram prog;
    bool compiled = false;
    double* T = nullptr;
    double* S = nullptr;
    std::vector<uint64_t> stage1_bnd, stage3_bnd;
    int device = 0;
    // per-stage timing
    bool timing = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool pending = false;
    double stage_ms[3] = {0, 0, 0};
    uint64_t timed_calls = 0;
    // FP64 emulated on the INT8 tensor cores (built on first use)
    int slices = 7;
    int solve_prec = DMRGB200_PREC_FP64;  // precision of the H psi inside dmrgb200_solve
    OzProgram* oz1 = nullptr;
    OzProgram* oz3 = nullptr;
    void* oz_scratch = nullptr;   // stage-1 digit planes (the constant ones persist between calls)
    uint64_t oz_scratch_size = 0;
    void* oz_scratch3 = nullptr;  // stage-3 digit planes
    uint64_t oz_scratch3_size = 0;
    int* oz_err = nullptr;        // wait-timeout words of emulated stage 1 and stage 3
    // Jacobi-Davidson: solver mode and the cached solver graph
    int solver_mode = DMRGB200_SOLVER_GRAPH;
    void* jd = nullptr;
    // H psi with host buffers (built on first use): split program, device copies of x
    // and y, a copy stream and its events
    static constexpr uint32_t PIPE_PARTS = 4;
    bool pipe_built = false;
    PipelineProgram pipe;
    double* hx = nullptr;
    double* hy = nullptr;
    cudaStream_t copy_stream = nullptr, capture_stream = nullptr;
    cudaEvent_t pev[2 * PIPE_PARTS + 2] = {};
    // the whole host-buffer sequence as one CUDA graph, captured for one (x_host, y_host)
    // pair: 26 API calls per H psi cost more host time than the device takes
    cudaGraphExec_t pipe_exec = nullptr;
    const double* pipe_x = nullptr;
    double* pipe_y = nullptr;
    // boundary step: the lowered program of the last output binding, its T / S scratch
    // (reused while a caller keeps writing the same output boundary buffer)
    bool step_valid = false;
    std::vector<uint64_t> step_outp;
    DeviceProgram step_prog;
    double* step_T = nullptr;
    double* step_S = nullptr;
    void drop_step() {
        if (step_valid) free_program(step_prog);
        cudaFree(step_T);
        cudaFree(step_S);
        step_T = step_S = nullptr;
        step_valid = false;
        step_outp.clear();
    }
    // density matrix with the perturbation (dmrgb200_step_alpha_dm): the grouped GEMM
    // of the last dm binding
    bool dm_valid = false;
    std::vector<uint64_t> dm_ptrs;
    GemmDev dm_gemm;
    void drop_dm() {
        if (dm_valid) free_gemm(dm_gemm);
        dm_valid = false;
        dm_ptrs.clear();
    }
    // cuBLAS handle of the per-block comparison path (dmrgb200_hpsi_per_block)
    void* blas = nullptr;
    // adjoint program (built on first use)
    bool adj_built = false;
    std::string adj_err;
    AdjointProgram adj;

    void collect() {
        if (!pending) return;
        cudaEventSynchronize(ev[3]);
        for (int i = 0; i < 3; ++i) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
            stage_ms[i] += ms;
        }
        ++timed_calls;
        pending = false;
    }
};

namespace {

thread_local std::string g_last_error;

dmrgb200_status fail(dmrgb200_status s, std::string const& msg) {
    g_last_error = msg;
    return s;
}

dmrgb200_status cuda_fail(cudaError_t e, const char* where) {
    return fail(e == cudaErrorMemoryAllocation ? DMRGB200_OUT_OF_MEMORY : DMRGB200_DEVICE_ERROR,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define DMRGB200_TRY try {
#define DMRGB200_CATCH                                                              \
    }                                                                               \
    catch (std::bad_alloc const&) {                                                 \
        return fail(DMRGB200_OUT_OF_MEMORY, "host allocation failed");              \
    }                                                                               \
    catch (std::exception const& ex) {                                              \
        return fail(DMRGB200_INVALID_ARGUMENT, ex.what());                          \
    }

Symm to_symm(dmrgb200_symmetry s) {
    switch (s) {
        case DMRGB200_U1: return Symm::U1;
        case DMRGB200_TWOU1: return Symm::TwoU1;
        case DMRGB200_SU2U1: return Symm::SU2U1;
    }
    throw std::runtime_error("unknown symmetry");
}

Index to_index(const dmrgb200_index_desc* d) {
    if (!d) throw std::runtime_error("null index description");
    Index ix;
    for (uint32_t i = 0; i < d->n; ++i) {
        Charge c(d->charges[2 * i], d->charges[2 * i + 1]);
        if (ix.position(c) != ix.size()) throw std::runtime_error("duplicate charge in index");
        ix.push(c, d->sizes[i]);
    }
    return ix;
}

template <class T>
std::vector<T> vec(const T* p, size_t n) {
    if (n && !p) throw std::runtime_error("null array in plan description");
    return std::vector<T>(p, p + n);
}

void desc_to_flat(const dmrgb200_plan_desc* d, FlatPlan& f) {
    f.kind = d->kind;
    f.g_t = vec(d->g_t, size_t(d->n_groups) + 1);
    f.g_c = vec(d->g_c, size_t(d->n_groups) + 1);
    f.in_rows = vec(d->in_rows, d->n_in_blocks);
    f.in_cols = vec(d->in_cols, d->n_in_blocks);
    f.in_off = vec(d->in_off, d->n_in_blocks);
    f.in_size = d->in_size;
    f.out_rows = vec(d->out_rows, d->n_out_blocks);
    f.out_cols = vec(d->out_cols, d->n_out_blocks);
    f.out_off = vec(d->out_off, d->n_out_blocks);
    f.out_size = d->out_size;
    f.t_lb = vec(d->t_lb, d->n_t);
    f.t_col = vec(d->t_col, d->n_t);
    f.t_ci = vec(d->t_ci, d->n_t);
    f.t_trans = vec(d->t_trans, d->n_t);
    f.t_nb = vec(d->t_nb, d->n_t);
    f.t_brows = vec(d->t_brows, d->n_t);
    f.t_bcols = vec(d->t_bcols, d->n_t);
    if (d->kind == DMRGB200_PLAN_LEFT_STEP) f.t_width = vec(d->t_width, d->n_t);
    f.c_lb = vec(d->c_lb, d->n_cohorts);
    f.c_rb = vec(d->c_rb, d->n_cohorts);
    f.c_ls = vec(d->c_ls, d->n_cohorts);
    f.c_rs = vec(d->c_rs, d->n_cohorts);
    f.c_nsrows = vec(d->c_nsrows, d->n_cohorts);
    f.c_stripe = vec(d->c_stripe, d->n_cohorts);
    f.c_unit = vec(d->c_unit, size_t(d->n_cohorts) + 1);
    if (d->kind == DMRGB200_PLAN_HPSI) {
        f.c_ci = vec(d->c_ci, d->n_cohorts);
        f.c_trans = vec(d->c_trans, d->n_cohorts);
        f.c_out_ci.assign(d->n_cohorts, 0);
    } else {
        f.c_ci.assign(d->n_cohorts, 0);
        f.c_trans.assign(d->n_cohorts, 0);
        f.c_out_ci = vec(d->c_out_ci, d->n_cohorts);
    }
    f.u_offset = vec(d->u_offset, d->n_units);
    f.u_ms = vec(d->u_ms, d->n_units);
    f.u_line = vec(d->u_line, size_t(d->n_units) + 1);
    f.l_b1 = vec(d->l_b1, d->n_lines);
    f.l_term = vec(d->l_term, size_t(d->n_lines) + 1);
    f.term_alpha = vec(d->term_alpha, d->n_terms);
    f.term_t = vec(d->term_t, d->n_terms);
    f.term_col = vec(d->term_col, d->n_terms);
}

dmrgb200_status alloc_scratch(dmrgb200_plan_s* p) {
    cudaError_t e;
    if (p->prog.t_elems && (e = cudaMalloc(&p->T, p->prog.t_elems * sizeof(double))) != cudaSuccess)
        return cuda_fail(e, "T scratch allocation");
    if (p->prog.s_elems && (e = cudaMalloc(&p->S, p->prog.s_elems * sizeof(double))) != cudaSuccess)
        return cuda_fail(e, "S scratch allocation");
    return DMRGB200_OK;
}

std::vector<uint64_t> view_ptrs(const dmrgb200_boundary_view* v) {
    if (!v) return {};
    if (v->n_cohorts && !v->cohort_ptr) throw std::runtime_error("boundary view without cohort pointers");
    std::vector<uint64_t> p(v->n_cohorts);
    for (uint32_t i = 0; i < v->n_cohorts; ++i) p[i] = reinterpret_cast<uint64_t>(v->cohort_ptr[i]);
    return p;
}

std::string check_bound(FlatPlan const& f, std::vector<uint64_t> const& s1, std::vector<uint64_t> const& s3) {
    for (uint32_t t = 0; t < f.n_t(); ++t)
        if (f.t_ci[t] >= s1.size() || !s1[f.t_ci[t]]) return "T task reads a boundary cohort without storage";
    if (f.kind == KIND_HPSI)
        for (uint32_t c = 0; c < f.n_cohorts(); ++c)
            if (f.c_ci[c] >= s3.size() || !s3[f.c_ci[c]]) return "cohort reads a left cohort without storage";
    return std::string();
}

dmrgb200_status finish_plan(std::unique_ptr<dmrgb200_plan_s>& p, dmrgb200_plan_t* out) {
    std::string err = p->flat.validate();
    if (!err.empty()) return fail(DMRGB200_INVALID_PLAN, err);
    err = check_bound(p->flat, p->stage1_bnd, p->stage3_bnd);
    if (!err.empty()) return fail(DMRGB200_INVALID_PLAN, err);
    cudaGetDevice(&p->device);
    if (p->flat.kind == KIND_HPSI) {
        compile_program(p->flat, p->stage3_bnd, p->stage1_bnd, {}, p->prog, true, true);
        cudaError_t e = upload_program(p->prog);
        if (e != cudaSuccess) {
            free_program(p->prog);
            return cuda_fail(e, "plan upload");
        }
        p->compiled = true;
        dmrgb200_status s = alloc_scratch(p.get());
        if (s != DMRGB200_OK) {
            free_program(p->prog);
            cudaFree(p->T);
            cudaFree(p->S);
            return s;
        }
    }
    *out = p.release();
    return DMRGB200_OK;
}

// Execute a step plan whose output cohort pointers are `outp`.  The lowered program
// (row-stacked stage 1 for right steps, grouped S build) and its T / S scratch are
// kept with the plan and reused while the output binding stays the same, so a sweep
// that rewrites one boundary buffer per bond lowers each step once; the grouped GEMMs
// of a program of at least 50 MFLOP are autotuned once.  Synchronises the stream.
bool capturing(cudaStream_t st);

dmrgb200_status run_step(dmrgb200_plan_s* p, const double* ket, const double* bra, std::vector<uint64_t> const& outp,
                         cudaStream_t stream) {
    for (uint32_t c = 0; c < p->flat.n_cohorts(); ++c)
        if (p->flat.c_out_ci[c] >= outp.size() || !outp[p->flat.c_out_ci[c]])
            return fail(DMRGB200_INVALID_ARGUMENT, "output boundary view misses a cohort");
    cudaError_t e;
    if (!p->step_valid || p->step_outp != outp) {
        p->drop_step();
        compile_program(p->flat, {}, p->stage1_bnd, outp, p->step_prog, true, true);
        if ((e = upload_program(p->step_prog)) != cudaSuccess) {
            free_program(p->step_prog);
            return cuda_fail(e, "step plan upload");
        }
        p->step_valid = true;
        p->step_outp = outp;
        if (p->step_prog.t_elems && (e = cudaMalloc(&p->step_T, p->step_prog.t_elems * sizeof(double))) != cudaSuccess) {
            p->drop_step();
            return cuda_fail(e, "step T scratch");
        }
        if (p->step_prog.s_elems && (e = cudaMalloc(&p->step_S, p->step_prog.s_elems * sizeof(double))) != cudaSuccess) {
            p->drop_step();
            return cuda_fail(e, "step S scratch");
        }
        static const bool tune = [] {
            const char* v = std::getenv("DMRGB200_AUTOTUNE");
            return !(v && v[0] == '0');
        }();
        if (tune && p->flat.flops() >= 50000000ull && !capturing(stream)) {
            // the variants run the whole step (outputs included): the run below rewrites them
            if ((e = tune_program(p->step_prog, reinterpret_cast<uint64_t>(ket), reinterpret_cast<uint64_t>(bra),
                                  p->step_T, p->step_S, stream)) != cudaSuccess) {
                p->drop_step();
                return cuda_fail(e, "step autotuning");
            }
        }
    }
    e = run_program(p->step_prog, reinterpret_cast<uint64_t>(ket), reinterpret_cast<uint64_t>(bra), p->step_T,
                    p->step_S, stream, p->timing ? p->ev : nullptr);
    cudaError_t e2 = cudaStreamSynchronize(stream);
    if (p->timing && e == cudaSuccess && e2 == cudaSuccess) {
        p->pending = true;  // the device time of the three stages, without the host-side lowering
        p->collect();
    }
    const bool timed_out = e2 == cudaSuccess && sbuild_timed_out(p->step_prog);
    if (e != cudaSuccess) return cuda_fail(e, "step launch");
    if (e2 != cudaSuccess) return cuda_fail(e2, "step execution");
    if (timed_out) return fail(DMRGB200_TIMEOUT, "step S build: a bulk-copy wait timed out");
    return DMRGB200_OK;
}

// Emulation tables and digit-plane scratch of a plan (host work and allocations:
// outside any stream capture).  A new scratch drops the cached constant digit
// planes; the calls that change the slice count (and so the scratch a captured
// solver graph used) drop that graph themselves.
cudaError_t emu_prepare(dmrgb200_plan_s* plan) {
    if (!plan->oz1) {
        // stage 1 on the stacked row-table problems when the plan has them (one problem per
        // boundary cohort instead of one per T task)
        plan->oz1 = oz_build(plan->prog.stage1);
        plan->oz3 = oz_build(plan->prog.stage3);
        if (!plan->oz1 || !plan->oz3) return cudaErrorMemoryAllocation;
    }
    if (!plan->oz_err) {
        cudaError_t e = cudaMalloc(&plan->oz_err, 2 * sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(plan->oz_err, 0, 2 * sizeof(int));
        if (e != cudaSuccess) return e;
    }
    auto ensure = [&](OzProgram* oz, void*& buf, uint64_t& size) -> cudaError_t {
        const uint64_t need = oz_scratch_bytes(oz, plan->slices);
        if (need <= size) return cudaSuccess;
        cudaFree(buf);
        buf = nullptr;
        size = 0;
        oz_invalidate(oz);
        cudaError_t e = cudaMalloc(&buf, need);
        if (e != cudaSuccess) return e;
        size = need;
        return cudaSuccess;
    };
    cudaError_t e = ensure(plan->oz1, plan->oz_scratch, plan->oz_scratch_size);
    if (e == cudaSuccess) e = ensure(plan->oz3, plan->oz_scratch3, plan->oz_scratch3_size);
    return e;
}

// Stage 1 and stage 3 on the INT8 tensor cores (Ozaki split with plan->slices digit
// planes), the S build in FP64 between them.  Stream-ordered: a pipeline wait that
// timed out is recorded in the device error words and reported by the next
// dmrgb200_plan_check or dmrgb200_solve.
cudaError_t emu_launch(dmrgb200_plan_s* plan, const double* x, double* y, cudaStream_t st) {
    Bases bs{};
    bs.b[BUF_IN] = reinterpret_cast<uint64_t>(x);
    bs.b[BUF_OUT] = reinterpret_cast<uint64_t>(y);
    bs.b[BUF_T] = reinterpret_cast<uint64_t>(plan->T);
    bs.b[BUF_S] = reinterpret_cast<uint64_t>(plan->S);
    cudaError_t e = oz_run(plan->oz1, bs, plan->slices, plan->oz_scratch, plan->oz_err, st);
    if (e == cudaSuccess) e = run_sbuild(plan->prog, plan->T, plan->S, st);
    if (e == cudaSuccess) e = oz_run(plan->oz3, bs, plan->slices, plan->oz_scratch3, plan->oz_err + 1, st);
    return e;
}

bool capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

dmrgb200_status hpsi_emulated(dmrgb200_plan_s* plan, const double* x, double* y, cudaStream_t st) {
    const bool ready = plan->oz1 && plan->oz_scratch && plan->oz_scratch3;
    if (!ready && capturing(st))
        return fail(DMRGB200_NOT_SUPPORTED, "the first emulated H psi of a plan allocates its digit planes: make it "
                                            "before capturing the stream");
    cudaError_t e = ready ? cudaSuccess : emu_prepare(plan);
    if (e != cudaSuccess) return cuda_fail(e, "emulation tables and scratch");
    e = emu_launch(plan, x, y, st);
    if (e != cudaSuccess) return cuda_fail(e, "emulated H psi");
    return DMRGB200_OK;
}

// Wait-timeout words of a plan's kernels, read after the stream is synchronised and
// cleared: bit 0 the S build, bit 1 emulated stage 1, bit 2 emulated stage 3.
int read_error_words(dmrgb200_plan_s* plan) {
    int bits = 0;
    if (plan->compiled && sbuild_timed_out(plan->prog)) bits |= 1;
    auto oz_word = [&](OzProgram* oz, int* w) -> int {
        if (!oz || !w) return 0;
        int v = 0;
        if (cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
        if (v) {
            cudaMemset(w, 0, sizeof(int));
            oz_invalidate(oz);  // the digit planes of a stopped run may be incomplete
        }
        return v != 0;
    };
    if (plan->oz_err && oz_word(plan->oz1, plan->oz_err)) bits |= 2;
    if (plan->oz_err && oz_word(plan->oz3, plan->oz_err + 1)) bits |= 4;
    return bits;
}

dmrgb200_status timeout_status(int bits) {
    if (!bits) return DMRGB200_OK;
    std::string where = (bits & 1) ? "S build (bulk-copy ring)" : (bits & 2) ? "emulated stage 1" : "emulated stage 3";
    return fail(DMRGB200_TIMEOUT, where + ": a bounded wait ran out; the results of the calls since the last check "
                                          "are not valid");
}

}  // namespace

namespace dmrgb200 {
dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg) { return fail(s, msg); }
cudaError_t plan_hpsi_launch(dmrgb200_plan_t plan, const double* x, double* y, cudaStream_t stream) {
    if (plan->flat.kind != KIND_HPSI || !plan->compiled) return cudaErrorInvalidValue;
    if (plan->solve_prec == DMRGB200_PREC_FP64_EMULATED) {
        if (!plan->oz_scratch3) {
            if (capturing(stream)) return cudaErrorStreamCaptureUnsupported;
            cudaError_t e = emu_prepare(plan);
            if (e != cudaSuccess) return e;
        }
        return emu_launch(plan, x, y, stream);
    }
    return run_program(plan->prog, reinterpret_cast<uint64_t>(x), reinterpret_cast<uint64_t>(y), plan->T, plan->S,
                       stream);
}
void noalloc_desc_to_flat(const dmrgb200_plan_desc* d, FlatPlan& f) { desc_to_flat(d, f); }
int plan_solver_mode(dmrgb200_plan_t plan) { return plan->solver_mode; }
int plan_error_words(dmrgb200_plan_t plan) { return read_error_words(plan); }
// Before a solve: an emulated plan whose boundary digit planes were dropped (new boundary
// values) makes them again eagerly, outside the solver graph (which only splits psi and S);
// x is read and y written as scratch.
cudaError_t plan_refresh_constants(dmrgb200_plan_t plan, const double* x, double* y, cudaStream_t stream) {
    if (plan->solve_prec != DMRGB200_PREC_FP64_EMULATED || !plan->oz1 || !plan->oz_scratch3) return cudaSuccess;
    if (oz_constants_ready(plan->oz1) && oz_constants_ready(plan->oz3)) return cudaSuccess;
    if (capturing(stream)) return cudaErrorStreamCaptureUnsupported;
    return emu_launch(plan, x, y, stream);
}
// Autotune the plan's grouped GEMMs once, outside any stream capture (DMRGB200_AUTOTUNE=0
// keeps the default variant, and so do plans below 50 MFLOP per H psi).
cudaError_t plan_ensure_tuned(dmrgb200_plan_t plan, const double* x, double* y, cudaStream_t stream) {
    if (!plan->compiled) return cudaSuccess;
    if (plan->solve_prec == DMRGB200_PREC_FP64_EMULATED) {
        // tables, scratch and the constant (boundary) digit planes before any capture: one
        // emulated H psi splits the boundaries, later ones (captured or not) only psi and S
        const bool fresh = !plan->oz_scratch3;
        cudaError_t e = emu_prepare(plan);
        if (e == cudaSuccess && (fresh || !oz_constants_ready(plan->oz1) || !oz_constants_ready(plan->oz3)) &&
            !capturing(stream))
            e = emu_launch(plan, x, y, stream);
        return e;
    }
    if (plan->prog.tuned) return cudaSuccess;
    static const bool enabled = [] {
        const char* v = std::getenv("DMRGB200_AUTOTUNE");
        return !(v && v[0] == '0');
    }();
    // small plans keep the default variant: tuning would cost more than it saves
    if (!enabled || plan->flat.flops() < 50000000ull) {
        plan->prog.tuned = true;
        return cudaSuccess;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return cudaSuccess;
    return tune_program(plan->prog, reinterpret_cast<uint64_t>(x), reinterpret_cast<uint64_t>(y), plan->T, plan->S,
                        stream);
}
void** plan_jd_cache(dmrgb200_plan_t plan) { return &plan->jd; }
FlatPlan const& plan_flat(dmrgb200_plan_t plan) { return plan->flat; }
DeviceProgram const& plan_program(dmrgb200_plan_t plan) { return plan->prog; }
std::vector<uint64_t> const& plan_stage1_bnd(dmrgb200_plan_t plan) { return plan->stage1_bnd; }
std::vector<uint64_t> const& plan_stage3_bnd(dmrgb200_plan_t plan) { return plan->stage3_bnd; }
double* plan_T(dmrgb200_plan_t plan) { return plan->compiled ? plan->T : nullptr; }
double* plan_S(dmrgb200_plan_t plan) { return plan->S; }
void*& plan_blas_handle(dmrgb200_plan_t plan) { return plan->blas; }
}  // namespace dmrgb200

extern "C" {

const char* dmrgb200_status_string(dmrgb200_status s) {
    switch (s) {
        case DMRGB200_OK: return "ok";
        case DMRGB200_INVALID_ARGUMENT: return "invalid argument";
        case DMRGB200_INVALID_PLAN: return "invalid plan";
        case DMRGB200_OUT_OF_MEMORY: return "out of memory";
        case DMRGB200_DEVICE_ERROR: return "device error";
        case DMRGB200_TIMEOUT: return "timeout";
        case DMRGB200_NUMERIC: return "numeric error";
        case DMRGB200_NOT_SUPPORTED: return "not supported";
    }
    return "unknown status";
}

const char* dmrgb200_last_error(void) { return g_last_error.c_str(); }

int dmrgb200_abi_version(void) { return 1; }

double dmrgb200_wigner6j(int a, int b, int c, int d, int e, int f) { return wigner6j(a, b, c, d, e, f); }
double dmrgb200_wigner9j(int a, int b, int c, int d, int e, int f, int g, int h, int i) {
    return wigner9j(a, b, c, d, e, f, g, h, i);
}
void dmrgb200_set_coupling(int a, int b, int c, int d, int e, int f, int g, int h, int i, double init,
                           double couplings[4]) {
    set_coupling(a, b, c, d, e, f, g, h, i, init, couplings);
}

dmrgb200_status dmrgb200_context_create(int device, dmrgb200_context_t* out) {
    if (!out) return fail(DMRGB200_INVALID_ARGUMENT, "null output");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    auto* c = new dmrgb200_context_s;
    c->device = device;
    *out = c;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_context_destroy(dmrgb200_context_t ctx) {
    delete ctx;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_create(dmrgb200_context_t ctx, const dmrgb200_plan_desc* d,
                                     const dmrgb200_boundary_view* left, const dmrgb200_boundary_view* other,
                                     dmrgb200_plan_t* out) {
    DMRGB200_TRY
    if (!ctx || !d || !out) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    auto p = std::make_unique<dmrgb200_plan_s>();
    desc_to_flat(d, p->flat);
    if (d->kind == DMRGB200_PLAN_HPSI) {
        p->stage3_bnd = view_ptrs(left);
        p->stage1_bnd = view_ptrs(other);
    } else if (d->kind == DMRGB200_PLAN_LEFT_STEP) {
        p->stage1_bnd = view_ptrs(left);
    } else {
        p->stage1_bnd = view_ptrs(other);
    }
    return finish_plan(p, out);
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_calibrate(int what, double* value) {
    if (!value || what != 0) return fail(DMRGB200_INVALID_ARGUMENT, "unknown calibration");
    *value = calibrate_fp64_tflops();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "calibration");
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_validate(const dmrgb200_plan_desc* d) {
    DMRGB200_TRY
    if (!d) return fail(DMRGB200_INVALID_ARGUMENT, "null plan description");
    if (d->kind < DMRGB200_PLAN_HPSI || d->kind > DMRGB200_PLAN_RIGHT_STEP)
        return fail(DMRGB200_INVALID_PLAN, "unknown plan kind");
    FlatPlan f;
    desc_to_flat(d, f);
    std::string err = f.validate();
    if (!err.empty()) return fail(DMRGB200_INVALID_PLAN, err);
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_plan_create_batched(dmrgb200_context_t ctx, uint32_t n, const dmrgb200_plan_desc* descs,
                                             const dmrgb200_boundary_view* lefts,
                                             const dmrgb200_boundary_view* rights, uint64_t* in_base,
                                             uint64_t* total_size, dmrgb200_plan_t* out) {
    DMRGB200_TRY
    if (!ctx || !descs || !lefts || !rights || !out || n == 0) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    std::vector<FlatPlan> plans(n);
    std::vector<uint32_t> lbase(n), rbase(n);
    auto p = std::make_unique<dmrgb200_plan_s>();
    for (uint32_t i = 0; i < n; ++i) {
        if (descs[i].kind != DMRGB200_PLAN_HPSI) return fail(DMRGB200_INVALID_PLAN, "batched plans must be H psi plans");
        desc_to_flat(&descs[i], plans[i]);
        std::string err = plans[i].validate();
        if (!err.empty()) return fail(DMRGB200_INVALID_PLAN, "instance " + std::to_string(i) + ": " + err);
        lbase[i] = uint32_t(p->stage3_bnd.size());
        rbase[i] = uint32_t(p->stage1_bnd.size());
        auto lp = view_ptrs(&lefts[i]), rp = view_ptrs(&rights[i]);
        p->stage3_bnd.insert(p->stage3_bnd.end(), lp.begin(), lp.end());
        p->stage1_bnd.insert(p->stage1_bnd.end(), rp.begin(), rp.end());
    }
    std::vector<uint64_t> ib, ob;
    p->flat = merge_plans(plans, lbase, rbase, ib, ob);
    if (in_base)
        for (uint32_t i = 0; i < n; ++i) in_base[i] = ib[i];
    if (total_size) *total_size = p->flat.in_size;
    return finish_plan(p, out);
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_plan_destroy(dmrgb200_plan_t plan) {
    if (!plan) return DMRGB200_OK;
    if (plan->compiled) free_program(plan->prog);
    if (plan->adj_built) free_adjoint(plan->adj);
    if (plan->pipe_built) {
        free_pipeline(plan->pipe);
        cudaFree(plan->hx);
        cudaFree(plan->hy);
        if (plan->pipe_exec) cudaGraphExecDestroy(plan->pipe_exec);
        for (auto& e : plan->pev)
            if (e) cudaEventDestroy(e);
        if (plan->copy_stream) cudaStreamDestroy(plan->copy_stream);
        if (plan->capture_stream) cudaStreamDestroy(plan->capture_stream);
    }
    jd_graph_free(plan->jd);
    blas_handle_free(plan->blas);
    plan->drop_step();
    plan->drop_dm();
    oz_free(plan->oz1);
    oz_free(plan->oz3);
    cudaFree(plan->oz_scratch);
    cudaFree(plan->oz_scratch3);
    cudaFree(plan->oz_err);
    for (auto& e : plan->ev)
        if (e) cudaEventDestroy(e);
    cudaFree(plan->T);
    cudaFree(plan->S);
    delete plan;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_flops(dmrgb200_plan_t plan, uint64_t* flops) {
    if (!plan || !flops) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    *flops = plan->flat.flops();
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_scratch_bytes(dmrgb200_plan_t plan, uint64_t* bytes) {
    if (!plan || !bytes) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    *bytes = (plan->prog.t_elems + plan->prog.s_elems) * sizeof(double);
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_hpsi(dmrgb200_plan_t plan, const double* x, double* y, dmrgb200_precision prec,
                              void* cuda_stream) {
    if (!plan || !x || !y) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (plan->flat.kind != KIND_HPSI) return fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
    if (prec == DMRGB200_PREC_FP64_EMULATED) return hpsi_emulated(plan, x, y, static_cast<cudaStream_t>(cuda_stream));
    if (prec != DMRGB200_PREC_FP64) return fail(DMRGB200_INVALID_ARGUMENT, "unknown precision");
    if (plan->timing) plan->collect();
    {
        cudaError_t te = plan_ensure_tuned(plan, x, y, static_cast<cudaStream_t>(cuda_stream));
        if (te != cudaSuccess) return cuda_fail(te, "grouped GEMM autotuning");
    }
    cudaError_t e = run_program(plan->prog, reinterpret_cast<uint64_t>(x), reinterpret_cast<uint64_t>(y), plan->T,
                                plan->S, static_cast<cudaStream_t>(cuda_stream), plan->timing ? plan->ev : nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "hpsi launch");
    if (plan->timing) plan->pending = true;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_hpsi_host(dmrgb200_plan_t plan, const double* x_host, double* y_host, void* cuda_stream) {
    DMRGB200_TRY
    if (!plan || !x_host || !y_host) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (plan->flat.kind != KIND_HPSI || !plan->compiled) return fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e;
    if (!plan->pipe_built) {
        plan->pipe_built = true;  // released by dmrgb200_plan_destroy, also after a failure here
        if ((e = compile_pipeline(plan->flat, plan->stage3_bnd, plan->stage1_bnd, plan->PIPE_PARTS, plan->pipe)) !=
            cudaSuccess)
            return cuda_fail(e, "host-buffer program");
        const size_t nx = std::max<uint64_t>(plan->flat.in_size, 1), ny = std::max<uint64_t>(plan->flat.out_size, 1);
        if ((e = cudaMalloc(&plan->hx, nx * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc(&plan->hy, ny * sizeof(double))) != cudaSuccess ||
            // H psi writes only block elements: the padding copied back stays zero
            (e = cudaMemset(plan->hy, 0, ny * sizeof(double))) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&plan->copy_stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&plan->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "host-buffer scratch");
        for (auto& ev : plan->pev)
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "host-buffer events");
    }
    if (!plan->hx || !plan->copy_stream) return fail(DMRGB200_DEVICE_ERROR, "host-buffer program unavailable");
    if ((e = plan_ensure_tuned(plan, plan->hx, plan->hy, st)) != cudaSuccess)
        return cuda_fail(e, "grouped GEMM autotuning");
    if (!plan->pipe_exec || plan->pipe_x != x_host || plan->pipe_y != y_host) {
        // (re)capture for these host buffers on the plan's own stream
        if (plan->pipe_exec) cudaGraphExecDestroy(plan->pipe_exec);
        plan->pipe_exec = nullptr;
        cudaGraph_t g = nullptr;
        cudaStream_t cs = plan->capture_stream;
        if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_fail(e, "host-buffer capture");
        cudaError_t er = run_pipeline(plan->prog, plan->pipe, x_host, y_host, plan->hx, plan->hy, plan->T, plan->S, cs,
                                      plan->copy_stream, plan->pev);
        e = cudaStreamEndCapture(cs, &g);
        if (er != cudaSuccess || e != cudaSuccess) {
            // not capturable (pageable host buffers, for one): run the sequence directly
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            e = run_pipeline(plan->prog, plan->pipe, x_host, y_host, plan->hx, plan->hy, plan->T, plan->S, st,
                             plan->copy_stream, plan->pev);
            return e == cudaSuccess ? DMRGB200_OK : cuda_fail(e, "host-buffer H psi");
        }
        e = cudaGraphInstantiate(&plan->pipe_exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            plan->pipe_exec = nullptr;
            return cuda_fail(e, "host-buffer graph");
        }
        plan->pipe_x = x_host;
        plan->pipe_y = y_host;
    }
    if ((e = cudaGraphLaunch(plan->pipe_exec, st)) != cudaSuccess) return cuda_fail(e, "host-buffer H psi");
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_hpsi_adjoint(dmrgb200_plan_t plan, const double* w, const double* x, double* gx,
                                      double* galpha, void* cuda_stream) {
    DMRGB200_TRY
    if (!plan || !w || (galpha && !x)) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (plan->flat.kind != KIND_HPSI) return fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
    if (!plan->adj_built) {
        plan->adj_err = compile_adjoint(plan->flat, plan->stage3_bnd, plan->stage1_bnd, plan->prog, plan->adj);
        if (plan->adj_err.empty()) {
            cudaError_t e = upload_adjoint(plan->adj);
            if (e != cudaSuccess) {
                free_adjoint(plan->adj);
                return cuda_fail(e, "adjoint program upload");
            }
        }
        plan->adj_built = true;
    }
    if (!plan->adj_err.empty()) return fail(DMRGB200_INVALID_PLAN, "no adjoint for this plan: " + plan->adj_err);
    cudaError_t e = run_adjoint(plan->prog, plan->adj, reinterpret_cast<uint64_t>(w), reinterpret_cast<uint64_t>(x),
                                gx, plan->flat.in_size, galpha, plan->T, plan->S,
                                static_cast<cudaStream_t>(cuda_stream));
    if (e != cudaSuccess) return cuda_fail(e, "adjoint launch");
    return DMRGB200_OK;
    DMRGB200_CATCH
}

// The captured graphs of a plan (the solver graph, the host-buffer H psi) launch the GEMM
// variants chosen when they were captured: a new choice drops them (captured again on use).
static void drop_variant_graphs(dmrgb200_plan_t plan) {
    jd_graph_free(plan->jd);
    plan->jd = nullptr;
    if (plan->pipe_exec) cudaGraphExecDestroy(plan->pipe_exec);
    plan->pipe_exec = nullptr;
    plan->pipe_x = nullptr;
    plan->pipe_y = nullptr;
}

dmrgb200_status dmrgb200_plan_autotune(dmrgb200_plan_t plan, const double* x, double* y, void* cuda_stream,
                                       int32_t variants[2]) {
    if (!plan || !x || !y) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (plan->flat.kind != KIND_HPSI) return fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
    plan->prog.tuned = false;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e = tune_program(plan->prog, reinterpret_cast<uint64_t>(x), reinterpret_cast<uint64_t>(y), plan->T,
                                 plan->S, st);
    drop_variant_graphs(plan);
    if (e != cudaSuccess) return cuda_fail(e, "grouped GEMM autotuning");
    if (variants) {
        variants[0] = plan->prog.var1;
        variants[1] = plan->prog.var3;
    }
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_set_gemm_variants(dmrgb200_plan_t plan, int32_t stage1, int32_t stage3) {
    if (!plan) return fail(DMRGB200_INVALID_ARGUMENT, "null plan");
    if (stage1 < 0 || stage1 >= N_GEMM_VARIANTS || stage3 < 0 || stage3 >= N_GEMM_VARIANTS)
        return fail(DMRGB200_INVALID_ARGUMENT, "variant index out of range");
    if (plan->flat.kind != KIND_HPSI || !plan->compiled) return fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
    plan->prog.var1 = stage1;
    plan->prog.var3 = stage3;
    plan->prog.tuned = true;
    drop_variant_graphs(plan);
    return DMRGB200_OK;
}

const char* dmrgb200_gemm_variant_name(int variant) { return gemm_variant_name(variant); }
int dmrgb200_gemm_variant_count(void) { return N_GEMM_VARIANTS; }

dmrgb200_status dmrgb200_plan_set_solver(dmrgb200_plan_t plan, int mode) {
    if (!plan || (mode != DMRGB200_SOLVER_GRAPH && mode != DMRGB200_SOLVER_STEPWISE))
        return fail(DMRGB200_INVALID_ARGUMENT, "unknown solver mode");
    plan->solver_mode = mode;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_set_slices(dmrgb200_plan_t plan, int slices) {
    if (!plan || slices < 2 || slices > 8) return fail(DMRGB200_INVALID_ARGUMENT, "slices must be 2..8");
    if (slices != plan->slices) {
        plan->slices = slices;
        oz_free(plan->oz1);
        oz_free(plan->oz3);
        plan->oz1 = plan->oz3 = nullptr;
        jd_graph_free(plan->jd);  // a captured emulated solve used the old digit planes
        plan->jd = nullptr;
    }
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_set_wait_limit(uint64_t ns) {
    g_wait_limit_ns.store(ns ? ns : 2000000000ull, std::memory_order_relaxed);
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_set_precision(dmrgb200_plan_t plan, int prec) {
    if (!plan) return fail(DMRGB200_INVALID_ARGUMENT, "null plan");
    if (prec != DMRGB200_PREC_FP64 && prec != DMRGB200_PREC_FP64_EMULATED)
        return fail(DMRGB200_INVALID_ARGUMENT, "unknown precision");
    if (prec != plan->solve_prec) {
        plan->solve_prec = prec;
        jd_graph_free(plan->jd);  // the cached solver graph captured the other H psi
        plan->jd = nullptr;
    }
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_boundaries_changed(dmrgb200_plan_t plan) {
    if (!plan) return fail(DMRGB200_INVALID_ARGUMENT, "null plan");
    oz_invalidate(plan->oz1);
    oz_invalidate(plan->oz3);
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_check(dmrgb200_plan_t plan, void* cuda_stream) {
    if (!plan) return fail(DMRGB200_INVALID_ARGUMENT, "null plan");
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(cuda_stream));
    if (e != cudaSuccess) return cuda_fail(e, "plan check");
    return timeout_status(read_error_words(plan));
}

dmrgb200_status dmrgb200_plan_tune_slices(dmrgb200_plan_t plan, const double* x, double target, void* cuda_stream,
                                          int* slices, double* rel_err) {
    DMRGB200_TRY
    if (!plan || !x || !(target > 0.0)) return fail(DMRGB200_INVALID_ARGUMENT, "null argument or target <= 0");
    if (plan->flat.kind != KIND_HPSI || !plan->compiled) return fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    const uint64_t n = std::max<uint64_t>(plan->flat.out_size, 1);
    double *y64 = nullptr, *ye = nullptr, *dot = nullptr;
    cudaError_t e = cudaMalloc(&y64, 2 * n * sizeof(double) + 2 * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(e, "slice tuning buffers");
    ye = y64 + n;
    dot = ye + n;
    struct Free {
        double* p;
        ~Free() { cudaFree(p); }
    } guard{y64};
    if ((e = cudaMemsetAsync(y64, 0, 2 * n * sizeof(double), st)) != cudaSuccess) return cuda_fail(e, "slice tuning");
    if ((e = run_program(plan->prog, reinterpret_cast<uint64_t>(x), reinterpret_cast<uint64_t>(y64), plan->T, plan->S,
                         st)) != cudaSuccess)
        return cuda_fail(e, "slice tuning: FP64 H psi");
    const int s0 = plan->slices;
    int chosen = 8;
    double chosen_err = -1.0;
    for (int sl = 3; sl <= 8; ++sl) {
        plan->slices = sl;
        oz_free(plan->oz1);
        oz_free(plan->oz3);
        plan->oz1 = plan->oz3 = nullptr;
        if ((e = emu_prepare(plan)) != cudaSuccess) return cuda_fail(e, "slice tuning: emulation scratch");
        if ((e = emu_launch(plan, x, ye, st)) != cudaSuccess) return cuda_fail(e, "slice tuning: emulated H psi");
        if ((e = diff_norms(ye, y64, n, dot, st)) != cudaSuccess) return cuda_fail(e, "slice tuning: norms");
        double h[2] = {0, 0};
        if ((e = cudaMemcpyAsync(h, dot, 2 * sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_fail(e, "slice tuning");
        dmrgb200_status ts = timeout_status(read_error_words(plan));
        if (ts != DMRGB200_OK) {
            plan->slices = s0;
            return ts;
        }
        const double err = h[1] > 0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
        if (err <= target || sl == 8) {
            chosen = sl;
            chosen_err = err;
            break;
        }
    }
    // keep the chosen slice count (its digit planes are the ones now in the scratch)
    plan->slices = chosen;
    jd_graph_free(plan->jd);
    plan->jd = nullptr;
    if (slices) *slices = chosen;
    if (rel_err) *rel_err = chosen_err;
    if (chosen_err > target) return fail(DMRGB200_NUMERIC, "no slice count up to 8 meets the target error");
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_plan_set_timing(dmrgb200_plan_t plan, int enable) {
    if (!plan) return fail(DMRGB200_INVALID_ARGUMENT, "null plan");
    if (enable && !plan->ev[0])
        for (auto& e : plan->ev) {
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return cuda_fail(r, "event creation");
        }
    plan->collect();
    plan->timing = enable != 0;
    plan->stage_ms[0] = plan->stage_ms[1] = plan->stage_ms[2] = 0.0;
    plan->timed_calls = 0;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_plan_stage_times(dmrgb200_plan_t plan, double ms[3], uint64_t flops[3], uint64_t* calls) {
    if (!plan) return fail(DMRGB200_INVALID_ARGUMENT, "null plan");
    plan->collect();
    if (ms)
        for (int i = 0; i < 3; ++i) ms[i] = plan->stage_ms[i];
    if (flops) plan->flat.stage_flops(flops);
    if (calls) *calls = plan->timed_calls;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_step_alpha_dm(dmrgb200_plan_t plan, const double* ket, const double* bra,
                                       const dmrgb200_boundary_view* dm, double alpha, void* cuda_stream) {
    DMRGB200_TRY
    if (!plan || !ket || !bra || !dm) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (!(alpha >= 0.0)) return fail(DMRGB200_INVALID_ARGUMENT, "alpha must be >= 0");
    FlatPlan const& p = plan->flat;
    const bool left = p.kind == KIND_LEFT;
    if (!left && p.kind != KIND_RIGHT) return fail(DMRGB200_INVALID_PLAN, "alpha_dm needs a left or right step plan");
    const uint32_t nb = uint32_t(p.out_rows.size());
    std::vector<uint64_t> ptrs = view_ptrs(dm);
    if (ptrs.size() < nb) return fail(DMRGB200_INVALID_ARGUMENT, "dm view has fewer blocks than the bra");
    ptrs.resize(nb);
    for (uint32_t b = 0; b < nb; ++b)
        if (!ptrs[b] && (left ? p.out_rows[b] : p.out_cols[b]))
            return fail(DMRGB200_INVALID_ARGUMENT, "dm view misses a block");
    for (uint32_t c = 0; c < p.n_cohorts(); ++c) {
        const uint32_t b = left ? p.c_lb[c] : p.c_rb[c];
        if (b >= nb || p.c_stripe[c] != (left ? p.out_rows[b] : p.out_cols[b]))
            return fail(DMRGB200_INVALID_PLAN, "cohort stripe differs from its bra block");
    }
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e;
    if (!plan->step_valid) {
        // stages 1 and 2 of the step program; its stage 3 (never launched here) gets
        // placeholder output addresses, so a later dmrgb200_step_execute lowers it again
        uint32_t nout = 0;
        for (uint32_t c = 0; c < p.n_cohorts(); ++c) nout = std::max(nout, p.c_out_ci[c] + 1);
        std::vector<uint64_t> placeholder(nout, 8);
        compile_program(p, {}, plan->stage1_bnd, placeholder, plan->step_prog, true, true);
        if ((e = upload_program(plan->step_prog)) != cudaSuccess) {
            free_program(plan->step_prog);
            return cuda_fail(e, "alpha_dm step upload");
        }
        plan->step_valid = true;
        plan->step_outp = placeholder;
        if (plan->step_prog.t_elems &&
            (e = cudaMalloc(&plan->step_T, plan->step_prog.t_elems * sizeof(double))) != cudaSuccess) {
            plan->drop_step();
            return cuda_fail(e, "alpha_dm T scratch");
        }
        if (plan->step_prog.s_elems &&
            (e = cudaMalloc(&plan->step_S, plan->step_prog.s_elems * sizeof(double))) != cudaSuccess) {
            plan->drop_step();
            return cuda_fail(e, "alpha_dm S scratch");
        }
    }
    if (!plan->dm_valid || plan->dm_ptrs != ptrs) {
        plan->drop_dm();
        GemmList gl;
        build_alpha_dm(p, ptrs, gl);
        if ((e = upload_gemm(gl, plan->dm_gemm)) != cudaSuccess) return cuda_fail(e, "alpha_dm tables");
        plan->dm_valid = true;
        plan->dm_ptrs = ptrs;
    }
    const uint64_t ki = reinterpret_cast<uint64_t>(ket), bo = reinterpret_cast<uint64_t>(bra);
    if ((e = run_stages12(plan->step_prog, ki, bo, plan->step_T, plan->step_S, stream)) != cudaSuccess)
        return cuda_fail(e, "alpha_dm S build");
    if ((e = scale_buffer(plan->step_S, plan->step_prog.s_elems, std::sqrt(alpha), stream)) != cudaSuccess)
        return cuda_fail(e, "alpha_dm scale");
    Bases bs{};
    bs.b[BUF_OUT] = bo;
    bs.b[BUF_S] = reinterpret_cast<uint64_t>(plan->step_S);
    if ((e = launch_gemm(plan->dm_gemm, bs, stream)) != cudaSuccess) return cuda_fail(e, "alpha_dm GEMM");
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_step_execute(dmrgb200_plan_t plan, const double* ket, const double* bra,
                                      const dmrgb200_boundary_view* out, void* cuda_stream) {
    DMRGB200_TRY
    if (!plan || !ket || !bra || !out) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    if (plan->flat.kind == KIND_HPSI) return fail(DMRGB200_INVALID_PLAN, "plan is not a boundary-step plan");
    return run_step(plan, ket, bra, view_ptrs(out), static_cast<cudaStream_t>(cuda_stream));
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_mpo_create(const dmrgb200_mpo_desc* d, dmrgb200_mpo_t* out) {
    DMRGB200_TRY
    if (!d || !out) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    auto m = std::make_unique<dmrgb200_mpo_s>();
    m->symm = to_symm(d->symm);
    MPOTensor& t = m->mpo;
    t.row_dim = d->row_dim;
    t.col_dim = d->col_dim;
    if (d->left_spin) t.left_spin.assign(d->left_spin, d->left_spin + d->row_dim);
    if (d->right_spin) t.right_spin.assign(d->right_spin, d->right_spin + d->col_dim);
    t.left_herm = d->left_herm ? Hermitian(std::vector<unsigned>(d->left_herm, d->left_herm + d->row_dim),
                                           std::vector<int>(d->left_phase, d->left_phase + d->row_dim))
                               : Hermitian(d->row_dim);
    t.right_herm = d->right_herm ? Hermitian(std::vector<unsigned>(d->right_herm, d->right_herm + d->col_dim),
                                             std::vector<int>(d->right_phase, d->right_phase + d->col_dim))
                                 : Hermitian(d->col_dim);
    for (uint32_t o = 0; o < d->n_ops; ++o) {
        SiteOp op;
        op.spin = d->op_spin ? d->op_spin[o] : 0;
        for (uint32_t k = d->op_block[o]; k < d->op_block[o + 1]; ++k) {
            OpBlock blk;
            blk.left = Charge(d->blk_in[2 * k], d->blk_in[2 * k + 1]);
            blk.right = Charge(d->blk_out[2 * k], d->blk_out[2 * k + 1]);
            for (uint32_t e = d->blk_entry[k]; e < d->blk_entry[k + 1]; ++e)
                blk.entries.push_back(SparseEntry{d->e_row[e], d->e_col[e], d->e_row_spin ? d->e_row_spin[e] : 0,
                                                  d->e_col_spin ? d->e_col_spin[e] : 0, d->e_coeff[e]});
            op.blocks.push_back(std::move(blk));
        }
        t.ops.push_back(std::move(op));
    }
    t.rows.assign(t.row_dim, {});
    t.cols.assign(t.col_dim, {});
    for (uint32_t i = 0; i < d->n_terms; ++i) {
        uint32_t b1 = d->term_b1[i], b2 = d->term_b2[i];
        if (b1 >= t.row_dim || b2 >= t.col_dim || d->term_op[i] >= d->n_ops)
            return fail(DMRGB200_INVALID_ARGUMENT, "MPO term index out of range");
        auto& row = t.rows[b1];
        if (row.empty() || row.back().other != b2) {
            if (!row.empty() && row.back().other > b2)
                return fail(DMRGB200_INVALID_ARGUMENT, "MPO terms must be sorted by (b1, b2)");
            row.push_back(MPOEntry{b2, {}});
        }
        row.back().terms.push_back(TermRef{d->term_op[i], d->term_scale[i], i});
    }
    for (uint32_t b1 = 0; b1 < t.row_dim; ++b1)
        for (auto const& e : t.rows[b1]) t.cols[e.other].push_back(MPOEntry{b1, e.terms});
    *out = m.release();
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_mpo_destroy(dmrgb200_mpo_t mpo) {
    delete mpo;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_bindex_create_edge(dmrgb200_symmetry symm, const dmrgb200_index_desc* index,
                                            uint32_t aux_dim, dmrgb200_bindex_t* out) {
    DMRGB200_TRY
    if (!index || !out || aux_dim == 0) return fail(DMRGB200_INVALID_ARGUMENT, "invalid argument");
    Index ix = to_index(index);
    auto b = std::make_unique<dmrgb200_bindex_s>();
    b->idx = BoundaryIndex(to_symm(symm), ix, ix);
    for (unsigned i = 0; i < ix.size(); ++i) {
        std::vector<long> off(aux_dim);
        for (uint32_t a = 0; a < aux_dim; ++a) off[a] = long(a) * ix.block_size(i) * ix.block_size(i);
        b->idx.add_cohort(i, i, off);
    }
    b->layout();
    *out = b.release();
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_bindex_destroy(dmrgb200_bindex_t b) {
    delete b;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_bindex_info(dmrgb200_bindex_t b, uint32_t* n_cohorts, uint32_t* aux_dim,
                                     uint64_t* n_elements) {
    if (!b) return fail(DMRGB200_INVALID_ARGUMENT, "null boundary index");
    if (n_cohorts) *n_cohorts = b->idx.n_cohorts();
    if (aux_dim) *aux_dim = uint32_t(b->idx.aux_dim());
    if (n_elements) *n_elements = b->n_elems;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_bindex_describe(dmrgb200_bindex_t b, uint32_t* lb, uint32_t* rb, uint8_t* tr,
                                         uint64_t* storage_off, uint32_t* lsize, uint32_t* rsize,
                                         uint32_t* nblocks, int64_t* offsets, double* conj_scales,
                                         uint8_t* transposes) {
    if (!b) return fail(DMRGB200_INVALID_ARGUMENT, "null boundary index");
    BoundaryIndex const& ix = b->idx;
    size_t aux = ix.aux_dim();
    std::vector<uint32_t> clb(ix.n_cohorts(), 0), crb(ix.n_cohorts(), 0);
    for (unsigned l = 0; l < ix.bra().size(); ++l)
        for (unsigned r = 0; r < ix.ket().size(); ++r) {
            unsigned ci = ix.cohort_index(l, r);
            if (ci < ix.n_cohorts()) {
                clb[ci] = l;
                crb[ci] = r;
            }
        }
    for (unsigned ci = 0; ci < ix.n_cohorts(); ++ci) {
        if (lb) lb[ci] = clb[ci];
        if (rb) rb[ci] = crb[ci];
        if (tr) tr[ci] = ix.tr(ci);
        if (storage_off) storage_off[ci] = b->coh_off[ci];
        if (lsize) lsize[ci] = uint32_t(ix.left_size(ci));
        if (rsize) rsize[ci] = uint32_t(ix.right_size(ci));
        if (nblocks) nblocks[ci] = uint32_t(ix.n_blocks(ci));
        for (size_t a = 0; a < aux; ++a) {
            if (offsets) offsets[ci * aux + a] = ix.offset(ci, unsigned(a));
            if (conj_scales) conj_scales[ci * aux + a] = ix.conjugate_scale(ci, unsigned(a));
            if (transposes) transposes[ci * aux + a] = ix.trans(ci, unsigned(a));
        }
    }
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_schedule_hpsi(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                       const dmrgb200_index_desc* right_i, dmrgb200_mpo_t mpo,
                                       dmrgb200_bindex_t L, dmrgb200_bindex_t R, dmrgb200_schedule_t* out) {
    DMRGB200_TRY
    if (!mpo || !L || !R || !out) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    Index ph = to_index(phys), li = to_index(left_i), ri = to_index(right_i);
    Schedule s = create_contraction_schedule(mpo->symm, ph, li, ri, L->idx, R->idx, mpo->mpo);
    auto sc = std::make_unique<dmrgb200_schedule_s>();
    sc->flat = flatten_hpsi(s, right_paired_layout(ph, li, ri), L->idx, R->idx);
    std::string err = sc->flat.validate();
    if (!err.empty()) return fail(DMRGB200_INVALID_PLAN, "builder produced an inconsistent plan: " + err);
    *out = sc.release();
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_schedule_left_step(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                            const dmrgb200_index_desc* right_i, dmrgb200_mpo_t mpo,
                                            dmrgb200_bindex_t L, int symmetric, dmrgb200_schedule_t* out,
                                            dmrgb200_bindex_t* new_index) {
    DMRGB200_TRY
    if (!mpo || !L || !out || !new_index) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    Index ph = to_index(phys), li = to_index(left_i), ri = to_index(right_i);
    auto nb = std::make_unique<dmrgb200_bindex_s>();
    Schedule s = left_step_schedule(mpo->symm, ph, li, ri, li, ri, L->idx, mpo->mpo, symmetric != 0, nb->idx);
    nb->layout();
    auto sc = std::make_unique<dmrgb200_schedule_s>();
    sc->flat = flatten_left_step(s, right_paired_layout(ph, li, ri), left_paired_layout(ph, li, ri), ri, L->idx,
                                 nb->idx);
    std::string err = sc->flat.validate();
    if (!err.empty()) return fail(DMRGB200_INVALID_PLAN, "builder produced an inconsistent plan: " + err);
    *out = sc.release();
    *new_index = nb.release();
    return DMRGB200_OK;
    DMRGB200_CATCH
}

dmrgb200_status dmrgb200_schedule_right_step(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                             const dmrgb200_index_desc* right_i, dmrgb200_mpo_t mpo,
                                             dmrgb200_bindex_t R, int symmetric, dmrgb200_schedule_t* out,
                                             dmrgb200_bindex_t* new_index) {
    DMRGB200_TRY
    if (!mpo || !R || !out || !new_index) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    Index ph = to_index(phys), li = to_index(left_i), ri = to_index(right_i);
    auto nb = std::make_unique<dmrgb200_bindex_s>();
    Schedule s = right_step_schedule(mpo->symm, ph, li, ri, li, R->idx, mpo->mpo, symmetric != 0, nb->idx);
    nb->layout();
    auto sc = std::make_unique<dmrgb200_schedule_s>();
    TensorLayout rp = right_paired_layout(ph, li, ri);
    sc->flat = flatten_right_step(s, rp, rp, R->idx, nb->idx);
    std::string err = sc->flat.validate();
    if (!err.empty()) return fail(DMRGB200_INVALID_PLAN, "builder produced an inconsistent plan: " + err);
    *out = sc.release();
    *new_index = nb.release();
    return DMRGB200_OK;
    DMRGB200_CATCH
}

static void export_flat(FlatPlan const& f, dmrgb200_plan_desc* d);

dmrgb200_status dmrgb200_schedule_export(dmrgb200_schedule_t sc, dmrgb200_plan_desc* d) {
    if (!sc || !d) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    export_flat(sc->flat, d);
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_schedule_flops(dmrgb200_schedule_t sc, uint64_t* flops) {
    if (!sc || !flops) return fail(DMRGB200_INVALID_ARGUMENT, "null argument");
    *flops = sc->flat.flops();
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_schedule_term_sources(dmrgb200_schedule_t sc, uint32_t* term_src, double* term_dscale) {
    if (!sc) return fail(DMRGB200_INVALID_ARGUMENT, "null schedule");
    FlatPlan const& f = sc->flat;
    if (f.kind != KIND_HPSI || f.term_src.size() != f.n_terms())
        return fail(DMRGB200_NOT_SUPPORTED, "term provenance is recorded for H psi schedules only");
    if (term_src) std::copy(f.term_src.begin(), f.term_src.end(), term_src);
    if (term_dscale) std::copy(f.term_dscale.begin(), f.term_dscale.end(), term_dscale);
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_schedule_destroy(dmrgb200_schedule_t sc) {
    delete sc;
    return DMRGB200_OK;
}

dmrgb200_status dmrgb200_tensor_layout(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                       const dmrgb200_index_desc* right_i, int left_paired, uint32_t* n_blocks,
                                       uint32_t* rows, uint32_t* cols, uint64_t* offsets, uint64_t* total) {
    DMRGB200_TRY
    Index ph = to_index(phys), li = to_index(left_i), ri = to_index(right_i);
    TensorLayout t = left_paired ? left_paired_layout(ph, li, ri) : right_paired_layout(ph, li, ri);
    if (n_blocks) *n_blocks = uint32_t(t.rows.size());
    for (size_t b = 0; b < t.rows.size(); ++b) {
        if (rows) rows[b] = t.rows[b];
        if (cols) cols[b] = t.cols[b];
        if (offsets) offsets[b] = t.off[b];
    }
    if (total) *total = t.total;
    return DMRGB200_OK;
    DMRGB200_CATCH
}

static void export_flat(FlatPlan const& f, dmrgb200_plan_desc* d) {
    std::memset(d, 0, sizeof(*d));
    d->kind = dmrgb200_plan_kind(f.kind);
    d->n_groups = f.n_groups();
    d->g_t = f.g_t.data();
    d->g_c = f.g_c.data();
    d->n_in_blocks = uint32_t(f.in_rows.size());
    d->in_rows = f.in_rows.data();
    d->in_cols = f.in_cols.data();
    d->in_off = f.in_off.data();
    d->in_size = f.in_size;
    d->n_out_blocks = uint32_t(f.out_rows.size());
    d->out_rows = f.out_rows.data();
    d->out_cols = f.out_cols.data();
    d->out_off = f.out_off.data();
    d->out_size = f.out_size;
    d->n_t = f.n_t();
    d->t_lb = f.t_lb.data();
    d->t_col = f.t_col.data();
    d->t_ci = f.t_ci.data();
    d->t_trans = f.t_trans.data();
    d->t_nb = f.t_nb.data();
    d->t_brows = f.t_brows.data();
    d->t_bcols = f.t_bcols.data();
    d->t_width = f.t_width.empty() ? nullptr : f.t_width.data();
    d->n_cohorts = f.n_cohorts();
    d->c_lb = f.c_lb.data();
    d->c_rb = f.c_rb.data();
    d->c_ls = f.c_ls.data();
    d->c_rs = f.c_rs.data();
    d->c_ci = f.c_ci.data();
    d->c_trans = f.c_trans.data();
    d->c_nsrows = f.c_nsrows.data();
    d->c_stripe = f.c_stripe.data();
    d->c_out_ci = f.c_out_ci.data();
    d->c_unit = f.c_unit.data();
    d->n_units = f.n_units();
    d->u_offset = f.u_offset.data();
    d->u_ms = f.u_ms.data();
    d->u_line = f.u_line.data();
    d->n_lines = f.n_lines();
    d->l_b1 = f.l_b1.data();
    d->l_term = f.l_term.data();
    d->n_terms = f.n_terms();
    d->term_alpha = f.term_alpha.data();
    d->term_t = f.term_t.data();
    d->term_col = f.term_col.data();
}

}  // extern "C"
