/*
 * dmrgb200 — B200 (sm_100a) implementation of the QCMaquis DMRG hot path
 * behind a C ABI: the symmetry-blocked effective-Hamiltonian product H·psi and
 * the left/right boundary updates.
 *
 * Conventions
 *  - All numeric data is FP64, column-major, as in the reference's
 *    alps::numeric::matrix (dmrg/framework/alps/matrix/matrix.ipp:122).
 *  - Device pointers are plain CUDA device addresses; host pointers are plain
 *    host addresses.  No torch or C++ types cross this interface.
 *  - Every call returns dmrgb200_status; a call never exits the process.
 *    dmrgb200_last_error() returns a thread-local message for the last failure.
 *  - Calls are stream-ordered on the stream given (NULL = legacy default stream)
 *    and thread-compatible: one context per host thread.
 *
 * Two ways to obtain a plan:
 *  (1) dmrgb200_plan_create(): the caller flattens its own schedule
 *      (the reference's ScheduleNew / MPSBlock / Cohort) into
 *      dmrgb200_plan_desc.  This is the drop-in seam for the reference's
 *      C++ host code.
 *  (2) dmrgb200_*_plan_build(): the library's own schedule builder (a C++
 *      restatement of the reference's create_contraction_schedule and the
 *      lshtm_* / rshtm_* builders) from index, MPO and boundary descriptions.
 */
#ifndef DMRGB200_H
#define DMRGB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    DMRGB200_OK = 0,
    DMRGB200_INVALID_ARGUMENT = 1,
    DMRGB200_INVALID_PLAN = 2,
    DMRGB200_OUT_OF_MEMORY = 3,
    DMRGB200_DEVICE_ERROR = 4,
    DMRGB200_TIMEOUT = 5,
    DMRGB200_NUMERIC = 6,
    DMRGB200_NOT_SUPPORTED = 7
} dmrgb200_status;

typedef enum {
    DMRGB200_PREC_FP64 = 0,          /* native FP64 */
    DMRGB200_PREC_FP64_EMULATED = 1  /* split-precision FP64 emulation on the tensor cores */
} dmrgb200_precision;

typedef enum {
    DMRGB200_PLAN_HPSI = 0,        /* H·psi (super_hamil_mv) */
    DMRGB200_PLAN_LEFT_STEP = 1,   /* overlap_mpo_left_step */
    DMRGB200_PLAN_RIGHT_STEP = 2   /* overlap_mpo_right_step */
} dmrgb200_plan_kind;

typedef enum { DMRGB200_U1 = 1, DMRGB200_TWOU1 = 2, DMRGB200_SU2U1 = 3 } dmrgb200_symmetry;

typedef struct dmrgb200_context_s* dmrgb200_context_t;
typedef struct dmrgb200_plan_s* dmrgb200_plan_t;
typedef struct dmrgb200_mpo_s* dmrgb200_mpo_t;

const char* dmrgb200_status_string(dmrgb200_status s);
const char* dmrgb200_last_error(void);
int dmrgb200_abi_version(void);

/* ---- context ------------------------------------------------------------ */
/* Replaces accelerator::gpu / accelerator::device setup
 * (dmrg/framework/dmrg/solver/accelerator.h:36-135, accelerator.cpp:52-328). */
dmrgb200_status dmrgb200_context_create(int device, dmrgb200_context_t* out);
dmrgb200_status dmrgb200_context_destroy(dmrgb200_context_t ctx);

/* ---- flat plan description (the drop-in seam) ---------------------------- */
/* A flattened ScheduleNew (dmrg/framework/dmrg/solver/tasks.h:287-348).
 * Index arrays are host pointers; the library copies what it needs.
 *
 * Blocks ("in" = the right-paired input tensor psi / ket; "out" = the output
 * vector for H·psi, the bra tensor for boundary steps):
 *   element (r, c) of block b lives at base + off[b] + r + c*rows[b].
 * T tasks (MPSBlock::t_schedule, tasks.h:234-239): task t combines a column
 *   slice of in-block t_lb[t] (first column t_col[t]) with boundary cohort
 *   t_ci[t] (storage cohort ci_eff) that holds t_nb[t] blocks of logical size
 *   t_brows[t] x t_bcols[t] (stored transposed when t_trans[t]).
 *   H·psi / right step (MPSBlock::create_T, tasks.cpp:650-705):
 *     T_b = in[:, t_col + (0..t_brows)] * B_b            (rows x t_bcols)
 *   left step (MPSBlock::create_T_left, tasks.cpp:545-601):
 *     T_b = B_b * in[:, t_col + (0..t_width)] restricted to t_bcols rows
 *                                                        (t_brows x t_width)
 * Cohorts (Cohort, tasks.h:50-190): c_lb / c_rb / c_ls / c_rs as in the
 *   reference (for H·psi: input block, output block, their row counts),
 *   c_ci / c_trans the other boundary's storage cohort (H·psi only),
 *   c_nsrows S row blocks, c_stripe S columns, units [c_unit[c], c_unit[c+1]).
 *   For step plans c_out_ci is the new boundary's cohort index.
 * Units (SUnit): u_offset, u_ms, lines [u_line[u], u_line[u+1]).
 * Lines (one per b2s entry): l_b1 (S row block), terms [l_term[l], l_term[l+1]).
 * Terms: alpha, T task index (global), boundary column (tidx pair).
 * Task groups (one MPSBlock each): T tasks [g_t[g], g_t[g+1]) and cohorts
 * [g_c[g], g_c[g+1]); a cohort's terms reference T tasks of its own group. */
typedef struct {
    dmrgb200_plan_kind kind;
    uint32_t n_groups;
    const uint32_t* g_t; /* n_groups + 1 */
    const uint32_t* g_c; /* n_groups + 1 */
    uint32_t n_in_blocks;
    const uint32_t* in_rows;
    const uint32_t* in_cols;
    const uint64_t* in_off;
    uint64_t in_size;
    uint32_t n_out_blocks;
    const uint32_t* out_rows;
    const uint32_t* out_cols;
    const uint64_t* out_off;
    uint64_t out_size;

    uint32_t n_t;
    const uint32_t* t_lb;
    const uint32_t* t_col;
    const uint32_t* t_ci;
    const uint8_t* t_trans;
    const uint32_t* t_nb;
    const uint32_t* t_brows;
    const uint32_t* t_bcols;
    const uint32_t* t_width; /* left step only (may be NULL otherwise) */

    uint32_t n_cohorts;
    const uint32_t* c_lb;
    const uint32_t* c_rb;
    const uint32_t* c_ls;
    const uint32_t* c_rs;
    const uint32_t* c_ci;
    const uint8_t* c_trans;
    const uint32_t* c_nsrows;
    const uint32_t* c_stripe;
    const uint32_t* c_out_ci;
    const uint32_t* c_unit; /* n_cohorts + 1 */

    uint32_t n_units;
    const uint32_t* u_offset;
    const uint32_t* u_ms;
    const uint32_t* u_line; /* n_units + 1 */

    uint32_t n_lines;
    const uint32_t* l_b1;
    const uint32_t* l_term; /* n_lines + 1 */

    uint32_t n_terms;
    const double* term_alpha;
    const uint32_t* term_t;
    const uint32_t* term_col;
} dmrgb200_plan_desc;

/* Boundary cohort storage bound to a plan: n_cohorts device pointers, one per
 * cohort index ci (NULL for Hermitian-complement cohorts without storage);
 * replaces BoundaryView (dmrg/framework/dmrg/solver/solver.h:38-43). */
typedef struct {
    uint32_t n_cohorts;
    const double* const* cohort_ptr; /* host array of device pointers */
} dmrgb200_boundary_view;

/* Build an executable plan from a flattened schedule.  For H·psi, `left` is
 * the left boundary L and `other` the right boundary R (both stay resident and
 * must outlive the plan).  For a left step `left` is the input boundary; for a
 * right step `other` is.  Replaces ScheduleNew::stage_gpu (tasks.cpp:918-977). */
dmrgb200_status dmrgb200_plan_create(dmrgb200_context_t ctx, const dmrgb200_plan_desc* desc,
                                     const dmrgb200_boundary_view* left, const dmrgb200_boundary_view* other,
                                     dmrgb200_plan_t* out);
dmrgb200_status dmrgb200_plan_destroy(dmrgb200_plan_t plan);

/* Host-only structural validation of a plan description (no device needed):
 * array lengths, index ranges, slice bounds and shape consistency.  Returns
 * DMRGB200_INVALID_PLAN with a message for inconsistent input. */
dmrgb200_status dmrgb200_plan_validate(const dmrgb200_plan_desc* desc);

/* Batched H·psi (independent site problems in one plan): n H·psi plan
 * descriptions with their left / right boundary views are concatenated so that
 * each stage of dmrgb200_hpsi is one launch over the tiles of all instances.
 * Instance i's vector occupies the elements [in_base[i], in_base[i] + size_i)
 * of the batched x and y (128-element aligned), returned in in_base (n entries,
 * may be NULL); dmrgb200_plan_flops reports the sum over instances.  No
 * counterpart in the reference, which runs one site problem at a time. */
dmrgb200_status dmrgb200_plan_create_batched(dmrgb200_context_t ctx, uint32_t n, const dmrgb200_plan_desc* descs,
                                             const dmrgb200_boundary_view* lefts,
                                             const dmrgb200_boundary_view* rights, uint64_t* in_base,
                                             uint64_t* total_size, dmrgb200_plan_t* out);

/* Algorithmic FP64 flop count of one execution, the reference's formula
 * (Cohort::n_flops tasks.cpp:388-398 + MPSBlock::n_flops :777-796). */
dmrgb200_status dmrgb200_plan_flops(dmrgb200_plan_t plan, uint64_t* flops);
/* Device scratch (T and S intermediates) the plan holds, in bytes. */
dmrgb200_status dmrgb200_plan_scratch_bytes(dmrgb200_plan_t plan, uint64_t* bytes);

/* ---- H·psi -------------------------------------------------------------- */
/* y = H_eff x for a DMRGB200_PLAN_HPSI plan.  x and y are device vectors laid
 * out as the plan's in/out blocks (DavidsonVector layout,
 * davidson_vector.cpp:87-152); y's block elements are overwritten, its padding
 * is left untouched.  Replaces super_hamil_mv (super_hamil_mv.hpp:100-155) and
 * ietl::mult (ietl_interface_dv.h:112-118).  DMRGB200_PREC_FP64_EMULATED runs
 * the T and cohort contractions on the INT8 tensor cores (Ozaki split, see
 * dmrgb200_plan_set_slices) and the S build in FP64, stream-ordered like the
 * FP64 path.  The first emulated call of a plan allocates its digit-plane
 * scratch (make it before capturing the stream; DMRGB200_NOT_SUPPORTED
 * otherwise) and makes the digit planes of the boundaries, which later calls
 * reuse (the boundaries of a site problem do not change while it is solved);
 * dmrgb200_plan_set_slices with a new slice count makes them again.  Kernel
 * waits that run out are recorded on the device and reported by the next
 * dmrgb200_plan_check or dmrgb200_solve. */
dmrgb200_status dmrgb200_hpsi(dmrgb200_plan_t plan, const double* x, double* y, dmrgb200_precision prec,
                              void* cuda_stream);

/* H·psi with the reference's launch pattern, for comparison with the grouped
 * kernels: one cuBLAS DGEMM per T task (per stored block for transposed cohorts)
 * as MPSBlock::create_T_gpu (dmrg/framework/dmrg/solver/tasks.cpp:707-752), the
 * library's S build, and one cuBLAS DGEMM per cohort into its output block as
 * Cohort::contract_gpu (tasks.cpp:315-344), all on cuda_stream.  y's block
 * elements are overwritten.  *launches (may be NULL) receives the number of
 * launches made.  Same sums as dmrgb200_hpsi up to the addition order inside
 * the library GEMMs. */
dmrgb200_status dmrgb200_hpsi_per_block(dmrgb200_plan_t plan, const double* x, double* y, void* cuda_stream,
                                        uint64_t* launches);

/* Autotuning of the grouped FP64 GEMMs: every variant (pipeline depth x CTAs
 * per SM) is timed on the plan's stage-1 and stage-3 tile lists and the
 * fastest is kept per stage.  The first FP64 dmrgb200_hpsi / dmrgb200_solve of
 * a plan of at least 50 MFLOP per H·psi does this by itself (environment
 * DMRGB200_AUTOTUNE=0 keeps the default variant); this call re-tunes now, using x (in layout) and y (out
 * layout, overwritten), and returns the chosen variant per stage.  No
 * counterpart in the reference (its cuBLAS calls are untuned). */
dmrgb200_status dmrgb200_plan_autotune(dmrgb200_plan_t plan, const double* x, double* y, void* cuda_stream,
                                       int32_t variants[2]);
const char* dmrgb200_gemm_variant_name(int variant);
/* Number of grouped-GEMM variants (valid variant indices are 0 .. count - 1). */
int dmrgb200_gemm_variant_count(void);
/* Pin the grouped-GEMM variant of stage 1 and of stage 3 of an H·psi plan (each 0 ..
 * dmrgb200_gemm_variant_count() - 1) instead of the autotuner's choice: later calls use
 * them and do not tune the plan (dmrgb200_plan_autotune re-tunes).  The sums are the same
 * for every variant up to the order of the K steps.  No counterpart in the reference. */
dmrgb200_status dmrgb200_plan_set_gemm_variants(dmrgb200_plan_t plan, int32_t stage1, int32_t stage3);

/* H·psi with host buffers, the counterpart of the reference's super_hamil_mv on
 * host DavidsonVectors (solver/super_hamil_mv.hpp:100-155): x_host (the plan's in
 * layout, in_size doubles) is copied to the device, y_host (out layout, out_size
 * doubles) receives H·psi.  Stage 1 runs in four parts by input range and stage 3
 * in four parts by output range, so the copies of one range overlap the products
 * of another; the result is bitwise that of dmrgb200_hpsi.  Pin the host buffers
 * (cudaHostAlloc / cudaHostRegister) for the copies to overlap.  Stream-ordered on
 * cuda_stream: synchronise it before reading y_host.  The first call builds the
 * split program and device copies of x and y (kept by the plan); the sequence is
 * captured as one CUDA graph per (x_host, y_host) pair, so reusing the same host
 * buffers costs one graph launch per call. */
dmrgb200_status dmrgb200_hpsi_host(dmrgb200_plan_t plan, const double* x_host, double* y_host, void* cuda_stream);

/* Adjoint of H·psi (no counterpart in the reference, which has no derivative
 * code).  With the plan's terms y = sum_k alpha_k H_k x, one call gives
 *   gx          = H^T w                      (the plan's in layout; may be NULL)
 *   galpha[k]   = <w | H_k x>  = d<w|H x>/d alpha_k, k in plan term order
 *                                            (device, n_terms doubles; may be NULL)
 * in native FP64: T = x-slices * R (create_T), G = L^T w per cohort (the
 * transpose of contract), galpha[k] = <G cell, T cell> (the transpose of
 * create_s_r), gT = sum_k alpha_k G cells, gx = gT * R^T (the transpose of
 * create_T).  w uses the out layout and x the in layout.  gx is overwritten over
 * its whole padded range (uncovered columns and padding become zero).  For a
 * Hermitian effective Hamiltonian (a Hermitian MPO with boundaries of one MPS)
 * H^T w = H w, and d<psi|H|psi>/d psi = 2 H psi.  Derivatives with respect to
 * the MPO term scales follow from galpha and dmrgb200_schedule_term_sources.
 * Bitwise reproducible; returns DMRGB200_INVALID_PLAN for plans whose T-task
 * slices of one input block overlap (no such plan comes from the builders). */
dmrgb200_status dmrgb200_hpsi_adjoint(dmrgb200_plan_t plan, const double* w, const double* x, double* gx,
                                      double* galpha, void* cuda_stream);

/* Synchronise `cuda_stream` and report the device-side error words of the plan's
 * kernels since the last check (bounded waits of the grouped S build and of the
 * emulated stages that ran out): DMRGB200_TIMEOUT if any did (the results of
 * those calls are not valid; the words are cleared and the plan stays usable),
 * DMRGB200_OK otherwise.  The asynchronous dmrgb200_hpsi calls report such
 * failures only here.  No counterpart in the reference, whose kernels do not
 * wait on the device. */
dmrgb200_status dmrgb200_plan_check(dmrgb200_plan_t plan, void* cuda_stream);

/* Limit, in nanoseconds, of the device-side waits for pipeline data in the
 * grouped S build and the emulated stages (bulk copies completing on shared-memory
 * barriers); 0 restores the default of 2 s.  A wait that runs out sets the plan's
 * error word, the kernel lets the copies and MMAs it has in flight complete (with a
 * fixed 2 s limit), releases its tensor memory and returns; dmrgb200_plan_check or
 * dmrgb200_solve then reports DMRGB200_TIMEOUT and the plan stays usable.
 * Process-wide; read at every launch (a captured solver graph keeps the value of
 * its capture).  No counterpart in the reference, whose kernels do not wait on the
 * device. */
dmrgb200_status dmrgb200_set_wait_limit(uint64_t ns);

/* The boundary buffers bound to the plan were rewritten in place (a sweep that
 * keeps one buffer per bond and reuses the plan): the emulated path drops the digit
 * planes it keeps of the boundaries and makes them again on its next call (FP64
 * execution keeps nothing derived from the boundary values).  No counterpart in
 * the reference, which rebuilds its schedules at every site. */
dmrgb200_status dmrgb200_plan_boundaries_changed(dmrgb200_plan_t plan);

/* Precision of the H·psi inside dmrgb200_solve (default DMRGB200_PREC_FP64):
 * with DMRGB200_PREC_FP64_EMULATED the contractions of every H·psi run emulated
 * on the INT8 tensor cores while orthogonalisation, Rayleigh-Ritz, residuals and
 * energies stay in native FP64.  Changing it drops the plan's cached solver
 * graph. */
dmrgb200_status dmrgb200_plan_set_precision(dmrgb200_plan_t plan, int prec);

/* Slice count from an error target: H·psi of x (the plan's in layout) in FP64
 * against emulated H·psi with 3, 4, ... 8 digit planes; the smallest count whose
 * relative error ||y_emu - y_fp64|| / ||y_fp64|| is at most `target` is kept
 * (as by dmrgb200_plan_set_slices) and returned with its error.
 * DMRGB200_NUMERIC if 8 planes miss the target (8 is kept).  Synchronises the
 * stream. */
dmrgb200_status dmrgb200_plan_tune_slices(dmrgb200_plan_t plan, const double* x, double target, void* cuda_stream,
                                          int* slices, double* rel_err);

/* Digit planes per operand (2..8, default 7) used by DMRGB200_PREC_FP64_EMULATED:
 * the relative error of each emulated contraction is about 2^(-7 slices) of
 * its row / column maxima (7: below 1e-13, 6: about 1e-11, 5: about 1e-9). */
dmrgb200_status dmrgb200_plan_set_slices(dmrgb200_plan_t plan, int slices);

/* Per-stage timing of H·psi executions and boundary steps: when enabled, every
 * dmrgb200_hpsi / dmrgb200_step_execute call records CUDA events around its
 * stages on the call's stream (device time only, not the host-side lowering of
 * a step plan).
 * dmrgb200_plan_stage_times synchronises the last recorded events and returns
 * the accumulated milliseconds and the number of timed calls; stage 0 = T
 * GEMMs (create_T), 1 = S build (create_s_r), 2 = cohort contraction
 * (contract).  Algorithmic flops per stage per call are returned in flops[3]. */
dmrgb200_status dmrgb200_plan_set_timing(dmrgb200_plan_t plan, int enable);
dmrgb200_status dmrgb200_plan_stage_times(dmrgb200_plan_t plan, double ms[3], uint64_t flops[3], uint64_t* calls);

/* Roofline calibration on the current device: what = 0 measures the FP64
 * tensor-core (DMMA) rate of a register-resident loop in TFLOP/s.  Used as the
 * denominator of the native-FP64 roofline. */
dmrgb200_status dmrgb200_calibrate(int what, double* value);

/* ---- SU(2) recoupling utilities (arguments are twice the angular momenta) --- */
/* The coefficients the SU2U1 schedule builder folds into alpha: Wigner 6j and
 * 9j symbols (the reference links GSL's gsl_sf_coupling_6j/9j,
 * block_matrix/symmetry/gsl_coupling.h:30-34) and the four reduced-matrix-element
 * couplings of set_coupling (gsl_coupling.h:72-92). */
double dmrgb200_wigner6j(int two_j1, int two_j2, int two_j3, int two_j4, int two_j5, int two_j6);
double dmrgb200_wigner9j(int two_j1, int two_j2, int two_j3, int two_j4, int two_j5, int two_j6, int two_j7,
                         int two_j8, int two_j9);
void dmrgb200_set_coupling(int a, int b, int c, int d, int e, int f, int g, int h, int i, double init,
                           double couplings[4]);

/* ---- plain FP64 GEMM on the grouped DMMA kernel --------------------------- */
/* C = A * B (column-major FP64, A M x K, B K x N) with grouped-GEMM variant
 * `variant` (0 .. dmrgb200_gemm_variant_count() - 1, see
 * dmrgb200_gemm_variant_name) as one problem; for
 * measuring the H·psi kernel on regular shapes.  No counterpart in the
 * reference (it calls BLAS).  Allocates its tile tables per call; returns
 * after completion. */
dmrgb200_status dmrgb200_dgemm_f64(uint32_t M, uint32_t N, uint32_t K, const double* A, uint64_t lda,
                                   const double* B, uint64_t ldb, double* C, uint64_t ldc, int variant,
                                   void* cuda_stream);

/* ---- FP64 GEMM emulated on the INT8 tensor cores --------------------------- */
/* C = A * B (column-major FP64, A M x K, B K x N) computed with `slices`
 * (2..8) signed 7-bit digit planes per operand on tcgen05 INT8 MMAs with exact
 * INT32 accumulation and FP64 recombination (Ozaki scheme, integer variant);
 * relative accuracy about 2^(-7 slices) of the row/column maxima.  K beyond
 * 2^17 / slices accumulates in exact INT32 chunks of that length, summed in
 * FP64.  Stream-ordered; returns after completion. */
dmrgb200_status dmrgb200_dgemm_emulated(uint32_t M, uint32_t N, uint32_t K, const double* A, uint64_t lda,
                                        const double* B, uint64_t ldb, double* C, uint64_t ldc, int slices,
                                        void* cuda_stream);

/* ---- two-site split on the device ----------------------------------------- */
/* Thin SVD of every block of a block matrix: for block i (column-major,
 * rows[i] x cols[i], ld rows[i], device memory) writes U (rows x k, ld rows),
 * the singular values s (k, descending) and V^T (k x cols, ld k), k =
 * min(rows, cols); replaces the per-block loop of svd(block_matrix)
 * (dmrg/framework/dmrg/block_matrix/block_matrix_algorithms.h:95-113).  The
 * pointer arrays are host arrays of device pointers.  One-sided Jacobi in FP64:
 * singular values to high relative accuracy; the U columns of zero singular
 * values are zero.  Blocks with a zero extent are skipped.  Stream-ordered;
 * returns after completion (DMRGB200_NUMERIC if the sweeps do not converge). */
dmrgb200_status dmrgb200_block_svd(uint32_t n_blocks, const uint32_t* rows, const uint32_t* cols,
                                   const double* const* a, double* const* u, double* const* s,
                                   double* const* vt, void* cuda_stream);

typedef enum { DMRGB200_SCALE_NONE = 0, DMRGB200_SCALE_ROWS = 1, DMRGB200_SCALE_COLS = 2 } dmrgb200_scale_mode;

/* dst[dst_off + i + j dst_ld] = src[src_off + i + j src_ld] (times
 * scale[scale_off + i] for DMRGB200_SCALE_ROWS, scale[scale_off + j] for
 * DMRGB200_SCALE_COLS), 0 <= i < rows, 0 <= j < cols; offsets in elements. */
typedef struct {
    uint64_t src_off, dst_off, scale_off;
    uint32_t src_ld, dst_ld;
    uint32_t rows, cols;
    uint32_t scale_mode, reserved;
} dmrgb200_block_copy;

/* Block copies between device buffers: the gather of the two-site matrix
 * Theta and the scatter of U, S V^T (or U S, V^T) into the site tensors
 * (TwoSiteTensor::split_mps_l2r / split_mps_r2l,
 * dmrg/framework/dmrg/mp_tensors/twositetensor.hpp:153-200).  `copies` is a host
 * array that may be released on return; destinations must not overlap; the
 * offsets are not checked against the buffers.  Stream-ordered; the upload of
 * the descriptors from pageable memory may first wait for the stream. */
dmrgb200_status dmrgb200_copy_blocks(uint32_t n, const dmrgb200_block_copy* copies, const double* src, double* dst,
                                     const double* scale, void* cuda_stream);

/* ---- eigensolver ---------------------------------------------------------- */
/* Lowest eigenpair of H_eff by Jacobi-Davidson in FP64 on the device
 * (solve<double>, dmrg/framework/dmrg/solver/solver.cpp:13-28 ->
 * solve_ietl_jcd, solver/ietl_jacobi_davidson.h:35-76 -> ietl/jacobi.h:386-520,
 * with ietl_jcd_gmres = 0): MGS with refinement (kappa 0.25), projection of the
 * n_ortho orthogonal vectors (host array of device vectors), Rayleigh-Ritz,
 * convergence |r| <= tol |theta| or |r| < tol, at most max_iter (1..32) H·psi
 * applications.  x0 and x_out are device vectors of n doubles in the plan's
 * block layout with zero padding.  *energy = theta (no core energy). */
typedef struct {
    uint32_t iterations;
    int32_t converged;
    double residual;
    double hpsi_ms;  /* device time in H·psi (stepwise solver; 0 for the graph solver) */
    double solve_ms; /* device time of the whole solve */
} dmrgb200_solve_stats;
dmrgb200_status dmrgb200_solve(dmrgb200_plan_t plan, uint64_t n, const double* x0, const double* const* ortho,
                               uint32_t n_ortho, double tol, uint32_t max_iter, double* energy, double* x_out,
                               dmrgb200_solve_stats* stats, void* cuda_stream);

/* How dmrgb200_solve drives the iteration.
 * DMRGB200_SOLVER_GRAPH (default): all scalars stay on the device and the whole
 *   solve is one CUDA graph launch (one iteration = the body of a conditional
 *   WHILE node), built on the first solve and reused while n, max_iter,
 *   n_ortho and tol stay the same; one host synchronisation per solve.
 * DMRGB200_SOLVER_STEPWISE: the host reads the scalars each iteration (as the
 *   reference's solver does) and times each H·psi. */
enum { DMRGB200_SOLVER_GRAPH = 0, DMRGB200_SOLVER_STEPWISE = 1 };
dmrgb200_status dmrgb200_plan_set_solver(dmrgb200_plan_t plan, int mode);

/* ---- H·psi for callers that cannot allocate device memory --------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * when they need an H·psi (a custom allocator or memory pool owns the device
 * memory and forbids further allocations, or the host only hands the library
 * pre-placed buffers): y = H_eff x from the flat plan description, the caller's
 * device boundaries (left = L, right = R) and device vectors x, y, with every
 * other device byte (lowered tile tables and the T / S intermediates) taken
 * from one static device array of DMRGB200_NOALLOC_BYTES that each GPU loading
 * the library holds until the process exits.  The call allocates no device
 * memory.  Plans needing more than that return DMRGB200_OUT_OF_MEMORY with a
 * message giving the required size.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current; under
 * CUDA's lazy module loading (the default since CUDA 12.2) that lookup is also
 * when the array is placed in device memory, so the first call on a device
 * needs DMRGB200_NOALLOC_BYTES of free device memory (DMRGB200_OUT_OF_MEMORY
 * otherwise): make it before a pool or allocator takes the memory.  All calls
 * share the one array (it keeps the last call's contents; nothing in it needs
 * to start at zero), so calls whose executions overlap on the GPU race:
 * serialise them, e.g. on one stream.  The call copies its tables from host
 * memory and synchronises `cuda_stream` before returning, so it must not be
 * made while that stream is being captured. */
#define DMRGB200_NOALLOC_BYTES (64ull << 20)
dmrgb200_status dmrgb200_hpsi_noalloc(const dmrgb200_plan_desc* desc, const dmrgb200_boundary_view* left,
                                      const dmrgb200_boundary_view* right, const double* x, double* y,
                                      void* cuda_stream);

/* ---- boundary steps on a flattened plan --------------------------------- */
/* Execute a LEFT_STEP / RIGHT_STEP plan.  ket: right-paired device tensor
 * (plan in-blocks); bra: left-paired (left step) or right-paired (right step)
 * device tensor (plan out-blocks); out: device pointers of the new boundary's
 * cohorts (indexed by c_out_ci); every stored element of those cohorts is
 * written.
 * Replaces the GPU branches of overlap_mpo_left_step / overlap_mpo_right_step
 * (move_boundary.hpp:215-259, :342-384). */
dmrgb200_status dmrgb200_step_execute(dmrgb200_plan_t plan, const double* ket, const double* bra,
                                      const dmrgb200_boundary_view* out, void* cuda_stream);

/* Density matrix of a two-site split with the state prediction (perturbation) on a
 * LEFT_STEP / RIGHT_STEP plan built for the two-site tensor Theta viewed as one site
 * (ket = bra = Theta; left step: site 1 with the middle index as its right bond,
 * right step: site 2 with the middle index as its left bond; boundary skipping off):
 *   left step:  dm[b] = Theta_b Theta_b^T + alpha sum_{c: c_lb = b} S_c S_c^T
 *   right step: dm[b] = Theta_b^T Theta_b + alpha sum_{c: c_rb = b} S_c^T S_c
 * for every bra block b (left-paired blocks for the left step, right-paired for the
 * right step); S_c is the cohort's S of the step.  ket and bra are Theta in the
 * layouts dmrgb200_step_execute takes (ket right-paired; bra left-paired for the left
 * step, right-paired for the right step).  dm->cohort_ptr[b] is a device
 * stripe_b x stripe_b column-major block (stripe_b = out_rows[b] for the left step,
 * out_cols[b] for the right step), overwritten; alpha >= 0.  Stream-ordered (the
 * host-side lowering happens on the first call with a given dm binding).
 * Replaces the GPU side of alpha_dm / alpha_dm_right with alpha_dm_direct and
 * Cohort::lbtm / rbtm (prediction.hpp:41-69, move_boundary.hpp:38-143,
 * tasks.cpp:346-380), used by predict_split_l2r / r2l (prediction.hpp:152-240). */
dmrgb200_status dmrgb200_step_alpha_dm(dmrgb200_plan_t plan, const double* ket, const double* bra,
                                       const dmrgb200_boundary_view* dm, double alpha, void* cuda_stream);

/* ---- library-side schedule builder (host only) -------------------------- */
/* Index description: n sectors, charges[2*i+0..1] (U1 uses component 0),
 * sizes[i]. */
typedef struct {
    uint32_t n;
    const int32_t* charges;
    const uint32_t* sizes;
} dmrgb200_index_desc;

/* MPO tensor description (MPOTensor, dmrg/framework/dmrg/mp_tensors/mpotensor.h:45-135).
 * Terms (b1, b2, op, scale) must be sorted by (b1, b2); several terms may share
 * (b1, b2).  Operators: op_block[o]..op_block[o+1] index blocks; block k has
 * input charge blk_in[2k..], output charge blk_out[2k..] and entries
 * blk_entry[k]..blk_entry[k+1] (row, col, row spin, col spin, coeff) in
 * row-major order (SparseOperator, block_matrix/sparse_operator.h:35-235).
 * Spins and Hermitian data may be NULL (no SU2, no Hermitian partners). */
typedef struct {
    dmrgb200_symmetry symm;
    uint32_t row_dim, col_dim;
    const int32_t* left_spin;
    const int32_t* right_spin;
    const uint32_t* left_herm;   /* partner index or UINT32_MAX */
    const int32_t* left_phase;
    const uint32_t* right_herm;
    const int32_t* right_phase;
    uint32_t n_terms;
    const uint32_t* term_b1;
    const uint32_t* term_b2;
    const uint32_t* term_op;
    const double* term_scale;
    uint32_t n_ops;
    const int32_t* op_spin;
    const uint32_t* op_block; /* n_ops + 1 */
    const int32_t* blk_in;
    const int32_t* blk_out;
    const uint32_t* blk_entry; /* n_blocks + 1 */
    const uint32_t* e_row;
    const uint32_t* e_col;
    const int32_t* e_row_spin;
    const int32_t* e_col_spin;
    const double* e_coeff;
} dmrgb200_mpo_desc;

typedef struct dmrgb200_bindex_s* dmrgb200_bindex_t;     /* boundary index */
typedef struct dmrgb200_schedule_s* dmrgb200_schedule_t; /* host-side flat plan */

dmrgb200_status dmrgb200_mpo_create(const dmrgb200_mpo_desc* desc, dmrgb200_mpo_t* out);
dmrgb200_status dmrgb200_mpo_destroy(dmrgb200_mpo_t mpo);

/* Boundary index (BoundaryIndex, mp_tensors/boundary.h:76-234) with the
 * library's storage layout: every cohort with storage occupies
 * cohort_size doubles at a 32-double aligned storage offset of one buffer of
 * n_elements doubles.  The caller owns the buffer (host or device).
 * Edge index: the reference's Boundary(ud, ld, ad) (boundary.h:257-283), one
 * diagonal cohort per sector with aux_dim blocks; its values are all ones. */
dmrgb200_status dmrgb200_bindex_create_edge(dmrgb200_symmetry symm, const dmrgb200_index_desc* index,
                                            uint32_t aux_dim, dmrgb200_bindex_t* out);
dmrgb200_status dmrgb200_bindex_destroy(dmrgb200_bindex_t b);
dmrgb200_status dmrgb200_bindex_info(dmrgb200_bindex_t b, uint32_t* n_cohorts, uint32_t* aux_dim,
                                     uint64_t* n_elements);
/* Per cohort ci: bra block, ket block, tr flag, storage offset (UINT64_MAX
 * without storage), left/right size, n_blocks; per (ci, b): offset (-1 absent),
 * conjugate scale, transposed flag.  Any output pointer may be NULL. */
dmrgb200_status dmrgb200_bindex_describe(dmrgb200_bindex_t b, uint32_t* lb, uint32_t* rb, uint8_t* tr,
                                         uint64_t* storage_off, uint32_t* lsize, uint32_t* rsize,
                                         uint32_t* nblocks, int64_t* offsets, double* conj_scales,
                                         uint8_t* transposes);

/* H·psi schedule (create_contraction_schedule, site_hamil_schedule.hpp:40-93)
 * for a right-paired psi with the given physical, left and right indices. */
dmrgb200_status dmrgb200_schedule_hpsi(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                       const dmrgb200_index_desc* right_i, dmrgb200_mpo_t mpo,
                                       dmrgb200_bindex_t L, dmrgb200_bindex_t R, dmrgb200_schedule_t* out);
/* Left-step schedule (overlap_mpo_left_step, move_boundary.hpp:147-279) for a
 * site tensor with bra = ket indices; returns the new boundary index. */
dmrgb200_status dmrgb200_schedule_left_step(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                            const dmrgb200_index_desc* right_i, dmrgb200_mpo_t mpo,
                                            dmrgb200_bindex_t L, int symmetric, dmrgb200_schedule_t* out,
                                            dmrgb200_bindex_t* new_index);
/* Right-step schedule (overlap_mpo_right_step, move_boundary.hpp:281-404). */
dmrgb200_status dmrgb200_schedule_right_step(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                             const dmrgb200_index_desc* right_i, dmrgb200_mpo_t mpo,
                                             dmrgb200_bindex_t R, int symmetric, dmrgb200_schedule_t* out,
                                             dmrgb200_bindex_t* new_index);
/* Flat description of a schedule (arrays owned by the schedule). */
dmrgb200_status dmrgb200_schedule_export(dmrgb200_schedule_t s, dmrgb200_plan_desc* desc);
dmrgb200_status dmrgb200_schedule_flops(dmrgb200_schedule_t s, uint64_t* flops);
/* Provenance of the exported terms of an H·psi schedule, in plan term order:
 * term_src[k] = index of the MPO term (in the dmrgb200_mpo_desc order) that
 * produced term k and term_dscale[k] = d alpha_k / d term_scale[term_src[k]]
 * (alpha is linear in each term scale: it is coefficient * SU2 coupling *
 * boundary conjugate scales * term scale, op_iterate.hpp:37-69,
 * site_hamil_tasks.hpp:120-125).  So d<w|H x>/d term_scale[j] =
 * sum over k with term_src[k] = j of term_dscale[k] * galpha[k].  Arrays hold
 * n_terms entries; either may be NULL. */
dmrgb200_status dmrgb200_schedule_term_sources(dmrgb200_schedule_t s, uint32_t* term_src, double* term_dscale);
dmrgb200_status dmrgb200_schedule_destroy(dmrgb200_schedule_t s);

/* Block layout of an MPS tensor: right-paired (left_paired = 0: one block per
 * left sector, rows = left size, cols = sum over sigma of d_sigma * right size)
 * or left-paired (one block per right sector).  Offsets are 128-element padded
 * (davidson_vector.cpp:96-97).  Arrays have room for the number of blocks
 * (left_i->n or right_i->n); *n_blocks receives the count and *total the size. */
dmrgb200_status dmrgb200_tensor_layout(const dmrgb200_index_desc* phys, const dmrgb200_index_desc* left_i,
                                       const dmrgb200_index_desc* right_i, int left_paired, uint32_t* n_blocks,
                                       uint32_t* rows, uint32_t* cols, uint64_t* offsets, uint64_t* total);

#ifdef __cplusplus
}
#endif

#endif /* DMRGB200_H */
