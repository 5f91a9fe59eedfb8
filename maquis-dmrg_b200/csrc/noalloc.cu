// H·psi without any device allocation.
//
// Some callers cannot call cudaMalloc at the point where they need an H·psi:
// code that runs while a custom allocator or memory pool owns the device memory
// and forbids further allocations, hosts that only hand the library pre-placed
// buffers, and callers in contexts where an allocation could block or fail
// (e.g. while other work holds nearly all HBM).  dmrgb200_hpsi_noalloc serves
// them: it takes the flat plan description and the caller's device buffers
// (boundaries, x, y), and places everything else it needs -- the lowered tile
// and line tables and the T / S intermediates -- in one file-scope device array
// of fixed size, DMRGB200_NOALLOC_BYTES, that every GPU loading the library
// holds until the process exits.
//
// With CUDA's lazy module loading (the default since CUDA 12.2) the array is
// placed in device memory when its module is loaded on a device, which happens
// at the first cudaGetSymbolAddress below, i.e. on the first call on that
// device.  That first call therefore needs DMRGB200_NOALLOC_BYTES of free
// device memory: make it (with any plan that fits) before a pool or allocator
// takes the memory.  A failed placement is reported as DMRGB200_OUT_OF_MEMORY.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dmrgb200.h"
#include "device.hpp"
#include "plan.hpp"

namespace dmrgb200 {
// defined in capi.cpp
dmrgb200_status noalloc_fail(dmrgb200_status s, std::string const& msg);
void noalloc_desc_to_flat(const dmrgb200_plan_desc* d, FlatPlan& f);
}  // namespace dmrgb200

using namespace dmrgb200;

namespace {

constexpr size_t kScratchBytes = DMRGB200_NOALLOC_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// device address of the static array for the current device (looked up once per device)
dmrgb200_status scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(DMRGB200_NOT_SUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();  // reset the runtime's last-error state
            return noalloc_fail(DMRGB200_OUT_OF_MEMORY,
                                "placing the static scratch of dmrgb200_hpsi_noalloc (" +
                                    std::to_string(kScratchBytes) + " bytes) on this device failed: out of memory");
        }
        if (e != cudaSuccess || !p)
            return noalloc_fail(DMRGB200_DEVICE_ERROR,
                                std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return DMRGB200_OK;
}

template <class T>
size_t place(size_t& cursor, std::vector<T> const& v) {
    size_t off = (cursor + 255) / 256 * 256;
    cursor = off + v.size() * sizeof(T);
    return off;
}

}  // namespace

extern "C" dmrgb200_status dmrgb200_hpsi_noalloc(const dmrgb200_plan_desc* desc, const dmrgb200_boundary_view* left,
                                                 const dmrgb200_boundary_view* right, const double* x, double* y,
                                                 void* cuda_stream) {
    try {
        if (!desc || !left || !right || !x || !y) return noalloc_fail(DMRGB200_INVALID_ARGUMENT, "null argument");
        if (desc->kind != DMRGB200_PLAN_HPSI) return noalloc_fail(DMRGB200_INVALID_PLAN, "plan is not an H psi plan");
        FlatPlan f;
        noalloc_desc_to_flat(desc, f);
        std::string err = f.validate();
        if (!err.empty()) return noalloc_fail(DMRGB200_INVALID_PLAN, err);
        std::vector<uint64_t> lp(left->n_cohorts), rp(right->n_cohorts);
        for (uint32_t i = 0; i < left->n_cohorts; ++i) lp[i] = reinterpret_cast<uint64_t>(left->cohort_ptr[i]);
        for (uint32_t i = 0; i < right->n_cohorts; ++i) rp[i] = reinterpret_cast<uint64_t>(right->cohort_ptr[i]);
        for (uint32_t t = 0; t < f.n_t(); ++t)
            if (f.t_ci[t] >= rp.size() || !rp[f.t_ci[t]])
                return noalloc_fail(DMRGB200_INVALID_PLAN, "T task reads a right cohort without storage");
        for (uint32_t c = 0; c < f.n_cohorts(); ++c)
            if (f.c_ci[c] >= lp.size() || !lp[f.c_ci[c]])
                return noalloc_fail(DMRGB200_INVALID_PLAN, "cohort reads a left cohort without storage");

        DeviceProgram prog;
        compile_program(f, lp, rp, {}, prog);

        // layout inside the static array: tables, then T, then S (256-byte aligned)
        size_t cur = 0;
        size_t o_p1 = place(cur, prog.stage1.probs), o_s1 = place(cur, prog.stage1.segs),
               o_t1 = place(cur, prog.stage1.tiles), o_p3 = place(cur, prog.stage3.probs),
               o_s3 = place(cur, prog.stage3.segs), o_t3 = place(cur, prog.stage3.tiles), o_l = place(cur, prog.lines),
               o_k = place(cur, prog.terms), o_li = place(cur, prog.litems);
        size_t o_T = (cur + 255) / 256 * 256;
        size_t o_S = (o_T + prog.t_elems * sizeof(double) + 255) / 256 * 256;
        size_t need = o_S + prog.s_elems * sizeof(double);
        if (need > kScratchBytes)
            return noalloc_fail(DMRGB200_OUT_OF_MEMORY,
                                "plan needs " + std::to_string(need) + " bytes of scratch; the static area of "
                                "dmrgb200_hpsi_noalloc holds " + std::to_string(kScratchBytes) + " bytes");

        void* base = nullptr;
        dmrgb200_status st = scratch_address(&base);
        if (st != DMRGB200_OK) return st;
        unsigned char* b = static_cast<unsigned char*>(base);
        cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
        auto put = [&](size_t off, const void* src, size_t bytes) -> cudaError_t {
            if (!bytes) return cudaSuccess;
            return cudaMemcpyAsync(b + off, src, bytes, cudaMemcpyHostToDevice, stream);
        };
        cudaError_t e = cudaSuccess;
        e = e == cudaSuccess ? put(o_p1, prog.stage1.probs.data(), prog.stage1.probs.size() * sizeof(DevProb)) : e;
        e = e == cudaSuccess ? put(o_s1, prog.stage1.segs.data(), prog.stage1.segs.size() * sizeof(DevSeg)) : e;
        e = e == cudaSuccess ? put(o_t1, prog.stage1.tiles.data(), prog.stage1.tiles.size() * sizeof(DevTile)) : e;
        e = e == cudaSuccess ? put(o_p3, prog.stage3.probs.data(), prog.stage3.probs.size() * sizeof(DevProb)) : e;
        e = e == cudaSuccess ? put(o_s3, prog.stage3.segs.data(), prog.stage3.segs.size() * sizeof(DevSeg)) : e;
        e = e == cudaSuccess ? put(o_t3, prog.stage3.tiles.data(), prog.stage3.tiles.size() * sizeof(DevTile)) : e;
        e = e == cudaSuccess ? put(o_l, prog.lines.data(), prog.lines.size() * sizeof(DevSLine)) : e;
        e = e == cudaSuccess ? put(o_k, prog.terms.data(), prog.terms.size() * sizeof(DevSTerm)) : e;
        e = e == cudaSuccess ? put(o_li, prog.litems.data(), prog.litems.size() * sizeof(DevSItem)) : e;
        if (e != cudaSuccess)
            return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("table upload: ") + cudaGetErrorString(e));
        prog.d_p1 = reinterpret_cast<DevProb*>(b + o_p1);
        prog.d_s1 = reinterpret_cast<DevSeg*>(b + o_s1);
        prog.d_t1 = reinterpret_cast<DevTile*>(b + o_t1);
        prog.d_p3 = reinterpret_cast<DevProb*>(b + o_p3);
        prog.d_s3 = reinterpret_cast<DevSeg*>(b + o_s3);
        prog.d_t3 = reinterpret_cast<DevTile*>(b + o_t3);
        prog.d_lines = reinterpret_cast<DevSLine*>(b + o_l);
        prog.d_terms = reinterpret_cast<DevSTerm*>(b + o_k);
        prog.d_litems = reinterpret_cast<DevSItem*>(b + o_li);
        prog.n_t1 = uint32_t(prog.stage1.tiles.size());
        prog.n_t3 = uint32_t(prog.stage3.tiles.size());
        prog.n_lines = uint32_t(prog.lines.size());
        prog.n_litems = uint32_t(prog.litems.size());
        e = run_program(prog, reinterpret_cast<uint64_t>(x), reinterpret_cast<uint64_t>(y),
                        reinterpret_cast<double*>(b + o_T), reinterpret_cast<double*>(b + o_S), stream);
        if (e != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("launch: ") + cudaGetErrorString(e));
        // the host tables must outlive the pageable-memory copies above
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return noalloc_fail(DMRGB200_DEVICE_ERROR, std::string("execution: ") + cudaGetErrorString(e));
        return DMRGB200_OK;
    } catch (std::exception const& ex) {
        return noalloc_fail(DMRGB200_INVALID_ARGUMENT, ex.what());
    }
}
