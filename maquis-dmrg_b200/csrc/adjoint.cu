// Adjoint of the H psi plan in native FP64.
//
// The forward product is y = sum_c L_c S_c with S_c cells = sum_k alpha_k T
// cells and T_t = x-slice * R_t (create_T, create_s_r, contract;
// solver/tasks.cpp:650-705, 466-494, 286-313).  Its transpose runs the stages
// backwards on the same scratch buffers:
//   G_c  = L_c^T w                 grouped GEMM, into the S scratch
//   galpha[k] = <G cell(k), T cell(k)>   (T from the forward stage 1 on x)
//   gT cell   = sum_k alpha_k G cell(k)  into the T scratch (after galpha)
//   gx slice  = sum over the slice's T tasks of gT_t R_t^T   grouped GEMM
// Every output (G cell, galpha entry, gT block, gx tile) has exactly one
// writer, so the result is bitwise reproducible without atomics.
#include <algorithm>
#include <map>
#include <tuple>

#include "device.hpp"

namespace dmrgb200 {

namespace {

// galpha: one warp per term, fixed-order lane sums and a butterfly reduction
__global__ void __launch_bounds__(256) alpha_grad(const DevATerm* __restrict__ at, uint32_t n,
                                                  const double* __restrict__ G, const double* __restrict__ T,
                                                  double* __restrict__ galpha) {
    const uint32_t lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (uint32_t i = blockIdx.x * warps + (threadIdx.x >> 5); i < n; i += gridDim.x * warps) {
        const DevATerm a = at[i];
        double s = 0.0;
        if (a.rows) {
            // column-major walk in steps of 32 without per-element division
            const uint32_t dr = 32u % a.rows, dc = 32u / a.rows;
            uint32_t r = lane % a.rows, c = lane / a.rows;
            while (c < a.cols) {
                s = fma(G[a.g_base + r + uint64_t(c) * a.ld_g], T[a.t_base + r + uint64_t(c) * a.ld_t], s);
                r += dr;
                c += dc;
                if (r >= a.rows) {
                    r -= a.rows;
                    ++c;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) galpha[a.k] = s;
    }
}

// gT: one block per T block; every element is the alpha-weighted sum of its
// G sources in plan term order (a block without sources becomes zero)
__global__ void __launch_bounds__(256) tgrad_cells(const DevSLine* __restrict__ lines,
                                                   const DevGTerm* __restrict__ terms, uint32_t n_lines,
                                                   double* __restrict__ gT, const double* __restrict__ G) {
    for (uint32_t li = blockIdx.x; li < n_lines; li += gridDim.x) {
        const DevSLine L = lines[li];
        if (!L.rows) continue;
        // column-major walk in steps of blockDim.x without per-element division
        const uint32_t di = blockDim.x % L.rows, dc = blockDim.x / L.rows;
        uint32_t i = threadIdx.x % L.rows, c = threadIdx.x / L.rows;
        while (c < L.cols) {
            double v = 0.0;
            for (uint32_t t = L.term_begin; t < L.term_end; ++t) {
                const DevGTerm tm = terms[t];
                v += tm.alpha * G[tm.g_base + i + uint64_t(c) * tm.ld];
            }
            gT[L.s_base + i + uint64_t(c) * L.ld_s] = v;
            i += di;
            c += dc;
            if (i >= L.rows) {
                i -= L.rows;
                ++c;
            }
        }
    }
}

// galpha of the terms of grouped units (DevSGroup, built for the forward S build):
// gram[entry * SG_LINES + j] = <G line j of the group, T source of the entry>, one
// warp per (group, batch of AG_BATCH entries).  Per 128-element chunk every lane holds
// the group's 16 lines' G values of its 4 elements; per entry it forms 16 partial
// products, which a reduce-scatter butterfly (16 shuffles) sums over the warp so that
// lanes 2j, 2j+1 end with line j's total; the chunks add up in order, so the result is
// bitwise reproducible.  A term's galpha is then its (entry, line) slot.
constexpr int AG_BATCH = 16;
static_assert(SG_LINES == 16, "the butterfly below scatters 16 lines over the warp");
__device__ __forceinline__ double sum16_scatter(double const (&p)[SG_LINES], uint32_t lane) {
    const bool h1 = (lane >> 4) & 1u, h2 = (lane >> 3) & 1u, h3 = (lane >> 2) & 1u, h4 = (lane >> 1) & 1u;
    double q[8], r[4], t[2];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double send = h1 ? p[k] : p[8 + k];
        q[k] = (h1 ? p[8 + k] : p[k]) + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double send = h2 ? q[k] : q[4 + k];
        r[k] = (h2 ? q[4 + k] : q[k]) + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double send = h3 ? r[k] : r[2 + k];
        t[k] = (h3 ? r[2 + k] : r[k]) + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    double v = (h4 ? t[1] : t[0]) + __shfl_xor_sync(0xffffffffu, h4 ? t[0] : t[1], 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v;  // the line (lane >> 1) & 15
}

__global__ void __launch_bounds__(128) gram_groups(const DevSGroup* __restrict__ groups,
                                                   const DevSItem* __restrict__ items, uint32_t n_items,
                                                   const uint64_t* __restrict__ ent_t, const double* __restrict__ G,
                                                   const double* __restrict__ T, double* __restrict__ gram) {
    const uint32_t lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (uint32_t it = blockIdx.x * wpb + (threadIdx.x >> 5); it < n_items; it += gridDim.x * wpb) {
        const DevSItem I = items[it];
        const DevSGroup Gr = groups[I.group];
        const uint32_t n = Gr.rows * Gr.cols, nb = min(uint32_t(AG_BATCH), Gr.ent_end - I.e0);
        const uint64_t my_tb = lane < nb ? ent_t[I.e0 + lane] : 0;
        double acc[AG_BATCH];
#pragma unroll
        for (int b = 0; b < AG_BATCH; ++b) acc[b] = 0.0;
        for (uint32_t c0 = 0; c0 < n; c0 += 32 * SG_EPT) {
            double g[SG_LINES][SG_EPT];
            uint32_t el[SG_EPT];
            bool in[SG_EPT];
#pragma unroll
            for (int u = 0; u < SG_EPT; ++u) {
                el[u] = c0 + lane + 32u * u;
                in[u] = el[u] < n;
                const uint32_t col = in[u] ? el[u] / Gr.rows : 0, i = in[u] ? el[u] - col * Gr.rows : 0;
                const double* src = G + Gr.s_base + i + uint64_t(col) * Gr.ld_s;
#pragma unroll
                for (int j = 0; j < SG_LINES; ++j)
                    g[j][u] = (in[u] && uint32_t(j) < Gr.nlines) ? src[uint64_t(j) * Gr.line_stride] : 0.0;
            }
#pragma unroll
            for (int b = 0; b < AG_BATCH; ++b) {
                if (uint32_t(b) >= nb) break;
                const uint64_t tb = __shfl_sync(0xffffffffu, my_tb, b);
                double t[SG_EPT];
#pragma unroll
                for (int u = 0; u < SG_EPT; ++u) t[u] = in[u] ? T[tb + el[u]] : 0.0;
                double p[SG_LINES];
#pragma unroll
                for (int j = 0; j < SG_LINES; ++j) {
                    double a = 0.0;
#pragma unroll
                    for (int u = 0; u < SG_EPT; ++u) a = fma(g[j][u], t[u], a);
                    p[j] = a;
                }
                acc[b] += sum16_scatter(p, lane);
            }
        }
#pragma unroll
        for (int b = 0; b < AG_BATCH; ++b)
            if (uint32_t(b) < nb && (lane & 1u) == 0) gram[uint64_t(I.e0 + b) * SG_LINES + (lane >> 1)] = acc[b];
    }
}

// gT of T blocks taken as cell groups (DevTGroup): one warp per 128 elements of a
// group; each lane keeps TG_CELLS x SG_EPT accumulators (one per cell) and reads
// every G line of the group once for all its cells; cells sum their lines in the
// group's entry order.
__global__ void __launch_bounds__(256) tgrad_groups(const DevTGroup* __restrict__ groups,
                                                    const DevSItem* __restrict__ items, uint32_t n_items,
                                                    const uint64_t* __restrict__ ent_g,
                                                    const uint32_t* __restrict__ ent_ld,
                                                    const double* __restrict__ ent_a, const double* __restrict__ G,
                                                    double* __restrict__ gT) {
    const uint32_t lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (uint32_t it = blockIdx.x * wpb + (threadIdx.x >> 5); it < n_items; it += gridDim.x * wpb) {
        const DevSItem I = items[it];
        const DevTGroup Gr = groups[I.group];
        const uint32_t n = Gr.rows * Gr.cols;
        uint32_t el[SG_EPT], ri[SG_EPT], ci[SG_EPT];
        bool in[SG_EPT];
#pragma unroll
        for (int u = 0; u < SG_EPT; ++u) {
            el[u] = I.e0 + lane + 32u * u;
            in[u] = el[u] < n;
            ci[u] = in[u] ? el[u] / Gr.rows : 0;
            ri[u] = in[u] ? el[u] - ci[u] * Gr.rows : 0;
        }
        double acc[TG_CELLS][SG_EPT];
#pragma unroll
        for (int j = 0; j < TG_CELLS; ++j)
#pragma unroll
            for (int u = 0; u < SG_EPT; ++u) acc[j][u] = 0.0;
        for (uint32_t k = Gr.ent_begin; k < Gr.ent_end; ++k) {
            const double* g = G + ent_g[k];
            const uint64_t ld = ent_ld[k];
            double v[SG_EPT];
#pragma unroll
            for (int u = 0; u < SG_EPT; ++u) v[u] = in[u] ? g[ri[u] + ci[u] * ld] : 0.0;
            const double2* a2 = reinterpret_cast<const double2*>(ent_a + uint64_t(k) * TG_CELLS);
#pragma unroll
            for (int h = 0; h < TG_CELLS / 2; ++h) {
                const double2 x = a2[h];
#pragma unroll
                for (int u = 0; u < SG_EPT; ++u) {
                    acc[2 * h][u] = fma(x.x, v[u], acc[2 * h][u]);
                    acc[2 * h + 1][u] = fma(x.y, v[u], acc[2 * h + 1][u]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < SG_EPT; ++u) {
            if (!in[u]) continue;
#pragma unroll
            for (int c = 0; c < TG_CELLS; ++c)
                if (uint32_t(c) < Gr.ncells)
                    gT[Gr.out_base + uint64_t(c) * n + el[u]] = ((Gr.mask >> c) & 1u) ? acc[c][u] : 0.0;
        }
    }
}

__global__ void __launch_bounds__(256) gram_scatter(const uint32_t* __restrict__ k, const uint32_t* __restrict__ slot,
                                                    uint32_t n, const double* __restrict__ gram,
                                                    double* __restrict__ galpha) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        galpha[k[i]] = gram[slot[i]];
}

template <class T>
cudaError_t up(std::vector<T> const& v, T** d) {
    *d = nullptr;
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(d, v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

std::string compile_adjoint(FlatPlan const& p, std::vector<uint64_t> const& stage3_bnd,
                            std::vector<uint64_t> const& stage1_bnd, DeviceProgram const& fwd, AdjointProgram& a) {
    a = AdjointProgram();
    if (p.kind != KIND_HPSI) return "the adjoint exists for H psi plans only";
    const uint32_t nt = p.n_t(), nc = p.n_cohorts();
    std::vector<uint64_t> t_off = t_offsets(p, nullptr);
    std::vector<uint64_t> s_off = s_offsets(p, nullptr);

    // ---- G = L^T w per cohort (transpose of the stage-3 contraction) ----
    for (uint32_t c = 0; c < nc; ++c) {
        const uint32_t ls = p.c_ls[c], rs = p.c_rs[c], ns = p.c_nsrows[c], ob = p.c_rb[c];
        if (p.c_stripe[c] != p.out_cols[ob] || rs != p.out_rows[ob]) return "cohort shape differs from its output block";
        const uint64_t lbase = stage3_bnd.at(p.c_ci[c]) / 8;
        DevProb pr;
        DevSeg sg{};
        sg.B = dev_op(BUF_W, p.out_off[ob], rs, false);
        sg.K = rs;
        pr.N = p.c_stripe[c];
        uint32_t nbatch = 1;
        if (!p.c_trans[c]) {
            // L_c is rs x (ns*ls) with leading dimension rs: read it transposed
            pr.M = ns * ls;
            sg.A = dev_op(BUF_ABS, lbase, rs, true);
            pr.C = dev_op(BUF_S, s_off[c], ns * ls, false);
        } else {
            // stored blocks are ls x rs (used transposed forward): G row block b = block_b * w
            pr.M = ls;
            sg.A = dev_op(BUF_ABS, lbase, ls, false, uint64_t(ls) * rs);
            pr.C = dev_op(BUF_S, s_off[c], ns * ls, false, ls);
            nbatch = ns;
        }
        pr.seg_begin = uint32_t(a.g3.segs.size());
        a.g3.segs.push_back(sg);
        pr.seg_end = uint32_t(a.g3.segs.size());
        a.g3.probs.push_back(pr);
        gemm_add_tiles(a.g3, uint32_t(a.g3.probs.size() - 1), nbatch);
    }
    gemm_sort_tiles(a.g3);

    // ---- term cells: galpha sources and gT sources ----
    // every term must read one whole T block: ms = T block width, column on a block boundary
    std::vector<std::vector<uint32_t>> block_terms;  // per (t, b), flattened below
    std::vector<uint64_t> tb_base(nt + 1, 0);
    for (uint32_t t = 0; t < nt; ++t) tb_base[t + 1] = tb_base[t] + p.t_nb[t];
    block_terms.resize(tb_base[nt]);
    a.aterms.reserve(p.n_terms());
    for (uint32_t c = 0; c < nc; ++c) {
        const uint32_t ls = p.c_ls[c], ns = p.c_nsrows[c];
        for (uint32_t u = p.c_unit[c]; u < p.c_unit[c + 1]; ++u)
            for (uint32_t l = p.u_line[u]; l < p.u_line[u + 1]; ++l)
                for (uint32_t k = p.l_term[l]; k < p.l_term[l + 1]; ++k) {
                    const uint32_t t = p.term_t[k], w = p.t_bcols[t];
                    if (p.in_rows[p.t_lb[t]] != ls) return "term T rows differ from its cohort";
                    if (p.u_ms[u] != w || (w && p.term_col[k] % w)) return "term does not read one whole T block";
                    const uint32_t b = w ? p.term_col[k] / w : 0;
                    if (w && b >= p.t_nb[t]) return "term T block out of range";
                    DevATerm at{};
                    at.g_base = s_off[c] + uint64_t(p.l_b1[l]) * ls + uint64_t(p.u_offset[u]) * ns * ls;
                    at.t_base = t_off[t] + uint64_t(p.term_col[k]) * ls;
                    at.rows = ls;
                    at.cols = p.u_ms[u];
                    at.ld_g = ns * ls;
                    at.ld_t = ls;
                    at.k = k;
                    a.aterms.push_back(at);
                    if (w) block_terms[tb_base[t] + b].push_back(uint32_t(a.aterms.size() - 1));
                }
    }
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t M = p.in_rows[p.t_lb[t]], N = p.t_bcols[t];
        // up to 8 consecutive blocks of the task as one cell group over the union of
        // their G lines, where that issues at most twice the term walk's multiply-adds
        // (and the blocks average 4 or more terms); the other blocks keep the walk
        std::vector<char> grouped_b(p.t_nb[t], 0);
        if (uint64_t(M) * N)
            for (uint32_t b0 = 0; b0 < p.t_nb[t]; b0 += TG_CELLS) {
                const uint32_t ncell = std::min<uint32_t>(TG_CELLS, p.t_nb[t] - b0);
                uint64_t nterms = 0;
                for (uint32_t c = 0; c < ncell; ++c) nterms += block_terms[tb_base[t] + b0 + c].size();
                if (nterms < 4ull * ncell) continue;
                std::map<std::pair<uint64_t, uint32_t>, uint32_t> slot;  // (g_base, ld_g) in address order
                for (uint32_t c = 0; c < ncell; ++c)
                    for (uint32_t i : block_terms[tb_base[t] + b0 + c])
                        slot.emplace(std::make_pair(a.aterms[i].g_base, a.aterms[i].ld_g), 0u);
                if (uint64_t(slot.size()) * TG_CELLS > 2 * nterms) continue;
                DevTGroup G{};
                G.out_base = t_off[t] + uint64_t(b0) * M * N;
                G.rows = M;
                G.cols = N;
                G.ncells = ncell;
                G.ent_begin = uint32_t(a.tg_g.size());
                uint32_t e = G.ent_begin;
                for (auto& kv : slot) {
                    kv.second = e++;
                    a.tg_g.push_back(kv.first.first);
                    a.tg_ld.push_back(kv.first.second);
                    a.tg_a.insert(a.tg_a.end(), TG_CELLS, 0.0);
                }
                G.ent_end = e;
                for (uint32_t c = 0; c < ncell; ++c)
                    for (uint32_t i : block_terms[tb_base[t] + b0 + c]) {
                        DevATerm const& at = a.aterms[i];
                        a.tg_a[uint64_t(slot[{at.g_base, at.ld_g}]) * TG_CELLS + c] += p.term_alpha[at.k];
                        G.mask |= 1u << c;
                    }
                const uint32_t gi = uint32_t(a.tgroups.size());
                a.tgroups.push_back(G);
                for (uint64_t e0 = 0; e0 < uint64_t(M) * N; e0 += 32 * SG_EPT)
                    a.tg_items.push_back(DevSItem{gi, uint32_t(e0)});
                for (uint32_t c = 0; c < ncell; ++c) grouped_b[b0 + c] = 1;
            }
        for (uint32_t b = 0; b < p.t_nb[t]; ++b) {
            if (grouped_b[b]) continue;
            DevSLine L{};
            L.s_base = t_off[t] + uint64_t(b) * M * N;
            L.ld_s = M;
            L.rows = M;
            L.cols = N;
            L.ld_t = M;
            L.term_begin = uint32_t(a.gterms.size());
            for (uint32_t i : block_terms[tb_base[t] + b]) {
                DevATerm const& at = a.aterms[i];
                a.gterms.push_back(DevGTerm{p.term_alpha[at.k], at.g_base, at.ld_g, 0});
            }
            L.term_end = uint32_t(a.gterms.size());
            if (uint64_t(M) * N) a.tlines.push_back(L);
        }
    }

    // ---- gx slices: sum over the slice's T tasks of gT_t R_t^T (transpose of stage 1) ----
    std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> slices;  // (block, column) -> tasks
    for (uint32_t t = 0; t < nt; ++t) slices[{p.t_lb[t], p.t_col[t]}].push_back(t);
    uint32_t prev_lb = UINT32_MAX;
    uint64_t prev_end = 0;
    for (auto const& kv : slices) {
        const uint32_t lb = kv.first.first, col = kv.first.second;
        const uint32_t M = p.in_rows[lb], W = p.t_brows[kv.second.front()];
        for (uint32_t t : kv.second)
            if (p.t_brows[t] != W) return "T tasks of one slice differ in width";
        if (lb == prev_lb && col < prev_end) return "T-task slices of an input block overlap";
        prev_lb = lb;
        prev_end = uint64_t(col) + W;
        DevProb pr;
        pr.M = M;
        pr.N = W;
        pr.C = dev_op(BUF_OUT, p.in_off[lb] + uint64_t(col) * M, M, false);
        pr.seg_begin = uint32_t(a.g1.segs.size());
        for (uint32_t t : kv.second) {
            const uint32_t Nf = p.t_bcols[t], nb = p.t_nb[t];
            const uint64_t bnd = stage1_bnd.at(p.t_ci[t]) / 8;
            if (!p.t_trans[t]) {
                // R_t is W x (nb*Nf) with leading dimension W: read it transposed
                DevSeg sg{};
                sg.A = dev_op(BUF_T, t_off[t], M, false);
                sg.B = dev_op(BUF_ABS, bnd, W, true);
                sg.K = nb * Nf;
                a.g1.segs.push_back(sg);
            } else {
                // stored blocks are Nf x W (used transposed forward): one segment per block
                for (uint32_t b = 0; b < nb; ++b) {
                    DevSeg sg{};
                    sg.A = dev_op(BUF_T, t_off[t] + uint64_t(b) * M * Nf, M, false);
                    sg.B = dev_op(BUF_ABS, bnd + uint64_t(b) * W * Nf, Nf, false);
                    sg.K = Nf;
                    a.g1.segs.push_back(sg);
                }
            }
        }
        pr.seg_end = uint32_t(a.g1.segs.size());
        a.g1.probs.push_back(pr);
        gemm_add_tiles(a.g1, uint32_t(a.g1.probs.size() - 1), 1);
    }
    gemm_sort_tiles(a.g1);

    // ---- galpha of grouped units from the groups' Gram blocks; the rest term by term ----
    std::vector<char> grouped(p.n_terms(), 0);
    for (uint32_t k : fwd.gterm_k) grouped[k] = 1;
    for (DevATerm const& at : a.aterms)
        if (!grouped[at.k]) a.aterms_walk.push_back(at);
    for (uint32_t gi = 0; gi < fwd.groups.size(); ++gi)
        for (uint32_t e = fwd.groups[gi].ent_begin; e < fwd.groups[gi].ent_end; e += AG_BATCH)
            a.gram_items.push_back(DevSItem{gi, e});
    a.gram_k = fwd.gterm_k;
    a.gram_slot = fwd.gterm_slot;
    a.gram_elems = uint64_t(fwd.gent_t.size()) * SG_LINES;
    return std::string();
}

cudaError_t upload_adjoint(AdjointProgram& a) {
    cudaError_t e;
    if ((e = upload_gemm(a.g3, a.d3)) != cudaSuccess) return e;
    if ((e = upload_gemm(a.g1, a.d1)) != cudaSuccess) return e;
    if ((e = up(a.aterms_walk, &a.d_aterms)) != cudaSuccess) return e;
    if ((e = up(a.gram_items, &a.d_gram_items)) != cudaSuccess) return e;
    if ((e = up(a.tgroups, &a.d_tgroups)) != cudaSuccess) return e;
    if ((e = up(a.tg_items, &a.d_tg_items)) != cudaSuccess) return e;
    if ((e = up(a.tg_g, &a.d_tg_g)) != cudaSuccess) return e;
    if ((e = up(a.tg_ld, &a.d_tg_ld)) != cudaSuccess) return e;
    if ((e = up(a.tg_a, &a.d_tg_a)) != cudaSuccess) return e;
    a.n_tg_items = uint32_t(a.tg_items.size());
    if ((e = up(a.gram_k, &a.d_gram_k)) != cudaSuccess) return e;
    if ((e = up(a.gram_slot, &a.d_gram_slot)) != cudaSuccess) return e;
    if (a.gram_elems && (e = cudaMalloc(&a.d_gram, a.gram_elems * sizeof(double))) != cudaSuccess) return e;
    a.n_gram_items = uint32_t(a.gram_items.size());
    a.n_gram_terms = uint32_t(a.gram_k.size());
    if ((e = up(a.tlines, &a.d_tlines)) != cudaSuccess) return e;
    if ((e = up(a.gterms, &a.d_gterms)) != cudaSuccess) return e;
    a.n_aterms = uint32_t(a.aterms_walk.size());
    a.n_tlines = uint32_t(a.tlines.size());
    return cudaSuccess;
}

void free_adjoint(AdjointProgram& a) {
    free_gemm(a.d3);
    free_gemm(a.d1);
    cudaFree(a.d_aterms);
    cudaFree(a.d_tlines);
    cudaFree(a.d_gterms);
    cudaFree(a.d_gram_items);
    cudaFree(a.d_tgroups);
    cudaFree(a.d_tg_items);
    cudaFree(a.d_tg_g);
    cudaFree(a.d_tg_ld);
    cudaFree(a.d_tg_a);
    a.d_tgroups = nullptr;
    a.d_tg_items = nullptr;
    a.d_tg_g = nullptr;
    a.d_tg_ld = nullptr;
    a.d_tg_a = nullptr;
    cudaFree(a.d_gram_k);
    cudaFree(a.d_gram_slot);
    cudaFree(a.d_gram);
    a.d_gram_items = nullptr;
    a.d_gram_k = nullptr;
    a.d_gram_slot = nullptr;
    a.d_gram = nullptr;
    a.d_aterms = nullptr;
    a.d_tlines = nullptr;
    a.d_gterms = nullptr;
}

cudaError_t run_adjoint(DeviceProgram const& fwd, AdjointProgram const& a, uint64_t w, uint64_t x, double* gx,
                        uint64_t gx_elems, double* galpha, double* T, double* S, cudaStream_t stream) {
    Bases bs{};
    bs.b[BUF_IN] = x;
    bs.b[BUF_OUT] = reinterpret_cast<uint64_t>(gx);
    bs.b[BUF_T] = reinterpret_cast<uint64_t>(T);
    bs.b[BUF_S] = reinterpret_cast<uint64_t>(S);
    bs.b[BUF_W] = w;
    const uint32_t sms = uint32_t(device_sm_count());
    cudaError_t e;
    if (!gx && !galpha) return cudaSuccess;
    GemmDev d3 = a.d3, d1 = a.d1;  // the transposed stages use the forward stages' tuned variants
    d3.var = fwd.var3;
    d1.var = fwd.var1;
    if ((e = launch_gemm(d3, bs, stream)) != cudaSuccess) return e;  // G into S
    if (galpha) {
        GemmDev f1;
        f1.p = fwd.d_p1;
        f1.s = fwd.d_s1;
        f1.t = fwd.d_t1;
        f1.n = fwd.n_t1;
        f1.x = fwd.x1;
        f1.r = fwd.d_r1;
        f1.var = fwd.var1;
        if ((e = launch_gemm(f1, bs, stream)) != cudaSuccess) return e;  // T = x-slices * R
        if (a.n_aterms) {
            uint32_t grid = std::min<uint32_t>((a.n_aterms + 7) / 8, sms * 8);
            alpha_grad<<<grid, 256, 0, stream>>>(a.d_aterms, a.n_aterms, S, T, galpha);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (a.n_gram_items) {
            uint32_t grid = std::min<uint32_t>((a.n_gram_items + 3) / 4, sms * 8);
            gram_groups<<<grid, 128, 0, stream>>>(fwd.d_groups, a.d_gram_items, a.n_gram_items, fwd.d_gent_t, S, T,
                                                  a.d_gram);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            grid = std::min<uint32_t>((a.n_gram_terms + 255) / 256, sms * 8);
            gram_scatter<<<grid, 256, 0, stream>>>(a.d_gram_k, a.d_gram_slot, a.n_gram_terms, a.d_gram, galpha);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    if (gx) {
        if (a.n_tlines) {
            uint32_t grid = std::min<uint32_t>(a.n_tlines, sms * 8);
            tgrad_cells<<<grid, 256, 0, stream>>>(a.d_tlines, a.d_gterms, a.n_tlines, T, S);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (a.n_tg_items) {
            uint32_t grid = std::min<uint32_t>((a.n_tg_items + 7) / 8, sms * 4);
            tgrad_groups<<<grid, 256, 0, stream>>>(a.d_tgroups, a.d_tg_items, a.n_tg_items, a.d_tg_g, a.d_tg_ld,
                                                   a.d_tg_a, S, T);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if ((e = cudaMemsetAsync(gx, 0, gx_elems * sizeof(double), stream)) != cudaSuccess) return e;
        if ((e = launch_gemm(d1, bs, stream)) != cudaSuccess) return e;  // gx = gT * R^T
    }
    return cudaSuccess;
}

}  // namespace dmrgb200
