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

// D (8 x 8, two values per lane) += A (8 x 4) * B (4 x 8) on the FP64 tensor cores
__device__ __forceinline__ void dmma_f64(double& c0, double& c1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

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

// gT of the T blocks outside cell groups: one warp per 128 elements of a block (a
// block without sources becomes zero).  Each lane owns four elements (lane + 32 u) and
// sums the block's terms in plan term order; the terms (alpha, G cell, leading dimension)
// are read 32 at a time, one per lane, and handed round by shuffles, so a lane keeps four
// independent G loads in flight per term and no block barrier is needed.
__global__ void __launch_bounds__(256) tgrad_cells(const DevSLine* __restrict__ lines,
                                                   const DevGTerm* __restrict__ terms,
                                                   const DevSItem* __restrict__ items, uint32_t n_items,
                                                   double* __restrict__ gT, const double* __restrict__ G) {
    const uint32_t lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (uint32_t it = blockIdx.x * wpb + (threadIdx.x >> 5); it < n_items; it += gridDim.x * wpb) {
        const DevSItem I = items[it];
        const DevSLine L = lines[I.group];
        const uint32_t n = L.rows * L.cols;
        uint32_t ri[SG_EPT], ci[SG_EPT];
        bool in[SG_EPT];
        double v[SG_EPT];
#pragma unroll
        for (int u = 0; u < SG_EPT; ++u) {
            const uint32_t e = I.e0 + lane + 32u * u;
            in[u] = e < n;
            ci[u] = in[u] ? e / L.rows : 0;
            ri[u] = in[u] ? e - ci[u] * L.rows : 0;
            v[u] = 0.0;
        }
        for (uint32_t t0 = L.term_begin; t0 < L.term_end; t0 += 32) {
            const uint32_t nt = min(32u, L.term_end - t0);
            DevGTerm my{0.0, 0, 0, 0};
            if (lane < nt) my = terms[t0 + lane];
            for (uint32_t t = 0; t < nt; ++t) {
                const double a = __shfl_sync(0xffffffffu, my.alpha, t);
                const uint64_t gb = __shfl_sync(0xffffffffu, my.g_base, t);
                const uint32_t ld = __shfl_sync(0xffffffffu, my.ld, t);
#pragma unroll
                for (int u = 0; u < SG_EPT; ++u)
                    if (in[u]) v[u] += a * G[gb + ri[u] + uint64_t(ci[u]) * ld];
            }
        }
#pragma unroll
        for (int u = 0; u < SG_EPT; ++u)
            if (in[u]) gT[L.s_base + ri[u] + uint64_t(ci[u]) * L.ld_s] = v[u];
    }
}

// galpha of the terms of grouped units (DevSGroup, built for the forward S build):
// gram[entry * SG_LINES + j] = <G line j of the group, T source of the entry>, one
// warp per (group, batch of AG_BATCH entries).  The Gram block of the batch, 16 lines x
// 32 entries, is a product (lines x elements) * (elements x entries) on the FP64 tensor
// cores: DMMA m8n8k4 over 8 lines x 8 entries per tile, four elements per K step, each
// lane loading its lines' and its entries' element (lane & 3) of the step from global
// memory (8 rows x 32 bytes per warp load), so a G element loaded once serves 32 entries.
// A batch of at most 16 entries skips the upper entry tiles (warp-uniform).  Two
// accumulator sets take alternate K steps and are added at the end, in a fixed order, so
// the result is bitwise reproducible.  A term's galpha is then its (entry, line) slot.
constexpr int AG_BATCH = 32;
static_assert(SG_LINES == 16, "2 line tiles of 8");

template <int ET>  // entry tiles of 8
__device__ __forceinline__ void gram_batch(DevSGroup const& Gr, uint32_t e0, uint32_t nb,
                                           const uint64_t* __restrict__ ent_t, const double* __restrict__ G,
                                           const double* __restrict__ T, double* __restrict__ gram, uint32_t g,
                                           uint32_t q) {
    const uint32_t n = Gr.rows * Gr.cols;
    // this lane's rows of the A (lines g, 8 + g) and B (entries 8 j + g) fragments
    const bool l0 = g < Gr.nlines, l1 = 8 + g < Gr.nlines;
    const double* G0 = G + Gr.s_base + uint64_t(g) * Gr.line_stride;
    const double* G1 = G0 + 8ull * Gr.line_stride;
    const double* Tj[ET];
    bool bj[ET];
#pragma unroll
    for (int j = 0; j < ET; ++j) {
        bj[j] = uint32_t(8 * j) + g < nb;
        Tj[j] = T + (bj[j] ? ent_t[e0 + 8 * j + g] : 0);
    }
    double acc[2][2][ET][2];  // [set][line tile][entry tile][pair]
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < ET; ++j) acc[s][i][j][0] = acc[s][i][j][1] = 0.0;
    // element e = 4 step + q of the lane, at (row r, column c) of the lines' cells
    uint32_t e = q, c = q / max(Gr.rows, 1u), r = q - c * Gr.rows;
    const uint32_t dc = 4u / max(Gr.rows, 1u), dr = 4u - dc * Gr.rows;
    for (uint32_t st = 0; st * 4 < n; st += 2) {
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const bool in = e < n;
            const uint64_t go = r + uint64_t(c) * Gr.ld_s;
            const double a0 = (in && l0) ? G0[go] : 0.0, a1 = (in && l1) ? G1[go] : 0.0;
#pragma unroll
            for (int j = 0; j < ET; ++j) {
                const double t = (in && bj[j]) ? Tj[j][e] : 0.0;
                dmma_f64(acc[s][0][j][0], acc[s][0][j][1], a0, t);
                dmma_f64(acc[s][1][j][0], acc[s][1][j][1], a1, t);
            }
            e += 4;
            r += dr;
            c += dc;
            if (r >= Gr.rows) {
                r -= Gr.rows;
                ++c;
            }
        }
    }
    // D tile (line tile i, entry tile j): line 8 i + g, entries 8 j + 2 q + h
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < ET; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t ent = uint32_t(8 * j) + 2u * q + uint32_t(h);
                if (ent < nb)
                    gram[uint64_t(e0 + ent) * SG_LINES + uint32_t(8 * i) + g] = acc[0][i][j][h] + acc[1][i][j][h];
            }
}

__global__ void __launch_bounds__(128) gram_groups(const DevSGroup* __restrict__ groups,
                                                   const DevSItem* __restrict__ items, uint32_t n_items,
                                                   const uint64_t* __restrict__ ent_t, const double* __restrict__ G,
                                                   const double* __restrict__ T, double* __restrict__ gram) {
    const uint32_t lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const uint32_t g = lane >> 2, q = lane & 3;
    for (uint32_t it = blockIdx.x * wpb + (threadIdx.x >> 5); it < n_items; it += gridDim.x * wpb) {
        const DevSItem I = items[it];
        const DevSGroup Gr = groups[I.group];
        const uint32_t nb = min(uint32_t(AG_BATCH), Gr.ent_end - I.e0);
        if (nb > 16)
            gram_batch<4>(Gr, I.e0, nb, ent_t, G, T, gram, g, q);
        else
            gram_batch<2>(Gr, I.e0, nb, ent_t, G, T, gram, g, q);
    }
}

// gT of T blocks taken as cell groups (DevTGroup): one warp per 128 elements of a
// group.  The chunk of every cell is one product (elements x G lines) * (G lines x
// cells) on the FP64 tensor cores (DMMA m8n8k4: 8 elements x 8 cells x 4 lines per
// instruction; the chunk in two passes of 8 element tiles), so every G line of the group
// is read once per pass for all its cells; the lines enter four per K step in the group's
// entry order (lines past the end as zeros).
__global__ void __launch_bounds__(256) tgrad_groups(const DevTGroup* __restrict__ groups,
                                                    const DevSItem* __restrict__ items, uint32_t n_items,
                                                    const uint64_t* __restrict__ ent_g,
                                                    const uint32_t* __restrict__ ent_ld,
                                                    const double* __restrict__ ent_a, const double* __restrict__ G,
                                                    double* __restrict__ gT) {
    static_assert(TG_CELLS == 8, "one DMMA tile of cells");
    constexpr int MT = 8;  // element tiles per pass: a 128-element chunk in two passes of 64
    const uint32_t lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const uint32_t g = lane >> 2, q = lane & 3;
    for (uint32_t it = blockIdx.x * wpb + (threadIdx.x >> 5); it < n_items; it += gridDim.x * wpb) {
        const DevSItem I = items[it];
        const DevTGroup Gr = groups[I.group];
        const uint32_t n = Gr.rows * Gr.cols;
        for (uint32_t half = 0; half < 32u * SG_EPT; half += 8u * MT) {
            const uint32_t eb = I.e0 + half;
            if (eb >= n) break;
            // this lane's elements eb + 8 i + g: row and column in the G lines' cells
            uint32_t ri[MT], ci[MT];
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const uint32_t e = eb + uint32_t(8 * i) + g;
                ci[i] = e < n ? e / Gr.rows : 0xffffffffu;  // beyond the block: no load
                ri[i] = e < n ? e - ci[i] * Gr.rows : 0;
            }
            double acc[MT][2];
#pragma unroll
            for (int i = 0; i < MT; ++i) acc[i][0] = acc[i][1] = 0.0;
            // the line of K step k0 + 4 (its address, leading dimension and alpha) is read
            // while step k0 multiplies, so the two dependent loads of a step overlap the last
            auto line = [&](uint32_t k0, const double*& gk, uint64_t& ld, double& b) {
                const uint32_t k = k0 + q;
                const bool live = k < Gr.ent_end;
                gk = live ? G + ent_g[k] : nullptr;
                ld = live ? ent_ld[k] : 0;
                b = live ? ent_a[uint64_t(k) * TG_CELLS + g] : 0.0;
            };
            const double* gk;
            uint64_t ld;
            double b;
            line(Gr.ent_begin, gk, ld, b);
            for (uint32_t k0 = Gr.ent_begin; k0 < Gr.ent_end; k0 += 4) {
                double a[MT];
#pragma unroll
                for (int i = 0; i < MT; ++i) a[i] = (gk && ci[i] != 0xffffffffu) ? gk[ri[i] + ci[i] * ld] : 0.0;
                const double bk = b;
                line(k0 + 4, gk, ld, b);
#pragma unroll
                for (int i = 0; i < MT; ++i) dmma_f64(acc[i][0], acc[i][1], a[i], bk);
            }
            // D tile i: element eb + 8 i + g, cells 2 q + h
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const uint32_t e = eb + uint32_t(8 * i) + g;
                if (e >= n) continue;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t c = 2u * q + uint32_t(h);
                    if (c < Gr.ncells)
                        gT[Gr.out_base + uint64_t(c) * n + e] = ((Gr.mask >> c) & 1u) ? acc[i][h] : 0.0;
                }
            }
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
        // their G lines, where that issues at most four times the term walk's
        // multiply-adds (on the tensor cores they cost far less than the walk's) and the
        // blocks average 4 or more terms; the other blocks keep the walk
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
                if (uint64_t(slot.size()) * TG_CELLS > 4 * nterms) continue;
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
            if (uint64_t(M) * N) {
                for (uint64_t e0 = 0; e0 < uint64_t(M) * N; e0 += 32 * SG_EPT)
                    a.tl_items.push_back(DevSItem{uint32_t(a.tlines.size()), uint32_t(e0)});
                a.tlines.push_back(L);
            }
        }
    }
    // cell groups in the order of the first G line they read (their lines are listed in
    // address order): groups of different T tasks that read the same G lines run side by
    // side, so a line's chunk comes from DRAM once and from L2 for the others
    {
        std::vector<uint32_t> order(a.tgroups.size());
        for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
        auto first_g = [&](uint32_t gi) {
            DevTGroup const& G = a.tgroups[gi];
            return G.ent_end > G.ent_begin ? a.tg_g[G.ent_begin] : 0ull;
        };
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return first_g(x) < first_g(y); });
        a.tg_items.clear();
        for (uint32_t gi : order) {
            const uint64_t n = uint64_t(a.tgroups[gi].rows) * a.tgroups[gi].cols;
            for (uint64_t e0 = 0; e0 < n; e0 += 32 * SG_EPT) a.tg_items.push_back(DevSItem{gi, uint32_t(e0)});
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
    if ((e = up(a.tl_items, &a.d_tl_items)) != cudaSuccess) return e;
    a.n_tl_items = uint32_t(a.tl_items.size());
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
    cudaFree(a.d_tl_items);
    a.d_tl_items = nullptr;
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
        if (a.n_tl_items) {
            uint32_t grid = std::min<uint32_t>((a.n_tl_items + 7) / 8, sms * 8);
            tgrad_cells<<<grid, 256, 0, stream>>>(a.d_tlines, a.d_gterms, a.d_tl_items, a.n_tl_items, T, S);
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
