// bsg_density1b: m-scheme one-body transition densities <f| a+_c a_d |i> for
// every pair of a set of states, protons and neutrons, in one pass.
//
// The reference (src/bdenslib3.f90:14-311, driven by
// master_density1b_bundled, src/bdenslib1.f90:1506-1607) walks P1B / N1B
// opbundles: for each one-body jump it sums vec1(statei) * vec2(statef) over
// the conjugate SDs of the other species (an arithmetic progression of basis
// states) and adds the sum times the jump phase to p1bopme(cop, dop) (for 'b'
// bundles the roles of the two states swap and the label is transposed).  It
// handles one (initial, final) pair per call.
//
// Here the host turns every (bundle, jump) into a segment (first row on the
// final-state side, first row on the initial-state side, stride, count,
// phase), sorts the segments by output label and cuts each label's segments
// into chunks of about the same number of rows.  One CTA per chunk stages
// up to 256 rows of all states (interleaved, so a row of all states is
// contiguous) in shared memory and accumulates the nstates x nstates products
// in FP64; a second kernel sums the chunks of each label in chunk order.  No
// atomics: bitwise repeatable.

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "bsg_internal.h"

namespace bsg {

namespace {

constexpr int kDenThreads = 256;
constexpr int kDenMaxStates = 32;   // pairs per thread <= 4

struct DSeg {
    int64_t row_f, row_i;   // 0-based first rows: final-state side, initial-state side
    int64_t step;           // row stride between consecutive conjugate SDs
    int32_t cnt;            // conjugate SDs (rows) in this segment
    int32_t item0;          // rows of the chunk before this segment
    int32_t sign;           // jump phase
    int32_t pad;
};
static_assert(sizeof(DSeg) == 40, "DSeg layout");

struct DChunk {
    int32_t seg0, seg1;     // segment range
    int32_t nitems;         // rows in the chunk
    int32_t label;          // output label (species-combined)
};

// [dim x ns] column-major -> [dim x nsp] interleaved (row of all states
// contiguous, nsp = ns rounded up to even, the padding state zero): every row
// starts on a 16-byte boundary
__global__ void k_interleave(const double *__restrict__ cols, double *__restrict__ x, int64_t dim, int ns, int nsp) {
    const int64_t n = dim * nsp;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = e / nsp;
        const int k = (int)(e - row * nsp);
        x[e] = k < ns ? cols[(int64_t)k * dim + row] : 0.0;
    }
}

__host__ __device__ inline int den_nsp(int ns) { return (ns + 1) & ~1; }
// rows staged per pass: tile * nsp <= 1024 doubles per side and buffer, so
// that 32 KB of shared memory per CTA leaves room for 6 CTAs per SM
__host__ __device__ inline int den_tile(int ns) {
    int t = (1024 / den_nsp(ns)) / 32 * 32;
    return t < 32 ? 32 : (t > kDenThreads ? kDenThreads : t);
}
// shared layout: two buffers of (final rows, initial rows) [tile][nsp] and
// their row signs; the per-thread partial sums reuse the buffers at the end
inline size_t den_smem(int ns) {
    const int tile = den_tile(ns), nsp = den_nsp(ns);
    return sizeof(double) * (size_t)(4 * tile * nsp + 2 * tile);
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// One CTA per chunk, passes of `tile` rows, double-buffered: while the
// threads multiply pass p out of one buffer, the copies of pass p+1 are in
// flight into the other (cp.async, 16 bytes each, no registers held).  In
// each pass thread t maps row t of the pass to (final row, initial row,
// sign), walking forward from the segment the previous pass ended in, and
// copies both rows of all states.  Each thread then accumulates a 2 x 2 block
// of (final, initial) pairs over its share of the rows: the h*h blocks
// (h = nsp/2) take G = 256 / (h*h) row groups, summed in group order at the
// end.
__global__ void __launch_bounds__(kDenThreads, 6) k_density_chunks(const DSeg *__restrict__ segs,
                                                              const DChunk *__restrict__ chunks,
                                                              const double *__restrict__ x, int ns,
                                                              double *__restrict__ partial) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int nsp = den_nsp(ns), tile = den_tile(ns);
    double *buf = reinterpret_cast<double *>(smem);     // [2 buffers][2 sides][tile][nsp]
    double *s_sg = buf + (size_t)4 * tile * nsp;        // [2 buffers][tile]
    __shared__ int s_next[2];
    const DChunk ch = chunks[blockIdx.x];
    const int t = threadIdx.x;
    const int h = nsp >> 1, nbk = h * h, groups = kDenThreads / nbk;
    const int g = t / nbk, bk = t - g * nbk;
    const int f0 = 2 * (bk / h), i0 = 2 * (bk % h);
    const int npass = (ch.nitems + tile - 1) / tile;
    auto issue = [&](int p, int seg) {
        const int base = p * tile, nrow = min(tile, ch.nitems - base), b = p & 1;
        if (t < nrow) {
            const int item = base + t;
            int s = seg;
            while (s + 1 < ch.seg1 && segs[s + 1].item0 <= item) ++s;
            const DSeg sgm = segs[s];
            const int64_t c = item - sgm.item0;
            const double *rf = x + (sgm.row_f + c * sgm.step) * nsp;
            const double *ri = x + (sgm.row_i + c * sgm.step) * nsp;
            double *df = buf + ((size_t)(2 * b) * tile + t) * nsp;
            double *di = buf + ((size_t)(2 * b + 1) * tile + t) * nsp;
            for (int k = 0; k < nsp; k += 2) {
                cp_async16(df + k, rf + k);
                cp_async16(di + k, ri + k);
            }
            s_sg[b * tile + t] = (double)sgm.sign;
            if (t == nrow - 1) s_next[b] = s;
        }
        cp_async_commit();
    };
    // two accumulator sets (alternate rows of a thread), summed at the end:
    // independent FMA chains
    double a00 = 0.0, a01 = 0.0, a10 = 0.0, a11 = 0.0;
    double b00 = 0.0, b01 = 0.0, b10 = 0.0, b11 = 0.0;
    if (npass > 0) issue(0, ch.seg0);
    __syncthreads();
    for (int p = 0; p < npass; ++p) {
        if (p + 1 < npass) {
            issue(p + 1, s_next[p & 1]);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();   // pass p's rows and signs are in shared memory
        const int nrow = min(tile, ch.nitems - p * tile), b = p & 1;
        const double *__restrict__ F = buf + (size_t)(2 * b) * tile * nsp;
        const double *__restrict__ I = F + (size_t)tile * nsp;
        const double *__restrict__ S = s_sg + b * tile;
        if (g < groups) {
            int r = g;
            for (; r + groups < nrow; r += 2 * groups) {
                const int q = r + groups;
                const double2 xf = *reinterpret_cast<const double2 *>(F + r * nsp + f0);
                const double2 yi = *reinterpret_cast<const double2 *>(I + r * nsp + i0);
                const double2 xg = *reinterpret_cast<const double2 *>(F + q * nsp + f0);
                const double2 yj = *reinterpret_cast<const double2 *>(I + q * nsp + i0);
                const double sg = S[r], sh = S[q];
                const double y0 = sg * yi.x, y1 = sg * yi.y, z0 = sh * yj.x, z1 = sh * yj.y;
                a00 = fma(xf.x, y0, a00);
                a01 = fma(xf.x, y1, a01);
                a10 = fma(xf.y, y0, a10);
                a11 = fma(xf.y, y1, a11);
                b00 = fma(xg.x, z0, b00);
                b01 = fma(xg.x, z1, b01);
                b10 = fma(xg.y, z0, b10);
                b11 = fma(xg.y, z1, b11);
            }
            if (r < nrow) {
                const double2 xf = *reinterpret_cast<const double2 *>(F + r * nsp + f0);
                const double2 yi = *reinterpret_cast<const double2 *>(I + r * nsp + i0);
                const double sg = S[r];
                const double y0 = sg * yi.x, y1 = sg * yi.y;
                a00 = fma(xf.x, y0, a00);
                a01 = fma(xf.x, y1, a01);
                a10 = fma(xf.y, y0, a10);
                a11 = fma(xf.y, y1, a11);
            }
        }
        __syncthreads();   // buffer b is free for pass p+2
    }
    double *s_red = buf;   // all copies have landed: the buffers are free
    s_red[4 * t + 0] = a00 + b00;
    s_red[4 * t + 1] = a01 + b01;
    s_red[4 * t + 2] = a10 + b10;
    s_red[4 * t + 3] = a11 + b11;
    __syncthreads();
    const int np = ns * ns;
    for (int p = t; p < np; p += kDenThreads) {
        const int f = p / ns, i = p - f * ns;
        const int b = (f >> 1) * h + (i >> 1), sub = ((f & 1) << 1) | (i & 1);
        double v = 0.0;
        for (int q = 0; q < groups; ++q) v += s_red[4 * (q * nbk + b) + sub];
        partial[(int64_t)blockIdx.x * np + p] = v;
    }
}

// out[p * nlab + label] = sum over the label's chunks, in chunk order
__global__ void k_density_reduce(const double *__restrict__ partial, const int32_t *__restrict__ lab_chunk0,
                                 const int32_t *__restrict__ lab_ids, int np, double *__restrict__ out_p,
                                 int nlab_p, double *__restrict__ out_n, int nlab_n) {
    const int u = blockIdx.x;
    const int c0 = lab_chunk0[u], c1 = lab_chunk0[u + 1];
    const int label = lab_ids[u];
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        double s = 0.0;
        for (int c = c0; c < c1; ++c) s += partial[(int64_t)c * np + p];
        if (label < nlab_p) out_p[(int64_t)p * nlab_p + label] = s;
        else out_n[(int64_t)p * nlab_n + (label - nlab_p)] = s;
    }
}

struct RawSeg {
    int32_t label;
    int64_t row_f, row_i, step;
    int64_t cnt;
    int32_t sign;
};

// One segment per (bundle, jump), every index checked: the rows of the
// conjugate SDs are the arithmetic progressions the reference walks
// (src/bdenslib3.f90:58-100 for P1B, :206-265 for N1B); 'b' bundles swap the
// final and initial rows and transpose the label.  Labels are species-combined:
// protons c*nqp + d, neutrons nqp^2 + c*nqn + d.
int build_segments(bsg_ctx *ctx, const bsg_density_tables *dt, std::vector<RawSeg> &raw) {
    const int64_t dim = ctx->dim;
    const int nl_p = ctx->t.nhsps_pl, nq_p = ctx->t.nhsps_pl + ctx->t.nhsps_pr;
    const int nl_n = ctx->t.nhsps_nl, nq_n = ctx->t.nhsps_nl + ctx->t.nhsps_nr;
    const int nlab_p = nq_p * nq_p;
    int st;
    // pstart / nstart (host copies of the uploaded tables)
    std::vector<int64_t> pstart(ctx->t.nsd_p), nstart(ctx->t.nsd_n);
    cudaError_t e = cudaMemcpy(pstart.data(), ctx->raw[0].p, 8 * pstart.size(), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(nstart.data(), ctx->raw[1].p, 8 * nstart.size(), cudaMemcpyDeviceToHost);
    if ((st = cuda_check(ctx, e, "density tables: table copy"))) return st;

    // ---- segments: one per (bundle, jump), validated
    auto comb = [](int lab, int nl, int nq) -> int {
        if (lab < 0) return -lab <= nl ? -lab - 1 : -1;
        return (lab > 0 && lab <= nq - nl) ? nl + lab - 1 : -1;
    };
    for (int64_t b = 0; b < dt->nbundles; ++b) {
        const int op = dt->optype[b], hc = dt->hchar[b];
        if (op != BSG_OP_P1B && op != BSG_OP_N1B)
            return set_err(ctx, BSG_ERR_BAD_TABLE, "density tables: bundle " + std::to_string(b + 1) + " has an optype other than P1B/N1B");
        if (hc != BSG_H_FWD && hc != BSG_H_BWD && hc != BSG_H_HERM)
            return set_err(ctx, BSG_ERR_BAD_TABLE, "density tables: bad hchar in bundle " + std::to_string(b + 1));
        const bool pro = op == BSG_OP_P1B;
        const int64_t cs = dt->cstride[b];
        const int64_t j0 = pro ? dt->pxstart[b] : dt->nxstart[b], j1 = pro ? dt->pxend[b] : dt->nxend[b];
        const int64_t c0 = pro ? dt->nxstart[b] : dt->pxstart[b], c1 = pro ? dt->nxend[b] : dt->pxend[b];
        const int64_t njumps = pro ? dt->np1b : dt->nn1b;
        const int64_t nconj = pro ? ctx->t.nsd_n : ctx->t.nsd_p;
        if (cs < 1 || j0 < 1 || j1 > njumps || c0 < 1 || c1 > nconj)
            return set_err(ctx, BSG_ERR_OOB_INDEX, "density tables: bundle " + std::to_string(b + 1) + " range outside its table");
        if (j1 < j0 || c1 < c0) continue;
        const int64_t nc = (c1 + cs - c0) / cs;
        int64_t first, step;
        if (pro) {
            // statei = isd + (nstart(c0 - cs + 1) - 1) + cs * k, k = 1..nc
            const int64_t a = c0 - cs + 1;
            if (a < 1) return set_err(ctx, BSG_ERR_OOB_INDEX, "density tables: P1B conjugate start below 1");
            first = nstart[a - 1] - 1 + cs;   // + isd, 1-based
            step = cs;
        } else {
            // statei = isd + pstart(c0) + pstride * (k - 1)
            first = pstart[c0 - 1];
            step = nc > 1 ? pstart[c0 - 1 + cs] - pstart[c0 - 1] : 0;
        }
        const int64_t *isd = pro ? dt->p1b_isd : dt->n1b_isd, *fsd = pro ? dt->p1b_fsd : dt->n1b_fsd;
        const int16_t *cop = pro ? dt->p1b_cop : dt->n1b_cop, *dop = pro ? dt->p1b_dop : dt->n1b_dop;
        const int8_t *ph = pro ? dt->p1b_phase : dt->n1b_phase;
        const int nl = pro ? nl_p : nl_n, nq = pro ? nq_p : nq_n;
        for (int64_t j = j0 - 1; j < j1; ++j) {
            const int qc = comb(cop[j], nl, nq), qd = comb(dop[j], nl, nq);
            if (qc < 0 || qd < 0)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "density tables: jump " + std::to_string(j + 1) + " label outside nhsps");
            if (ph[j] != 1 && ph[j] != -1)
                return set_err(ctx, BSG_ERR_BAD_TABLE, "density tables: jump " + std::to_string(j + 1) + " phase not +-1");
            const int64_t ri = isd[j] + first - 1, rf = fsd[j] + first - 1;   // 0-based
            const int64_t li = ri + step * (nc - 1), lf = rf + step * (nc - 1);
            if (std::min({ri, rf, li, lf}) < 0 || std::max({ri, rf, li, lf}) >= dim)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "density tables: jump " + std::to_string(j + 1) + " reaches a state outside the basis");
            RawSeg s;
            const bool bwd = hc == BSG_H_BWD;
            s.label = (pro ? 0 : nlab_p) + (bwd ? qd * nq + qc : qc * nq + qd);
            s.row_f = bwd ? ri : rf;
            s.row_i = bwd ? rf : ri;
            s.step = step;
            s.cnt = nc;
            s.sign = ph[j];
            raw.push_back(s);
        }
    }
    return BSG_OK;
}

// ---- one-body operator application (applyP1Bopbundled_g /
// applyN1Bopbundled_g, src/bdenslib3.f90:319-584): vout(statef) +=
// pot(cop, dop) * phase * vin(statei), 'b' bundles the other way round.
// Organised by output rows: the segments that write the same row progression
// (same first row, stride and count: the jumps into one final SD of one
// bundle) form a group; every row belongs to at most one group per species,
// so each CTA owns its rows and sums its group's segments in a fixed order.
struct AGroup {
    int64_t out0, step;
    int32_t cnt, seg0, seg1, pad;
};
struct ASeg {
    int64_t in0;
    double coef;
};
struct AItem {
    int32_t group, c0;
};
constexpr int kApplyRows = 4;                       // rows per thread
constexpr int kApplyChunk = kApplyRows * 256;       // rows per CTA

__global__ void __launch_bounds__(256) k_apply1b(const AGroup *__restrict__ groups, const ASeg *__restrict__ segs,
                                               const AItem *__restrict__ items, const double *__restrict__ vin,
                                               double *__restrict__ vout, int64_t dim) {
    __shared__ ASeg s_seg[128];
    const AItem it = items[blockIdx.x];
    const AGroup g = groups[it.group];
    const double *__restrict__ x = vin + (int64_t)blockIdx.y * dim;
    double *__restrict__ y = vout + (int64_t)blockIdx.y * dim;
    int64_t c[kApplyRows];
    bool ok[kApplyRows];
    double acc[kApplyRows];
#pragma unroll
    for (int u = 0; u < kApplyRows; ++u) {
        c[u] = (int64_t)it.c0 + threadIdx.x + 256 * u;
        ok[u] = c[u] < g.cnt;
        acc[u] = 0.0;
    }
    for (int s0 = g.seg0; s0 < g.seg1; s0 += 128) {
        const int n = min(128, g.seg1 - s0);
        __syncthreads();
        if ((int)threadIdx.x < n) s_seg[threadIdx.x] = segs[s0 + threadIdx.x];
        __syncthreads();
        for (int q = 0; q < n; ++q) {
            const int64_t b = s_seg[q].in0;
            const double w = s_seg[q].coef;
#pragma unroll
            for (int u = 0; u < kApplyRows; ++u)
                if (ok[u]) acc[u] = fma(w, x[b + c[u] * g.step], acc[u]);
        }
    }
#pragma unroll
    for (int u = 0; u < kApplyRows; ++u)
        if (ok[u]) y[g.out0 + c[u] * g.step] += acc[u];
}

// Neutron groups: the rows of a group step by the neutron-sector size, so the
// row-parallel kernel above reads one word per 32-byte sector.  Here thread t
// takes group g0 + t (consecutive groups of a bundle write consecutive
// states: one final neutron SD each) and kApplyCols of its rows; the gathers
// of one proton SD's neutron slice stay in L1.  The sum per row runs over the
// group's segments in the same order as in k_apply1b.
constexpr int kApplyCols = 8;
struct ATItem {
    int32_t g0, ng, c0, pad;
};

__global__ void __launch_bounds__(256) k_apply1b_t(const AGroup *__restrict__ groups, const ASeg *__restrict__ segs,
                                                 const ATItem *__restrict__ items, const double *__restrict__ vin,
                                                 double *__restrict__ vout, int64_t dim) {
    const ATItem it = items[blockIdx.x];
    if ((int)threadIdx.x >= it.ng) return;
    const AGroup g = groups[it.g0 + threadIdx.x];
    const int nc = min(kApplyCols, g.cnt - it.c0);
    if (nc <= 0) return;
    const double *__restrict__ x = vin + (int64_t)blockIdx.y * dim + (int64_t)it.c0 * g.step;
    double *__restrict__ y = vout + (int64_t)blockIdx.y * dim + g.out0 + (int64_t)it.c0 * g.step;
    double acc[kApplyCols];
#pragma unroll
    for (int u = 0; u < kApplyCols; ++u) acc[u] = 0.0;
    for (int q = g.seg0; q < g.seg1; ++q) {
        const ASeg sg = segs[q];
#pragma unroll
        for (int u = 0; u < kApplyCols; ++u)
            if (u < nc) acc[u] = fma(sg.coef, x[sg.in0 + (int64_t)u * g.step], acc[u]);
    }
#pragma unroll
    for (int u = 0; u < kApplyCols; ++u)
        if (u < nc) y[(int64_t)u * g.step] += acc[u];
}

}  // namespace

}  // namespace bsg

using namespace bsg;

extern "C" int bsg_density1b(bsg_ctx *ctx, const bsg_density_tables *dt, const double *vecs, int nstates,
                             double *p1bopme, double *n1bopme) {
    if (!ctx) return BSG_ERR_ARG;
    if (!dt || !vecs || !p1bopme || !n1bopme)
        return set_err(ctx, BSG_ERR_ARG, "bsg_density1b: null argument");
    if (nstates < 1 || nstates > kDenMaxStates)
        return set_err(ctx, BSG_ERR_ARG, "bsg_density1b: nstates must be 1..32");
    const int ns = nstates, np = ns * ns;
    const int64_t dim = ctx->dim;
    const int nq_p = ctx->t.nhsps_pl + ctx->t.nhsps_pr, nq_n = ctx->t.nhsps_nl + ctx->t.nhsps_nr;
    const int nlab_p = nq_p * nq_p, nlab_n = nq_n * nq_n;
    std::memset(p1bopme, 0, sizeof(double) * (size_t)np * nlab_p);
    std::memset(n1bopme, 0, sizeof(double) * (size_t)np * nlab_n);
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (st) return st;

    std::vector<RawSeg> raw;
    if ((st = build_segments(ctx, dt, raw))) return st;
    std::stable_sort(raw.begin(), raw.end(), [](const RawSeg &a, const RawSeg &b) { return a.label < b.label; });
    int64_t total = 0;
    for (auto &s : raw) total += s.cnt;
    if (total == 0) return BSG_OK;

    // ---- chunks of about `per` rows, one label each
    const int64_t per = std::max<int64_t>(1024, std::min<int64_t>(1 << 20, total / (148 * 16) + 1));
    std::vector<DSeg> segs;
    std::vector<DChunk> chunks;
    std::vector<int32_t> lab_chunk0, lab_ids;
    int cur_label = -1;
    for (const RawSeg &r : raw) {
        int64_t done = 0;
        while (done < r.cnt) {
            if (r.label != cur_label || chunks.back().nitems >= per) {
                if (r.label != cur_label) {
                    lab_chunk0.push_back((int32_t)chunks.size());
                    lab_ids.push_back(r.label);
                    cur_label = r.label;
                }
                DChunk c;
                c.seg0 = c.seg1 = (int32_t)segs.size();
                c.nitems = 0;
                c.label = r.label;
                chunks.push_back(c);
            }
            DChunk &c = chunks.back();
            const int64_t take = std::min<int64_t>(r.cnt - done, per - c.nitems);
            DSeg d;
            d.row_f = r.row_f + done * r.step;
            d.row_i = r.row_i + done * r.step;
            d.step = r.step;
            d.cnt = (int32_t)take;
            d.item0 = c.nitems;
            d.sign = r.sign;
            d.pad = 0;
            segs.push_back(d);
            c.seg1 = (int32_t)segs.size();
            c.nitems += (int32_t)take;
            done += take;
        }
    }
    lab_chunk0.push_back((int32_t)chunks.size());
    if (chunks.size() > (size_t)INT32_MAX / 2 || segs.size() > (size_t)INT32_MAX / 2)
        return set_err(ctx, BSG_ERR_UNSUPPORTED, "bsg_density1b: too many segments");

    // ---- device work
    DevBuf d_cols, d_x, d_segs, d_chunks, d_part, d_l0, d_lid, d_outp, d_outn;
    auto release = [&]() {
        dev_free(d_cols); dev_free(d_x); dev_free(d_segs); dev_free(d_chunks); dev_free(d_part);
        dev_free(d_l0); dev_free(d_lid); dev_free(d_outp); dev_free(d_outn);
    };
    const size_t vbytes = sizeof(double) * (size_t)dim * ns;
    if ((st = dev_alloc(ctx, d_cols, vbytes)) || (st = dev_alloc(ctx, d_x, sizeof(double) * (size_t)dim * den_nsp(ns))) ||
        (st = upload(ctx, d_segs, segs.data(), sizeof(DSeg) * segs.size())) ||
        (st = upload(ctx, d_chunks, chunks.data(), sizeof(DChunk) * chunks.size())) ||
        (st = dev_alloc(ctx, d_part, sizeof(double) * (size_t)np * chunks.size())) ||
        (st = upload(ctx, d_l0, lab_chunk0.data(), sizeof(int32_t) * lab_chunk0.size())) ||
        (st = upload(ctx, d_lid, lab_ids.data(), sizeof(int32_t) * lab_ids.size())) ||
        (st = dev_alloc(ctx, d_outp, sizeof(double) * (size_t)np * std::max(1, nlab_p))) ||
        (st = dev_alloc(ctx, d_outn, sizeof(double) * (size_t)np * std::max(1, nlab_n)))) {
        release();
        return st;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(d_cols.p, vecs, vbytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_outp.p, 0, d_outp.bytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_outn.p, 0, d_outn.bytes, s);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, s);
    if (e == cudaSuccess) {
        k_interleave<<<148 * 8, 256, 0, s>>>((const double *)d_cols.p, (double *)d_x.p, dim, ns, den_nsp(ns));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        const size_t sm = den_smem(ns);
        e = cudaFuncSetAttribute(k_density_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e == cudaSuccess) {
            k_density_chunks<<<(unsigned)chunks.size(), kDenThreads, sm, s>>>(
                (const DSeg *)d_segs.p, (const DChunk *)d_chunks.p, (const double *)d_x.p, ns, (double *)d_part.p);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) {
        k_density_reduce<<<(unsigned)lab_ids.size(), 256, 0, s>>>(
            (const double *)d_part.p, (const int32_t *)d_l0.p, (const int32_t *)d_lid.p, np,
            (double *)d_outp.p, nlab_p, (double *)d_outn.p, nlab_n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
    if (e == cudaSuccess && nlab_p)
        e = cudaMemcpyAsync(p1bopme, d_outp.p, sizeof(double) * (size_t)np * nlab_p, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && nlab_n)
        e = cudaMemcpyAsync(n1bopme, d_outn.p, sizeof(double) * (size_t)np * nlab_n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (e == cudaSuccess) {
        ctx->stats.density_ms = ms;
        ctx->stats.density_rows = total;
        ctx->stats.density_launches = 3;
    }
    st = cuda_check(ctx, e, "bsg_density1b");
    release();
    return st;
}

extern "C" int bsg_apply1b(bsg_ctx *ctx, const bsg_density_tables *dt, const double *ppot, const double *npot,
                           const double *vin, double *vout, int nvec) {
    if (!ctx) return BSG_ERR_ARG;
    if (!dt || !vin || !vout) return set_err(ctx, BSG_ERR_ARG, "bsg_apply1b: null argument");
    if (nvec < 1 || nvec > 65535) return set_err(ctx, BSG_ERR_ARG, "bsg_apply1b: nvec must be 1..65535");
    const int64_t dim = ctx->dim;
    const int nq_p = ctx->t.nhsps_pl + ctx->t.nhsps_pr;
    const int nlab_p = nq_p * nq_p;
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (st) return st;
    std::vector<RawSeg> raw;
    if ((st = build_segments(ctx, dt, raw))) return st;

    // ---- groups per species: segments with the same output progression
    std::vector<AGroup> groups[2];
    std::vector<ASeg> segs;
    std::vector<int64_t> order(raw.size());
    std::iota(order.begin(), order.end(), 0);
    auto species = [&](const RawSeg &r) { return r.label < nlab_p ? 0 : 1; };
    auto coef_of = [&](const RawSeg &r) {
        const double *pot = species(r) == 0 ? ppot : npot;
        const int lab = species(r) == 0 ? r.label : r.label - nlab_p;
        return pot ? pot[lab] * (double)r.sign : 0.0;
    };
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        const RawSeg &x = raw[a], &y = raw[b];
        const int sx = species(x), sy = species(y);
        if (sx != sy) return sx < sy;
        if (x.row_f != y.row_f) return x.row_f < y.row_f;
        if (x.step != y.step) return x.step < y.step;
        return x.cnt < y.cnt;
    });
    for (size_t k = 0; k < order.size(); ++k) {
        const RawSeg &r = raw[order[k]];
        const double w = coef_of(r);
        if (w == 0.0) continue;
        if (r.cnt > INT32_MAX) return set_err(ctx, BSG_ERR_UNSUPPORTED, "bsg_apply1b: conjugate range above 2^31");
        auto &gv = groups[species(r)];
        if (gv.empty() || gv.back().out0 != r.row_f || gv.back().step != r.step || gv.back().cnt != r.cnt ||
            gv.back().seg1 != (int32_t)segs.size()) {
            AGroup g;
            g.out0 = r.row_f; g.step = r.step; g.cnt = (int32_t)r.cnt;
            g.seg0 = g.seg1 = (int32_t)segs.size();
            g.pad = 0;
            gv.push_back(g);
        }
        segs.push_back(ASeg{r.row_i, w});
        gv.back().seg1 = (int32_t)segs.size();
    }
    // one writer per row and species (checked on a bitmap of the basis)
    std::vector<uint64_t> seen((size_t)(dim + 63) / 64);
    for (int sp = 0; sp < 2; ++sp) {
        std::fill(seen.begin(), seen.end(), 0ull);
        for (const AGroup &g : groups[sp])
            for (int64_t c = 0; c < g.cnt; ++c) {
                const int64_t r = g.out0 + c * g.step;
                uint64_t &w = seen[(size_t)(r >> 6)];
                const uint64_t bit = 1ull << (r & 63);
                if (w & bit)
                    return set_err(ctx, BSG_ERR_UNSUPPORTED, "bsg_apply1b: two jump groups write the same basis state");
                w |= bit;
            }
    }
    // protons: row chunks of one group per CTA; neutrons: 256 consecutive
    // groups per CTA, kApplyCols rows each
    std::vector<AItem> items[2];
    for (size_t gi = 0; gi < groups[0].size(); ++gi)
        for (int64_t c0 = 0; c0 < groups[0][gi].cnt; c0 += kApplyChunk)
            items[0].push_back(AItem{(int32_t)gi, (int32_t)c0});
    std::vector<ATItem> titems;
    for (size_t g0 = 0; g0 < groups[1].size(); g0 += 256) {
        const int ng = (int)std::min<size_t>(256, groups[1].size() - g0);
        int32_t cmax = 0;
        for (int t = 0; t < ng; ++t) cmax = std::max(cmax, groups[1][g0 + t].cnt);
        for (int32_t c0 = 0; c0 < cmax; c0 += kApplyCols) titems.push_back(ATItem{(int32_t)g0, ng, c0, 0});
    }

    DevBuf d_in, d_out, d_g[2], d_it[2], d_seg;
    auto release = [&]() {
        dev_free(d_in); dev_free(d_out); dev_free(d_seg);
        for (int sp = 0; sp < 2; ++sp) { dev_free(d_g[sp]); dev_free(d_it[sp]); }
    };
    const size_t vbytes = sizeof(double) * (size_t)dim * nvec;
    if ((st = dev_alloc(ctx, d_in, vbytes)) || (st = dev_alloc(ctx, d_out, vbytes)) ||
        (st = upload(ctx, d_seg, segs.data(), sizeof(ASeg) * segs.size()))) {
        release();
        return st;
    }
    for (int sp = 0; sp < 2 && !st; ++sp)
        st = upload(ctx, d_g[sp], groups[sp].data(), sizeof(AGroup) * groups[sp].size());
    if (!st) st = upload(ctx, d_it[0], items[0].data(), sizeof(AItem) * items[0].size());
    if (!st) st = upload(ctx, d_it[1], titems.data(), sizeof(ATItem) * titems.size());
    if (st) { release(); return st; }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(d_in.p, vin, vbytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_out.p, 0, vbytes, s);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, s);
    // protons, then neutrons: the two passes write the same states
    if (e == cudaSuccess && !items[0].empty()) {
        k_apply1b<<<dim3((unsigned)items[0].size(), (unsigned)nvec), 256, 0, s>>>(
            (const AGroup *)d_g[0].p, (const ASeg *)d_seg.p, (const AItem *)d_it[0].p, (const double *)d_in.p,
            (double *)d_out.p, dim);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !titems.empty()) {
        k_apply1b_t<<<dim3((unsigned)titems.size(), (unsigned)nvec), 256, 0, s>>>(
            (const AGroup *)d_g[1].p, (const ASeg *)d_seg.p, (const ATItem *)d_it[1].p, (const double *)d_in.p,
            (double *)d_out.p, dim);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(vout, d_out.p, vbytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (e == cudaSuccess) ctx->stats.apply1b_ms = ms;
    st = cuda_check(ctx, e, "bsg_apply1b");
    release();
    return st;
}
