// bsg_grad: Hellmann-Feynman gradient of eigenvalues with respect to every
// uncoupled matrix element (the transposed-jump contraction of the two-body
// densities, src/bdenslib4.f90:129-729; the tile body is grad_tile.cuh).
//
// One launch covers every (system, state, row tile) item: bsg_grad is the
// one-system case of grad_many, bsg_batch_grad (batch.cu) the many-system
// one.  Sums are 128-bit fixed point updated with integer atomics, so the
// gradient is bitwise repeatable and does not depend on how the work is
// split: a system's gradient is the same alone or inside a batch.

#include <algorithm>
#include <string>
#include <vector>

#include "grad_tile.cuh"

namespace bsg {

struct GradDesc {
    RowArgs a;
    GradArgs g;
    const double *psi;
};
struct GradItem {
    int32_t desc;   // (system, state)
    int32_t tile;
};

__global__ void k_fix_to_double(const unsigned long long *__restrict__ acc, double *__restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = fix_value(acc + 2 * i);
}

template <int ITEMS>
__global__ void __launch_bounds__(kGradWarps * 32) k_grad_items(const GradDesc *__restrict__ desc,
                                                                const GradItem *__restrict__ items, int mstride) {
    double *Aw, *stage_v;
    int *stage_k;
    grad_smem(mstride, Aw, stage_k, stage_v);
    const GradItem it = items[blockIdx.x];
    const GradDesc *D = desc + it.desc;
    grad_tile<ITEMS>(D->a, D->g, D->psi, D->a.tiles[it.tile], Aw, stage_k, stage_v);
}

namespace {
constexpr int kGradItems = 4;  // 128-position tiles
}

int grad_many(bsg_ctx *const *ctxs, int nsys, const double *const *evecs, int nstates, double *const *dpp,
              double *const *dnn, double *const *dpn, double *const *dspe_p, double *const *dspe_n, cudaStream_t s,
              std::string &err, double *kernel_ms) {
    auto fail = [&](int code, const std::string &m) {
        err = m;
        return code;
    };
    if (nsys < 1 || nstates < 1 || !evecs || !dpp || !dnn || !dpn) return fail(BSG_ERR_ARG, "null argument");
    for (int i = 0; i < nsys; ++i)
        if (ctxs[i]->threebody)
            return fail(BSG_ERR_UNSUPPORTED, "the adjoint covers two-body contexts only (hmatpp, hmatnn, hmatpn)");
    // per (system, state): psi offset, accumulator offsets; per system: sizes
    std::vector<int64_t> psi_off(nsys), acc_off((size_t)nsys * nstates);
    std::vector<int64_t> nlab(nsys);
    int64_t npsi = 0, nacc = 0;
    int32_t max_nbd = 0;
    std::vector<const TileSet *> ts(nsys);
    std::vector<GradItem> items;
    for (int s2 = 0; s2 < nsys; ++s2) {
        bsg_ctx *c = ctxs[s2];
        if (!evecs[s2] || !dpp[s2] || !dnn[s2] || !dpn[s2]) return fail(BSG_ERR_ARG, "null output for a system");
        const bool spe = c->t.call_spe && dspe_p && dspe_n && dspe_p[s2] && dspe_n[s2];
        c->last_status = BSG_OK;
        ts[s2] = get_tiles(c, 32 * kGradItems);
        if (!ts[s2]) return fail(c->last_status ? c->last_status : BSG_ERR_NOMEM, "tiles: " + c->last_error);
        max_nbd = std::max(max_nbd, c->args.max_nbd);
        psi_off[s2] = npsi;
        npsi += c->dim * nstates;
        nlab[s2] = c->t.nmatpp + c->t.nmatnn + c->t.nmatpn + (spe ? c->t.nsd_p + c->t.nsd_n : 0);
        for (int k = 0; k < nstates; ++k) {
            acc_off[(size_t)s2 * nstates + k] = nacc;
            nacc += nlab[s2];
        }
    }
    // 8 per-warp FP64 bin tables and staging within 227 KB of shared memory
    if (max_nbd > 3392) return fail(BSG_ERR_UNSUPPORTED, "a neutron sector jump has more than 3392 distinct (b,d) pairs");
    const int mstride = (max_nbd + 1) & ~1;
    // items heaviest tiles first (the tile lists are already in that order
    // per system); interleave states so that concurrent CTAs share records
    for (int s2 = 0; s2 < nsys; ++s2)
        for (int t = 0; t < ts[s2]->ntiles; ++t)
            for (int k = 0; k < nstates; ++k) items.push_back(GradItem{s2 * nstates + k, t});
    bsg_ctx *c0 = ctxs[0];
    DevBuf psi, acc, out, descb, itemb;
    auto cleanup = [&]() {
        dev_free(psi); dev_free(acc); dev_free(out); dev_free(descb); dev_free(itemb);
    };
    int st;
    if ((st = dev_alloc(c0, psi, sizeof(double) * (size_t)std::max<int64_t>(npsi, 1))) ||
        (st = dev_alloc(c0, acc, 16 * (size_t)std::max<int64_t>(nacc, 1))) ||
        (st = dev_alloc(c0, out, sizeof(double) * (size_t)std::max<int64_t>(nacc, 1)))) {
        cleanup();
        return fail(st, "device allocation: " + c0->last_error);
    }
    std::vector<GradDesc> desc((size_t)nsys * nstates);
    for (int s2 = 0; s2 < nsys; ++s2) {
        bsg_ctx *c = ctxs[s2];
        const bool spe = c->t.call_spe && dspe_p && dspe_n && dspe_p[s2] && dspe_n[s2];
        for (int k = 0; k < nstates; ++k) {
            GradDesc &d = desc[(size_t)s2 * nstates + k];
            d.a = c->args;
            d.a.tiles = (const Tile *)ts[s2]->buf.p;
            d.a.ntiles = ts[s2]->ntiles;
            unsigned long long *base = (unsigned long long *)acc.p + 2 * acc_off[(size_t)s2 * nstates + k];
            d.g.pp_op = (const int32_t *)c->pp_op.p;
            d.g.pp_ph = (const int8_t *)c->pp_ph.p;
            d.g.nnrec_op = (const int32_t *)c->nnrec_op.p;
            d.g.nnrec_ph = (const int8_t *)c->nnrec_ph.p;
            d.g.pp = base;
            d.g.nn = d.g.pp + 2 * c->t.nmatpp;
            d.g.pn = d.g.nn + 2 * c->t.nmatnn;
            d.g.spe_p = spe ? d.g.pn + 2 * c->t.nmatpn : nullptr;
            d.g.spe_n = spe ? d.g.spe_p + 2 * c->t.nsd_p : nullptr;
            d.psi = (const double *)psi.p + psi_off[s2] + (int64_t)k * c->dim;
        }
    }
    if ((st = upload(c0, descb, desc.data(), sizeof(GradDesc) * desc.size())) ||
        (st = upload(c0, itemb, items.data(), sizeof(GradItem) * std::max<size_t>(items.size(), 1)))) {
        cleanup();
        return fail(st, "upload: " + c0->last_error);
    }
    cudaError_t e = cudaSuccess;
    for (int s2 = 0; s2 < nsys && e == cudaSuccess; ++s2)
        e = cudaMemcpyAsync((double *)psi.p + psi_off[s2], evecs[s2], sizeof(double) * ctxs[s2]->dim * nstates,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(acc.p, 0, acc.bytes, s);
    const size_t smem = grad_smem_bytes(mstride);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_grad_items<kGradItems>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    if (e == cudaSuccess && !items.empty()) {
        k_grad_items<kGradItems><<<(unsigned)items.size(), kGradWarps * 32, smem, s>>>(
            (const GradDesc *)descb.p, (const GradItem *)itemb.p, mstride);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && nacc > 0) {
        k_fix_to_double<<<(unsigned)std::min<int64_t>((nacc + 255) / 256, 4096), 256, 0, s>>>(
            (const unsigned long long *)acc.p, (double *)out.p, nacc);
        e = cudaGetLastError();
    }
    cudaEventRecord(e1, s);
    // outputs: per system, state-major blocks [state][label]
    for (int s2 = 0; s2 < nsys && e == cudaSuccess; ++s2) {
        bsg_ctx *c = ctxs[s2];
        const bool spe = c->t.call_spe && dspe_p && dspe_n && dspe_p[s2] && dspe_n[s2];
        for (int k = 0; k < nstates && e == cudaSuccess; ++k) {
            const double *o = (const double *)out.p + acc_off[(size_t)s2 * nstates + k];
            auto cp = [&](double *dst, const double *src, int64_t cnt) {
                if (e == cudaSuccess && cnt > 0)
                    e = cudaMemcpyAsync(dst, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost, s);
            };
            cp(dpp[s2] + k * c->t.nmatpp, o, c->t.nmatpp);
            cp(dnn[s2] + k * c->t.nmatnn, o + c->t.nmatpp, c->t.nmatnn);
            cp(dpn[s2] + k * c->t.nmatpn, o + c->t.nmatpp + c->t.nmatnn, c->t.nmatpn);
            if (spe) {
                const int64_t b0 = c->t.nmatpp + c->t.nmatnn + c->t.nmatpn;
                cp(dspe_p[s2] + k * c->t.nsd_p, o + b0, c->t.nsd_p);
                cp(dspe_n[s2] + k * c->t.nsd_n, o + b0 + c->t.nsd_p, c->t.nsd_n);
            }
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (kernel_ms && e == cudaSuccess) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        *kernel_ms = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cleanup();
    if (e != cudaSuccess) return fail(e == cudaErrorMemoryAllocation ? BSG_ERR_NOMEM : BSG_ERR_CUDA,
                                      std::string("adjoint: ") + cudaGetErrorString(e));
    return BSG_OK;
}

}  // namespace bsg

using namespace bsg;

extern "C" int bsg_grad(bsg_ctx *ctx, const double *evecs, int nstates, double *dpp, double *dnn, double *dpn,
                        double *dspe_p, double *dspe_n) {
    if (!ctx) return BSG_ERR_ARG;
    if (!evecs || nstates < 1 || !dpp || !dnn || !dpn)
        return set_err(ctx, BSG_ERR_ARG, "bsg_grad: null argument or nstates < 1");
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (st) return st;
    bsg_ctx *cs[1] = {ctx};
    const double *ev[1] = {evecs};
    double *p[1] = {dpp}, *nn[1] = {dnn}, *pn[1] = {dpn}, *sp[1] = {dspe_p}, *sn[1] = {dspe_n};
    std::string err;
    double ms = 0.0;
    st = grad_many(cs, 1, ev, nstates, p, nn, pn, sp, sn, ctx->stream, err, &ms);
    if (st) return set_err(ctx, st, "bsg_grad: " + err);
    ctx->stats.grad_ms = ms;
    return BSG_OK;
}
