// bsg_grad: Hellmann-Feynman gradient of eigenvalues with respect to every
// uncoupled matrix element, dE_k/dhmat(label) = sum over every appearance of
// the label in H of phase * psi_k(out) * psi_k(in).
//
// This is the traversal of the two-body densities applyh{PP,NN,PN}bundled_den
// (src/bdenslib4.f90:129-729: dmat(op) += vout(f)*vin(i)*phase) with both
// vectors equal to the eigenvector, run over the same row tiles and
// (row, warp) slots as the matvec: PP contributions reduce a row-segment dot
// product per jump; PN contributions accumulate per distinct (b,d) label pair
// in shared memory and flush one atomic per pair and proton jump; NN records
// and SPE terms go straight to their bins.  Every f and b appearance is
// visited, so hermitian halves and the 1/2 on diagonal pair labels are
// accounted for exactly as in the matvec.

#include <vector>

#include "bsg_internal.h"

namespace bsg {

struct GradArgs {
    const int32_t *pp_op;
    const int8_t *pp_ph;
    const int32_t *nnrec_op;
    const int8_t *nnrec_ph;
    double *dpp, *dnn, *dpn, *dspe_p, *dspe_n;
};

constexpr int kGradWarps = kRowWarps;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int ITEMS>
__global__ void __launch_bounds__(kGradWarps * 32) k_grad(const RowArgs a, const GradArgs g,
                                                          const double *__restrict__ psi, const int mstride) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *__restrict__ Aw = reinterpret_cast<double *>(smem) + (size_t)warp * mstride;
    const Tile tile = a.tiles[blockIdx.x];
    const int row = tile.row;
    const int64_t roff = a.row_off[row];
    const int slot = row * kGradWarps + warp;
    int pos[ITEMS];
    bool valid[ITEMS];
    double pout[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int local = lane + 32 * i;
        pos[i] = tile.pos0 + local;
        valid[i] = local < tile.npos;
        pout[i] = valid[i] ? psi[roff + pos[i]] : 0.0;
    }
    // ---- PP: dpp[op] += ph * sum_pos psi[row+pos] psi[q+pos]
    for (int c = a.pp_ptr[slot]; c < a.pp_ptr[slot + 1]; ++c) {
        const PPContrib pc = a.pp[c];
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (valid[i] && pos[i] >= pc.lo && pos[i] <= pc.hi) s += pout[i] * psi[pc.q_off + pos[i]];
        s = warp_sum(s);
        if (lane == 0 && s != 0.0) atomicAdd(g.dpp + g.pp_op[c] - 1, (double)g.pp_ph[c] * s);
    }
    // ---- NN: dnn[op_r] += ph_r * psi[row+pos] psi[row+in_r]
    for (int c = a.nn_ptr[slot]; c < a.nn_ptr[slot + 1]; ++c) {
        const NOp op = a.nops[a.nn[c].nop];
        const int32_t *__restrict__ ptr = a.nptr + op.ptr_base;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            if (!valid[i] || pos[i] >= op.nout) continue;
            const int k0 = ptr[pos[i]], k1 = ptr[pos[i] + 1];
            for (int k = k0; k < k1; ++k) {
                const int64_t r = op.rec_base + k;
                const double v = pout[i] * psi[roff + a.nnrec[r].in];
                atomicAdd(g.dnn + g.nnrec_op[r] - 1, (double)g.nnrec_ph[r] * v);
            }
        }
    }
    // ---- PN: dpn[cpn(b,a)+dpn(d,c)] += php * phn * psi[row+pos] psi[q+in]
    for (int c = a.pn_ptr[slot]; c < a.pn_ptr[slot + 1]; ++c) {
        const PNContrib pc = a.pn[c];
        const NOp op = a.nops[pc.nop];
        for (int k = lane; k < op.nbd; k += 32) Aw[k] = 0.0;
        __syncwarp();
        const int32_t *__restrict__ ptr = a.nptr + op.ptr_base;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            if (!valid[i] || pos[i] >= op.nout) continue;
            const int k0 = ptr[pos[i]], k1 = ptr[pos[i] + 1];
            for (int k = k0; k < k1; ++k) {
                const PNRec r = a.pnrec[op.rec_base + k];
                const double v = pout[i] * psi[pc.q_off + r.in] * (double)r.ph;
                atomicAdd(Aw + r.k, v);
            }
        }
        __syncwarp();
        const int acol = pc.acol * a.ld_cpn, ccol = pc.ccol * a.ld_cpn;
        for (int k = lane; k < op.nbd; k += 32) {
            const double v = Aw[k];
            if (v != 0.0) {
                const BDPair bd = a.bd[op.bd_base + k];
                const int idx = a.cpn[bd.b + acol] + a.dpn[bd.d + ccol];
                atomicAdd(g.dpn + idx - 1, (double)pc.php * v);
            }
        }
        __syncwarp();
    }
    // ---- SPE: d/dpspe_h(ip) and d/dnspe_h(in) of sum psi^2 (pspe + nspe)
    if (g.dspe_p) {
        for (int c = a.spe_ptr[slot]; c < a.spe_ptr[slot + 1]; ++c) {
            const SPEContrib sc = a.spe[c];
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (valid[i] && pos[i] >= sc.lo && pos[i] <= sc.hi) {
                    const double p2 = pout[i] * pout[i];
                    s += p2;
                    atomicAdd(g.dspe_n + sc.n0 + (pos[i] - sc.lo), p2);
                }
            }
            s = warp_sum(s);
            if (lane == 0 && s != 0.0) atomicAdd(g.dspe_p + row, s);
        }
    }
}

}  // namespace bsg

using namespace bsg;

extern "C" int bsg_grad(bsg_ctx *ctx, const double *evecs, int nstates, double *dpp, double *dnn, double *dpn,
                        double *dspe_p, double *dspe_n) {
    if (!ctx) return BSG_ERR_ARG;
    if (!evecs || nstates < 1 || !dpp || !dnn || !dpn)
        return set_err(ctx, BSG_ERR_ARG, "bsg_grad: null argument or nstates < 1");
    const bool spe = ctx->t.call_spe && dspe_p && dspe_n;
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (st) return st;
    const int64_t n = ctx->dim;
    const size_t npp = (size_t)ctx->t.nmatpp, nnn = (size_t)ctx->t.nmatnn, npn = (size_t)ctx->t.nmatpn;
    const size_t nsp = (size_t)ctx->t.nsd_p, nsn = (size_t)ctx->t.nsd_n;
    DevBuf psi, gpp, gnn, gpn, gsp, gsn;
    constexpr int ITEMS = 4;
    ctx->last_status = BSG_OK;
    const TileSet *ts = get_tiles(ctx, 32 * ITEMS);
    if (!ts) return ctx->last_status ? ctx->last_status : BSG_ERR_NOMEM;
    if ((st = dev_alloc(ctx, psi, sizeof(double) * n)) || (st = dev_alloc(ctx, gpp, sizeof(double) * npp)) ||
        (st = dev_alloc(ctx, gnn, sizeof(double) * nnn)) || (st = dev_alloc(ctx, gpn, sizeof(double) * npn)) ||
        (st = dev_alloc(ctx, gsp, sizeof(double) * nsp)) || (st = dev_alloc(ctx, gsn, sizeof(double) * nsn))) {
        dev_free(psi); dev_free(gpp); dev_free(gnn); dev_free(gpn); dev_free(gsp); dev_free(gsn);
        return st;
    }
    RowArgs a = ctx->args;
    a.tiles = (const Tile *)ts->buf.p;
    a.ntiles = ts->ntiles;
    GradArgs g;
    g.pp_op = (const int32_t *)ctx->pp_op.p;
    g.pp_ph = (const int8_t *)ctx->pp_ph.p;
    g.nnrec_op = (const int32_t *)ctx->nnrec_op.p;
    g.nnrec_ph = (const int8_t *)ctx->nnrec_ph.p;
    g.dpp = (double *)gpp.p;
    g.dnn = (double *)gnn.p;
    g.dpn = (double *)gpn.p;
    g.dspe_p = spe ? (double *)gsp.p : nullptr;
    g.dspe_n = spe ? (double *)gsn.p : nullptr;
    const int mstride = (a.max_nbd + 1) & ~1;
    // 8 per-warp FP64 tables within the 227 KB of shared memory per CTA
    if (a.max_nbd > 3392) {
        dev_free(psi); dev_free(gpp); dev_free(gnn); dev_free(gpn); dev_free(gsp); dev_free(gsn);
        return set_err(ctx, BSG_ERR_UNSUPPORTED, "bsg_grad: a neutron sector jump has more than 3392 distinct (b,d) pairs");
    }
    const size_t smem = sizeof(double) * (size_t)kGradWarps * (mstride > 0 ? mstride : 2);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaFuncSetAttribute(k_grad<ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (int k = 0; k < nstates && e == cudaSuccess; ++k) {
        e = cudaMemcpyAsync(psi.p, evecs + (size_t)k * n, sizeof(double) * n, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(gpp.p, 0, gpp.bytes, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(gnn.p, 0, gnn.bytes, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(gpn.p, 0, gpn.bytes, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(gsp.p, 0, gsp.bytes, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(gsn.p, 0, gsn.bytes, s);
        if (e == cudaSuccess && ts->ntiles > 0) {
            k_grad<ITEMS><<<ts->ntiles, kGradWarps * 32, smem, s>>>(a, g, (const double *)psi.p, mstride);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && npp) e = cudaMemcpyAsync(dpp + k * npp, gpp.p, sizeof(double) * npp, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && nnn) e = cudaMemcpyAsync(dnn + k * nnn, gnn.p, sizeof(double) * nnn, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && npn) e = cudaMemcpyAsync(dpn + k * npn, gpn.p, sizeof(double) * npn, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && spe) e = cudaMemcpyAsync(dspe_p + k * nsp, gsp.p, sizeof(double) * nsp, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && spe) e = cudaMemcpyAsync(dspe_n + k * nsn, gsn.p, sizeof(double) * nsn, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    st = cuda_check(ctx, e, "bsg_grad");
    dev_free(psi); dev_free(gpp); dev_free(gnn); dev_free(gpn); dev_free(gsp); dev_free(gsn);
    return st;
}
