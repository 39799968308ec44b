// Row-tile body of the adjoint (Hellmann-Feynman gradient), shared by the
// single-system bsg_grad and the batched bsg_batch_grad.
//
// dE_k/dhmat(label) = sum over every appearance of the label in H of
// phase * psi_k(out) * psi_k(in): the traversal of the two-body densities
// applyh{PP,NN,PN}bundled_den (src/bdenslib4.f90:129-729, dmat(op) +=
// vout(f)*vin(i)*phase) with both vectors equal to the eigenvector, run over
// the matvec's row tiles and (row, warp) slots, so every f/b appearance,
// hermitian half and 1/2 on diagonal pair labels counts as in the matvec.
//
// Determinism: every global sum is a 128-bit two's-complement fixed-point
// number with 64 fraction bits, updated with 64-bit integer atomics (low word,
// carry into the high word).  Integer addition is associative, so the result
// does not depend on the order in which CTAs arrive; doubles convert exactly
// down to 2^-64.  Per-warp PN bins are summed in lane order.
#pragma once

#include "bsg_internal.h"

namespace bsg {

constexpr int kGradWarps = kRowWarps;

struct GradArgs {
    const int32_t *pp_op;         // hmatpp label of each PP contribution
    const int8_t *pp_ph;          // its jump phase
    const int32_t *nnrec_op;      // hmatnn label of each NN record
    const int8_t *nnrec_ph;       // its jump phase
    // fixed-point accumulators, (lo, hi) words per label: acc[2i], acc[2i+1]
    unsigned long long *pp, *nn, *pn, *spe_p, *spe_n;
};

// acc += v exactly (to 2^-64), order-independent
__device__ __forceinline__ void fix_add(unsigned long long *acc, double v) {
    if (v == 0.0) return;
    const double fl = floor(v);
    const double fr = v - fl;  // [0, 1), exact for |v| < 2^52
    const unsigned long long lo = __double2ull_rz(fr * 18446744073709551616.0);
    const unsigned long long hi = (unsigned long long)(long long)fl;
    const unsigned long long old = atomicAdd(acc, lo);
    atomicAdd(acc + 1, hi + (old + lo < old ? 1ull : 0ull));
}

__device__ __forceinline__ double fix_value(const unsigned long long *acc) {
    return (double)(long long)acc[1] + (double)acc[0] * 5.421010862427522170e-20;  // 2^-64
}

__device__ __forceinline__ double grad_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One tile of one output row for one state.  Aw: this warp's FP64 bins for
// the distinct (b,d) pairs of a PN operator (mstride doubles); stage_k /
// stage_v: this warp's 32-entry staging area for the lane-order bin sums.
template <int ITEMS>
__device__ __forceinline__ void grad_tile(const RowArgs &a, const GradArgs &g, const double *__restrict__ psi,
                                          const Tile tile, double *__restrict__ Aw, int *__restrict__ stage_k,
                                          double *__restrict__ stage_v) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
        s = grad_warp_sum(s);
        if (lane == 0) fix_add(g.pp + 2 * (size_t)(g.pp_op[c] - 1), (double)g.pp_ph[c] * s);
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
                fix_add(g.nn + 2 * (size_t)(g.nnrec_op[r] - 1), (double)g.nnrec_ph[r] * v);
            }
        }
    }
    // ---- PN: dpn[cpn(b,a)+dpn(d,c)] += php * phn * psi[row+pos] psi[q+in]
    // Records are walked in warp-wide steps; in each step the lanes that hit
    // the same (b,d) bin are added in lane order by the lowest of them.
    for (int c = a.pn_ptr[slot]; c < a.pn_ptr[slot + 1]; ++c) {
        const PNContrib pc = a.pn[c];
        const NOp op = a.nops[pc.nop];
        for (int k = lane; k < op.nbd; k += 32) Aw[k] = 0.0;
        __syncwarp();
        const int32_t *__restrict__ ptr = a.nptr + op.ptr_base;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            int k0 = 0, n = 0;
            if (valid[i] && pos[i] < op.nout) {
                k0 = ptr[pos[i]];
                n = ptr[pos[i] + 1] - k0;
            }
            const int nmax = __reduce_max_sync(0xffffffffu, n);
            for (int j = 0; j < nmax; ++j) {
                int key = -1;
                double v = 0.0;
                if (j < n) {
                    const PNRec r = a.pnrec[op.rec_base + k0 + j];
                    v = pout[i] * psi[pc.q_off + r.in] * (double)r.ph;
                    key = r.k;
                }
                stage_k[lane] = key;
                stage_v[lane] = v;
                const unsigned grp = __match_any_sync(0xffffffffu, key);
                __syncwarp();
                if (key >= 0 && lane == __ffs(grp) - 1) {
                    double s = 0.0;
                    for (unsigned m = grp; m; m &= m - 1) s += stage_v[__ffs(m) - 1];
                    Aw[key] += s;
                }
                __syncwarp();
            }
        }
        for (int k = lane; k < op.nbd; k += 32) {
            const double v = Aw[k];
            if (v != 0.0) {
                const BDPair bd = a.bd[op.bd_base + k];
                const int idx = a.cpn[bd.b + pc.aoff] + a.dpn[bd.d + pc.coff];
                fix_add(g.pn + 2 * (size_t)(idx - 1), (double)pc.php * v);
            }
        }
        __syncwarp();
    }
    // ---- SPE: d/dpspe_h(ip) and d/dnspe_h(in) of sum psi^2 (pspe + nspe)
    if (g.spe_p) {
        for (int c = a.spe_ptr[slot]; c < a.spe_ptr[slot + 1]; ++c) {
            const SPEContrib sc = a.spe[c];
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (valid[i] && pos[i] >= sc.lo && pos[i] <= sc.hi) {
                    const double p2 = pout[i] * pout[i];
                    s += p2;
                    fix_add(g.spe_n + 2 * (size_t)(sc.n0 + (pos[i] - sc.lo)), p2);
                }
            }
            s = grad_warp_sum(s);
            if (lane == 0) fix_add(g.spe_p + 2 * (size_t)row, s);
        }
    }
}

// shared memory of one adjoint CTA: 8 warps' bins, then their staging areas
__host__ __device__ constexpr size_t grad_smem_bytes(int mstride) {
    return sizeof(double) * (size_t)kGradWarps * (size_t)(mstride > 0 ? mstride : 2) +
           (sizeof(double) + sizeof(int)) * (size_t)kGradWarps * 32;
}

__device__ __forceinline__ void grad_smem(int mstride, double *&Aw, int *&stage_k, double *&stage_v) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int ms = mstride > 0 ? mstride : 2;
    double *base = reinterpret_cast<double *>(smem);
    Aw = base + (size_t)warp * ms;
    stage_v = base + (size_t)kGradWarps * ms + (size_t)warp * 32;
    stage_k = reinterpret_cast<int *>(base + (size_t)kGradWarps * ms + (size_t)kGradWarps * 32) + warp * 32;
}

}  // namespace bsg
