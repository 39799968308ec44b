// Row-tile body of the output-stationary applyH, shared by the single-system
// kernel (applyh_kernels.cu) and the persistent batched kernel (batch.cu).
#pragma once

#include <type_traits>

#include "bsg_internal.h"

namespace bsg {

template <typename T, int NB, bool FULL>
struct Vec {
    // load NB consecutive elements of vector data starting at p
    static __device__ __forceinline__ void load(const T *__restrict__ p, T (&x)[NB]) {
#pragma unroll
        for (int v = 0; v < NB; ++v) x[v] = __ldg(p + v);
    }
};
template <>
struct Vec<float, 4, true> {
    static __device__ __forceinline__ void load(const float *__restrict__ p, float (&x)[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    }
};
template <>
struct Vec<float, 8, true> {
    static __device__ __forceinline__ void load(const float *__restrict__ p, float (&x)[8]) {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
        const float4 b = __ldg(reinterpret_cast<const float4 *>(p) + 1);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    }
};
template <>
struct Vec<float, 16, true> {
    static __device__ __forceinline__ void load(const float *__restrict__ p, float (&x)[16]) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float4 a = __ldg(reinterpret_cast<const float4 *>(p) + k);
            x[4 * k] = a.x; x[4 * k + 1] = a.y; x[4 * k + 2] = a.z; x[4 * k + 3] = a.w;
        }
    }
};
template <>
struct Vec<float, 2, true> {
    static __device__ __forceinline__ void load(const float *__restrict__ p, float (&x)[2]) {
        const float2 a = __ldg(reinterpret_cast<const float2 *>(p));
        x[0] = a.x; x[1] = a.y;
    }
};
template <int NB>
struct VecD2 {
    static __device__ __forceinline__ void load(const double *__restrict__ p, double (&x)[NB]) {
#pragma unroll
        for (int k = 0; k < NB / 2; ++k) {
            const double2 a = __ldg(reinterpret_cast<const double2 *>(p) + k);
            x[2 * k] = a.x; x[2 * k + 1] = a.y;
        }
    }
};
template <> struct Vec<double, 2, true> : VecD2<2> {};
template <> struct Vec<double, 4, true> : VecD2<4> {};
template <> struct Vec<double, 8, true> : VecD2<8> {};
template <> struct Vec<double, 16, true> : VecD2<16> {};

constexpr int kWarps = kRowWarps;

// Record k of an output position is read at column[kRecStride * k].  The row
// kernels walk the sliced copy, where the lanes of a warp read adjacent
// records (tiles start on multiples of 32, so pos & 31 == lane).  The
// position-sorted walk (stride 1) gives the records of a position in the same
// order and stays available for other traversals.
template <typename T, int NB> constexpr bool kSliced = true;
template <typename T, int NB> constexpr int kRecStride = kSliced<T, NB> ? 32 : 1;
// the column base and the range of k for one output position; csr = the
// operator's position-sorted records, [k0, k1) this position's range there
template <typename T, int NB>
__device__ __forceinline__ void record_column(const RowArgs &a, const NOp &op, const int2 *csr, int k0, int k1,
                                              int pos, int lane, const int2 *&col, int &k, int &kend) {
    if constexpr (kSliced<T, NB>) {
        col = a.sell + op.sell_base + __ldg(a.slice_off + op.slice_base + (pos >> 5)) + lane;
        k = 0;
        kend = k1 - k0;
    } else {
        col = csr;
        k = k0;
        kend = k1;
    }
}

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// One CTA = one tile of one output row: positions pos0 + lane + 32*i.  Warp w
// handles the contributions assigned to slot (row, w) at setup (balanced by
// estimated work) and accumulates in registers (SACC below: in its own shared
// entries between record walks); the eight partial sums are
// added in fixed warp order at the end, so the result does not depend on
// scheduling.
// ld: elements between consecutive states (the block size nb); v0: first
// vector column handled by this launch; FULL: ld == NB and aligned base.
// mstride: floats of per-warp shared memory for the PN matrix-element table.
// what the tile does with its sums: store them, add them to the output, or
// store them as FP64 columns (RowArgs::cols_out) for the Lanczos history.
// Separate instantiations keep the common store free of the other modes'
// registers.
enum RowOut { kStore = 0, kAccumulate = 1, kColumns = 2 };

// REC32: walk the 32-bit sliced records (RowArgs::sell32) instead of the
// 8-byte ones; the decoded values, and so the sums, are the same bit for bit.
// SACC: between the PP and SPE passes the running sums live in this thread's
// entries of `part` instead of registers; each NN / PN record walk loads its
// item's sum, accumulates in registers and stores it back.  The operations
// and their order are unchanged (bitwise the same sums); what changes is that
// the ITEMS sums are not live across the walks.
template <typename T, int NB, int ITEMS, bool FULL, int OUT = kStore, bool REC32 = false, bool SACC = false>
__device__ __forceinline__ void row_tile(const RowArgs &a, const Tile tile, const T *__restrict__ vin,
                                         T *__restrict__ vout, const int ld_, const int v0_,
                                         float *__restrict__ Mw, T *__restrict__ part) {
    // dense layout: the stride is the compile-time block size and the column
    // offset is zero, so gather addresses need no runtime multiply
    const int ld = FULL ? NB : ld_;
    const int v0 = FULL ? 0 : v0_;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = tile.row;
    const int64_t roff = a.row_off[row];

    // position of item i: p0 + 32 i, in the tile while 32 i < lim (derived
    // from two registers instead of held per item: the 32-register kernels
    // spill less)
    T acc[ITEMS][NB];
    const int p0 = tile.pos0 + lane, lim = tile.npos - lane;
#define BSG_POS(i) (p0 + 32 * (i))
#define BSG_VALID(i) (32 * (i) < lim)
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
#pragma unroll
        for (int v = 0; v < NB; ++v) acc[i][v] = T(0);
    }

    // ---- PP: out[pos] += me * in[q_off + pos]   (src/bapplyhlibOMP.f90:1068-1241)
    {
        const int slot = row * kWarps + warp;
        const int c1 = a.pp_ptr[slot + 1];
        for (int c = a.pp_ptr[slot]; c < c1; ++c) {
            const PPContrib pc = a.pp[c];
            const T me = (T)pc.me;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (BSG_VALID(i) && BSG_POS(i) >= pc.lo && BSG_POS(i) <= pc.hi) {
                    T x[NB];
                    Vec<T, NB, FULL>::load(vin + (size_t)(pc.q_off + BSG_POS(i)) * ld + v0, x);
#pragma unroll
                    for (int v = 0; v < NB; ++v) acc[i][v] += me * x[v];
                }
            }
        }
    }
    // item i's sums: mine[32 * i * NB + v], this thread's entries of part
    constexpr int TP = 32 * ITEMS;
    T *__restrict__ mine = part + ((size_t)warp * TP + lane) * NB;
    if constexpr (SACC) {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
#pragma unroll
            for (int v = 0; v < NB; ++v) mine[32 * i * NB + v] = acc[i][v];
    }
    // ---- NN: out[pos] += sum r.me * in[row + r.in]   (:1012-1066)
    {
        const int slot = row * kWarps + warp;
        const int c1 = a.nn_ptr[slot + 1];
        const T *__restrict__ src = vin + (size_t)roff * ld + v0;
        for (int c = a.nn_ptr[slot]; c < c1; ++c) {
            const NOp op = a.nops[a.nn[c].nop];
            const int32_t *__restrict__ ptr = a.nptr + op.ptr_base;
            const int2 *__restrict__ rec = reinterpret_cast<const int2 *>(a.nnrec + op.rec_base);
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (!BSG_VALID(i) || BSG_POS(i) >= op.nout) continue;
                const int k0 = __ldg(ptr + BSG_POS(i)), k1 = __ldg(ptr + BSG_POS(i) + 1);
                T sv[NB];
                if constexpr (SACC) {
#pragma unroll
                    for (int v = 0; v < NB; ++v) sv[v] = mine[32 * i * NB + v];
                }
                T (&A)[NB] = SACC ? sv : acc[i];
                auto put = [&]() {
                    if constexpr (SACC) {
#pragma unroll
                        for (int v = 0; v < NB; ++v) mine[32 * i * NB + v] = sv[v];
                    }
                };
                // NN takes the 32-bit records for FP64 vectors only: for FP32
                // the extra hmatnn load per record cost more than the halved
                // record bytes saved (pf 6p6n: 143.8 against 139.2 ms)
                if constexpr (REC32 && std::is_same<T, double>::value) {
                    // input position | hmatnn label - 1 | phase sign
                    const uint32_t *c32 =
                        a.sell32 + op.sell_base + __ldg(a.slice_off + op.slice_base + (BSG_POS(i) >> 5)) + lane;
                    const int n = k1 - k0;
                    int k = 0;
                    for (; k + 1 < n; k += 2) {
                        const uint32_t r0 = __ldg(c32 + 32 * k), r1 = __ldg(c32 + 32 * (k + 1));
                        T x0[NB], x1[NB];
                        Vec<T, NB, FULL>::load(src + (size_t)(r0 & 0xffffu) * ld, x0);
                        Vec<T, NB, FULL>::load(src + (size_t)(r1 & 0xffffu) * ld, x1);
                        const T m0 = (T)__int_as_float(__float_as_int(__ldg(a.hmatnn + ((r0 >> 16) & 0x7fffu))) ^
                                                       (int)(r0 & 0x80000000u));
                        const T m1 = (T)__int_as_float(__float_as_int(__ldg(a.hmatnn + ((r1 >> 16) & 0x7fffu))) ^
                                                       (int)(r1 & 0x80000000u));
#pragma unroll
                        for (int v = 0; v < NB; ++v) { A[v] += m0 * x0[v]; A[v] += m1 * x1[v]; }
                    }
                    if (k < n) {
                        const uint32_t r0 = __ldg(c32 + 32 * k);
                        T x0[NB];
                        Vec<T, NB, FULL>::load(src + (size_t)(r0 & 0xffffu) * ld, x0);
                        const T m0 = (T)__int_as_float(__float_as_int(__ldg(a.hmatnn + ((r0 >> 16) & 0x7fffu))) ^
                                                       (int)(r0 & 0x80000000u));
#pragma unroll
                        for (int v = 0; v < NB; ++v) A[v] += m0 * x0[v];
                    }
                    put();
                    continue;
                }
                const int2 *col;
                int k, n;
                record_column<T, NB>(a, op, rec, k0, k1, BSG_POS(i), lane, col, k, n);
                for (; k + 1 < n; k += 2) {
                    const int2 r0 = __ldg(col + kRecStride<T, NB> * k), r1 = __ldg(col + kRecStride<T, NB> * (k + 1));
                    T x0[NB], x1[NB];
                    Vec<T, NB, FULL>::load(src + (size_t)r0.x * ld, x0);
                    Vec<T, NB, FULL>::load(src + (size_t)r1.x * ld, x1);
                    const T m0 = (T)__int_as_float(r0.y), m1 = (T)__int_as_float(r1.y);
#pragma unroll
                    for (int v = 0; v < NB; ++v) { A[v] += m0 * x0[v]; A[v] += m1 * x1[v]; }
                }
                if (k < n) {
                    const int2 r0 = __ldg(col + kRecStride<T, NB> * k);
                    T x0[NB];
                    Vec<T, NB, FULL>::load(src + (size_t)r0.x * ld, x0);
                    const T m0 = (T)__int_as_float(r0.y);
#pragma unroll
                    for (int v = 0; v < NB; ++v) A[v] += m0 * x0[v];
                }
                put();
            }
        }
    }
    // ---- PN: out[pos] += sum hmatpn(cpn(b,a)+dpn(d,c))*php*phn * in[q_off + r.in]  (:1242-1442)
    // The warp first tabulates hmatpn(cpn(b,a)+dpn(d,c))*php for the proton
    // jump's (a,c) and every distinct neutron (b,d) of the operator; a record
    // then costs one shared load, the neutron phase is its sign bit.
    {
        const int slot = row * kWarps + warp;
        const int c1 = a.pn_ptr[slot + 1];
        for (int c = a.pn_ptr[slot]; c < c1; ++c) {
            const PNContrib pc = a.pn[c];
            const NOp op = a.nops[pc.nop];
            for (int k = lane; k < op.nbd; k += 32) {
                const BDPair bd = a.bd[op.bd_base + k];
                const int idx = __ldg(a.cpn + bd.b + pc.aoff) + __ldg(a.dpn + bd.d + pc.coff);
                float xme = __ldg(a.hmatpn + idx - 1);
                Mw[k] = xme * pc.php;
            }
            __syncwarp();
            const int32_t *__restrict__ ptr = a.nptr + op.ptr_base;
            const int2 *__restrict__ rec = reinterpret_cast<const int2 *>(a.pnrec + op.rec_base);
            const T *__restrict__ src = vin + (size_t)pc.q_off * ld + v0;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (!BSG_VALID(i) || BSG_POS(i) >= op.nout) continue;
                const int k0 = __ldg(ptr + BSG_POS(i)), k1 = __ldg(ptr + BSG_POS(i) + 1);
                T sv[NB];
                if constexpr (SACC) {
#pragma unroll
                    for (int v = 0; v < NB; ++v) sv[v] = mine[32 * i * NB + v];
                }
                T (&A)[NB] = SACC ? sv : acc[i];
                auto put = [&]() {
                    if constexpr (SACC) {
#pragma unroll
                        for (int v = 0; v < NB; ++v) mine[32 * i * NB + v] = sv[v];
                    }
                };
                if constexpr (REC32) {
                    // input position | (b,d) index | neutron phase sign
                    const uint32_t *c32 =
                        a.sell32 + op.sell_base + __ldg(a.slice_off + op.slice_base + (BSG_POS(i) >> 5)) + lane;
                    const int n = k1 - k0;
                    int k = 0;
                    for (; k + 1 < n; k += 2) {
                        const uint32_t r0 = __ldg(c32 + 32 * k), r1 = __ldg(c32 + 32 * (k + 1));
                        T x0[NB], x1[NB];
                        Vec<T, NB, FULL>::load(src + (size_t)(r0 & 0xffffu) * ld, x0);
                        Vec<T, NB, FULL>::load(src + (size_t)(r1 & 0xffffu) * ld, x1);
                        const T m0 = (T)__int_as_float(__float_as_int(Mw[(r0 >> 16) & 0x7fffu]) ^ (int)(r0 & 0x80000000u));
                        const T m1 = (T)__int_as_float(__float_as_int(Mw[(r1 >> 16) & 0x7fffu]) ^ (int)(r1 & 0x80000000u));
#pragma unroll
                        for (int v = 0; v < NB; ++v) { A[v] += m0 * x0[v]; A[v] += m1 * x1[v]; }
                    }
                    if (k < n) {
                        const uint32_t r0 = __ldg(c32 + 32 * k);
                        T x0[NB];
                        Vec<T, NB, FULL>::load(src + (size_t)(r0 & 0xffffu) * ld, x0);
                        const T m0 = (T)__int_as_float(__float_as_int(Mw[(r0 >> 16) & 0x7fffu]) ^ (int)(r0 & 0x80000000u));
#pragma unroll
                        for (int v = 0; v < NB; ++v) A[v] += m0 * x0[v];
                    }
                    put();
                    continue;
                }
                const int2 *col;
                int k, n;
                record_column<T, NB>(a, op, rec, k0, k1, BSG_POS(i), lane, col, k, n);
                for (; k + 1 < n; k += 2) {
                    const int2 r0 = __ldg(col + kRecStride<T, NB> * k), r1 = __ldg(col + kRecStride<T, NB> * (k + 1));
                    T x0[NB], x1[NB];
                    Vec<T, NB, FULL>::load(src + (size_t)r0.x * ld, x0);
                    Vec<T, NB, FULL>::load(src + (size_t)r1.x * ld, x1);
                    // neutron phase: int8 at bits 16..23, its sign moved to bit 31
                    const float f0 = __int_as_float(__float_as_int(Mw[r0.y & 0xffff]) ^ ((r0.y << 8) & 0x80000000));
                    const float f1 = __int_as_float(__float_as_int(Mw[r1.y & 0xffff]) ^ ((r1.y << 8) & 0x80000000));
                    const T m0 = (T)f0, m1 = (T)f1;
#pragma unroll
                    for (int v = 0; v < NB; ++v) { A[v] += m0 * x0[v]; A[v] += m1 * x1[v]; }
                }
                if (k < n) {
                    const int2 r0 = __ldg(col + kRecStride<T, NB> * k);
                    T x0[NB];
                    Vec<T, NB, FULL>::load(src + (size_t)r0.x * ld, x0);
                    const float f0 = __int_as_float(__float_as_int(Mw[r0.y & 0xffff]) ^ ((r0.y << 8) & 0x80000000));
                    const T m0 = (T)f0;
#pragma unroll
                    for (int v = 0; v < NB; ++v) A[v] += m0 * x0[v];
                }
                put();
            }
            __syncwarp();
        }
    }
    // ---- SPE: out[pos] += (pspe + nspe) * in[pos]   (:988-1011)
    if constexpr (SACC) {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
#pragma unroll
            for (int v = 0; v < NB; ++v) acc[i][v] = mine[32 * i * NB + v];
    }
    {
        const int slot = row * kWarps + warp;
        const int c1 = a.spe_ptr[slot + 1];
        for (int c = a.spe_ptr[slot]; c < c1; ++c) {
            const SPEContrib sc = a.spe[c];
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (BSG_VALID(i) && BSG_POS(i) >= sc.lo && BSG_POS(i) <= sc.hi) {
                    const float e = sc.pspe + __ldg(a.nspe + sc.n0 + (BSG_POS(i) - sc.lo));
                    T x[NB];
                    Vec<T, NB, FULL>::load(vin + (size_t)(roff + BSG_POS(i)) * ld + v0, x);
#pragma unroll
                    for (int v = 0; v < NB; ++v) acc[i][v] += x[v] * (T)e;
                }
            }
        }
    }
    // ---- fixed-order reduction over the warps, single write per element
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
#pragma unroll
        for (int v = 0; v < NB; ++v) part[((size_t)warp * TP + lane + 32 * i) * NB + v] = acc[i][v];
    __syncthreads();
    const int nel = tile.npos * NB;
    if constexpr (OUT == kColumns) {
        // FP64 columns: consecutive threads take consecutive positions of one
        // column (coalesced stores); each element summed as below
        for (int e = threadIdx.x; e < nel; e += kWarps * 32) {
            const int v = e / tile.npos, lp = e - v * tile.npos;
            const int idx = lp * NB + v;
            T s = part[idx];
#pragma unroll
            for (int w = 1; w < kWarps; ++w) s += part[(size_t)w * TP * NB + idx];
            a.cols_out[(size_t)(v0 + v) * a.cols_ld + roff + tile.pos0 + lp] = (double)s;
        }
    } else {
        for (int e = threadIdx.x; e < nel; e += kWarps * 32) {
            T s = part[e];
#pragma unroll
            for (int w = 1; w < kWarps; ++w) s += part[(size_t)w * TP * NB + e];
            const int lp = e / NB, v = e - lp * NB;
            T *o = vout + (size_t)(roff + tile.pos0 + lp) * ld + v0 + v;
            if constexpr (OUT == kAccumulate)
                *o = *o + s;
            else
                *o = s;
        }
    }
}


#undef BSG_POS
#undef BSG_VALID

}  // namespace bsg
