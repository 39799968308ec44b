// Output-stationary applyH kernels for sm_100a.
//
// The reference (src/bapplyhlibOMP.f90:882-1657) walks opbundles and
// scatters `vout(statef) += xme*vin(statei)`, keeping OpenMP threads apart
// with per-thread output ranges (getLoadDist) and repeated filtered scans.
// Here every CTA owns one tile of one output row (a proton SD with its
// contiguous run of neutron partners, pstart(ip) + nstart(in)).  It gathers
// all contributions to that tile -- PP as coalesced row AXPYs, NN and PN
// through neutron operators whose records are sorted by output position --
// in registers, and writes each output element exactly once.  There are no
// atomics and the summation order is fixed, so results are bitwise
// repeatable; the vector traffic is one gathered read per operation and one
// write per output element.
//
// Arithmetic follows the reference: the matrix element is formed in float
// (hmat * phase, src/bapplyhlibOMP.f90:1093-1095, :1269-1272) and promoted
// to the vector type; FP32 vectors accumulate in FP32, FP64 vectors in FP64.

#include <type_traits>

#include "applyh_tile.cuh"

namespace bsg {

template <typename T, int NB, int ITEMS, bool FULL, int OUT, bool REC32 = false, bool SACC = false>
__device__ __forceinline__ void rows_body(const RowArgs &a, const T *__restrict__ vin, T *__restrict__ vout,
                                          const int ld, const int v0, const int mstride) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    float *__restrict__ Mw = reinterpret_cast<float *>(smem) + (size_t)warp * mstride;
    T *__restrict__ part = reinterpret_cast<T *>(smem + align16(sizeof(float) * (size_t)kWarps * mstride));
    row_tile<T, NB, ITEMS, FULL, OUT, REC32, SACC>(a, a.tiles[blockIdx.x], vin, vout, ld, v0, Mw, part);
}

// OUT: store, accumulate, or FP64 columns (RowOut in applyh_tile.cuh)
template <typename T, int NB, int ITEMS, bool FULL, int OUT>
__global__ void __launch_bounds__(kWarps * 32) k_rows(const RowArgs a, const T *__restrict__ vin,
                                                      T *__restrict__ vout, const int ld, const int v0,
                                                      const int mstride) {
    rows_body<T, NB, ITEMS, FULL, OUT>(a, vin, vout, ld, v0, mstride);
}

// single vectors: at most 40 registers, so that 6 CTAs of 256 threads stay
// resident per SM to hide the gather latency (measured faster than the
// compiler's own choice of 48 registers, the small spills included).  FP32
// tiles of 256 positions (long rows) go further, to 32 registers and 8 CTAs:
// pf 4p4n 1.80 -> 1.61 ms, while short rows lose more to the spills.
// REC32: the 32-bit sliced records (half the record bytes of the L1 stream).
// With 4 or more items per lane the running sums stay in shared memory during
// the NN and PN record walks (row_tile's SACC): spill loads of the 8-item
// kernel 372 -> 64 bytes, and pf 6p6n 141.1 -> 133.1 ms, bitwise the same
// output.  FP64 keeps its sums in registers: there the extra shared traffic
// cost more than the spills (sd 6p6n 81.1 -> 87.2 us).
template <int ITEMS, bool FULL, int OUT, bool REC32>
__global__ void __launch_bounds__(kWarps * 32, ITEMS >= 8 ? 8 : 6) k_rows_f1(const RowArgs a, const float *__restrict__ vin,
                                                            float *__restrict__ vout, const int ld, const int v0,
                                                            const int mstride) {
    rows_body<float, 1, ITEMS, FULL, OUT, REC32, (ITEMS >= 4)>(a, vin, vout, ld, v0, mstride);
}
template <int ITEMS, bool FULL, int OUT, bool REC32>
__global__ void __launch_bounds__(kWarps * 32, 6) k_rows_d1(const RowArgs a, const double *__restrict__ vin,
                                                            double *__restrict__ vout, const int ld, const int v0,
                                                            const int mstride) {
    rows_body<double, 1, ITEMS, FULL, OUT, REC32>(a, vin, vout, ld, v0, mstride);
}

template <typename T, int NB, int ITEMS, bool FULL, int OUT, bool REC32>
constexpr auto rows_kernel() {
    if constexpr (std::is_same<T, float>::value && NB == 1)
        return k_rows_f1<ITEMS, FULL, OUT, REC32>;
    else if constexpr (std::is_same<T, double>::value && NB == 1)
        return k_rows_d1<ITEMS, FULL, OUT, REC32>;
    else
        return k_rows<T, NB, ITEMS, FULL, OUT>;
}

template <typename T, int NB, int ITEMS>
static int launch_one(bsg_ctx *ctx, const T *vin, T *vout, int ld, int v0, int accumulate,
                      cudaStream_t s, TileLookup lookup, double *cols) {
    ctx->last_status = BSG_OK;
    const TileSet *ts = lookup ? lookup(ctx, 32 * ITEMS) : get_tiles(ctx, 32 * ITEMS);
    // the status the failing lookup recorded (a refused size is BSG_ERR_ARG)
    if (!ts) return ctx->last_status ? ctx->last_status : BSG_ERR_NOMEM;
    if (ts->ntiles == 0) return BSG_OK;
    RowArgs a = ctx->args;
    a.tiles = (const Tile *)ts->buf.p;
    a.ntiles = ts->ntiles;
    a.accumulate = accumulate;
    a.cols_out = cols;
    a.cols_ld = ctx->dim;
    const int mstride = (a.max_nbd + 3) & ~3;
    const size_t smem = align16(sizeof(float) * (size_t)kWarps * mstride) +
                        sizeof(T) * (size_t)kWarps * 32 * ITEMS * NB;
    // aligned vector loads only when each state's NB values are contiguous and
    // the base pointer is 16-byte aligned
    const bool full = (ld == NB) && ((reinterpret_cast<uintptr_t>(vin) & 15u) == 0);
    cudaError_t e;
    auto allow = [&](const void *fn) -> cudaError_t {
        size_t &cur = ctx->smem_allowed[fn];
        if (cur >= smem) return cudaSuccess;
        const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (r == cudaSuccess) cur = smem;
        return r;
    };
    auto go = [&](auto k) -> cudaError_t {
        cudaError_t r = allow((const void *)k);
        if (r == cudaSuccess) k<<<ts->ntiles, kWarps * 32, smem, s>>>(a, vin, vout, ld, v0, mstride);
        return r;
    };
    // single vectors walk the 32-bit records when the context has them
    auto pick = [&](auto rec32) -> cudaError_t {
        constexpr bool R = decltype(rec32)::value && NB == 1;
        if (cols) return go(rows_kernel<T, NB, ITEMS, true, kColumns, R>());
        if (full)
            return accumulate ? go(rows_kernel<T, NB, ITEMS, true, kAccumulate, R>())
                              : go(rows_kernel<T, NB, ITEMS, true, kStore, R>());
        return accumulate ? go(rows_kernel<T, NB, ITEMS, false, kAccumulate, R>())
                          : go(rows_kernel<T, NB, ITEMS, false, kStore, R>());
    };
    // FP32 reads only the PN part of the 32-bit records; FP64 also their NN labels
    if (NB == 1 && a.sell32 && (std::is_same<T, float>::value || ctx->rec32_nn))
        e = pick(std::true_type{});
    else
        e = pick(std::false_type{});
    if (e != cudaSuccess) return cuda_check(ctx, e, "applyh smem attribute");
    return cuda_check(ctx, cudaGetLastError(), "applyh kernel launch");
}

// tile width: 32*ITEMS positions, ITEMS the smallest power of two covering the
// median row, capped so that ITEMS*NB accumulators stay in registers
template <typename T, int NB>
static int launch_nb(bsg_ctx *ctx, const T *vin, T *vout, int ld, int v0, int accumulate, cudaStream_t s,
                     TileLookup lk, double *cols = nullptr) {
    // nb = 8 measured fastest at two positions per lane (pf 4p4n: 5.10 ms at
    // one, 4.86 at two, 5.08 at four); single FP64 vectors at four (pf 6p6n:
    // 194.4 ms against 219.5 at eight, pf 4p4n 2.11 against 2.30 ms), single
    // FP32 vectors at eight (pf 6p6n 138.9 against 159.0 ms at four)
    constexpr int cap = NB >= 16 ? 1 : (NB >= 4 ? 2 : (NB == 2 ? 4 : (std::is_same<T, double>::value ? 4 : 8)));
    int items = 1;
    while (items < cap && 32 * items < ctx->median_rowlen) items *= 2;
    if (items >= 8 && cap >= 8) return launch_one<T, NB, (cap >= 8 ? 8 : 1)>(ctx, vin, vout, ld, v0, accumulate, s, lk, cols);
    if (items >= 4 && cap >= 4) return launch_one<T, NB, (cap >= 4 ? 4 : 1)>(ctx, vin, vout, ld, v0, accumulate, s, lk, cols);
    if (items >= 2 && cap >= 2) return launch_one<T, NB, (cap >= 2 ? 2 : 1)>(ctx, vin, vout, ld, v0, accumulate, s, lk, cols);
    return launch_one<T, NB, 1>(ctx, vin, vout, ld, v0, accumulate, s, lk, cols);
}

template <typename T>
static int launch_typed(bsg_ctx *ctx, const T *vin, T *vout, int nb, int accumulate, cudaStream_t s,
                        TileLookup lk) {
    switch (nb) {
    case 1: return launch_nb<T, 1>(ctx, vin, vout, nb, 0, accumulate, s, lk);
    case 2: return launch_nb<T, 2>(ctx, vin, vout, nb, 0, accumulate, s, lk);
    case 4: return launch_nb<T, 4>(ctx, vin, vout, nb, 0, accumulate, s, lk);
    case 8: return launch_nb<T, 8>(ctx, vin, vout, nb, 0, accumulate, s, lk);
    case 16: return launch_nb<T, 16>(ctx, vin, vout, nb, 0, accumulate, s, lk);
    default: {
        // other block sizes: one column pass per vector (strided layout)
        int st = BSG_OK;
        for (int v0 = 0; v0 < nb && st == BSG_OK; ++v0) st = launch_nb<T, 1>(ctx, vin, vout, nb, v0, accumulate, s, lk);
        return st;
    }
    }
}

int launch_applyh_cols(bsg_ctx *ctx, const void *vin, double *cols, int nb, int prec, cudaStream_t s) {
    if (ctx->args.max_nbd > 5120)
        return set_err(ctx, BSG_ERR_UNSUPPORTED, "a neutron sector jump has more than 5120 distinct (b,d) pairs");
    if ((reinterpret_cast<uintptr_t>(vin) & 15u) != 0 || !cols)
        return set_err(ctx, BSG_ERR_ARG, "applyH to columns: misaligned input or no output");
    if (prec == BSG_PREC_FP32) {
        const float *x = (const float *)vin;
        switch (nb) {
        case 1: return launch_nb<float, 1>(ctx, x, nullptr, 1, 0, 0, s, nullptr, cols);
        case 2: return launch_nb<float, 2>(ctx, x, nullptr, 2, 0, 0, s, nullptr, cols);
        case 4: return launch_nb<float, 4>(ctx, x, nullptr, 4, 0, 0, s, nullptr, cols);
        case 8: return launch_nb<float, 8>(ctx, x, nullptr, 8, 0, 0, s, nullptr, cols);
        case 16: return launch_nb<float, 16>(ctx, x, nullptr, 16, 0, 0, s, nullptr, cols);
        }
    } else {
        const double *x = (const double *)vin;
        switch (nb) {
        case 1: return launch_nb<double, 1>(ctx, x, nullptr, 1, 0, 0, s, nullptr, cols);
        case 2: return launch_nb<double, 2>(ctx, x, nullptr, 2, 0, 0, s, nullptr, cols);
        case 4: return launch_nb<double, 4>(ctx, x, nullptr, 4, 0, 0, s, nullptr, cols);
        case 8: return launch_nb<double, 8>(ctx, x, nullptr, 8, 0, 0, s, nullptr, cols);
        case 16: return launch_nb<double, 16>(ctx, x, nullptr, 16, 0, 0, s, nullptr, cols);
        }
    }
    return set_err(ctx, BSG_ERR_ARG, "applyH to columns: nb must be 1, 2, 4, 8 or 16");
}

int launch_applyh(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int accumulate,
                  cudaStream_t s, TileLookup lk) {
    // the 8 per-warp PN tables must fit in shared memory beside the partial
    // sums (227 KB per CTA; 32 KB of partial sums at nb = 16, FP64)
    if (ctx->args.max_nbd > 5120)
        return set_err(ctx, BSG_ERR_UNSUPPORTED, "a neutron sector jump has more than 5120 distinct (b,d) pairs");
    if (prec == BSG_PREC_FP32)
        return launch_typed<float>(ctx, (const float *)vin, (float *)vout, nb, accumulate, s, lk);
    return launch_typed<double>(ctx, (const double *)vin, (double *)vout, nb, accumulate, s, lk);
}

}  // namespace bsg
