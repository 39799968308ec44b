// FP64 device kernels for the Lanczos loop.
//
//   k_multidot      C = A^T B for a few tall vectors (alpha, Gram-Schmidt
//                   coefficients, block overlaps): dot_product8 /
//                   br_orthogonalize's dot phase (src/breorthog.f90:658-891)
//   k_sub_gemv      W -= H C (the subtract phase of br_orthogonalize and the
//                   alpha projection of br_remove_prev_overlap)
//   k_transform     out = V Y (br_transform_basis, src/breorthog.f90:1211-1243)
//   k_bisect_arrow  lowest eigenvalues of the arrowhead-tridiagonal projected
//                   matrix of scalar Lanczos by Sturm counting (replaces the
//                   DSYEV 'N' / DSTEGR calls made for the convergence test)
//   k_pack/k_unpack history columns <-> interleaved applyH vectors
//
// All reductions are two-pass with a fixed grid and fixed summation order, so
// every coefficient is bitwise repeatable.
//
// History columns are stored in FP64 or, as with the reference's shipped
// lanc_prec = 4 (src/bmodules_main.f90:171), in FP32; every dot product and
// update accumulates in FP64 either way (dot_product8 and the REAL(...,8)
// sums of src/breorthog.f90:658-673, :1055-1116), and the working block W is
// always FP64.

#include <cuda_runtime.h>
#include <algorithm>
#include <stdint.h>

#include "lanczos_kernels.h"

namespace bsg {

constexpr int kDotThreads = 256;
constexpr int kDotTile = 512;      // rows per tile
// partial sums that the last CTA of a pass adds up itself; above this the
// separate k_reduce_partials grid is faster than one CTA
constexpr int64_t kFusedPartials = 32768;

// The CTA that finishes a pass last adds the partials up: out[p] = sum over g
// of partial[p*G + g], p < np, in k_reduce_partials' order (lanes take g =
// lane, lane + 32, ..., then the same shuffle tree), so the fused and the
// separate reduction give the same bits.  Every CTA calls it after writing
// its partials; the ticket counts the CTAs done and is left at zero for the
// next pass on the stream.  No CTA waits on another.
__device__ __forceinline__ void finish_partials(const double *partial, int np, int G, double *out, unsigned *ticket,
                                                unsigned nblocks) {
    __shared__ unsigned s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == nblocks - 1u) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int p = warp; p < np; p += nw) {
        const double *row = partial + (int64_t)p * G;
        double v = 0.0;
        // four loads in flight ahead of the additions, which stay in g order
        for (int g0 = lane; g0 < G; g0 += 128) {
            double x[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) x[u] = (g0 + 32 * u < G) ? __ldcg(row + g0 + 32 * u) : 0.0;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (g0 + 32 * u < G) v += x[u];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) out[p] = v;
    }
    if (threadIdx.x == 0) atomicExch(ticket, 0u);
}

// C[p] partials: pairs p = a*nB + b, a < nA, b < nB; A, B column-major with
// leading dimension ld (vector j at base + j*ld).  CTA (x, y) walks the row
// chunks x, x + gridDim.x, ... and the A vectors of chunk y (short vectors
// spread the A vectors over gridDim.y CTAs).  The chunk of B is staged in
// shared memory, column-major so that lanes read consecutive rows; warp w
// takes its vectors (two at a time for NB >= 4, halving the shared loads per
// multiply-add, and for FP32 columns with NB <= 2, doubling the loads in
// flight) and reads them coalesced, lanes keep NB partial sums per
// vector, and a warp reduction adds them into the CTA's shared accumulator
// (each (a,b) owned by one warp, added in chunk order).  The CTA writes
// partial[p * gridDim.x + x] for its vectors; with a ticket, the last CTA
// also writes out[p] (finish_partials).
template <typename TA, int NB, int PAIR>
__global__ void __launch_bounds__(kDotThreads) k_multidot(const TA *__restrict__ A, int nA,
                                                         const double *__restrict__ B, int64_t n, int64_t ld,
                                                         double *__restrict__ partial, double *__restrict__ out,
                                                         unsigned *__restrict__ ticket) {
    extern __shared__ double sm[];
    double *sB = sm;                       // [NB][kDotTile]
    double *sAcc = sm + kDotTile * NB;     // [nA][NB]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = kDotThreads / 32;
    const int per = (nA + gridDim.y - 1) / gridDim.y;
    const int a_lo = blockIdx.y * per, a_hi = min(nA, a_lo + per);
    for (int e = threadIdx.x; e < nA * NB; e += kDotThreads) sAcc[e] = 0.0;
    for (int64_t t0 = (int64_t)blockIdx.x * kDotTile; t0 < n; t0 += (int64_t)gridDim.x * kDotTile) {
        const int rows = (int)((n - t0) < kDotTile ? (n - t0) : kDotTile);
        __syncthreads();
        for (int e = threadIdx.x; e < rows * NB; e += kDotThreads) {
            const int b = e / rows, r = e - b * rows;
            sB[b * kDotTile + r] = B[(int64_t)b * ld + t0 + r];
        }
        __syncthreads();
        for (int a = a_lo + warp * PAIR; a < a_hi; a += nw * PAIR) {
            const bool two = PAIR == 2 && a + 1 < a_hi;
            const TA *__restrict__ col0 = A + (int64_t)a * ld + t0;
            const TA *__restrict__ col1 = two ? col0 + ld : col0;
            double acc0[NB], acc1[NB];
#pragma unroll
            for (int b = 0; b < NB; ++b) acc0[b] = acc1[b] = 0.0;
            // U rows per lane and step, loads first (the sum stays in row
            // order): eight for one or two FP32 vectors, whose passes are
            // bound by the loads in flight (measured; FP64 history columns
            // ran slower with eight)
            constexpr int U = (NB <= 2 && sizeof(TA) == 4) ? 8 : 4;
            int r = lane;
            for (; r + 32 * (U - 1) < rows; r += 32 * U) {
                double x0[U], x1[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    x0[u] = (double)__ldg(col0 + r + 32 * u);
                    x1[u] = PAIR == 2 ? (double)__ldg(col1 + r + 32 * u) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        const double y = sB[b * kDotTile + r + 32 * u];
                        acc0[b] = fma(x0[u], y, acc0[b]);
                        if (PAIR == 2) acc1[b] = fma(x1[u], y, acc1[b]);
                    }
            }
            for (; r < rows; r += 32) {
                const double x0 = (double)__ldg(col0 + r);
                const double x1 = PAIR == 2 ? (double)__ldg(col1 + r) : 0.0;
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    const double y = sB[b * kDotTile + r];
                    acc0[b] = fma(x0, y, acc0[b]);
                    if (PAIR == 2) acc1[b] = fma(x1, y, acc1[b]);
                }
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                double v = acc0[b];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) sAcc[a * NB + b] += v;
                if (PAIR == 2) {
                    double u = acc1[b];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
                    if (lane == 0 && two) sAcc[(a + 1) * NB + b] += u;
                }
            }
        }
    }
    __syncthreads();
    for (int e = a_lo * NB + threadIdx.x; e < a_hi * NB; e += kDotThreads)
        partial[(int64_t)e * gridDim.x + blockIdx.x] = sAcc[e];
    if (ticket) finish_partials(partial, nA * NB, gridDim.x, out, ticket, gridDim.x * gridDim.y);
}

// out[p] = sum over g of partial[p*G + g]: one warp per p, lanes take g = lane,
// lane+32, ... in order and a fixed shuffle tree combines them
__global__ void k_reduce_partials(const double *__restrict__ partial, int npairs, int G, double *__restrict__ out) {
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= npairs) return;
    double s = 0.0;
    for (int g = lane; g < G; g += 32) s += partial[(int64_t)p * G + g];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[p] = s;
}

// W[b] -= sum_j H[j] * C[j*nB + b]   (j < k), fused sum of squares of the
// result per column when sq != nullptr (partials per block, NB entries; with
// a ticket the last block adds them into sq_out)
template <typename TH, int NB>
__global__ void __launch_bounds__(256) k_sub_gemv(const TH *__restrict__ H, int k, const double *__restrict__ C,
                                                  double *__restrict__ W, int64_t n, int64_t ld,
                                                  double *__restrict__ sq, double *__restrict__ sq_out,
                                                  unsigned *__restrict__ ticket) {
    extern __shared__ double sC[];  // [k*NB] then [8][NB] warp sums
    for (int e = threadIdx.x; e < k * NB; e += blockDim.x) sC[e] = C[e];
    __syncthreads();
    double sqacc[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) sqacc[b] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[b] = 0.0;
        int j = 0;
        if constexpr (NB <= 2 && sizeof(TH) == 4) {
            // eight FP32 history rows loaded ahead of their multiply-adds,
            // which stay in j order: the pass of one or two vectors is bound
            // by the loads in flight (measured faster)
            for (; j + 8 <= k; j += 8) {
                double h[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) h[u] = (double)__ldg(H + (int64_t)(j + u) * ld + i);
#pragma unroll
                for (int u = 0; u < 8; ++u)
#pragma unroll
                    for (int b = 0; b < NB; ++b) acc[b] = fma(h[u], sC[(j + u) * NB + b], acc[b]);
            }
            for (; j < k; ++j) {
                const double h0 = (double)__ldg(H + (int64_t)j * ld + i);
#pragma unroll
                for (int b = 0; b < NB; ++b) acc[b] = fma(h0, sC[j * NB + b], acc[b]);
            }
        } else {
            // two rows per step (more raised the registers of FP64 passes
            // above the 6 CTAs per SM that stream_grid assumes)
            for (; j + 1 < k; j += 2) {
                const double h0 = (double)__ldg(H + (int64_t)j * ld + i),
                             h1 = (double)__ldg(H + (int64_t)(j + 1) * ld + i);
#pragma unroll
                for (int b = 0; b < NB; ++b) acc[b] = fma(h1, sC[(j + 1) * NB + b], fma(h0, sC[j * NB + b], acc[b]));
            }
            if (j < k) {
                const double h0 = (double)__ldg(H + (int64_t)j * ld + i);
#pragma unroll
                for (int b = 0; b < NB; ++b) acc[b] = fma(h0, sC[j * NB + b], acc[b]);
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const double w = W[(int64_t)b * ld + i] - acc[b];
            W[(int64_t)b * ld + i] = w;
            sqacc[b] = fma(w, w, sqacc[b]);
        }
    }
    if (!sq) return;
    double *red = sC + k * NB;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        double v = sqacc[b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp * NB + b] = v;
    }
    __syncthreads();
    if (threadIdx.x < NB) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w * NB + threadIdx.x];
        sq[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
    if (ticket) finish_partials(sq, NB, gridDim.x, sq_out, ticket, gridDim.x);
}

// out[l] = sum_j V[j] * Y[j*ldy + l], l < K (K <= 16 per launch)
// K is a template parameter so that the K accumulators live in registers
// xpack (optional): the result also as the interleaved applyH input of the
// next step (x[i*K + l], FP32 for xprec 4, FP64 for 8), as k_pack would make it
template <int K, typename TV, typename TO>
__global__ void __launch_bounds__(256) k_transform(const TV *__restrict__ V, int m, const double *__restrict__ Y,
                                                   int ldy, TO *__restrict__ out, int64_t n, int64_t ld,
                                                   int64_t ldo, void *__restrict__ xpack, int xprec) {
    extern __shared__ double sY[];  // [m][K]
    for (int e = threadIdx.x; e < m * K; e += blockDim.x) {
        const int j = e / K, l = e - j * K;
        sY[e] = Y[(int64_t)j * ldy + l];
    }
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc[K];
#pragma unroll
        for (int l = 0; l < K; ++l) acc[l] = 0.0;
        int j = 0;
        for (; j + 1 < m; j += 2) {
            const double v0 = (double)__ldg(V + (int64_t)j * ld + i), v1 = (double)__ldg(V + (int64_t)(j + 1) * ld + i);
#pragma unroll
            for (int l = 0; l < K; ++l) acc[l] = fma(v1, sY[(j + 1) * K + l], fma(v0, sY[j * K + l], acc[l]));
        }
        if (j < m) {
            const double v0 = (double)__ldg(V + (int64_t)j * ld + i);
#pragma unroll
            for (int l = 0; l < K; ++l) acc[l] = fma(v0, sY[j * K + l], acc[l]);
        }
#pragma unroll
        for (int l = 0; l < K; ++l) out[(int64_t)l * ldo + i] = (TO)acc[l];
        if (xpack) {
            if (xprec == 4) {
#pragma unroll
                for (int l = 0; l < K; ++l) static_cast<float *>(xpack)[i * K + l] = (float)acc[l];
            } else {
#pragma unroll
                for (int l = 0; l < K; ++l) static_cast<double *>(xpack)[i * K + l] = acc[l];
            }
        }
    }
}

// y[b] = s[b] * x[b] (scale columns), x and y may alias
template <typename TO>
__global__ void k_scale_cols(const double *x, TO *y, const double *__restrict__ s, int nB, int64_t n, int64_t ld) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int b = 0; b < nB; ++b) y[(int64_t)b * ld + i] = (TO)(x[(int64_t)b * ld + i] * s[b]);
}

// y = x / sqrt(sq[0]) when sq[0] > 0 (nothing written otherwise): the
// scalar normalization of the residual, with the norm left on the device
// (xpack as for k_transform)
template <typename TO>
__global__ void k_normalize_col(const double *__restrict__ x, TO *__restrict__ y, const double *__restrict__ sq,
                                int64_t n, void *__restrict__ xpack, int xprec) {
    const double q = sq[0];
    if (!(q > 0.0)) return;
    const double inv = 1.0 / sqrt(q);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = x[i] * inv;
        y[i] = (TO)v;
        if (xpack) {
            if (xprec == 4)
                static_cast<float *>(xpack)[i] = (float)v;
            else
                static_cast<double *>(xpack)[i] = v;
        }
    }
}

// interleaved applyH vector from nB history columns (TV -> T)
template <typename TV, typename T>
__global__ void k_pack(const TV *__restrict__ V, int nB, int64_t n, int64_t ld, T *__restrict__ x) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * nB; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = e / nB;
        const int b = (int)(e - s * nB);
        x[e] = (T)V[(int64_t)b * ld + s];
    }
}
template <typename T>
__global__ void k_unpack(const T *__restrict__ y, int nB, int64_t n, int64_t ld, double *__restrict__ W) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * nB; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = e / nB;
        const int b = (int)(e - s * nB);
        W[(int64_t)b * ld + s] = (double)y[e];
    }
}

// ---------------------------------------------------------- bisection ----
// number of eigenvalues below x of the symmetric arrowhead-tridiagonal T:
// T(i,i) = al[i]; T(i,k) = bt[i] for i < k (arrow, k = nthick);
// T(i,i+1) = bt[i] for k <= i < n-1.  Sylvester inertia of LDL^T(T - xI)
// eliminating the arrow diagonal first.
__device__ int sturm_count(int n, int k, const double *__restrict__ al, const double *__restrict__ bt,
                           double x, double pivmin) {
    int cnt = 0;
    double schur = 0.0;
    for (int i = 0; i < k; ++i) {
        double d = al[i] - x;
        if (fabs(d) < pivmin) d = -pivmin;
        if (d < 0) ++cnt;
        schur += bt[i] * bt[i] / d;
    }
    double d = al[k] - x - schur;
    if (fabs(d) < pivmin) d = -pivmin;
    if (d < 0) ++cnt;
    for (int i = k + 1; i < n; ++i) {
        const double b = bt[i - 1];
        d = al[i] - x - b * b / d;
        if (fabs(d) < pivmin) d = -pivmin;
        if (d < 0) ++cnt;
    }
    return cnt;
}

// one warp per wanted eigenvalue index j: multisection with 32 shifts a round
__global__ void k_bisect_arrow(int n, int k, const double *__restrict__ al, const double *__restrict__ bt,
                               int nwant, double glo, double ghi, double *__restrict__ ev) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nwant) return;
    const int j = warp;  // find the (j+1)-th smallest eigenvalue
    double lo = glo, hi = ghi;
    const double scale = fmax(fabs(glo), fabs(ghi));
    const double pivmin = fmax(1e-300, 1e-290 * scale * scale);
    for (int round = 0; round < 40; ++round) {
        if (hi - lo <= 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300) break;
        const double x = lo + (hi - lo) * (double)(lane + 1) / 33.0;
        const int c = sturm_count(n, k, al, bt, x, pivmin);
        // lanes whose shift has count <= j lie at or below the eigenvalue
        const unsigned below = __ballot_sync(0xffffffffu, c <= j);
        const int nb = __popc(below);  // shifts 0..nb-1 are below
        const double nlo = (nb == 0) ? lo : lo + (hi - lo) * (double)nb / 33.0;
        const double nhi = (nb == 32) ? hi : lo + (hi - lo) * (double)(nb + 1) / 33.0;
        // an interval a few ulps wide no longer shrinks: every shift rounds
        // onto an end point
        if (nlo == lo && nhi == hi) break;
        lo = nlo;
        hi = nhi;
    }
    if (lane == 0) ev[j] = 0.5 * (lo + hi);
}

// seeded pseudo-random normal columns (SplitMix64 of (seed, column, row) and
// Box-Muller), for block pivots and random restarts
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__global__ void k_random_cols(double *W, int nB, int64_t n, int64_t ld, uint64_t seed) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int b = 0; b < nB; ++b) {
            const uint64_t h = splitmix64(seed ^ splitmix64(((uint64_t)b << 48) ^ (uint64_t)i));
            const uint64_t h2 = splitmix64(h);
            const double u1 = ((double)(h >> 11) + 1.0) * (1.0 / 9007199254740992.0);
            const double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
            W[(int64_t)b * ld + i] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        }
}

// ---------------------------------------------------- inverse iteration ---
// Eigenvectors of the arrowhead-tridiagonal T (see sturm_count) for given
// eigenvalues: one thread per vector, three steps of inverse iteration
// (T - theta) x_{new} = x / |x|.  The arrow rows i < k are eliminated into
// row k (Schur complement), the remaining tridiagonal block is factored by
// Gaussian elimination with partial pivoting (the dgttrf/dgttrs scheme), and
// the arrow unknowns are recovered by back substitution.  Tiny pivots are
// replaced by +-pivmin.  work: 6*n doubles per vector.
__device__ void arrow_solve(int n, int k, const double *__restrict__ al, const double *__restrict__ bt, double th,
                            double pivmin, double *x, double *w) {
    const int m = n - k;
    double *dl = w, *d = w + n, *du = w + 2 * n, *du2 = w + 3 * n, *b = w + 4 * n;
    int *piv = reinterpret_cast<int *>(w + 5 * n);
    // Schur complement of the arrow block into row k
    double sdiag = 0.0, srhs = 0.0;
    for (int i = 0; i < k; ++i) {
        double di = al[i] - th;
        if (fabs(di) < pivmin) di = (di < 0 ? -pivmin : pivmin);
        sdiag += bt[i] * bt[i] / di;
        srhs += bt[i] * x[i] / di;
    }
    for (int i = 0; i < m; ++i) {
        d[i] = al[k + i] - th;
        b[i] = x[k + i];
        if (i + 1 < m) { dl[i] = bt[k + i]; du[i] = bt[k + i]; }
        du2[i] = 0.0;
    }
    d[0] -= sdiag;
    b[0] -= srhs;
    // factor with partial pivoting
    for (int i = 0; i + 1 < m; ++i) {
        if (fabs(d[i]) >= fabs(dl[i])) {
            piv[i] = i;
            if (fabs(d[i]) < pivmin) d[i] = (d[i] < 0 ? -pivmin : pivmin);
            const double f = dl[i] / d[i];
            dl[i] = f;
            d[i + 1] -= f * du[i];
        } else {
            piv[i] = i + 1;
            const double f = d[i] / dl[i];
            d[i] = dl[i];
            dl[i] = f;
            const double t = du[i];
            du[i] = d[i + 1];
            d[i + 1] = t - f * d[i + 1];
            if (i + 2 < m) {
                du2[i] = du[i + 1];
                du[i + 1] = -f * du[i + 1];
            }
        }
    }
    if (fabs(d[m - 1]) < pivmin) d[m - 1] = (d[m - 1] < 0 ? -pivmin : pivmin);
    // forward: L
    for (int i = 0; i + 1 < m; ++i) {
        if (piv[i] == i) {
            b[i + 1] -= dl[i] * b[i];
        } else {
            const double t = b[i];
            b[i] = b[i + 1];
            b[i + 1] = t - dl[i] * b[i + 1];
        }
    }
    // back: U
    b[m - 1] /= d[m - 1];
    if (m > 1) b[m - 2] = (b[m - 2] - du[m - 2] * b[m - 1]) / d[m - 2];
    for (int i = m - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i];
    // arrow unknowns
    const double xk = b[0];
    for (int i = 0; i < k; ++i) {
        double di = al[i] - th;
        if (fabs(di) < pivmin) di = (di < 0 ? -pivmin : pivmin);
        x[i] = (x[i] - bt[i] * xk) / di;
    }
    for (int i = 0; i < m; ++i) x[k + i] = b[i];
}

__global__ void k_inverse_iter_arrow(int n, int k, const double *__restrict__ al, const double *__restrict__ bt,
                                     const double *__restrict__ ev, int nvec, double scale, double *__restrict__ Z,
                                     double *__restrict__ work) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nvec) return;
    double *x = Z + (int64_t)j * n;  // column j (column-major n x nvec)
    double *w = work + (int64_t)j * 6 * n;
    const double pivmin = fmax(1e-300, 2.2e-16 * scale);
    // deterministic start vector with components in every direction
    for (int i = 0; i < n; ++i) x[i] = 1.0 + 0.5 * sin(0.7 * (double)(i + 1) + 1.3 * (double)(j + 1));
    for (int it = 0; it < 3; ++it) {
        double nrm = 0.0;
        for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
        nrm = 1.0 / sqrt(nrm);
        for (int i = 0; i < n; ++i) x[i] *= nrm;
        arrow_solve(n, k, al, bt, ev[j], pivmin, x, w);
    }
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
    nrm = 1.0 / sqrt(nrm);
    for (int i = 0; i < n; ++i) x[i] *= nrm;
}

// modified Gram-Schmidt of the nvec columns of Z (column-major n x nvec), in
// order, in one CTA (keeps nearly degenerate inverse-iteration vectors
// orthogonal)
__global__ void k_mgs(int n, int nvec, double *__restrict__ Z) {
    __shared__ double red[32];
    __shared__ double coef;
    for (int j = 0; j < nvec; ++j) {
        double *zj = Z + (int64_t)j * n;
        for (int i2 = 0; i2 < j; ++i2) {
            const double *zi = Z + (int64_t)i2 * n;
            double s = 0.0;
            for (int r = threadIdx.x; r < n; r += blockDim.x) s += zi[r] * zj[r];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
                coef = t;
            }
            __syncthreads();
            const double c = coef;
            for (int r = threadIdx.x; r < n; r += blockDim.x) zj[r] -= c * zi[r];
            __syncthreads();
        }
        double s = 0.0;
        for (int r = threadIdx.x; r < n; r += blockDim.x) s += zj[r] * zj[r];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
            coef = 1.0 / sqrt(t);
        }
        __syncthreads();
        const double c = coef;
        for (int r = threadIdx.x; r < n; r += blockDim.x) zj[r] *= c;
        __syncthreads();
    }
}

// ------------------------------------------------ Householder tridiagonal --
// In one CTA: A (n x n row-major, symmetric, lower part used) is reduced to
// tridiagonal form Q^T A Q (the dsytd2 scheme): d[0:n] diagonal, e[0:n-1]
// subdiagonal; reflector j is stored in V[j*n + (j+1 .. n-1)] with tau[j].
// work: 2*n doubles.
__global__ void __launch_bounds__(1024) k_tridiag(int n, double *__restrict__ A, double *__restrict__ d,
                                                  double *__restrict__ e, double *__restrict__ V,
                                                  double *__restrict__ tau, double *__restrict__ work) {
    __shared__ double red[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    double *p = work, *v = work + n;
    auto block_sum = [&](double x) -> double {
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        __syncthreads();
        if ((tid & 31) == 0) red[tid >> 5] = x;
        __syncthreads();
        double t = 0.0;
        for (int w = 0; w < (nt + 31) / 32; ++w) t += red[w];
        return t;
    };
    for (int j = 0; j + 2 < n; ++j) {
        const int m = n - j - 1;  // length of the column below the diagonal
        // x = A[j+1:, j]
        double ss = 0.0;
        for (int i = tid; i < m; i += nt) {
            const double xi = A[(j + 1 + i) * n + j];
            ss += (i > 0) ? xi * xi : 0.0;
        }
        const double sigma = block_sum(ss);  // sum of squares without x0
        const double x0 = A[(j + 1) * n + j];
        double alpha, t_;
        if (sigma == 0.0) {
            t_ = 0.0;
            alpha = x0;
        } else {
            const double nrm = sqrt(x0 * x0 + sigma);
            alpha = (x0 <= 0.0) ? nrm : -nrm;
            const double v0 = x0 - alpha;
            t_ = -v0 / alpha;             // tau = (alpha - x0)/alpha
            for (int i = tid; i < m; i += nt) v[i] = (i == 0) ? 1.0 : A[(j + 1 + i) * n + j] / v0;
        }
        if (tid == 0) {
            d[j] = A[j * n + j];
            e[j] = alpha;
            tau[j] = t_;
        }
        __syncthreads();
        if (t_ == 0.0) {
            for (int i = tid; i < m; i += nt) V[(int64_t)j * n + j + 1 + i] = (i == 0) ? 1.0 : 0.0;
            __syncthreads();
            continue;
        }
        for (int i = tid; i < m; i += nt) V[(int64_t)j * n + j + 1 + i] = v[i];
        // p = tau * A22 v: one warp per row, coalesced over the row
        {
            const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
            for (int r = warp; r < m; r += nw) {
                const double *row = A + (int64_t)(j + 1 + r) * n + (j + 1);
                double s2 = 0.0;
                for (int c = lane; c < m; c += 32) s2 += row[c] * v[c];
                for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                if (lane == 0) p[r] = t_ * s2;
            }
        }
        __syncthreads();
        double pv = 0.0;
        for (int i = tid; i < m; i += nt) pv += p[i] * v[i];
        const double K = 0.5 * t_ * block_sum(pv);
        // w = p - K v ; A22 -= v w^T + w v^T
        for (int i = tid; i < m; i += nt) p[i] -= K * v[i];
        __syncthreads();
        for (int e2 = tid; e2 < m * m; e2 += nt) {
            const int r = e2 / m, c = e2 - r * m;
            A[(j + 1 + r) * n + (j + 1 + c)] -= v[r] * p[c] + p[r] * v[c];
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            d[n - 2] = A[(n - 2) * n + (n - 2)];
            e[n - 2] = A[(n - 1) * n + (n - 2)];
        }
        d[n - 1] = A[(n - 1) * n + (n - 1)];
    }
}

// Z (n x nvec column-major) <- Q Z with Q = H_0 H_1 ... H_{n-3}
__global__ void k_apply_q(int n, int nvec, const double *__restrict__ V, const double *__restrict__ tau,
                          double *__restrict__ Z) {
    const int col = blockIdx.x;
    if (col >= nvec) return;
    double *z = Z + (int64_t)col * n;
    __shared__ double red[32];
    __shared__ double coef;
    for (int j = n - 3; j >= 0; --j) {
        const double t_ = tau[j];
        if (t_ == 0.0) continue;
        const double *v = V + (int64_t)j * n + j + 1;
        const int m = n - j - 1;
        double s = 0.0;
        for (int i = threadIdx.x; i < m; i += blockDim.x) s += v[i] * z[j + 1 + i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
            coef = t_ * t;
        }
        __syncthreads();
        const double c = coef;
        for (int i = threadIdx.x; i < m; i += blockDim.x) z[j + 1 + i] -= c * v[i];
        __syncthreads();
    }
}

// ------------------------------------------------------------- launchers --
cudaError_t random_cols(double *W, int nB, int64_t n, int64_t ld, uint64_t seed, cudaStream_t s) {
    k_random_cols<<<592, 256, 0, s>>>(W, nB, n, ld, seed);
    return cudaGetLastError();
}

int dot_grid(int64_t n) {
    int64_t tiles = (n + kDotTile - 1) / kDotTile;
    return (int)(tiles < kMaxDotGrid ? (tiles > 0 ? tiles : 1) : kMaxDotGrid);
}

// CTAs of the streaming passes: single vectors at 40 registers fit 6 CTAs of
// 256 per SM, and on long vectors (at least 592 row tiles) the extra loads in
// flight were measured faster (pf 4p4n); blocks of vectors stay at 4 per SM
template <int NB>
static int stream_grid(int64_t n) {
    return (NB == 1 && n >= (int64_t)592 * kDotTile) ? kMaxDotGrid : 592;
}

template <typename TA, int NB>
static cudaError_t multidot_nb(const TA *A, int nA, const double *B, int64_t n, int64_t ld, double *partial,
                               double *out, cudaStream_t s, unsigned *ticket) {
    const int64_t tiles = (n + kDotTile - 1) / kDotTile;
    const int G = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, stream_grid<NB>(n)));
    const int maxa = 4096 / NB;  // shared accumulator of at most 4096 doubles
    for (int a0 = 0; a0 < nA;) {
        const int na = (nA - a0) < maxa ? (nA - a0) : maxa;
        // short vectors (fewer row chunks than 4 CTAs per SM): spread the A
        // vectors over more CTAs, at least 8 vectors each
        const int gy = std::max(1, std::min((592 + G - 1) / G, na / 8));
        const size_t smem = sizeof(double) * ((size_t)kDotTile * NB + (size_t)na * NB);
        // few partials: the last CTA reduces them, no second launch
        unsigned *tk = (ticket && (int64_t)na * NB * G <= kFusedPartials) ? ticket : nullptr;
        double *o = out + (int64_t)a0 * NB;
        // two A vectors per warp pass halve the shared loads per multiply-add
        // for NB >= 4 and double the loads in flight for NB <= 2, once there
        // are enough vectors to keep all 8 warps of each CTA busy
        if ((NB >= 4 && na >= 16) || (NB <= 2 && sizeof(TA) == 4 && na >= 16 * gy)) {
            cudaFuncSetAttribute(k_multidot<TA, NB, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_multidot<TA, NB, 2><<<dim3(G, gy), kDotThreads, smem, s>>>(A + (int64_t)a0 * ld, na, B, n, ld, partial,
                                                                         o, tk);
        } else {
            cudaFuncSetAttribute(k_multidot<TA, NB, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_multidot<TA, NB, 1><<<dim3(G, gy), kDotThreads, smem, s>>>(A + (int64_t)a0 * ld, na, B, n, ld, partial,
                                                                         o, tk);
        }
        if (!tk) k_reduce_partials<<<(na * NB * 32 + 255) / 256, 256, 0, s>>>(partial, na * NB, G, o);
        a0 += na;
    }
    return cudaGetLastError();
}

template <typename TA>
static cudaError_t multidot_t(const TA *A, int nA, const double *B, int nB, int64_t n, int64_t ld, double *partial,
                              double *out, cudaStream_t s, unsigned *ticket) {
    if (nA <= 0 || nB <= 0) return cudaSuccess;
    switch (nB) {
    case 1: return multidot_nb<TA, 1>(A, nA, B, n, ld, partial, out, s, ticket);
    case 2: return multidot_nb<TA, 2>(A, nA, B, n, ld, partial, out, s, ticket);
    case 4: return multidot_nb<TA, 4>(A, nA, B, n, ld, partial, out, s, ticket);
    case 8: return multidot_nb<TA, 8>(A, nA, B, n, ld, partial, out, s, ticket);
    case 16: return multidot_nb<TA, 16>(A, nA, B, n, ld, partial, out, s, ticket);
    default:
        return cudaErrorInvalidValue;
    }
}

cudaError_t multidot(const void *A, int aprec, int nA, const double *B, int nB, int64_t n, int64_t ld,
                     double *partial, double *out, cudaStream_t s, unsigned *ticket) {
    if (aprec == 4) return multidot_t<float>((const float *)A, nA, B, nB, n, ld, partial, out, s, ticket);
    return multidot_t<double>((const double *)A, nA, B, nB, n, ld, partial, out, s, ticket);
}

cudaError_t multidot(const double *A, int nA, const double *B, int nB, int64_t n, int64_t ld, double *partial,
                     double *out, cudaStream_t s, unsigned *ticket) {
    return multidot_t<double>(A, nA, B, nB, n, ld, partial, out, s, ticket);
}

template <typename TH, int NB>
static cudaError_t sub_gemv_nb(const TH *H, int k, const double *C, double *W, int64_t n, int64_t ld,
                               double *sq_partial, double *sq_out, cudaStream_t s, unsigned *ticket) {
    const int G = stream_grid<NB>(n);
    // the sums of squares: the last block of the last pass adds them up when
    // there is a ticket, else a separate reduction
    unsigned *tk = (sq_partial && sq_out) ? ticket : nullptr;
    int j0 = 0;
    do {
        const int kk = (k - j0) < 512 ? (k - j0) : 512;
        const bool last = (j0 + kk >= k);
        const size_t smem = sizeof(double) * ((size_t)kk * NB + 8 * NB);
        cudaFuncSetAttribute(k_sub_gemv<TH, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(smem + 256));
        k_sub_gemv<TH, NB><<<G, 256, smem, s>>>(H + (int64_t)j0 * ld, kk, C + (int64_t)j0 * NB, W, n, ld,
                                                 last ? sq_partial : nullptr, sq_out, last ? tk : nullptr);
        j0 += kk;
    } while (j0 < k);
    if (sq_partial && sq_out && !tk)
        k_reduce_partials<<<(NB * 32 + 255) / 256, 256, 0, s>>>(sq_partial, NB, G, sq_out);
    return cudaGetLastError();
}

template <typename TH>
static cudaError_t sub_gemv_t(const TH *H, int k, const double *C, double *W, int nB, int64_t n, int64_t ld,
                              double *sq_partial, double *sq_out, cudaStream_t s, unsigned *ticket) {
    switch (nB) {
    case 1: return sub_gemv_nb<TH, 1>(H, k, C, W, n, ld, sq_partial, sq_out, s, ticket);
    case 2: return sub_gemv_nb<TH, 2>(H, k, C, W, n, ld, sq_partial, sq_out, s, ticket);
    case 4: return sub_gemv_nb<TH, 4>(H, k, C, W, n, ld, sq_partial, sq_out, s, ticket);
    case 8: return sub_gemv_nb<TH, 8>(H, k, C, W, n, ld, sq_partial, sq_out, s, ticket);
    case 16: return sub_gemv_nb<TH, 16>(H, k, C, W, n, ld, sq_partial, sq_out, s, ticket);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t sub_gemv(const void *H, int hprec, int k, const double *C, double *W, int nB, int64_t n, int64_t ld,
                     double *sq_partial, double *sq_out, cudaStream_t s, unsigned *ticket) {
    if (hprec == 4) return sub_gemv_t<float>((const float *)H, k, C, W, nB, n, ld, sq_partial, sq_out, s, ticket);
    return sub_gemv_t<double>((const double *)H, k, C, W, nB, n, ld, sq_partial, sq_out, s, ticket);
}

cudaError_t sub_gemv(const double *H, int k, const double *C, double *W, int nB, int64_t n, int64_t ld,
                     double *sq_partial, double *sq_out, cudaStream_t s, unsigned *ticket) {
    return sub_gemv_t<double>(H, k, C, W, nB, n, ld, sq_partial, sq_out, s, ticket);
}

template <typename TV, typename TO>
static cudaError_t transform_t(const TV *V, int m, const double *Y, int ldy, int K, TO *out, int64_t n, int64_t ld,
                               int64_t ldo, cudaStream_t s, void *xpack, int xprec) {
    if (xpack && K > 16) return cudaErrorInvalidValue;  // the packed copy needs one pass
    for (int l0 = 0; l0 < K; l0 += 16) {
        const int kk = (K - l0) < 16 ? (K - l0) : 16;
        // Y rows in chunks that fit shared memory: accumulate over row chunks
        if ((size_t)m * kk * sizeof(double) > 160 * 1024) return cudaErrorInvalidValue;
        const size_t smem = sizeof(double) * (size_t)m * kk;
        cudaError_t e = cudaSuccess;
        switch (kk) {
#define BSG_TRANSFORM_CASE(KT)                                                                              \
    case KT:                                                                                                \
        e = cudaFuncSetAttribute(k_transform<KT, TV, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                                 160 * 1024);                                                               \
        if (e == cudaSuccess)                                                                               \
            k_transform<KT, TV, TO><<<592, 256, smem, s>>>(V, m, Y + l0, ldy, out + (int64_t)l0 * ldo, n, ld, \
                                                            ldo, xpack, xprec);                             \
        break;
            BSG_TRANSFORM_CASE(1) BSG_TRANSFORM_CASE(2) BSG_TRANSFORM_CASE(3) BSG_TRANSFORM_CASE(4)
            BSG_TRANSFORM_CASE(5) BSG_TRANSFORM_CASE(6) BSG_TRANSFORM_CASE(7) BSG_TRANSFORM_CASE(8)
            BSG_TRANSFORM_CASE(9) BSG_TRANSFORM_CASE(10) BSG_TRANSFORM_CASE(11) BSG_TRANSFORM_CASE(12)
            BSG_TRANSFORM_CASE(13) BSG_TRANSFORM_CASE(14) BSG_TRANSFORM_CASE(15) BSG_TRANSFORM_CASE(16)
#undef BSG_TRANSFORM_CASE
        }
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t transform(const void *V, int vprec, int m, const double *Y, int ldy, int K, void *out, int oprec,
                      int64_t n, int64_t ld, int64_t ldo, cudaStream_t s, void *xpack, int xprec) {
    if (vprec == 4 && oprec == 4)
        return transform_t<float, float>((const float *)V, m, Y, ldy, K, (float *)out, n, ld, ldo, s, xpack, xprec);
    if (vprec == 4)
        return transform_t<float, double>((const float *)V, m, Y, ldy, K, (double *)out, n, ld, ldo, s, xpack, xprec);
    if (oprec == 4)
        return transform_t<double, float>((const double *)V, m, Y, ldy, K, (float *)out, n, ld, ldo, s, xpack, xprec);
    return transform_t<double, double>((const double *)V, m, Y, ldy, K, (double *)out, n, ld, ldo, s, xpack, xprec);
}

cudaError_t transform(const double *V, int m, const double *Y, int ldy, int K, double *out, int64_t n, int64_t ld,
                      int64_t ldo, cudaStream_t s, void *xpack, int xprec) {
    return transform_t<double, double>(V, m, Y, ldy, K, out, n, ld, ldo, s, xpack, xprec);
}

cudaError_t scale_cols(const double *x, void *y, int yprec, const double *sc, int nB, int64_t n, int64_t ld,
                       cudaStream_t s) {
    if (yprec == 4)
        k_scale_cols<float><<<592, 256, 0, s>>>(x, (float *)y, sc, nB, n, ld);
    else
        k_scale_cols<double><<<592, 256, 0, s>>>(x, (double *)y, sc, nB, n, ld);
    return cudaGetLastError();
}

cudaError_t scale_cols(const double *x, double *y, const double *sc, int nB, int64_t n, int64_t ld, cudaStream_t s) {
    return scale_cols(x, y, 8, sc, nB, n, ld, s);
}

cudaError_t normalize_col(const double *x, void *y, int yprec, const double *sq, int64_t n, cudaStream_t s,
                          void *xpack, int xprec) {
    if (yprec == 4)
        k_normalize_col<float><<<592, 256, 0, s>>>(x, (float *)y, sq, n, xpack, xprec);
    else
        k_normalize_col<double><<<592, 256, 0, s>>>(x, (double *)y, sq, n, xpack, xprec);
    return cudaGetLastError();
}

cudaError_t pack(const void *V, int vprec, int nB, int64_t n, int64_t ld, void *x, int prec, cudaStream_t s) {
    if (vprec == 4) {
        if (prec == 4)
            k_pack<float, float><<<1184, 256, 0, s>>>((const float *)V, nB, n, ld, (float *)x);
        else
            k_pack<float, double><<<1184, 256, 0, s>>>((const float *)V, nB, n, ld, (double *)x);
    } else {
        if (prec == 4)
            k_pack<double, float><<<1184, 256, 0, s>>>((const double *)V, nB, n, ld, (float *)x);
        else
            k_pack<double, double><<<1184, 256, 0, s>>>((const double *)V, nB, n, ld, (double *)x);
    }
    return cudaGetLastError();
}

cudaError_t unpack(const void *y, int nB, int64_t n, int64_t ld, double *W, int prec, cudaStream_t s) {
    if (prec == 4)
        k_unpack<float><<<1184, 256, 0, s>>>((const float *)y, nB, n, ld, W);
    else
        k_unpack<double><<<1184, 256, 0, s>>>((const double *)y, nB, n, ld, W);
    return cudaGetLastError();
}

cudaError_t inverse_iter_arrow(int n, int k, const double *al, const double *bt, const double *ev, int nvec,
                               double scale, double *Z, double *work, cudaStream_t s) {
    if (nvec <= 0) return cudaSuccess;
    k_inverse_iter_arrow<<<(nvec + 31) / 32, 32, 0, s>>>(n, k, al, bt, ev, nvec, scale, Z, work);
    k_mgs<<<1, 256, 0, s>>>(n, nvec, Z);
    return cudaGetLastError();
}

cudaError_t tridiag(int n, double *A, double *d, double *e, double *V, double *tau, double *work, cudaStream_t s) {
    k_tridiag<<<1, 1024, 0, s>>>(n, A, d, e, V, tau, work);
    return cudaGetLastError();
}

cudaError_t apply_q(int n, int nvec, const double *V, const double *tau, double *Z, cudaStream_t s) {
    if (n < 3 || nvec <= 0) return cudaSuccess;
    k_apply_q<<<nvec, 256, 0, s>>>(n, nvec, V, tau, Z);
    return cudaGetLastError();
}

cudaError_t bisect_arrow(int n, int k, const double *al, const double *bt, int nwant, double glo, double ghi,
                         double *ev, cudaStream_t s) {
    if (nwant <= 0) return cudaSuccess;
    const int threads = 32 * nwant;
    k_bisect_arrow<<<(threads + 255) / 256, 256, 0, s>>>(n, k, al, bt, nwant, glo, ghi, ev);
    return cudaGetLastError();
}

}  // namespace bsg
