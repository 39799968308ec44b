// Launchers of the FP64 Lanczos kernels (lanczos_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bsg {
// largest grid of the dot and update passes (partial buffers are sized by it)
constexpr int kMaxDotGrid = 888;
int dot_grid(int64_t n);
// Operands marked "prec" are history columns stored in FP32 (4) or FP64
// (8); every sum accumulates in FP64.
// out[a*nB + b] = A_a . B_b   (partial: scratch of nA*nB*dot_grid(n) doubles)
// ticket (optional): a device counter at zero, used by one pass at a time on
// the stream; with it the last CTA of a pass with few partials adds them up
// itself instead of a second launch, with the same summation order
cudaError_t multidot(const void *A, int aprec, int nA, const double *B, int nB, int64_t n, int64_t ld,
                     double *partial, double *out, cudaStream_t s, unsigned *ticket = nullptr);
cudaError_t multidot(const double *A, int nA, const double *B, int nB, int64_t n, int64_t ld, double *partial,
                     double *out, cudaStream_t s, unsigned *ticket = nullptr);
// W_b -= sum_j H_j C[j*nB+b]; optional column sums of squares of the result
// (sq_partial: nB*888 doubles, sq_out: nB doubles; ticket as for multidot)
cudaError_t sub_gemv(const void *H, int hprec, int k, const double *C, double *W, int nB, int64_t n, int64_t ld,
                     double *sq_partial, double *sq_out, cudaStream_t s, unsigned *ticket = nullptr);
cudaError_t sub_gemv(const double *H, int k, const double *C, double *W, int nB, int64_t n, int64_t ld,
                     double *sq_partial, double *sq_out, cudaStream_t s, unsigned *ticket = nullptr);
// out_l = sum_j V_j Y[j*ldy + l], l < K
// xpack (optional, K <= 16): the result also as the interleaved applyH input
// (FP32 for xprec 4, FP64 for 8), as pack() would make it
cudaError_t transform(const void *V, int vprec, int m, const double *Y, int ldy, int K, void *out, int oprec,
                      int64_t n, int64_t ld, int64_t ldo, cudaStream_t s, void *xpack = nullptr, int xprec = 8);
cudaError_t transform(const double *V, int m, const double *Y, int ldy, int K, double *out, int64_t n, int64_t ld,
                      int64_t ldo, cudaStream_t s, void *xpack = nullptr, int xprec = 8);
cudaError_t scale_cols(const double *x, void *y, int yprec, const double *sc, int nB, int64_t n, int64_t ld,
                       cudaStream_t s);
cudaError_t scale_cols(const double *x, double *y, const double *sc, int nB, int64_t n, int64_t ld, cudaStream_t s);
// y = x / sqrt(sq[0]) if sq[0] > 0, else y untouched (sq on the device)
cudaError_t normalize_col(const double *x, void *y, int yprec, const double *sq, int64_t n, cudaStream_t s,
                          void *xpack = nullptr, int xprec = 8);
cudaError_t pack(const void *V, int vprec, int nB, int64_t n, int64_t ld, void *x, int prec, cudaStream_t s);
cudaError_t unpack(const void *y, int nB, int64_t n, int64_t ld, double *W, int prec, cudaStream_t s);
// lowest nwant eigenvalues of the arrowhead-tridiagonal matrix
cudaError_t bisect_arrow(int n, int k, const double *al, const double *bt, int nwant, double glo, double ghi,
                         double *ev, cudaStream_t s);
// eigenvectors (columns of Z, column-major n x nvec) of the arrowhead-
// tridiagonal matrix for the given eigenvalues; work: 6*n*nvec doubles
cudaError_t inverse_iter_arrow(int n, int k, const double *al, const double *bt, const double *ev, int nvec,
                               double scale, double *Z, double *work, cudaStream_t s);
// Householder reduction of a dense symmetric matrix (row-major, destroyed)
// to tridiagonal d/e with reflectors V/tau; work: 2*n doubles
cudaError_t tridiag(int n, double *A, double *d, double *e, double *V, double *tau, double *work, cudaStream_t s);
// Z <- Q Z for the reflectors of tridiag
cudaError_t apply_q(int n, int nvec, const double *V, const double *tau, double *Z, cudaStream_t s);
}  // namespace bsg
