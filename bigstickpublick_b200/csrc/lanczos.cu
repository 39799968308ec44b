// bsg_lanczos: scalar and block Lanczos with full reorthogonalization and
// thick restart, everything on the device: the applyH call in FP32 or FP64,
// the Lanczos vectors stored in FP64 or FP32 (lanc_prec, as the reference's
// shipped lanc_prec = 4 stores them), every dot product, update, alpha,
// beta and the projected eigenproblem in FP64.
//
// Restates lanczos_p (src/blanczosmain.f90:1413-1793) and lanczos_block
// (:1804-2153):
//   * pivot: uniform 1/sqrt(dim) (initialize_lanczos_vector option 0,
//     src/blanczoslib.f90:825-831); block pivots are seeded pseudo-random
//     columns (the reference uses the compiler's random_number,
//     src/bblock_algebra.f90:107-113, which is not reproducible);
//   * each step: W = H V_i; alpha = V_i^T W; W -= V_i alpha
//     (br_remove_prev_overlap / grab_alpha_blockv2); one classical
//     Gram-Schmidt pass against every earlier history vector
//     (br_orthogonalize(1) / compute_W); scalar: beta = |W|, V_{i+1} = W/beta
//     (br_normalize); block: S = W^T W = U L U^T (nb x nb, decomposed on
//     the host like the reference's DSYEV), beta = L^1/2 U^T,
//     V_{i+1} = W U L^-1/2 (spectral_decomp, src/bblock_algebra.f90:684-856);
//   * beta collapse (beta < 1e-4 beta_prev) -> random restart against the
//     history (random_restart_with_history, src/breorthog.f90:1471-1482);
//     beta < 0.1 beta_prev -> second full Gram-Schmidt pass
//     (src/blanczosmain.f90:1634-1660);
//   * projected matrix: tridiagonal / band plus the arrow left by thick
//     restart (src/blanczoslib.f90:195-221); its lowest eigenvalues for the
//     convergence test come from Sturm bisection on the device, after a
//     Householder reduction of the band for the block recursion;
//   * convergence_test option 0 (src/blanczoslib.f90:2660-2800): mean energy
//     change over ncheck states, scaled by (1+restarts)/sqrt(ncheck+1),
//     below converge_tol;
//   * thick restart when the next step would be the niter-th.  Scalar
//     (thick_restart_sub_p, src/blanczoslib.f90:1656-1894): Ritz pairs of the
//     projected matrix without its last column, alpha_i = theta_i, coupling
//     beta_prev * y_last,i, basis V <- V Y (br_transform_basis), the last
//     Lanczos vector continues the recursion.  Block
//     (block_thick_restart_sub_p, :1923-2170): Ritz pairs of the whole
//     projected matrix, floor(nthick/nb)*nb of them kept, coupling
//     beta_last * Y[last block rows, kept], and the block made for the next
//     step continues.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bsg_internal.h"
#include "lanczos_kernels.h"

using namespace bsg;

namespace bsg {
cudaError_t random_cols(double *W, int nB, int64_t n, int64_t ld, uint64_t seed, cudaStream_t s);
}

namespace {

struct Lz {
    bsg_ctx *ctx;
    cudaStream_t s;
    int64_t n;
    int nb, prec;
    int hprec = 8;   // history storage: 8 FP64, 4 FP32 (lanc_prec)
    int maxcol;      // history columns
    DevBuf hist, W, X, tmp, partial, coef, sqp, sq, Adev, Vtmp, Zdev, wdev, al, bt, ev, M, tau, ework;
    DevBuf ticket;   // zeroed counter of the dot / update passes (their last CTA reduces)
    // scalar recursion: the next step's applyH is queued before the host has
    // read this step's alpha and beta, into W2; W and W2 swap when it is used
    DevBuf W2;
    cudaEvent_t es0[2] = {nullptr, nullptr}, es1[2] = {nullptr, nullptr}, eb = nullptr;
    unsigned *tk() { return (unsigned *)ticket.p; }
    DevBuf Ydev;     // Ritz coefficients of a thick restart (maxcol x 128)
    std::vector<double> T;  // host projected matrix (maxcol x maxcol), row-major
    float t_mv = 0, t_ort = 0, t_eig = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr, e4 = nullptr;
    // pinned staging for the per-step scalars read on the host (alpha block,
    // residual sums of squares): device->host copies into it stay
    // asynchronous, so a step synchronizes with the device once
    double *hpin = nullptr;
    // X already holds the next step's block, written by the kernel that made
    // it (the normalization or the block transform), so the step needs no pack
    bool x_ready = false;
    // alpha block, residual norms, W^T W and the block coefficients (nb <= 16
    // each), then the convergence test's eigenvalues, diagonal and arrow
    static constexpr int kPinAlpha = 0, kPinSq = 256, kPinS = 272, kPinM = 528, kPinW = 784;
    double *pin_w() { return hpin + kPinW; }
    double *pin_al() { return hpin + kPinW + maxcol; }
    double *pin_bt() { return hpin + kPinW + 2 * (size_t)maxcol; }
    size_t pin_doubles() const { return kPinW + 3 * (size_t)maxcol; }
    // side stream (highest priority) for the convergence test, which then
    // overlaps the next step's applyH
    cudaStream_t s2 = nullptr;
    cudaEvent_t econv = nullptr;
    DevBuf al2, bt2, w2;
    // block recursion: dense projected matrix (pinned), Householder work
    double *pinA = nullptr;
    DevBuf Adev2, Vtmp2, tau2, ework2;

    // history column j (FP32 or FP64 storage, hprec)
    void *col(int j) { return (char *)hist.p + (size_t)j * (size_t)n * (size_t)hprec; }
    double &Tm(int i, int j) { return T[(size_t)i * maxcol + j]; }
};

#define CK(expr)                                              \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return cuda_check(L.ctx, _e, #expr); \
    } while (0)
#define ST(expr)                 \
    do {                         \
        int _s = (expr);         \
        if (_s != BSG_OK) return _s; \
    } while (0)

float elapsed(Lz &L) {
    float ms = 0.f;
    cudaEventSynchronize(L.e1);
    cudaEventElapsedTime(&ms, L.e0, L.e1);
    return ms;
}

// Lowest `want` eigenpairs of the projected matrix T[0:m,0:m] on the device.
// Scalar Lanczos: T is arrowhead-tridiagonal (arrow of size k) -> Sturm
// bisection + inverse iteration.  Block Lanczos: T is dense (band + arrow) ->
// Householder tridiagonalization first, then the same, then the reflectors.
// w (host) gets the eigenvalues; Z (host, column-major m x want) the vectors.
// Gershgorin interval of T[0:m,0:m], padded; scale = max |end point|
void gershgorin(Lz &L, int m, double &glo, double &ghi, double &scale) {
    glo = 1e300;
    ghi = -1e300;
    for (int i = 0; i < m; ++i) {
        double r = 0.0;
        for (int j = 0; j < m; ++j)
            if (j != i) r += std::fabs(L.Tm(i, j));
        glo = std::min(glo, L.Tm(i, i) - r);
        ghi = std::max(ghi, L.Tm(i, i) + r);
    }
    scale = std::max(std::fabs(glo), std::fabs(ghi));
    const double pad = 1e-12 * scale + 1e-300;
    glo -= pad;
    ghi += pad;
}

// diagonal al[0:m] and arrow/sub-diagonal bt[0:m] of the scalar projected matrix
void arrow_inputs(Lz &L, int m, int k, double *al, double *bt) {
    for (int i = 0; i < m; ++i) al[i] = L.Tm(i, i);
    for (int i = 0; i < m; ++i) bt[i] = 0.0;
    for (int i = 0; i < k; ++i) bt[i] = L.Tm(k, i);
    for (int i = k; i + 1 < m; ++i) bt[i] = L.Tm(i + 1, i);
}

int eig_lowest(Lz &L, int m, int k, int want, std::vector<double> &w, std::vector<double> *Z) {
    want = std::min(want, m);
    double glo, ghi, scale;
    gershgorin(L, m, glo, ghi, scale);
    cudaEventRecord(L.e0, L.s);
    int kk = k;
    if (L.nb == 1) {
        std::vector<double> al(m), bt(std::max(m, 1), 0.0);
        arrow_inputs(L, m, k, al.data(), bt.data());
        CK(cudaMemcpyAsync(L.al.p, al.data(), sizeof(double) * m, cudaMemcpyHostToDevice, L.s));
        CK(cudaMemcpyAsync(L.bt.p, bt.data(), sizeof(double) * m, cudaMemcpyHostToDevice, L.s));
    } else {
        std::vector<double> A((size_t)m * m);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) A[(size_t)i * m + j] = 0.5 * (L.Tm(i, j) + L.Tm(j, i));
        CK(cudaMemcpyAsync(L.Adev.p, A.data(), sizeof(double) * m * m, cudaMemcpyHostToDevice, L.s));
        CK(tridiag(m, (double *)L.Adev.p, (double *)L.al.p, (double *)L.bt.p, (double *)L.Vtmp.p, (double *)L.tau.p,
                   (double *)L.ework.p, L.s));
        kk = 0;
    }
    CK(bisect_arrow(m, kk, (const double *)L.al.p, (const double *)L.bt.p, want, glo, ghi, (double *)L.wdev.p, L.s));
    w.resize(want);
    CK(cudaMemcpyAsync(w.data(), L.wdev.p, sizeof(double) * want, cudaMemcpyDeviceToHost, L.s));
    if (Z) {
        CK(inverse_iter_arrow(m, kk, (const double *)L.al.p, (const double *)L.bt.p, (const double *)L.wdev.p, want,
                              scale, (double *)L.Zdev.p, (double *)L.ework.p + 2 * (size_t)m, L.s));
        if (L.nb > 1) CK(apply_q(m, want, (const double *)L.Vtmp.p, (const double *)L.tau.p, (double *)L.Zdev.p, L.s));
        Z->resize((size_t)m * want);
        CK(cudaMemcpyAsync(Z->data(), L.Zdev.p, sizeof(double) * m * want, cudaMemcpyDeviceToHost, L.s));
    }
    cudaEventRecord(L.e1, L.s);
    CK(cudaStreamSynchronize(L.s));
    L.t_eig += elapsed(L);
    return BSG_OK;
}

// Queue the lowest `want` eigenvalues of the scalar projected matrix
// T[0:m,0:m] on the side stream (pinned inputs and result, no host wait);
// eig_collect() waits for them.
int eig_queue(Lz &L, int m, int k, int want) {
    want = std::min(want, m);
    double glo, ghi, scale;
    gershgorin(L, m, glo, ghi, scale);
    int kk = k;
    if (L.nb == 1) {
        arrow_inputs(L, m, k, L.pin_al(), L.pin_bt());
        CK(cudaMemcpyAsync(L.al2.p, L.pin_al(), sizeof(double) * m, cudaMemcpyHostToDevice, L.s2));
        CK(cudaMemcpyAsync(L.bt2.p, L.pin_bt(), sizeof(double) * m, cudaMemcpyHostToDevice, L.s2));
    } else {
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) L.pinA[(size_t)i * m + j] = 0.5 * (L.Tm(i, j) + L.Tm(j, i));
        CK(cudaMemcpyAsync(L.Adev2.p, L.pinA, sizeof(double) * m * m, cudaMemcpyHostToDevice, L.s2));
        CK(tridiag(m, (double *)L.Adev2.p, (double *)L.al2.p, (double *)L.bt2.p, (double *)L.Vtmp2.p,
                   (double *)L.tau2.p, (double *)L.ework2.p, L.s2));
        kk = 0;
    }
    CK(bisect_arrow(m, kk, (const double *)L.al2.p, (const double *)L.bt2.p, want, glo, ghi, (double *)L.w2.p, L.s2));
    CK(cudaMemcpyAsync(L.pin_w(), L.w2.p, sizeof(double) * want, cudaMemcpyDeviceToHost, L.s2));
    CK(cudaEventRecord(L.econv, L.s2));
    return BSG_OK;
}

int eig_collect(Lz &L, int want, std::vector<double> &w) {
    CK(cudaEventSynchronize(L.econv));
    w.assign(L.pin_w(), L.pin_w() + want);
    return BSG_OK;
}

// classical Gram-Schmidt of W (nb columns) against history columns [0, k);
// optional column sums of squares into host sq (synchronizes), or left in
// L.sq on the device (sq_on_device)
int cgs(Lz &L, int k, std::vector<double> *sq, bool sq_on_device = false) {
    double *C = (double *)L.coef.p;
    const bool want_sq = sq || sq_on_device;
    if (k > 0)
        CK(multidot(L.col(0), L.hprec, k, (const double *)L.W.p, L.nb, L.n, L.n, (double *)L.partial.p, C, L.s,
                    L.tk()));
    CK(sub_gemv(L.col(0), L.hprec, k, C, (double *)L.W.p, L.nb, L.n, L.n, want_sq ? (double *)L.sqp.p : nullptr,
                want_sq ? (double *)L.sq.p : nullptr, L.s, L.tk()));
    if (sq) {
        sq->resize(L.nb);
        CK(cudaMemcpyAsync(sq->data(), L.sq.p, sizeof(double) * L.nb, cudaMemcpyDeviceToHost, L.s));
        CK(cudaStreamSynchronize(L.s));
    }
    return BSG_OK;
}

// Eigen-decomposition of a small symmetric matrix (n <= 16, row-major A) by
// cyclic Jacobi rotations (Golub & Van Loan, Matrix Computations, 8.5):
// w ascending, Z row-major with column j the eigenvector of w[j].  The block
// recursion needs it once per step for W^T W; on the host it costs
// microseconds and no round trip to the device.
void host_sym_eig(int n, std::vector<double> A, std::vector<double> &w, std::vector<double> &Z) {
    std::vector<double> V((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < n; ++i) {
            diag += A[(size_t)i * n + i] * A[(size_t)i * n + i];
            for (int j = i + 1; j < n; ++j) off += A[(size_t)i * n + j] * A[(size_t)i * n + j];
        }
        if (off <= 1e-32 * diag || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (apq == 0.0) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < n; ++k) {  // columns p, q
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - sn * akq;
                    A[(size_t)k * n + q] = sn * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p, q
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - sn * aqk;
                    A[(size_t)q * n + k] = sn * apk + c * aqk;
                }
                A[(size_t)p * n + q] = A[(size_t)q * n + p] = 0.0;
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - sn * vkq;
                    V[(size_t)k * n + q] = sn * vkp + c * vkq;
                }
            }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return A[(size_t)x * n + x] < A[(size_t)y * n + y]; });
    w.resize(n);
    Z.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        w[j] = A[(size_t)idx[j] * n + idx[j]];
        for (int k = 0; k < n; ++k) Z[(size_t)k * n + j] = V[(size_t)k * n + idx[j]];
    }
}

// Block step from S = W^T W on the host: S = U L U^T, beta = L^1/2 U^T,
// V_{next} = W U L^-1/2 written to history column `dst`.  The coefficients go
// through pinned memory; nothing waits for the device.
int block_finish(Lz &L, int dst, const double *Shost, std::vector<double> &beta, double &lmin, double &lmax) {
    const int nb = L.nb;
    std::vector<double> A((size_t)nb * nb), w, Z;
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) A[(size_t)i * nb + j] = 0.5 * (Shost[(size_t)i * nb + j] + Shost[(size_t)j * nb + i]);
    host_sym_eig(nb, A, w, Z);
    lmin = w[0];
    lmax = w[nb - 1];
    beta.assign((size_t)nb * nb, 0.0);
    double *Mh = L.hpin + Lz::kPinM;
    for (int a = 0; a < nb; ++a) {
        const double l = std::max(w[a], 0.0);
        const double sl = std::sqrt(l), il = (l > 0.0) ? 1.0 / sl : 0.0;
        for (int c = 0; c < nb; ++c) {
            beta[(size_t)a * nb + c] = sl * Z[(size_t)c * nb + a];  // (L^1/2 U^T)[a][c] = sqrt(l_a) U[c][a]
            Mh[(size_t)c * nb + a] = Z[(size_t)c * nb + a] * il;     // (U L^-1/2)[c][a]
        }
    }
    CK(cudaMemcpyAsync(L.M.p, Mh, sizeof(double) * nb * nb, cudaMemcpyHostToDevice, L.s));
    CK(transform(L.W.p, 8, nb, (const double *)L.M.p, nb, nb, L.col(dst), L.hprec, L.n, L.n, L.n, L.s, L.X.p,
                 L.prec));
    L.x_ready = true;
    return BSG_OK;
}

// V_{next} (nb columns at history column `dst`) from W: scalar normalization
// or the block spectral decomposition; returns the beta block (nb x nb,
// row-major beta[a][c]) and the smallest overlap eigenvalue
int next_block(Lz &L, int dst, const std::vector<double> &sq, std::vector<double> &beta, double &lmin, double &lmax) {
    const int nb = L.nb;
    beta.assign((size_t)nb * nb, 0.0);
    if (nb == 1) {
        const double b = std::sqrt(std::max(sq[0], 0.0));
        beta[0] = b;
        lmin = lmax = sq[0];
        if (b == 0.0) return BSG_OK;
        const double inv = 1.0 / b;
        CK(cudaMemcpyAsync(L.M.p, &inv, sizeof(double), cudaMemcpyHostToDevice, L.s));
        CK(scale_cols((const double *)L.W.p, L.col(dst), L.hprec, (const double *)L.M.p, 1, L.n, L.n, L.s));
        return BSG_OK;
    }
    // S = W^T W, then the decomposition on the host
    CK(multidot((const double *)L.W.p, nb, (const double *)L.W.p, nb, L.n, L.n, (double *)L.partial.p,
                (double *)L.coef.p, L.s, L.tk()));
    CK(cudaMemcpyAsync(L.hpin + Lz::kPinS, L.coef.p, sizeof(double) * nb * nb, cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    return block_finish(L, dst, L.hpin + Lz::kPinS, beta, lmin, lmax);
}

int run(Lz &L, const bsg_lanczos_params *p, const double *pivot, double *evals, double *evecs, bsg_report *rep) {
    bsg_ctx *ctx = L.ctx;
    const int nb = L.nb;
    const int64_t n = L.n;
    const int nkeep = p->nkeep, niter = p->niter;
    const bool thick = (p->nthick_add > 0 || p->max_restarts > 0);
    const int nthick = std::min(nkeep + std::max(p->nthick_add, 0), niter * nb - 2 * nb);
    const int ncheck = std::max(1, p->ncheck > 0 ? p->ncheck : nkeep + 5);
    const double tol = p->converge_tol > 0 ? p->converge_tol : 1e-3;
    L.maxcol = niter * nb + nb;
    L.T.assign((size_t)L.maxcol * L.maxcol, 0.0);

    // ---- pivot block into history columns [0, nb)
    if (pivot) {
        // the interleaved pivot block as given, split into columns on the device
        CK(cudaMemcpyAsync(L.tmp.p, pivot, sizeof(double) * n * nb, cudaMemcpyHostToDevice, L.s));
        CK(unpack(L.tmp.p, nb, n, n, (double *)L.W.p, BSG_PREC_FP64, L.s));
    } else if (nb == 1) {
        std::vector<double> hp(n, 1.0 / std::sqrt((double)n));
        CK(cudaMemcpyAsync(L.W.p, hp.data(), sizeof(double) * n, cudaMemcpyHostToDevice, L.s));
        CK(cudaStreamSynchronize(L.s));
    } else {
        CK(random_cols((double *)L.W.p, nb, n, n, p->seed, L.s));
    }
    std::vector<double> sq, beta;
    double lmin, lmax;
    ST(cgs(L, 0, &sq));
    ST(next_block(L, 0, sq, beta, lmin, lmax));
    if (lmax <= 0.0 || lmin <= 1e-14 * lmax) return set_err(ctx, BSG_ERR_ARG, "pivot block is rank deficient");

    int cur = 0;          // first history column of the current block
    int mT = 0;           // size of the valid projected matrix
    int restarts = 0, rnd = 0, total = 0, matvecs = 0;
    int karrow = 0;       // arrow size of the projected matrix after a thick restart
    double beta_prev = -1.0;
    bool finished = false, converged = false;
    std::vector<double> eold, e;
    bool post_pending = false;  // e3 -> e4 of the last step not yet accounted
    bool spec_ready = false;    // W2 holds H col(cur), queued during the previous step
    int spair = 0;              // event pair of the next speculative applyH
    int iter = 0;         // block iterations in this cycle (the reference's iter)
    struct {
        bool active = false;
        int want = 0, iter = 0, total = 0, rnd = 0, cur = 0, mT = 0;
    } pend;               // convergence test queued on the side stream
    while (!finished) {
        ++iter;
        ++total;
        // ---- W = H V
        cudaEvent_t m0 = L.e0, m1 = L.e1;   // its start and end
        if (spec_ready) {
            // queued by the previous step, whose next vector stood
            std::swap(L.W, L.W2);
            m0 = L.es0[spair ^ 1];
            m1 = L.es1[spair ^ 1];
        } else {
            if (!L.x_ready) CK(pack(L.col(cur), L.hprec, nb, n, n, L.X.p, L.prec, L.s));
            CK(cudaEventRecord(L.e0, L.s));
            ST(launch_applyh_cols(ctx, L.X.p, (double *)L.W.p, nb, L.prec, L.s));  // W columns directly
            CK(cudaEventRecord(L.e1, L.s));
        }
        spec_ready = false;
        L.x_ready = false;
        ++matvecs;
        CK(cudaEventRecord(L.eb, L.s));
        // ---- alpha = V^T W ; W -= V alpha ; CGS against [0, cur), all queued
        // without a host round trip; the scalar recursion also normalizes
        // the residual on the device (V_{i+1} = W / |W|), which the
        // safeguards below redo in the rare steps where they trigger.
        // alpha is removed first, as br_remove_prev_overlap does: one pass
        // against [0, cur + nb) that takes alpha with the rest loses
        // orthogonality (measured: spurious Ritz values below the spectrum
        // after 40-150 steps)
        CK(multidot(L.col(cur), L.hprec, nb, (const double *)L.W.p, nb, n, n, (double *)L.partial.p,
                    (double *)L.coef.p, L.s, L.tk()));
        CK(cudaMemcpyAsync(L.hpin + Lz::kPinAlpha, L.coef.p, sizeof(double) * nb * nb, cudaMemcpyDeviceToHost, L.s));
        CK(sub_gemv(L.col(cur), L.hprec, nb, (const double *)L.coef.p, (double *)L.W.p, nb, n, n, nullptr, nullptr,
                    L.s, L.tk()));
        ST(cgs(L, cur, nullptr, true));
        CK(cudaMemcpyAsync(L.hpin + Lz::kPinSq, L.sq.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, L.s));
        if (nb == 1) {
            CK(normalize_col((const double *)L.W.p, L.col(cur + 1), L.hprec, (const double *)L.sq.p, n, L.s, L.X.p,
                             L.prec));
        } else {
            // W^T W for the block step, read back with alpha and the norms
            CK(multidot((const double *)L.W.p, nb, (const double *)L.W.p, nb, n, n, (double *)L.partial.p,
                        (double *)L.coef.p, L.s, L.tk()));
            CK(cudaMemcpyAsync(L.hpin + Lz::kPinS, L.coef.p, sizeof(double) * nb * nb, cudaMemcpyDeviceToHost, L.s));
        }
        CK(cudaEventRecord(L.e2, L.s));
        // ---- the next step's applyH, queued before the host reads this
        // step's alpha and beta (scalar recursion): the normalization above
        // just wrote its packed input.  It is kept when the next vector
        // stands, i.e. unless a safeguard below rewrites it, the run stops,
        // or a restart comes first (each of these clears x_ready)
        const bool spec = nb == 1 && cur + nb < niter * nb && !(thick && cur + 2 * nb > (niter - 1) * nb) &&
                          (int64_t)(cur + nb) < n;
        if (spec) {
            CK(cudaEventRecord(L.es0[spair], L.s));
            ST(launch_applyh_cols(ctx, L.X.p, (double *)L.W2.p, nb, L.prec, L.s));
            CK(cudaEventRecord(L.es1[spair], L.s));
        }
        CK(cudaEventSynchronize(L.e2));
        {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, m0, m1);
            L.t_mv += ms;
            cudaEventElapsedTime(&ms, L.eb, L.e2);
            L.t_ort += ms;
            if (post_pending) {  // the previous step's work after its synchronization
                cudaEventElapsedTime(&ms, L.e3, L.e4);
                L.t_ort += ms;
                post_pending = false;
            }
        }
        std::vector<double> alpha(L.hpin + Lz::kPinAlpha, L.hpin + Lz::kPinAlpha + (size_t)nb * nb);
        sq.assign(L.hpin + Lz::kPinSq, L.hpin + Lz::kPinSq + nb);
        cudaEventRecord(L.e3, L.s);
        // ---- scalar beta checks (src/blanczosmain.f90:1634-1660)
        if (nb == 1) {
            const double b = std::sqrt(std::max(sq[0], 0.0));
            beta.assign(1, b);
            L.x_ready = sq[0] > 0.0;  // the normalization wrote nothing otherwise
            if (iter > 1 && beta_prev > 0.0 && b < 1e-4 * beta_prev) {
                // random restart: keep the tiny beta, continue from a random
                // direction orthogonal to the whole history
                CK(random_cols((double *)L.W.p, 1, n, n, p->seed + 7919ull * (uint64_t)(rnd + 1), L.s));
                ST(cgs(L, cur + 1, &sq));
                ST(cgs(L, cur + 1, &sq));
                ++rnd;
                std::vector<double> b2;
                ST(next_block(L, cur + 1, sq, b2, lmin, lmax));
                L.x_ready = false;
            } else if (iter > 1 && beta_prev > 0.0 && b < 0.1 * beta_prev) {
                ST(cgs(L, cur + 1, &sq));  // second full pass, v_i included
                ST(next_block(L, cur + 1, sq, beta, lmin, lmax));
                L.x_ready = false;
            }
        } else {
            // block: guard against a rank-deficient residual block
            ST(block_finish(L, cur + nb, L.hpin + Lz::kPinS, beta, lmin, lmax));
            if (lmin <= 1e-20 * std::max(lmax, 1.0)) {
                CK(random_cols((double *)L.tmp.p, nb, n, n, p->seed + 104729ull * (uint64_t)(rnd + 1), L.s));
                const double eps = 1e-7 * std::sqrt(std::max(lmax, 1e-30));
                std::vector<double> e2(nb, eps);
                CK(cudaMemcpyAsync(L.M.p, e2.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, L.s));
                CK(scale_cols((const double *)L.tmp.p, (double *)L.tmp.p, (const double *)L.M.p, nb, n, n, L.s));
                // W += eps R, then orthogonalize again
                std::vector<double> one((size_t)nb * nb, 0.0);
                for (int b = 0; b < nb; ++b) one[(size_t)b * nb + b] = -1.0;
                CK(cudaMemcpyAsync(L.coef.p, one.data(), sizeof(double) * nb * nb, cudaMemcpyHostToDevice, L.s));
                CK(sub_gemv((const double *)L.tmp.p, nb, (const double *)L.coef.p, (double *)L.W.p, nb, n, n,
                            nullptr, nullptr, L.s));
                ST(cgs(L, cur + nb, &sq));
                ST(next_block(L, cur + nb, sq, beta, lmin, lmax));
                ++rnd;
            }
        }
        // no wait here: the host goes on with the projected matrix while the
        // device finishes the step; its time is read at the next sync
        CK(cudaEventRecord(L.e4, L.s));
        post_pending = true;
        // ---- projected matrix
        for (int a = 0; a < nb; ++a)
            for (int c = 0; c < nb; ++c) {
                const double v = 0.5 * (alpha[(size_t)a * nb + c] + alpha[(size_t)c * nb + a]);
                L.Tm(cur + a, cur + c) = v;
            }
        for (int a = 0; a < nb; ++a)
            for (int c = 0; c < nb; ++c) {
                L.Tm(cur + nb + a, cur + c) = beta[(size_t)a * nb + c];
                L.Tm(cur + c, cur + nb + a) = beta[(size_t)a * nb + c];
            }
        beta_prev = (nb == 1) ? beta[0] : 1.0;
        mT = cur + nb;
        cur += nb;
        // ---- eigenvalues and convergence (convergence_test option 0)
        auto conv_test = [&](const std::vector<double> &ev_) {
            bool hit = false;
            if ((int)eold.size() == (int)ev_.size()) {
                double ed = 0.0;
                for (size_t j = 0; j < ev_.size(); ++j) ed += std::fabs(eold[j] - ev_[j]);
                ed = ed / std::sqrt((double)ev_.size() + 1.0) * (1.0 + restarts);
                hit = ed < tol;
            }
            eold = ev_;
            return hit;
        };
        if (pend.active) {
            // the previous step's test ran beside this step's applyH; if it
            // converged, this step is discarded and the run ends where the
            // reference's would
            pend.active = false;
            ST(eig_collect(L, pend.want, e));
            if (conv_test(e)) {
                iter = pend.iter;
                total = pend.total;
                rnd = pend.rnd;
                cur = pend.cur;
                mT = pend.mT;
                finished = converged = true;
                break;
            }
        }
        if (cur >= niter * nb) finished = true;
        if (!p->fixed_iter && mT > ncheck && mT < (int64_t)n) {
            const bool restart_due = thick && !finished && cur + nb > (niter - 1) * nb;
            if (!finished && !restart_due) {
                ST(eig_queue(L, mT, karrow, ncheck));
                pend.active = true;
                pend.want = std::min(ncheck, mT);
                pend.iter = iter;
                pend.total = total;
                pend.rnd = rnd;
                pend.cur = cur;
                pend.mT = mT;
            } else {
                ST(eig_lowest(L, mT, karrow, ncheck, e, nullptr));
                if (conv_test(e)) finished = converged = true;
            }
        }
        if (mT >= (int64_t)n) { finished = true; converged = true; }  // Krylov space exhausted
        if (p->fixed_iter && finished) converged = true;
        if (spec && L.x_ready && !finished) {
            // the queued applyH stands unless the restart below moves the
            // continuation vector (it clears x_ready, checked again there)
            spec_ready = true;
            spair ^= 1;
        }
        // ---- thick restart
        if (thick && !finished && cur + nb > (niter - 1) * nb) {
            if (restarts >= p->max_restarts) {
                finished = true;
                break;
            }
            // scalar (thick_restart_sub_p): Ritz pairs of the projected matrix
            // without its last column, whose vector continues the recursion.
            // block (block_thick_restart_sub_p): Ritz pairs of the whole
            // projected matrix, whole blocks kept, and the block already made
            // for the next step (column mT) continues
            const int m = (nb == 1) ? mT - nb : mT;
            const int k = (nb == 1) ? std::min(nthick, m - 1) : (std::min(nthick, m - 1) / nb) * nb;
            std::vector<double> w, Z;          // Z column-major m x k
            ST(eig_lowest(L, m, karrow, k, w, &Z));
            // coupling rows: beta_prev block between block [m-nb, m) and [m, m+nb)
            std::vector<double> bp((size_t)nb * nb);
            for (int a = 0; a < nb; ++a)
                for (int c = 0; c < nb; ++c) bp[(size_t)a * nb + c] = L.Tm(m + a, m - nb + c);
            // V[0:k] = V[0:m] Y[:, 0:k] (through tmp), continuation block -> [k, k+nb)
            cudaEventRecord(L.e0, L.s);
            std::vector<double> Yk((size_t)m * k);
            for (int j = 0; j < m; ++j)
                for (int l = 0; l < k; ++l) Yk[(size_t)j * k + l] = Z[(size_t)l * m + j];
            // Y (m x k <= maxcol x 128) through the solve's own buffer: no
            // allocation per restart
            CK(cudaMemcpyAsync(L.Ydev.p, Yk.data(), sizeof(double) * Yk.size(), cudaMemcpyHostToDevice, L.s));
            CK(transform(L.col(0), L.hprec, m, (const double *)L.Ydev.p, k, k, L.tmp.p, L.hprec, n, n, n, L.s));
            CK(cudaMemcpyAsync(L.col(0), L.tmp.p, (size_t)L.hprec * n * k, cudaMemcpyDeviceToDevice, L.s));
            CK(cudaMemcpyAsync(L.col(k), L.col(m), (size_t)L.hprec * n * nb, cudaMemcpyDeviceToDevice, L.s));
            cudaEventRecord(L.e1, L.s);
            L.t_ort += elapsed(L);
            std::fill(L.T.begin(), L.T.end(), 0.0);
            for (int i = 0; i < k; ++i) L.Tm(i, i) = w[i];
            for (int a = 0; a < nb; ++a)
                for (int i = 0; i < k; ++i) {
                    double c_ = 0.0;
                    for (int c = 0; c < nb; ++c) c_ += bp[(size_t)a * nb + c] * Z[(size_t)i * m + (m - nb + c)];
                    L.Tm(k + a, i) = c_;
                    L.Tm(i, k + a) = c_;
                }
            cur = k;
            mT = k;
            karrow = k;
            ++restarts;
            // scalar: the continuation vector moved and its applyH input must
            // be packed again; block: the continuation is the block whose
            // packed input the last spectral step already wrote
            if (nb == 1) L.x_ready = false;
            spec_ready = false;
            iter = k / nb;
            beta_prev = -1.0;
        }
    }

    if (post_pending) {
        CK(cudaEventSynchronize(L.e4));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, L.e3, L.e4);
        L.t_ort += ms;
    }
    // ---- final Ritz pairs of T[0:mT] (lanczos_output, src/blanczoslib.f90:1268)
    std::vector<double> w, Z;          // Z column-major mT x nk
    const int nk = std::min(nkeep, mT);
    ST(eig_lowest(L, mT, karrow, nk, w, evecs ? &Z : nullptr));
    for (int j = 0; j < nkeep; ++j) evals[j] = (j < nk) ? w[j] : NAN;
    if (evecs) {
        std::vector<double> Yk((size_t)mT * nk);
        for (int j = 0; j < mT; ++j)
            for (int l = 0; l < nk; ++l) Yk[(size_t)j * nk + l] = Z[(size_t)l * mT + j];
        DevBuf Yd, out;
        ST(upload(ctx, Yd, Yk.data(), sizeof(double) * Yk.size()));
        int st2 = dev_alloc(ctx, out, sizeof(double) * (size_t)n * nk);
        if (st2) { dev_free(Yd); return st2; }
        cudaError_t te = transform(L.col(0), L.hprec, mT, (const double *)Yd.p, nk, nk, out.p, 8, n, n, n, L.s);
        if (te == cudaSuccess)
            te = cudaMemcpyAsync(evecs, out.p, sizeof(double) * (size_t)n * nk, cudaMemcpyDeviceToHost, L.s);
        if (te == cudaSuccess) te = cudaStreamSynchronize(L.s);
        dev_free(Yd);
        dev_free(out);
        CK(te);
        for (size_t i = (size_t)n * nk; i < (size_t)n * nkeep; ++i) evecs[i] = NAN;
    }
    if (rep) {
        rep->iterations = iter;
        rep->total_iterations = total;
        rep->restarts = restarts;
        rep->random_restarts = rnd;
        rep->matvecs = matvecs;
        rep->converged = converged ? 1 : 0;
        rep->t_matvec_ms = L.t_mv;
        rep->t_reorth_ms = L.t_ort;
        rep->t_eig_ms = L.t_eig;
    }
    return BSG_OK;
}

}  // namespace

extern "C" int bsg_lanczos(bsg_ctx *ctx, const bsg_lanczos_params *p, const double *pivot, double *evals,
                           double *evecs, bsg_report *rep) {
    if (!ctx) return BSG_ERR_ARG;
    if (!p || !evals) return set_err(ctx, BSG_ERR_ARG, "bsg_lanczos: null argument");
    if ((p->nb != 1 && p->nb != 2 && p->nb != 4 && p->nb != 8 && p->nb != 16) || p->nkeep < 1 || p->niter < 2 ||
        p->nkeep + std::max(p->nthick_add, 0) > 128 ||
        (p->matvec_prec != BSG_PREC_FP32 && p->matvec_prec != BSG_PREC_FP64) ||
        (p->lanc_prec != 0 && p->lanc_prec != BSG_PREC_FP32 && p->lanc_prec != BSG_PREC_FP64))
        return set_err(ctx, BSG_ERR_ARG, "bsg_lanczos: bad parameters");
    if ((int64_t)p->niter * p->nb + p->nb > 2048)
        return set_err(ctx, BSG_ERR_UNSUPPORTED, "bsg_lanczos: niter*nb above 2048 (projected matrix too large)");
    if ((int64_t)p->nkeep > ctx->dim) return set_err(ctx, BSG_ERR_ARG, "bsg_lanczos: nkeep > dim");
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (st) return st;
    Lz L;
    L.ctx = ctx;
    L.s = ctx->stream;
    L.n = ctx->dim;
    L.nb = p->nb;
    L.prec = p->matvec_prec;
    L.hprec = (p->lanc_prec == BSG_PREC_FP32) ? 4 : 8;
    const int niter_eff = (int)std::min<int64_t>(p->niter, (ctx->dim + p->nb - 1) / p->nb + 1);
    bsg_lanczos_params pp = *p;
    pp.niter = std::max(2, niter_eff);
    const int maxcol = pp.niter * L.nb + L.nb;
    const int N = maxcol;
    const size_t vb = sizeof(double) * (size_t)L.n;
    const size_t hb = (size_t)L.hprec * (size_t)L.n;  // one history column
    size_t need = hb * (size_t)maxcol + vb * (2 * L.nb + (size_t)std::max(L.nb, pp.nkeep + pp.nthick_add + 1)) +
                  (size_t)L.n * L.nb * (L.prec == 4 ? 4 : 8);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    if (need > fr) return set_err(ctx, BSG_ERR_NOMEM, "bsg_lanczos: history does not fit in device memory");
    const int G = dot_grid(L.n);
    const int ktmp = std::max(L.nb, pp.nkeep + std::max(pp.nthick_add, 0) + 1);
    if ((st = dev_alloc(ctx, L.hist, hb * maxcol)) || (st = dev_alloc(ctx, L.W, vb * L.nb)) ||
        (st = dev_alloc(ctx, L.tmp, vb * ktmp)) ||
        (st = dev_alloc(ctx, L.X, (size_t)L.n * L.nb * (L.prec == 4 ? 4 : 8))) ||
        (st = dev_alloc(ctx, L.partial, sizeof(double) * (size_t)4096 * G)) ||
        (st = dev_alloc(ctx, L.coef, sizeof(double) * (size_t)maxcol * L.nb)) ||
        (st = dev_alloc(ctx, L.sqp, sizeof(double) * 16 * kMaxDotGrid)) || (st = dev_alloc(ctx, L.sq, sizeof(double) * 16)) ||
        (st = dev_alloc(ctx, L.Adev, sizeof(double) * (size_t)N * N)) ||
        (st = dev_alloc(ctx, L.Vtmp, sizeof(double) * (size_t)N * N)) ||
        (st = dev_alloc(ctx, L.Zdev, sizeof(double) * (size_t)N * N)) || (st = dev_alloc(ctx, L.wdev, sizeof(double) * N)) ||
        (st = dev_alloc(ctx, L.al, sizeof(double) * N)) ||
        (st = dev_alloc(ctx, L.bt, sizeof(double) * N)) || (st = dev_alloc(ctx, L.ev, sizeof(double) * N)) ||
        (st = dev_alloc(ctx, L.M, sizeof(double) * 16 * 16)) || (st = dev_alloc(ctx, L.tau, sizeof(double) * N)) ||
        (st = dev_alloc(ctx, L.ework, sizeof(double) * ((size_t)2 * N + (size_t)6 * N * std::min(N, 128)))) ||
        (st = dev_alloc(ctx, L.ticket, 16)) || (L.nb == 1 && (st = dev_alloc(ctx, L.W2, vb))) ||
        (st = cuda_check(ctx, cudaMemsetAsync(L.ticket.p, 0, 16, L.s), "cudaMemsetAsync (pass ticket)"))) {
        // fall through to cleanup
    }
    L.maxcol = maxcol;
    if (!st && ((st = dev_alloc(ctx, L.al2, sizeof(double) * N)) || (st = dev_alloc(ctx, L.bt2, sizeof(double) * N)) ||
                (st = dev_alloc(ctx, L.w2, sizeof(double) * N)) ||
                (st = dev_alloc(ctx, L.Ydev, sizeof(double) * (size_t)N * 128)))) {
        // fall through to cleanup
    }
    if (!st && L.nb > 1 &&
        ((st = dev_alloc(ctx, L.Adev2, sizeof(double) * (size_t)N * N)) ||
         (st = dev_alloc(ctx, L.Vtmp2, sizeof(double) * (size_t)N * N)) || (st = dev_alloc(ctx, L.tau2, sizeof(double) * N)) ||
         (st = dev_alloc(ctx, L.ework2, sizeof(double) * 2 * (size_t)N)))) {
        // fall through to cleanup
    }
    if (!st && L.nb > 1)
        st = cuda_check(ctx, cudaHostAlloc((void **)&L.pinA, sizeof(double) * (size_t)N * N, cudaHostAllocDefault),
                        "cudaHostAlloc (Lanczos projected matrix)");
    if (!st) st = cuda_check(ctx, cudaHostAlloc((void **)&L.hpin, sizeof(double) * L.pin_doubles(), cudaHostAllocDefault),
                             "cudaHostAlloc (Lanczos staging)");
    // the side stream runs the convergence test's small eigen-solve beside the
    // next step's applyH; at the highest priority its few CTAs are scheduled
    // as soon as any SM has room, instead of after the applyH grid's
    // remaining CTAs
    if (!st) {
        int prio_lo = 0, prio_hi = 0;
        cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
        st = cuda_check(ctx, cudaStreamCreateWithPriority(&L.s2, cudaStreamNonBlocking, prio_hi), "cudaStreamCreate");
    }
    if (!st) {
        cudaEventCreate(&L.e0);
        cudaEventCreate(&L.e1);
        cudaEventCreate(&L.e2);
        cudaEventCreate(&L.e3);
        cudaEventCreate(&L.e4);
        cudaEventCreate(&L.eb);
        for (int i = 0; i < 2; ++i) {
            cudaEventCreate(&L.es0[i]);
            cudaEventCreate(&L.es1[i]);
        }
        cudaEventCreateWithFlags(&L.econv, cudaEventDisableTiming);
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, L.s);
        st = run(L, &pp, pivot, evals, evecs, rep);
        cudaEventRecord(t1, L.s);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        if (rep) rep->t_total_ms = ms;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        cudaEventDestroy(L.e0);
        cudaEventDestroy(L.e1);
        cudaEventDestroy(L.e2);
        cudaEventDestroy(L.e3);
        cudaEventDestroy(L.e4);
        cudaEventDestroy(L.eb);
        for (int i = 0; i < 2; ++i) {
            cudaEventDestroy(L.es0[i]);
            cudaEventDestroy(L.es1[i]);
        }
    }
    if (L.s2) {
        cudaStreamSynchronize(L.s2);
        cudaStreamDestroy(L.s2);
    }
    if (L.econv) cudaEventDestroy(L.econv);
    DevBuf *bufs[] = {&L.hist, &L.W, &L.X, &L.tmp, &L.partial, &L.coef, &L.sqp, &L.sq, &L.Adev,
                      &L.Vtmp, &L.Zdev, &L.wdev, &L.al, &L.bt, &L.ev, &L.M, &L.tau, &L.ework,
                      &L.al2, &L.bt2, &L.w2, &L.Adev2, &L.Vtmp2, &L.tau2, &L.ework2, &L.Ydev, &L.ticket,
                      &L.W2};
    cudaStreamSynchronize(L.s);
    for (DevBuf *b : bufs) dev_free(*b);
    if (L.hpin) cudaFreeHost(L.hpin);
    if (L.pinA) cudaFreeHost(L.pinA);
    return st;
}
