"""ORACLE -- test infrastructure only.

lanczos(): numpy restatement of BIGSTICK's scalar Lanczos (lanczos_p,
src/blanczosmain.f90:1413-1793) with lanc_prec = 8: uniform pivot
(src/blanczoslib.f90:825-831), alpha before reorthogonalization
(br_remove_prev_overlap, src/breorthog.f90:683-711), one classical
Gram-Schmidt pass against the earlier history (br_orthogonalize(1),
:831-891), beta = |r| (br_normalize, :758-783), eigenvalues of the
arrowhead-tridiagonal projected matrix (find_lanczos_eigenvalues,
src/blanczoslib.f90:143-376), convergence_test option 0 (:2660-2800) and
thick restart (thick_restart_sub_p, :1656-1894).

Note: with the uniform pivot the Krylov space inherits every symmetry the
pivot has; for N = Z nuclei with an isospin-conserving interaction the
uniform vector is symmetric under proton-neutron exchange, so only that
exchange class of states is reachable (the reference behaves the same way).
Pass a generic `pivot` to reach the whole spectrum.  The matvec is the oracle's
C restatement of applyHbundled_g (FP64 vectors, FP32 matrix elements).
"""
import numpy as np

from . import applyh_omp


def _projected(alpha, beta, k):
    """T from alpha[0:m], beta with the arrow of size k (src/blanczoslib.f90:195-212)."""
    m = len(alpha)
    T = np.diag(np.asarray(alpha, dtype=np.float64))
    for i in range(k):
        T[i, k] = T[k, i] = beta[i]
    for i in range(k, m - 1):
        T[i, i + 1] = T[i + 1, i] = beta[i]
    return T


def lanczos(tables, nkeep=10, niter=300, nthick_add=0, max_restarts=0, ncheck=None, tol=1e-3,
            fixed_iter=False, want_vectors=False, nthreads=None, matvec=None, pivot=None):
    n = tables.dim
    mv = matvec or (lambda v: applyh_omp(tables, v, nthreads=nthreads))
    ncheck = ncheck or (nkeep + 5)
    thick = nthick_add > 0 or max_restarts > 0
    nthick = nkeep + nthick_add
    V = np.zeros((niter + 1, n))
    V[0] = 1.0 / np.sqrt(n) if pivot is None else pivot
    V[0] /= np.linalg.norm(V[0])
    alpha, beta = [], []
    k_arrow = 0
    cur = 0
    restarts = 0
    eold = None
    it = 0
    total = 0
    finished = False
    while not finished:
        it += 1
        total += 1
        r = mv(V[cur])
        a = float(V[cur] @ r)
        r = r - a * V[cur]
        if cur > 0:
            c = V[:cur] @ r
            r = r - V[:cur].T @ c
        b = float(np.linalg.norm(r))
        if it > 1 and len(beta) and b < 0.1 * beta[-1]:
            c = V[:cur + 1] @ r
            r = r - V[:cur + 1].T @ c
            b = float(np.linalg.norm(r))
        alpha.append(a)
        beta.append(b)
        V[cur + 1] = r / b
        cur += 1
        mT = cur
        if cur >= niter:
            finished = True
        if not fixed_iter and mT > ncheck:
            e = np.linalg.eigvalsh(_projected(alpha, beta, k_arrow))[:ncheck]
            if eold is not None and len(eold) == len(e):
                ed = np.abs(eold - e).sum() / np.sqrt(len(e) + 1.0) * (1 + restarts)
                if ed < tol:
                    finished = True
            eold = e
        if thick and not finished and cur + 1 > niter - 1:
            if restarts >= max_restarts:
                break
            m = mT - 1
            k = min(nthick, m - 1)
            w, Y = np.linalg.eigh(_projected(alpha[:m], beta[:m], k_arrow))
            coupling = beta[m - 1] * Y[m - 1, :k]
            newV = Y[:, :k].T @ V[:m]
            cont = V[m].copy()
            V[:k] = newV
            V[k] = cont
            alpha = list(w[:k])
            beta = list(coupling)
            k_arrow = k
            cur = k
            restarts += 1
            it = k
    T = _projected(alpha, beta, k_arrow)
    w, Y = np.linalg.eigh(T)
    ev = w[:nkeep]
    vecs = (V[:len(alpha)].T @ Y[:, :nkeep]) if want_vectors else None
    return ev, vecs, {"iterations": it, "total_iterations": total, "restarts": restarts}


def _sym_upper(T):
    """The symmetric matrix DSYEV reads from the upper triangle of T."""
    return np.triu(T) + np.triu(T, 1).T


def lanczos_block(tables, nb, nkeep=10, niter=50, nthick_add=0, max_restarts=0, ncheck=None, tol=1e-3,
                  fixed_iter=False, want_vectors=False, nthreads=None, matvec=None, pivot=None):
    """numpy restatement of BIGSTICK's block Lanczos (lanczos_block,
    src/blanczosmain.f90:1804-2153, with mod_balg, src/bblock_algebra.f90
    :594-908, and block_thick_restart_sub_p, src/blanczoslib.f90:1923-2170),
    lanc_prec = 8, on the engine's iteration count convention (niter block
    iterations per cycle, history of niter*nb + nb vectors):

    * pivot block (dim x nb, interleaved as pivot[s*nb + v]) orthonormalized
      by spectral_decomp(0): S = P^T P = U L U^T, V_1 = P U L^-1/2;
    * step: W = H V_i; alpha by sequential projection (grab_alpha_blockv2:
      for each i, for each j, a = v_i . w_j, w_j -= a v_i); one classical
      Gram-Schmidt pass of every w_j against all earlier blocks (compute_W,
      br_orthogonalize_in_place); spectral_decomp: S = W^T W = U L U^T,
      beta = L^1/2 U^T, V_{i+1} = W U L^-1/2; alpha and beta into the band
      (add_alpha_Tmat / add_beta_Tmat), eigenvalues of its upper triangle;
    * convergence_test option 0 over ncheck states once more than ncheck
      columns exist;
    * thick restart when the next block would pass the cycle: Ritz pairs of
      the whole projected matrix, whole blocks kept (floor(nthick/nb)*nb
      vectors, the rest of nthick being overwritten by the continuation
      block), coupling beta_last * Y[last block rows, kept], V <- V Y, and the
      block already made for the next step continues the recursion.

    matvec(X) takes and returns a (dim, nb) array.  Returns (eigenvalues,
    eigenvectors or None, report)."""
    n = tables.dim
    if matvec is None:
        def matvec(X):
            return applyh_omp(tables, np.ascontiguousarray(X).reshape(-1), nb=nb,
                              nthreads=nthreads).reshape(n, nb)
    ncheck = ncheck or (nkeep + 5)
    thick = nthick_add > 0 or max_restarts > 0
    nthick = min(nkeep + nthick_add, niter * nb - 2 * nb)
    maxcol = niter * nb + nb
    V = np.zeros((maxcol, n))
    P = np.asarray(pivot, dtype=np.float64).reshape(n, nb).T
    w, U = np.linalg.eigh(P @ P.T)
    V[:nb] = (U / np.sqrt(w)).T @ P
    T = np.zeros((maxcol, maxcol))
    cur = mT = restarts = total = 0
    eold = None
    finished = converged = False
    while not finished:
        total += 1
        W = matvec(V[cur:cur + nb].T).T.copy()
        A = np.zeros((nb, nb))
        for i in range(nb):
            for j in range(nb):
                a = float(V[cur + i] @ W[j])
                W[j] -= a * V[cur + i]
                A[i, j] = a
        if cur > 0:
            C = V[:cur] @ W.T
            W -= (V[:cur].T @ C).T
        w, U = np.linalg.eigh(W @ W.T)
        beta = np.sqrt(w)[:, None] * U.T
        V[cur + nb:cur + 2 * nb] = (U / np.sqrt(w)).T @ W
        T[cur:cur + nb, cur:cur + nb] = A
        T[cur + nb:cur + 2 * nb, cur:cur + nb] = beta
        T[cur:cur + nb, cur + nb:cur + 2 * nb] = beta.T
        mT = cur + nb
        cur += nb
        if cur >= niter * nb:
            finished = True
        if not fixed_iter and mT > ncheck and mT < n:
            e = np.linalg.eigvalsh(_sym_upper(T[:mT, :mT]))[:ncheck]
            if eold is not None and len(eold) == len(e):
                ed = np.abs(eold - e).sum() / np.sqrt(len(e) + 1.0) * (1 + restarts)
                if ed < tol:
                    finished = converged = True
            eold = e
        if mT >= n:
            finished = converged = True
        if fixed_iter and finished:
            converged = True
        if thick and not finished and cur + nb > (niter - 1) * nb:
            if restarts >= max_restarts:
                break
            m = mT
            k = (min(nthick, m - 1) // nb) * nb
            w, Y = np.linalg.eigh(_sym_upper(T[:m, :m]))
            coupling = T[m:m + nb, m - nb:m] @ Y[m - nb:m, :k]
            newV = Y[:, :k].T @ V[:m]
            cont = V[m:m + nb].copy()
            V[:k] = newV
            V[k:k + nb] = cont
            T[:] = 0.0
            T[np.arange(k), np.arange(k)] = w[:k]
            T[k:k + nb, :k] = coupling
            T[:k, k:k + nb] = coupling.T
            cur = mT = k
            restarts += 1
    w, Y = np.linalg.eigh(_sym_upper(T[:mT, :mT]))
    ev = w[:nkeep]
    vecs = (V[:mT].T @ Y[:, :nkeep]) if want_vectors else None
    return ev, vecs, {"total_iterations": total, "restarts": restarts, "converged": int(converged)}
