"""ORACLE -- test infrastructure only.

numpy restatement of BIGSTICK's scalar Lanczos (lanczos_p,
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
