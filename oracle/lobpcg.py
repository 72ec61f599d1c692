"""Block eigensolver and orthonormalisation.

Oracle (test infrastructure only).  Restates PWDFT.jl:
  diag_LOBPCG.jl:1-28      diag_LOBPCG! over (ispin, ik)
  diag_LOBPCG.jl:51-225    diag_LOBPCG! per k-point, including the lock
                           branch (devals <= 10 eps) and its quirk that the
                           W[:, iact] projection (:131-132) is a no-op
  ortho_sqrt.jl:1-11       ortho_sqrt

Julia's Hermitian(A) reads the upper triangle; scipy is asked for the same.
"""
import numpy as np
import scipy.linalg as sla

from .ops import op_H, Kprec

EPS = np.finfo(np.float64).eps


def ortho_sqrt(psi):
    """ortho_sqrt.jl:1-4: psi * inv(sqrt(psi'psi))."""
    S = psi.conj().T @ psi
    w, U = sla.eigh(S, lower=False)
    return psi @ ((U / np.sqrt(w)) @ U.conj().T)


def ortho_cholesky(psi):
    """ortho_sqrt.jl:80-89: psi / U with psi'psi = U^H U."""
    U = np.linalg.cholesky(psi.conj().T @ psi).conj().T
    return np.linalg.solve(U.T, psi.T).T


def _herm_upper(A):
    """Hermitian(A) with the upper triangle (Julia default uplo=:U)."""
    U = np.triu(A)
    return U + np.triu(A, 1).conj().T


def _chol_upper(C):
    """cholesky(Hermitian(C)).U."""
    return sla.cholesky(_herm_upper(C), lower=False)


def _rdiv(W, R):
    """W / R for upper-triangular R, i.e. W * inv(R)."""
    return sla.solve_triangular(R, W.T, trans="T", lower=False).T


def diag_LOBPCG_k(Ham, X, ik=None, tol=1e-5, NiterMax=100, Nstates_conv=0, hop=None, stats=None):
    """diag_LOBPCG.jl:51-225.  X (Ngw, Nstates) is overwritten with the
    eigenvectors; returns the eigenvalues.  `hop(psi)` overrides op_H."""
    ik = Ham.ik if ik is None else ik
    H = hop if hop is not None else (lambda v: op_H(Ham, v, ik))
    prec = lambda v: Kprec(Ham, v, ik)
    Nbasis, Nstates = X.shape
    if Nstates_conv == 0:
        Nstates_conv = Nstates
    HX = H(X)
    P = np.zeros_like(X)
    HP = np.zeros_like(X)
    evals_old = np.zeros(Nstates)
    SMALL = 10.0 * EPS
    niter = 0
    for it in range(1, NiterMax + 1):
        niter = it
        XHX = _herm_upper(X.conj().T @ HX)
        evals = sla.eigh(XHX, eigvals_only=True)
        devals = np.abs(evals - evals_old)
        evals_old = evals.copy()
        R = HX - X @ XHX
        nconv = int(np.sum(devals < tol))
        ilock = np.nonzero(devals <= SMALL)[0]
        iact = np.nonzero(devals > SMALL)[0]
        Nlock, Nact = len(ilock), len(iact)
        if nconv >= Nstates_conv:
            break
        W = prec(R)
        if Nlock > 0:
            Xlock = X[:, ilock]
            # diag_LOBPCG.jl:126-133 computes a projected W column into a
            # local binding and discards it: no effect on W.
            X[:, iact] = X[:, iact] - Xlock @ (Xlock.conj().T @ X[:, iact])
            W[:, iact] = W[:, iact] - Xlock @ (Xlock.conj().T @ W[:, iact])
            HX[:, iact] = H(X[:, iact])
            HW = H(W[:, iact])
            HX[:, iact] = HX[:, iact] - Xlock @ (Xlock.conj().T @ HX[:, iact])
            HW = HW - Xlock @ (Xlock.conj().T @ HW)
            Wa = W[:, iact]
            C = Wa.conj().T @ Wa
            Rc = _chol_upper(C)
            Wa = _rdiv(Wa, Rc)
            W[:, iact] = Wa
            HW = _rdiv(HW, Rc)
            Q = np.hstack([X[:, iact], Wa])
            HQ = np.hstack([HX[:, iact], HW])
            T = _herm_upper(Q.conj().T @ HQ)
            G = _herm_upper(Q.conj().T @ Q)
            sd, S = sla.eigh(T, G, lower=False)
            U = S[:, :Nact]
            Xact = Q @ U
            X[:, :] = np.hstack([Xlock, Xact])
            T = _herm_upper(X.conj().T @ H(X))
            evalT, evecsT = sla.eigh(T, lower=False)
            X[:, :] = X @ evecsT
            HX = H(X)
        else:
            HW = H(W)
            C = W.conj().T @ W
            Rc = _chol_upper(C)
            W = _rdiv(W, Rc)
            HW = _rdiv(HW, Rc)
            if it > 1:
                Q = np.hstack([X, W, P])
                HQ = np.hstack([HX, HW, HP])
            else:
                Q = np.hstack([X, W])
                HQ = np.hstack([HX, HW])
            T = _herm_upper(Q.conj().T @ HQ)
            G = _herm_upper(Q.conj().T @ Q)
            sd, S = sla.eigh(T, G, lower=False)
            U = S[:, :Nstates]
            X[:, :] = Q @ U
            HX = HQ @ U
            if it > 1:
                s2 = slice(Nstates, 2 * Nstates)
                s3 = slice(2 * Nstates, 3 * Nstates)
                P = W @ U[s2, :] + P @ U[s3, :]
                HP = HW @ U[s2, :] + HP @ U[s3, :]
                C = P.conj().T @ P
                Rc = _chol_upper(C)
                P = _rdiv(P, Rc)
                HP = _rdiv(HP, Rc)
            else:
                P = W.copy()
                HP = HW.copy()
    S = X.conj().T @ HX
    S = _herm_upper(0.5 * (S + S.conj().T))
    evals, Qv = sla.eigh(S, lower=False)
    X[:, :] = X @ Qv
    if stats is not None:
        stats.append(niter)
    return evals


def diag_LOBPCG(Ham, psiks, tol=1e-5, NiterMax=100, Nstates_conv=0, stats=None):
    """diag_LOBPCG.jl:1-28 (Nspin = 1)."""
    Nk = Ham.pw.kpoints.Nkpt
    evals = np.zeros((psiks[0].shape[1], Nk))
    for ik in range(Nk):
        Ham.ik = ik
        evals[:, ik] = diag_LOBPCG_k(Ham, psiks[ik], ik, tol=tol, NiterMax=NiterMax,
                                     Nstates_conv=Nstates_conv, stats=stats)
    return evals
