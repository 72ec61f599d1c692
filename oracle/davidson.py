"""QE-style block Davidson eigensolver.

Oracle (test infrastructure only).  Restates PWDFT.jl
diag_davidson_qe_v2.jl:38-216 (diag_davidson_qe! for one k-point) for
norm-conserving pseudopotentials (op_S = identity, so S psi = psi).
"""
import numpy as np
import scipy.linalg as sla

from .ops import op_H, Kprec


def _herm_from_upper(A, n):
    """Diagonal made real, lower triangle := conj(upper) (diag_davidson_qe_v2.jl:139-149)."""
    B = A[:n, :n]
    d = np.real(np.diag(B)).copy()
    U = np.triu(B, 1)
    A[:n, :n] = U + U.conj().T + np.diag(d)


def diag_davidson_qe(Ham, evc, ik=None, EBANDS_THR=1e-8, NiterMax=40, hop=None):
    """evc (N, Nvec) is overwritten with the Ritz vectors; returns (evals, iterations)."""
    ik = Ham.ik if ik is None else ik
    H = hop if hop is not None else (lambda v: op_H(Ham, v, ik))
    N, Nvec = evc.shape
    Nvecx = 2 * Nvec
    psi = np.zeros((N, Nvecx), dtype=np.complex128)
    Hpsi = np.zeros_like(psi)
    Hc = np.zeros((Nvecx, Nvecx), dtype=np.complex128)
    Sc = np.zeros_like(Hc)
    vc = np.zeros_like(Hc)
    ew = np.zeros(Nvecx)
    is_conv = np.zeros(Nvec, dtype=bool)
    notcnv, nbase = Nvec, Nvec
    psi[:, :Nvec] = evc
    Hpsi[:, :Nvec] = H(psi[:, :Nvec])
    Hc[:nbase, :nbase] = psi[:, :nbase].conj().T @ Hpsi[:, :nbase]
    Sc[:nbase, :nbase] = psi[:, :nbase].conj().T @ psi[:, :nbase]
    w, v = sla.eigh(Hc[:Nvec, :Nvec], Sc[:Nvec, :Nvec], lower=False)
    ew[:Nvec] = w
    vc[:Nvec, :Nvec] = v
    evals = ew[:Nvec].copy()
    kter, dav_iter = 1, 0
    while kter <= NiterMax:
        dav_iter = kter
        npos = 0
        for ist in range(Nvec):
            if not is_conv[ist]:
                if npos != ist:
                    vc[:, npos] = vc[:, ist]
                ew[nbase + npos] = evals[ist]
                npos += 1
        nb1 = nbase
        V = vc[:nbase, :notcnv]
        corr = psi[:, :nbase] @ V
        corr = corr * (-ew[nbase:nbase + notcnv])[None, :]
        corr = corr + Hpsi[:, :nbase] @ V
        corr = Kprec(Ham, corr, ik)
        nrm = np.real(np.sum(np.conj(corr) * corr, axis=0))
        corr = corr / np.sqrt(nrm)[None, :]
        psi[:, nb1:nb1 + notcnv] = corr
        Hpsi[:, nb1:nb1 + notcnv] = H(corr)
        Hc[:nbase + notcnv, nb1:nb1 + notcnv] = psi[:, :nbase + notcnv].conj().T @ Hpsi[:, nb1:nb1 + notcnv]
        Sc[:nbase + notcnv, nb1:nb1 + notcnv] = psi[:, :nbase + notcnv].conj().T @ psi[:, nb1:nb1 + notcnv]
        nbase += notcnv
        _herm_from_upper(Hc, nbase)
        _herm_from_upper(Sc, nbase)
        w, v = sla.eigh(Hc[:nbase, :nbase], Sc[:nbase, :nbase], lower=False)
        ew[:nbase] = w
        vc[:nbase, :nbase] = v
        vc[:, Nvec:] = 0.0
        is_conv = np.abs(ew[:Nvec] - evals) < EBANDS_THR
        notcnv = int(np.sum(~is_conv))
        evals = ew[:Nvec].copy()
        if notcnv == 0 or nbase + notcnv > Nvecx or dav_iter == NiterMax:
            evc[:, :] = psi[:, :nbase] @ vc[:nbase, :Nvec]
            if notcnv == 0 or dav_iter == NiterMax:
                break
            Hnew = Hpsi[:, :nbase] @ vc[:nbase, :Nvec]
            psi[:, :Nvec] = evc
            Hpsi[:, :Nvec] = Hnew
            nbase = Nvec
            Hc[:, :nbase] = 0.0
            Sc[:, :nbase] = 0.0
            vc[:, :nbase] = 0.0
            Hc[np.arange(nbase), np.arange(nbase)] = evals
            Sc[np.arange(nbase), np.arange(nbase)] = 1.0
            vc[np.arange(nbase), np.arange(nbase)] = 1.0
        kter += 1
    return evals, dav_iter


def diag_davidson_qe_all(Ham, psiks, tol=1e-5, NiterMax=100):
    """diag_davidson_qe_v2.jl:6-34: every k-point (Nspin = 1), EBANDS_THR =
    tol; returns evals (Nstates, Nkpt)."""
    Nkpt = Ham.pw.kpoints.Nkpt
    evals = np.zeros((psiks[0].shape[1], Nkpt))
    for ik in range(Nkpt):
        Ham.ik = ik
        evals[:, ik], _ = diag_davidson_qe(Ham, psiks[ik], ik, EBANDS_THR=tol, NiterMax=NiterMax)
    return evals


def diag_davidson(Ham, X, ik=None, tol=1e-5, NiterMax=100, Nstates_conv=0, hop=None):
    """The 2-block Davidson of diag_davidson.jl:50-191 for one k-point: the
    basis is [X, R] with R the Kprec-preconditioned, normalised residuals;
    X (Nbasis, Nstates), orthonormal on entry, is overwritten with the Ritz
    vectors.  Returns (evals, iterations, converged)."""
    ik = Ham.ik if ik is None else ik
    H = hop if hop is not None else (lambda v: op_H(Ham, v, ik))
    Nbasis, Nstates = X.shape
    if Nstates_conv == 0:
        Nstates_conv = Nstates
    n = Nstates
    s1, s2 = slice(0, n), slice(n, 2 * n)
    HX = H(X)
    evals = np.real(np.sum(X.conj() * HX, axis=0))                      # :82-85
    R = evals[None, :] * X - HX                                          # :88-93
    res = np.sqrt(np.real(np.sum(R.conj() * R, axis=0)))
    EPS = np.finfo(np.float64).eps
    evals_old = evals.copy()
    Hred = np.zeros((2 * n, 2 * n), dtype=np.complex128)
    Sred = np.zeros_like(Hred)
    it = 0
    converged = False
    for it in range(1, NiterMax + 1):
        res_norm = np.where(EPS < res, 1.0 / np.where(res > 0, res, 1.0), 1.0)   # :107-117
        R = R * res_norm[None, :]
        R = Kprec(Ham, R, ik)                                            # :119
        HR = H(R)                                                        # :121
        if it == 1:                                                      # :124-131
            Hred[s1, s1] = X.conj().T @ HX
        else:
            Hred[s1, s1] = np.diag(evals.astype(np.complex128))
        Hred[s1, s2] = X.conj().T @ HR                                   # :133-136
        Hred[s2, s2] = R.conj().T @ HR
        Hred[s2, s1] = Hred[s1, s2].conj().T
        Sred[s1, s1] = np.eye(n)                                         # :138-141
        Sred[s1, s2] = X.conj().T @ R
        Sred[s2, s2] = R.conj().T @ R
        Sred[s2, s1] = Sred[s1, s2].conj().T
        Hred = 0.5 * (Hred + Hred.conj().T)                              # :143-144
        Sred = 0.5 * (Sred + Sred.conj().T)
        lam, Xr = sla.eigh(Hred, Sred, lower=False)                      # :146
        evals = lam[:n].copy()
        devals = np.abs(evals - evals_old)                               # :150-151
        nconv = int(np.sum(devals < tol))
        Xn = X @ Xr[s1, s1] + R @ Xr[s2, s1]                             # :153-154
        HX = HX @ Xr[s1, s1] + HR @ Xr[s2, s1]
        X[:, :] = Xn
        R = evals[None, :] * X - HX                                      # :157-162
        res = np.sqrt(np.real(np.sum(R.conj() * R, axis=0)))
        if nconv >= Nstates_conv:                                        # :170-176
            converged = True
            break
        evals_old = evals.copy()
    return evals, it, converged
