"""All-band preconditioned conjugate-gradient eigensolver.

Oracle (test infrastructure only).  Restates PWDFT.jl
  diag_Emin_PCG.jl:57-193   diag_Emin_PCG! for one k-point (band-energy
                            minimisation, beta choices I_CG_BETA 1-4, trial
                            step alpha_t, ortho_sqrt after every update,
                            final Rayleigh-Ritz rotation)
  calc_grad.jl:60-82        calc_grad_evals: H psi - psi (psi' H psi)
"""
import numpy as np
import scipy.linalg as sla

from .ops import op_H, Kprec
from .lobpcg import ortho_sqrt


def calc_grad_evals(Ham, psi, ik):
    """calc_grad.jl:60-82."""
    Hpsi = op_H(Ham, psi, ik)
    return Hpsi - psi @ (psi.conj().T @ Hpsi)


def _rdot(a, b):
    """real(sum(conj(a) .* b))"""
    return float(np.real(np.vdot(a, b)))


def diag_Emin_PCG(Ham, X, ik=None, tol=1e-5, NiterMax=100, Nstates_conv=0, tol_ebands=1e-4,
                  alpha_t=3e-5, I_CG_BETA=2):
    """X (Ngw, Nstates), orthonormal on entry, is overwritten with the Ritz
    vectors; returns (evals, iterations, converged)."""
    ik = Ham.ik if ik is None else ik
    Nstates = X.shape[1]
    if Nstates_conv == 0:
        Nstates_conv = Nstates
    d_old = np.zeros_like(X)
    g_old = np.zeros_like(X)
    Kg_old = np.zeros_like(X)
    beta = 0.0
    Ebands_old = 0.0
    evals = sla.eigvalsh(X.conj().T @ op_H(Ham, X, ik), lower=False)          # :92-95
    evals_old = evals.copy()
    converged = False
    it = 0
    for it in range(1, NiterMax + 1):
        g = calc_grad_evals(Ham, X, ik)                                        # :103-104
        Kg = Kprec(Ham, g, ik)
        if it != 1:                                                            # :106-116
            if I_CG_BETA == 1:
                beta = _rdot(g, Kg) / _rdot(g_old, Kg_old)
            elif I_CG_BETA == 2:
                beta = _rdot(g - g_old, Kg) / _rdot(g_old, Kg_old)
            elif I_CG_BETA == 3:
                beta = _rdot(g - g_old, Kg) / _rdot(g - g_old, d_old)
            else:
                beta = _rdot(g, Kg) / float(np.real(np.sum((g - g_old) * np.conj(d_old))))
        if beta < 0.0:                                                         # :117-119
            beta = 0.0
        d = -Kg + beta * d_old                                                 # :121
        Xc = ortho_sqrt(X + alpha_t * d)                                       # :123-124
        gt = calc_grad_evals(Ham, Xc, ik)
        denum = _rdot(g - gt, d)                                               # :126-131
        alpha = abs(alpha_t * _rdot(g, d) / denum) if denum != 0.0 else 0.0
        X[:, :] = ortho_sqrt(X + alpha * d)                                    # :134
        evals = sla.eigvalsh(X.conj().T @ op_H(Ham, X, ik), lower=False)      # :136-139
        Ebands = float(np.sum(evals))
        devals = np.abs(evals - evals_old)
        evals_old = evals.copy()
        nconv = int(np.sum(devals < tol))
        diffE = abs(Ebands - Ebands_old)
        if nconv >= Nstates_conv or diffE <= tol_ebands * Nstates:             # :154-167
            converged = True
            break
        g_old, d_old, Kg_old = g.copy(), d.copy(), Kg.copy()                   # :169-172
        Ebands_old = Ebands
    X[:, :] = ortho_sqrt(X)                                                    # :179-184
    lam, V = sla.eigh(X.conj().T @ op_H(Ham, X, ik), lower=False)
    X[:, :] = X @ V
    return lam, it, converged
