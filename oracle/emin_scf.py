"""Direct minimisation of the Kohn-Sham energy (Ismail-Beigi and Arias).

Oracle (test infrastructure only).  Restates PWDFT.jl
KS_solve_Emin_PCG.jl:27-270 for Nspin = 1: Gaussian starting density and
update!, an initial diag_LOBPCG! of 10 iterations (unless skipped), then per
step, every k-point: calc_grad (with occupations), Kprec, beta (1 Fletcher-
Reeves, 2 Polak-Ribiere, 3 Hestenes-Stiefel, 4 Dai-Yuan; 1 and 4 reset near
1, negative or NaN beta reset to 0), d = -Kg + beta d_old, trial point
ortho_sqrt(psi + alpha_t d); the trial density and potentials; the line-
minimising alpha from the trial gradient; psi = ortho_sqrt(psi + alpha d);
density, potentials and energies; |dE| < etot_conv_thr twice.  Ends with
the Rayleigh-Ritz rotation of every block.
The reference's Hestenes-Stiefel line reads g_old[ik] (an index slip that
only differs with spin); this restatement uses g_old[i], the same for
Nspin = 1.
"""
import numpy as np
import scipy.linalg as sla

from .ops import op_H, Kprec, calc_grad, calc_rhoe
from .lobpcg import ortho_sqrt, diag_LOBPCG
from .energies import calc_energies


def _rdot(a, b):
    return float(np.real(np.vdot(a, b)))


def KS_solve_Emin_PCG(Ham, psiks, alpha_t=3e-5, NiterMax=200, i_cg_beta=2, etot_conv_thr=1e-6,
                      skip_initial_diag=False, alpha_max=2.1, restrict_linmin=False, log=None):
    """psiks (list of (Ngw, Nstates)) is overwritten; returns (energies,
    evals (Nstates, Nkpt), iterations)."""
    Nkpt = Ham.pw.kpoints.Nkpt
    wk = Ham.pw.kpoints.wk
    Focc = Ham.Focc
    Rhoe = Ham.guess_rhoe()                                                    # :65-71
    Ham.update(Rhoe)                                                           # :73
    if not skip_initial_diag:                                                  # :75-79
        diag_LOBPCG(Ham, psiks, NiterMax=10)
    g = [None] * Nkpt
    Kg = [None] * Nkpt
    d = [None] * Nkpt
    g_old = [np.zeros_like(p) for p in psiks]
    d_old = [np.zeros_like(p) for p in psiks]
    Kg_old = [np.zeros_like(p) for p in psiks]
    psic = [None] * Nkpt
    beta = np.zeros(Nkpt)
    alpha = np.zeros(Nkpt)
    Etot_old = 0.0
    E = calc_energies(Ham, psiks, Rhoe)                                        # :97-101
    Nconverges = 0
    it = 0
    for it in range(1, NiterMax + 1):
        for i in range(Nkpt):                                                  # :130-179
            g[i] = calc_grad(Ham, psiks[i], i, Focc[:, i], wk[i])
            Kg[i] = Kprec(Ham, g[i], i)
            if it != 1:
                if i_cg_beta == 1:
                    beta[i] = _rdot(g[i], Kg[i]) / _rdot(g_old[i], Kg_old[i])
                    if abs(beta[i] - 1.0) < 0.2:
                        beta[i] = 0.0
                elif i_cg_beta == 2:
                    beta[i] = _rdot(g[i] - g_old[i], Kg[i]) / _rdot(g_old[i], Kg_old[i])
                elif i_cg_beta == 3:
                    beta[i] = _rdot(g[i] - g_old[i], Kg[i]) / _rdot(g[i] - g_old[i], d[i])
                else:
                    beta[i] = _rdot(g[i], Kg[i]) / float(np.real(np.sum((g[i] - g_old[i]) * np.conj(d_old[i]))))
                    if abs(beta[i] - 1.0) < 0.2:
                        beta[i] = 0.0
            if beta[i] < 0.0 or np.isnan(beta[i]):
                beta[i] = 0.0
            d[i] = -Kg[i] + beta[i] * d_old[i]
            psic[i] = ortho_sqrt(psiks[i] + alpha_t * d[i])
        Rhoe = calc_rhoe(Ham, psic, Focc)                                      # :181-183
        Ham.update(Rhoe)
        for i in range(Nkpt):                                                  # :185-207
            gt = calc_grad(Ham, psic[i], i, Focc[:, i], wk[i])
            denum = _rdot(g[i] - gt, d[i])
            alpha[i] = abs(alpha_t * _rdot(g[i], d[i]) / denum) if denum != 0.0 else 0.0
            if restrict_linmin and alpha[i] > alpha_max:
                alpha[i] = alpha_max
            psiks[i] = ortho_sqrt(psiks[i] + alpha[i] * d[i])
        Rhoe = calc_rhoe(Ham, psiks, Focc)                                     # :209-214
        Ham.update(Rhoe)
        E = calc_energies(Ham, psiks, Rhoe)
        diffE = Etot_old - E["Total"]
        if log is not None:
            log.append((it, E["Total"], diffE))
        Nconverges = Nconverges + 1 if abs(diffE) < etot_conv_thr else 0       # :226-238
        if Nconverges >= 2:
            break
        g_old = [x.copy() for x in g]
        d_old = [x.copy() for x in d]
        Kg_old = [x.copy() for x in Kg]
        Etot_old = E["Total"]
    evals = np.zeros((psiks[0].shape[1], Nkpt))                                # :247-256
    for i in range(Nkpt):
        psiks[i] = ortho_sqrt(psiks[i])
        lam, V = sla.eigh(psiks[i].conj().T @ op_H(Ham, psiks[i], i), lower=False)
        evals[:, i] = lam
        psiks[i] = psiks[i] @ V
    return E, evals, it
