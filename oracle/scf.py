"""Self-consistent field driver with Pulay density mixing.

Oracle (test infrastructure only).  Restates PWDFT.jl:
  KS_solve_SCF.jl:24-373   KS_solve_SCF! (Nspin = 1, LOBPCG, optional Fermi-Dirac
                           smearing: KS_solve_SCF.jl:218-223 with occupations.jl)
  mix_pulay.jl:1-41        mix_pulay!
  gen_wavefunc.jl:90-92    rand_Wavefunc (with a NumPy RNG: Julia's stream
                           cannot be reproduced)
"""
import numpy as np

from .lobpcg import diag_LOBPCG, ortho_sqrt
from .ops import calc_rhoe
from .energies import calc_energies
from .occupations import calc_Focc, calc_entropy

EPS = np.finfo(np.float64).eps


def rand_BlochWavefunc(Ham, seed=1234):
    """gen_wavefunc.jl:75-92: ortho_sqrt(rand(ComplexF64, Ngw, Nstates))."""
    rng = np.random.default_rng(seed)
    out = []
    for ik in range(Ham.pw.kpoints.Nkpt):
        ngw = Ham.pw.gvecw.Ngw[ik]
        psi = rng.random((ngw, Ham.Nstates)) + 1j * rng.random((ngw, Ham.Nstates))
        out.append(ortho_sqrt(psi))
    return out


def mix_pulay(x, gx, beta, X, F, it, mixdim, state):
    """mix_pulay.jl:1-41 (it is 1-based as in the reference)."""
    f = gx - x
    if it == 1:
        dx = x.copy()
        df = f.copy()
    else:
        dx = x - state["x_old"]
        df = f - state["f_old"]
    if it <= mixdim:
        X[:, it - 1] = dx
        F[:, it - 1] = df
    else:
        X[:, :-1] = X[:, 1:].copy()
        F[:, :-1] = F[:, 1:].copy()
        X[:, -1] = dx
        F[:, -1] = df
    state["x_old"] = x.copy()
    state["f_old"] = f.copy()
    if it > mixdim:
        addv = (X + beta * F) @ np.linalg.inv(F.T @ F) @ (F.T @ f)
        return x + beta * f - addv
    return x + beta * f


def KS_solve_SCF(Ham, psiks=None, betamix=0.2, NiterMax=100, mix_method="pulay",
                 mixdim=5, etot_conv_thr=1e-6, ethr_evals_last=1e-5, verbose=False,
                 diag=None, seed=1234, log=None, use_smearing=False, kT=1e-3):
    """KS_solve_SCF.jl:24-373.  `diag(Ham, psiks, tol, Nstates_conv)` may
    replace the LOBPCG call (used to drive the GPU solver through the same
    loop); `log` collects (iter, Etot, diffE, diffRhoe) rows."""
    pw = Ham.pw
    N = pw.Npoints
    if psiks is None:
        psiks = rand_BlochWavefunc(Ham, seed=seed)
    Rhoe = Ham.guess_rhoe()
    Ham.update(Rhoe)
    Etot_old = 0.0
    XX = np.zeros((N, mixdim))
    FF = np.zeros((N, mixdim))
    state = {}
    Nconverges = 0
    ethr = 0.1
    energies = None
    evals = None
    for it in range(1, NiterMax + 1):
        if it == 1:
            ethr = 0.1
        elif it == 2:
            ethr = 0.01
        else:
            ethr = max(ethr / 5.0, ethr_evals_last)
        if diag is None:
            evals = diag_LOBPCG(Ham, psiks, tol=ethr, Nstates_conv=Ham.Nstates_occ)
        else:
            evals = diag(Ham, psiks, ethr, Ham.Nstates_occ)
        if use_smearing:
            Ham.Focc, Ham.E_fermi = calc_Focc(Ham.Nelectrons, pw.kpoints.wk, kT, evals)
            Ham.mTS = calc_entropy(pw.kpoints.wk, kT, evals, Ham.E_fermi)
        Rhoe_new = calc_rhoe(Ham, psiks)
        diffRhoe = float(np.sum(np.abs(Rhoe_new - Rhoe))) / N
        if mix_method == "simple":
            Rhoe = betamix * Rhoe_new + (1 - betamix) * Rhoe
        elif mix_method == "pulay":
            Rhoe = mix_pulay(Rhoe, Rhoe_new, betamix, XX, FF, it, mixdim, state)
        else:
            raise ValueError(mix_method)
        Rhoe = np.where(Rhoe < EPS, EPS, Rhoe)
        Ham.update(Rhoe)
        energies = calc_energies(Ham, psiks, Rhoe)
        Etot = energies["Total"]
        diffE = abs(Etot - Etot_old)
        if verbose:
            print("SCF: %5d %18.10f %12.5e %12.5e" % (it, Etot, diffE, diffRhoe))
        if log is not None:
            log.append((it, Etot, diffE, diffRhoe))
        Nconverges = Nconverges + 1 if diffE < etot_conv_thr else 0
        if Nconverges >= 2:
            break
        Etot_old = Etot
    Ham.evals = evals
    return energies, psiks, Rhoe
