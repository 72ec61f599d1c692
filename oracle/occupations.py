"""Fermi-Dirac smearing: occupations, Fermi level, entropy term.

Oracle (test infrastructure only).  Restates PWDFT.jl occupations.jl
(Nspin = 1, collinear):
  wgauss         :71-83     Fermi function 1/(1 + e^-x), clamped at |x| > 200
  sumkg          :92-121    electrons below `ene`, 2 wk per k-point
  find_E_fermi   :126-192   bisection between min(evals) - 2kT and max(evals) + 2kT
  calc_Focc      :6-32      Focc = 2 wgauss((E_f - evals)/kT)
  w1gauss        :197-207   f log f + (1 - f) log(1 - f), 0 for |x| > 36
  calc_entropy   :222-245   mTS = sum 2 wk kT w1gauss((E_f - evals)/kT)
"""
import numpy as np

EPS = np.finfo(np.float64).eps


def wgauss(x):
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(over="ignore"):
        f = 1.0 / (1.0 + np.exp(-x))
    return np.where(x < -200.0, 0.0, np.where(x > 200.0, 1.0, f))


def sumkg(wk, kT, evals, ene):
    return float(np.sum(2.0 * np.asarray(wk) * wgauss((ene - evals) / kT).sum(axis=0)))


def find_E_fermi(Nelectrons, wk, kT, evals, NiterMax=300):
    Elw = evals[0, :].min() - 2 * kT
    Eup = evals[-1, :].max() + 2 * kT
    if sumkg(wk, kT, evals, Eup) - Nelectrons < -EPS or sumkg(wk, kT, evals, Elw) - Nelectrons > EPS:
        raise ValueError("Bounds for E_fermi is not found")
    SMALL = 1e-10
    Ef = 0.5 * (Eup + Elw)
    Ef_old = Ef
    for _ in range(NiterMax):
        mid = sumkg(wk, kT, evals, Ef)
        if abs(mid - Nelectrons) < SMALL:
            return Ef
        elif mid - Nelectrons < -SMALL:
            Elw = Ef
        else:
            Eup = Ef
        Ef = 0.5 * (Eup + Elw)
        if abs(Ef - Ef_old) < SMALL:
            return Ef
        Ef_old = Ef
    return Ef


def calc_Focc(Nelectrons, wk, kT, evals):
    """(Focc (Nstates, Nkpt), E_fermi)."""
    Ef = find_E_fermi(Nelectrons, wk, kT, evals)
    return 2.0 * wgauss((Ef - evals) / kT), Ef


def w1gauss(x):
    x = np.asarray(x, dtype=np.float64)
    ok = np.abs(x) <= 36.0
    f = 1.0 / (1.0 + np.exp(-np.where(ok, x, 0.0)))
    onemf = 1.0 - f
    return np.where(ok, f * np.log(f) + onemf * np.log(onemf), 0.0)


def calc_entropy(wk, kT, evals, E_fermi):
    return float(np.sum(2.0 * np.asarray(wk)[None, :] * kT * w1gauss((E_fermi - evals) / kT)))
