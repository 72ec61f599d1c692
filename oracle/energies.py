"""Total-energy components.

Oracle (test infrastructure only).  Restates PWDFT.jl:
  calc_energies.jl:7-58      calc_E_Ps_nloc (GTH)
  calc_energies.jl:245-333   calc_E_local / calc_E_xc (VWN, Nspin = 1)
  calc_energies.jl:342-375   calc_E_kin
  calc_E_NN.jl:60-172        calc_E_NN (Ewald)
  Energies.jl:30-34          sum(energies)
"""
import math
import numpy as np
from scipy.special import erfc

from .ham import calc_epsxc_VWN
from .ops import calc_betaNL_psi


def calc_E_kin(Ham, psiks):
    """calc_energies.jl:342-375."""
    E = 0.0
    for ik, psi in enumerate(psiks):
        Gw2 = Ham.pw.Gk2(ik)
        per_band = (np.abs(psi) ** 2 * Gw2[:, None]).sum(axis=0)
        E += Ham.pw.kpoints.wk[ik] * float(np.dot(Ham.Focc[:, ik], per_band))
    return 0.5 * E


def calc_E_Ps_nloc(Ham, psiks):
    """calc_energies.jl:7-58."""
    E = 0.0
    for ik, psi in enumerate(psiks):
        B = calc_betaNL_psi(Ham, psi, ik)          # (Nstates, Nbeta)
        enl = np.real(np.einsum("si,ij,sj->s", B.conj(), Ham.Dnl, B))
        E += Ham.pw.kpoints.wk[ik] * float(np.dot(Ham.Focc[:, ik], enl))
    return E


def calc_E_local(Ham, Rhoe):
    """calc_energies.jl:245-274 (+ calc_E_xc :276-333 for VWN and PBE)."""
    dVol = Ham.pw.CellVolume / Ham.pw.Npoints
    E_Hartree = 0.5 * float(np.dot(Ham.V_Hartree, Rhoe)) * dVol
    E_Ps_loc = float(np.dot(Ham.V_Ps_loc, Rhoe)) * dVol
    if getattr(Ham, "xcfunc", "VWN") == "PBE":
        from .pbe import calc_epsxc_PBE
        epsxc = calc_epsxc_PBE(Ham.pw, Rhoe)
    else:
        epsxc = calc_epsxc_VWN(Rhoe)
    E_xc = float(np.sum(epsxc * Rhoe)) * dVol
    return E_Ps_loc, E_Hartree, E_xc


def calc_E_NN(LatVecs, positions, atm2species, Zvals):
    """calc_E_NN.jl:60-172 (Ewald sum, returned in Hartree)."""
    t = [LatVecs[:, i] for i in range(3)]
    Omega = abs(np.linalg.det(LatVecs))
    RecVecs = 2 * np.pi * np.linalg.inv(LatVecs.T)
    g = [RecVecs[:, i] for i in range(3)]
    tm = [math.sqrt(float(np.dot(v, v))) for v in t]
    gm = [math.sqrt(float(np.dot(v, v))) for v in g]
    Natoms = positions.shape[1]
    gcut, ebsl = 2.0, 1e-8
    glast2 = gcut * gcut
    gexp = -math.log(ebsl)
    eta = math.sqrt(glast2 / gexp) / 2
    Z = np.array([Zvals[atm2species[ia]] for ia in range(Natoms)])
    x = float(np.sum(Z ** 2))
    totalcharge = float(np.sum(Z))
    ewald = -2 * eta * x / math.sqrt(math.pi) - math.pi * totalcharge ** 2 / (Omega * eta ** 2)
    tmax = math.sqrt(0.5 * gexp) / eta
    m = [int(round(tmax / tm[i] + 1.5)) for i in range(3)]
    ii, jj, kk = np.meshgrid(np.arange(-m[0], m[0] + 1), np.arange(-m[1], m[1] + 1),
                             np.arange(-m[2], m[2] + 1), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    T = np.outer(t[0], ii) + np.outer(t[1], jj) + np.outer(t[2], kk)
    origin = (np.abs(ii) + np.abs(jj) + np.abs(kk)) == 0
    for ia in range(Natoms):
        for ja in range(Natoms):
            d = positions[:, ia] - positions[:, ja]
            r = np.sqrt(((d[:, None] - T) ** 2).sum(axis=0))
            keep = ~origin if ia == ja else np.ones_like(origin)
            ewald += Z[ia] * Z[ja] * float(np.sum(erfc(r[keep] * eta) / r[keep]))
    m = [int(round(gcut / gm[i] + 1.5)) for i in range(3)]
    ii, jj, kk = np.meshgrid(np.arange(-m[0], m[0] + 1), np.arange(-m[1], m[1] + 1),
                             np.arange(-m[2], m[2] + 1), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    keep = (np.abs(ii) + np.abs(jj) + np.abs(kk)) != 0
    Gv = (np.outer(g[0], ii) + np.outer(g[1], jj) + np.outer(g[2], kk))[:, keep]
    G2 = (Gv ** 2).sum(axis=0)
    xg = 4 * np.pi / Omega * np.exp(-0.25 * G2 / eta ** 2) / G2
    for ia in range(Natoms):
        for ja in range(Natoms):
            d = positions[:, ia] - positions[:, ja]
            ewald += float(np.sum(xg * Z[ia] * Z[ja] * np.cos(d @ Gv)))
    return ewald * 0.5


def calc_energies(Ham, psiks, Rhoe):
    """calc_energies.jl:457-492.  Returns a dict of components; 'Total'
    follows Energies.jl:30-34 (the free energy: mTS, Ham.mTS, is added when
    smearing set it, and is 0 otherwise)."""
    E = {}
    E["Kinetic"] = calc_E_kin(Ham, psiks)
    E["Ps_loc"], E["Hartree"], E["XC"] = calc_E_local(Ham, Rhoe)
    E["Ps_nloc"] = calc_E_Ps_nloc(Ham, psiks) if Ham.NbetaNL > 0 else 0.0
    if Ham.E_NN is None:
        Ham.E_NN = calc_E_NN(Ham.atoms.LatVecs, Ham.atoms.positions, Ham.atoms.atm2species, Ham.Zvals)
    E["NN"] = Ham.E_NN
    E["mTS"] = getattr(Ham, "mTS", 0.0)
    E["Total"] = E["Kinetic"] + E["Ps_loc"] + E["Ps_nloc"] + E["Hartree"] + E["XC"] + E["NN"] + E["mTS"]
    return E
