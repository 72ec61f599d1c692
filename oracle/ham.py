"""Hamiltonian set-up, local potentials, XC and density guess.

Oracle (test infrastructure only).  Restates PWDFT.jl:
  Hamiltonian.jl:41-302, 337-405   constructor (GTH, dual=4, collinear)
  Hamiltonian.jl:510-545           update! (Nspin = 1)
  calc_strfact.jl:2-16             structure factor
  PsPotNL.jl:16-77, 147-195        betaNL and the prj2beta ordering
  Electrons.jl:120-262             Nstates / Focc
  guess_rhoe.jl:1-49, 208-308      gaussian starting density, atmlength
  Poisson_solve.jl:22-40           Poisson_solve!
  XC_funcs/XC_x_slater.jl, XC_funcs/XC_c_vwn.jl, LDA_VWN_internal.jl:33-52
"""
import os
import numpy as np
import scipy.fft as sfft

from .pwgrid import PWGrid, gen_kpoint_grid
from .gth import PsPot_GTH, eval_Vloc_G, eval_proj_G, Ylm_real, ZATOMS

WORKERS = os.cpu_count() or 1


def G_to_R(Ns, fG):
    """wrappers_fft.jl:114-123: backward FFT normalised by 1/N (ifft).
    fG is a flat array in the grid order ip = i + N1*(j + N2*k)."""
    N1, N2, N3 = Ns
    a = np.asarray(fG, dtype=np.complex128).reshape(fG.shape[:-1] + (N3, N2, N1))
    out = sfft.ifftn(a, axes=(-3, -2, -1), workers=WORKERS)
    return out.reshape(fG.shape)


def R_to_G(Ns, fR):
    """wrappers_fft.jl:125-134: forward FFT, unnormalised."""
    N1, N2, N3 = Ns
    a = np.asarray(fR, dtype=np.complex128).reshape(fR.shape[:-1] + (N3, N2, N1))
    out = sfft.fftn(a, axes=(-3, -2, -1), workers=WORKERS)
    return out.reshape(fR.shape)


class Atoms:
    """Atoms.jl:5-15.  positions: (3, Natoms) Cartesian bohr."""

    def __init__(self, symbols, positions, LatVecs):
        self.LatVecs = np.array(LatVecs, dtype=np.float64)
        self.positions = np.array(positions, dtype=np.float64)
        self.Natoms = self.positions.shape[1]
        self.atsymbs = list(symbols)
        species = []
        for s in symbols:
            if s not in species:
                species.append(s)
        self.SpeciesSymbols = species
        self.Nspecies = len(species)
        self.atm2species = np.array([species.index(s) for s in symbols], dtype=np.int64)

    @classmethod
    def from_frac(cls, symbols, frac, LatVecs):
        """Atoms.jl:56-60: positions = LatVecs * frac."""
        LatVecs = np.array(LatVecs, dtype=np.float64)
        return cls(symbols, LatVecs @ np.array(frac, dtype=np.float64), LatVecs)


def calc_strfact(positions, Nspecies, atm2species, G):
    """calc_strfact.jl:2-16 -> (Ng, Nspecies) complex."""
    Sf = np.zeros((G.shape[1], Nspecies), dtype=np.complex128)
    for ia in range(positions.shape[1]):
        GX = positions[0, ia] * G[0] + positions[1, ia] * G[1] + positions[2, ia] * G[2]
        Sf[:, atm2species[ia]] += np.cos(GX) - 1j * np.sin(GX)
    return Sf


def init_prj2beta(atoms, pspots):
    """PsPotNL.jl:147-195.  Returns NbetaNL and a dict
    (iprj, ia, l, m) -> ibeta (all 0-based) in the reference's order:
    atom, then l, then m, then projector."""
    prj2beta = {}
    n = 0
    for ia in range(atoms.Natoms):
        psp = pspots[atoms.atm2species[ia]]
        for l in range(psp.lmax + 1):
            for m in range(-l, l + 1):
                for iprj in range(psp.Nproj_l[l]):
                    prj2beta[(iprj, ia, l, m)] = n
                    n += 1
    return n, prj2beta


def nonlocal_triplets(atoms, pspots, prj2beta):
    """The (ibeta, jbeta, h_ij) entries visited by op_V_Ps_nloc.jl:59-76,
    in the reference's loop order."""
    trip = []
    for ia in range(atoms.Natoms):
        psp = pspots[atoms.atm2species[ia]]
        for l in range(psp.lmax + 1):
            for m in range(-l, l + 1):
                for iprj in range(psp.Nproj_l[l]):
                    for jprj in range(psp.Nproj_l[l]):
                        trip.append((prj2beta[(iprj, ia, l, m)], prj2beta[(jprj, ia, l, m)],
                                     psp.h[l, iprj, jprj]))
    return trip


def calc_betaNL(atoms, pspots, pw, prj2beta, NbetaNL):
    """PsPotNL.jl:40-69: betaNL[ik][igk, ibeta] =
    (-i)^l Ylm_real(l,m,G+k) eval_proj_G(l,iprj,|G+k|) exp(-i (G+k).tau_a)."""
    betaNL = []
    G = pw.gvec.G
    for ik in range(pw.kpoints.Nkpt):
        idx = pw.gvecw.idx_gw2g[ik]
        k = pw.kpoints.k[:, ik]
        g = G[:, idx] + k[:, None]
        Gm = np.sqrt(g[0] ** 2 + g[1] ** 2 + g[2] ** 2)
        B = np.zeros((len(idx), NbetaNL), dtype=np.complex128)
        for ia in range(atoms.Natoms):
            psp = pspots[atoms.atm2species[ia]]
            tau = atoms.positions[:, ia]
            GX = tau[0] * g[0] + tau[1] * g[1] + tau[2] * g[2]
            Sf = np.cos(GX) - 1j * np.sin(GX)
            for l in range(psp.lmax + 1):
                for m in range(-l, l + 1):
                    ylm = Ylm_real(l, m, g)
                    for iprj in range(psp.Nproj_l[l]):
                        ib = prj2beta[(iprj, ia, l, m)]
                        B[:, ib] = ((-1j) ** l) * ylm * eval_proj_G(psp, l, iprj + 1, Gm, pw.CellVolume) * Sf
        betaNL.append(B)
    return betaNL


def atmlength(zion, znucl):
    """guess_rhoe.jl:208-308 (densty = 0)."""
    coreel = znucl - zion
    nval = int(round(zion))
    if nval == 0:
        return 0.0
    if coreel < 0.5:
        tab, dflt = [0.6, 0.4, 0.3, 0.25], 0.2
    elif coreel < 2.5:
        tab, dflt = [1.8, 1.4, 1.0, 0.7, 0.6, 0.5, 0.4, 0.35], 0.3
    elif coreel < 10.5:
        tab, dflt = [2.0, 1.6, 1.25, 1.1, 1.0, 0.9, 0.8, 0.7, 0.7, 0.7], 0.6
    elif coreel < 12.5:
        tab, dflt = [1.9, 1.5, 1.15, 1.0, 0.9, 0.8, 0.7, 0.6, 0.6, 0.6], 0.5
    elif coreel < 18.5:
        tab, dflt = [2.0, 1.8, 1.5, 1.2, 1.0, 0.9, 0.85, 0.8, 0.75, 0.7, 0.65, 0.65], 0.6
    elif coreel < 28.5:
        tab, dflt = [1.5, 1.25, 1.15, 1.05, 1.00, 0.95, 0.95, 0.9, 0.9, 0.85, 0.85, 0.80, 0.8, 0.75], 0.7
    elif coreel < 36.5:
        tab, dflt = [2.0, 2.00, 1.60, 1.40, 1.25, 1.10, 1.00, 0.95, 0.90, 0.85, 0.80, 0.75], 0.7
    else:
        tab, dflt = [2.0, 2.00, 1.55, 1.25, 1.15, 1.10, 1.05, 1.0, 0.95, 0.9, 0.85, 0.85], 0.8
    return tab[nval - 1] if nval <= len(tab) else dflt


# ---------------------------------------------------------------- XC (LDA)

def xc_x_slater(rho):
    """XC_funcs/XC_x_slater.jl:1-18 (vectorised)."""
    rho = np.asarray(rho, dtype=np.float64)
    ok = rho > 1e-10
    pi34 = 0.6203504908994
    with np.errstate(divide="ignore", invalid="ignore"):
        rs = pi34 / np.cbrt(np.where(ok, rho, 1.0))
    f = -0.687247939924714
    alpha = 2.0 / 3.0
    ex = np.where(ok, f * alpha / rs, 0.0)
    vx = np.where(ok, 4.0 / 3.0 * f * alpha / rs, 0.0)
    return ex, vx


def xc_c_vwn(rho):
    """XC_funcs/XC_c_vwn.jl:1-28 (vectorised; no low-density cutoff)."""
    rho = np.asarray(rho, dtype=np.float64)
    pi34 = 0.6203504908994
    rs = pi34 / np.cbrt(rho)
    a, b, c, x0 = 0.0310907, 3.72744, 12.9352, -0.10498
    q = np.sqrt(4.0 * c - b * b)
    f1 = 2.0 * b / q
    f2 = b * x0 / (x0 * x0 + b * x0 + c)
    f3 = 2.0 * (2.0 * x0 + b) / q
    rs12 = np.sqrt(rs)
    fx = rs + b * rs12 + c
    qx = np.arctan(q / (2.0 * rs12 + b))
    ec = a * (np.log(rs / fx) + f1 * qx - f2 * (np.log((rs12 - x0) ** 2 / fx) + f3 * qx))
    tx = 2.0 * rs12 + b
    tt = tx * tx + q * q
    vc = ec - rs12 * a / 6.0 * (2.0 / rs12 - tx / fx - 4.0 * b / tt
                                - f2 * (2.0 / (rs12 - x0) - tx / fx - 4.0 * (2.0 * x0 + b) / tt))
    return ec, vc


def calc_epsxc_VWN(rho):
    """LDA_VWN_internal.jl:33-41."""
    return xc_x_slater(rho)[0] + xc_c_vwn(rho)[0]


def calc_Vxc_VWN(rho):
    """LDA_VWN_internal.jl:44-52."""
    return xc_x_slater(rho)[1] + xc_c_vwn(rho)[1]


# -------------------------------------------------------------- Hamiltonian

class Hamiltonian:
    """Hamiltonian.jl:41-302 / 337-405 for GTH pseudopotentials, dual = 4,
    Nspin_wf = Nspin_dens = 1, xcfunc = "VWN" or "PBE" (internal formulas,
    Hamiltonian.jl:270-277)."""

    def __init__(self, atoms, pspfiles, ecutwfc, meshk=(1, 1, 1), extra_states=None,
                 Nstates=None, kpoints=None, Ns=None, xcfunc="VWN", use_symmetry=False):
        if xcfunc not in ("VWN", "PBE"):
            raise ValueError("xcfunc must be 'VWN' or 'PBE'")
        self.xcfunc = xcfunc
        self.atoms = atoms
        self.pspots = [PsPot_GTH(f) for f in pspfiles]
        for isp, s in enumerate(atoms.SpeciesSymbols):
            if self.pspots[isp].atsymb != s:
                raise ValueError("pseudopotential order does not match species")
        self.sym = None
        if use_symmetry:
            # Hamiltonian.jl:53-85: SymmetryInfo(atoms), k-points reduced by its rotations
            from .symmetry import SymmetryInfo, gen_kpoint_grid as gen_sym_grid
            from .pwgrid import KPoints, recvecs_of
            self.sym = SymmetryInfo(atoms.LatVecs, atoms.positions, atoms.atm2species)
            if kpoints is None:
                nk, xk, wk, _ = gen_sym_grid(atoms.LatVecs, meshk, self.sym.s)
                kpoints = KPoints(nk, tuple(meshk), xk, wk, recvecs_of(atoms.LatVecs))
        if kpoints is None:
            if tuple(meshk) == (1, 1, 1):
                kpoints = None
            else:
                kpoints = gen_kpoint_grid(atoms.LatVecs, meshk)
        self.pw = pw = PWGrid(ecutwfc, atoms.LatVecs, kpoints=kpoints, Ns=Ns)
        if self.sym is not None and self.sym.Nsyms > 1:
            from .symmetry import RhoeSymmetrizer
            self.symz = RhoeSymmetrizer(atoms.LatVecs, pw.gvec.G, self.sym)
        self.Zvals = np.array([float(p.zval) for p in self.pspots])
        N = pw.Npoints
        # local pseudopotential: Hamiltonian.jl:113-141
        strf = calc_strfact(atoms.positions, atoms.Nspecies, atoms.atm2species, pw.gvec.G)
        Vg = np.zeros(N, dtype=np.complex128)
        for isp in range(atoms.Nspecies):
            Vgl = eval_Vloc_G(self.pspots[isp], pw.gvec.G2_shells)
            np.add.at(Vg, pw.gvec.idx_g2r, strf[:, isp] * Vgl[pw.gvec.idx_g2shells] / pw.CellVolume)
        self.V_Ps_loc = np.real(G_to_R(pw.Ns, Vg)) * N
        self.strf = strf
        # electrons: Electrons.jl:120-262 (Nspin_wf = 1, no smearing)
        Nel = float(sum(self.Zvals[atoms.atm2species]))
        self.Nelectrons = Nel
        nmin = int(round(Nel / 2))
        if nmin * 2 < Nel:
            nmin += 1
        if Nstates is None:
            Nstates = nmin + (extra_states or 0)
        self.Nstates = Nstates
        self.Nstates_occ = nmin
        Nkpt = pw.kpoints.Nkpt
        Focc = np.zeros((Nstates, Nkpt))
        Focc[:nmin - 1, :] = 2.0
        Focc[nmin - 1, :] = 1.0 if int(round(Nel)) % 2 == 1 else 2.0
        self.Focc = Focc
        # nonlocal projectors
        self.NbetaNL, self.prj2beta = init_prj2beta(atoms, self.pspots)
        self.nl_triplets = nonlocal_triplets(atoms, self.pspots, self.prj2beta)
        self.betaNL = calc_betaNL(atoms, self.pspots, pw, self.prj2beta, self.NbetaNL)
        D = np.zeros((self.NbetaNL, self.NbetaNL))
        for ib, jb, h in self.nl_triplets:
            D[ib, jb] += h
        self.Dnl = D
        # potentials
        self.V_Hartree = np.zeros(N)
        self.V_xc = np.zeros(N)
        self.V_Total = np.zeros(N)
        self.ik = 0
        self.ispin = 0
        self.E_NN = None

    # ------------------------------------------------------------ update!
    def update(self, Rhoe):
        """Hamiltonian.jl:510-545 (Nspin = 1)."""
        self.V_Hartree = Poisson_solve(self.pw, Rhoe)
        if self.xcfunc == "PBE":
            from .pbe import calc_Vxc_PBE
            self.V_xc = calc_Vxc_PBE(self.pw, Rhoe)
        else:
            self.V_xc = calc_Vxc_VWN(Rhoe)
        self.V_Total = self.V_Ps_loc + self.V_Hartree + self.V_xc

    def guess_rhoe(self):
        """guess_rhoe.jl:1-38."""
        pw, atoms = self.pw, self.atoms
        RhoeG = np.zeros(pw.Npoints, dtype=np.complex128)
        for ia in range(atoms.Natoms):
            isp = atoms.atm2species[ia]
            psp = self.pspots[isp]
            L = atmlength(float(psp.zval), float(ZATOMS[psp.atsymb]))
            np.add.at(RhoeG, pw.gvec.idx_g2r, psp.zval * self.strf[:, isp] * np.exp(-pw.gvec.G2 * L ** 2))
        Rhoe = np.real(G_to_R(pw.Ns, RhoeG))
        intRhoe = Rhoe.sum() * pw.CellVolume / pw.Npoints
        return Rhoe * self.Nelectrons / intRhoe


def Poisson_solve(pw, rhoR):
    """Poisson_solve.jl:22-40."""
    ctmp = R_to_G(pw.Ns, rhoR.astype(np.complex128))
    ctmp[0] = 0.0
    ip = pw.gvec.idx_g2r[1:]
    ctmp[ip] = 4 * np.pi * ctmp[ip] / pw.gvec.G2[1:]
    return np.real(G_to_R(pw.Ns, ctmp))
