"""Host-side Hamiltonian set-up for the device path.

In the deployment this is PWDFT.jl's own job (the Julia constructor
Hamiltonian(atoms, pspfiles, ecutwfc; ...), Hamiltonian.jl:337-405, runs on
the host and hands its index maps, potentials and projectors to the C ABI).
Python stands in for Julia here, so this module restates the set-up that the
operators need -- once per geometry, off the hot path:

  basis        FFT grid (PWGrid.jl:84-95), G-sphere and per-k sphere maps
               computed by libpwb200's bit-exact C++ builders
               (pw_gvec_build / pw_gvecw_build)
  GTH          file parser and the G-space formulas of PsPot_GTH.jl
               (:43-118, :164-189, :338-391) and Ylm_real.jl:5-107
  V_Ps_loc     Hamiltonian.jl:113-141
  betaNL, h_ij PsPotNL.jl:40-69, 147-195 and op_V_Ps_nloc.jl:59-76
"""
import ctypes as C
import math

import numpy as np

from ._lib import lib, check
from .context import Context

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)


# ------------------------------------------------------------------ basis
def grid_size(LatVecs, ecutrho):
    """PWGrid.jl:79-92 with good_fft_order from the library."""
    L = lib()
    Ns = []
    for i in range(3):
        n = 2 * int(round(math.sqrt(ecutrho / 2) * float(np.linalg.norm(LatVecs[:, i])) / math.pi)) + 1
        Ns.append(L.pw_good_fft_order(n))
    return tuple(Ns)


class Basis:
    """G-vectors of the density sphere and per-k wavefunction spheres."""

    def __init__(self, LatVecs, ecutwfc, kpts=None, Ns=None):
        L = lib()
        self.LatVecs = np.array(LatVecs, dtype=np.float64)
        self.ecutwfc = float(ecutwfc)
        self.ecutrho = 4.0 * self.ecutwfc
        self.RecVecs = 2 * np.pi * np.linalg.inv(np.ascontiguousarray(self.LatVecs.T))
        self.CellVolume = abs(float(np.linalg.det(self.LatVecs)))
        self.Ns = tuple(Ns) if Ns is not None else grid_size(self.LatVecs, self.ecutrho)
        self.Npoints = int(np.prod(self.Ns))
        Ns32 = (C.c_int32 * 3)(*self.Ns)
        R = np.asfortranarray(self.RecVecs)
        Ng = C.c_int64()
        check(L.pw_gvec_count(Ns32, R.ctypes.data_as(_dp), self.ecutrho, C.byref(Ng)))
        self.Ng = Ng.value
        self.G = np.zeros((self.Ng, 3))
        self.G2 = np.zeros(self.Ng)
        self.idx_g2r = np.zeros(self.Ng, dtype=np.int64)
        check(L.pw_gvec_build(Ns32, R.ctypes.data_as(_dp), self.ecutrho, self.Ng, self.G.ctypes.data_as(_dp),
                              self.G2.ctypes.data_as(_dp), self.idx_g2r.ctypes.data_as(_i64p)))
        if kpts is None:
            kpts = np.zeros((3, 1))
        self.kpts = np.asarray(kpts, dtype=np.float64).reshape(3, -1)
        self.Nkpt = self.kpts.shape[1]
        self.idx_gw2g, self.idx_gw2r, self.Gk2, self.Ngw = [], [], [], []
        for ik in range(self.Nkpt):
            kp = np.ascontiguousarray(self.kpts[:, ik])
            n = C.c_int64()
            i2g = np.zeros(self.Ng, dtype=np.int64)
            i2r = np.zeros(self.Ng, dtype=np.int64)
            g2 = np.zeros(self.Ng)
            check(L.pw_gvecw_build(self.Ng, self.G.ctypes.data_as(_dp), self.idx_g2r.ctypes.data_as(_i64p),
                                   kp.ctypes.data_as(_dp), self.ecutwfc, C.byref(n), i2g.ctypes.data_as(_i64p),
                                   i2r.ctypes.data_as(_i64p), g2.ctypes.data_as(_dp)))
            self.idx_gw2g.append(i2g[:n.value].copy())
            self.idx_gw2r.append(i2r[:n.value].copy())
            self.Gk2.append(g2[:n.value].copy())
            self.Ngw.append(n.value)
        # shells (PWGrid.jl:245-275)
        new = np.empty(self.Ng, dtype=bool)
        new[0] = False
        new[1:] = self.G2[1:] > self.G2[:-1] + 1e-8
        self.idx_g2shells = np.cumsum(new)
        self.G2_shells = np.concatenate([[self.G2[0]], self.G2[1:][new[1:]]])


# -------------------------------------------------------------------- GTH
class GTH:
    """PsPot_GTH.jl:43-118."""

    def __init__(self, filename):
        with open(filename) as f:
            tok = [ln.split() for ln in f.read().splitlines()]
        self.atsymb = tok[0][0]
        self.zval = sum(int(x) for x in tok[1][:4])
        self.rlocal = float(tok[2][0])
        nc = int(tok[2][1])
        self.c = np.zeros(4)
        self.c[:nc] = [float(x) for x in tok[3][:nc]]
        self.lmax = int(tok[4][0]) - 1
        self.rc = np.zeros(4)
        self.Nproj_l = np.zeros(4, dtype=np.int64)
        self.h = np.zeros((4, 3, 3))
        row = 5
        for l in range(self.lmax + 1):
            self.rc[l] = float(tok[row][0])
            self.Nproj_l[l] = int(float(tok[row][1]))
            row += 1
            for ii in range(self.Nproj_l[l]):
                vals = [float(x) for x in tok[row]]
                row += 1
                for k, jj in enumerate(range(ii, self.Nproj_l[l])):
                    self.h[l, ii, jj] = self.h[l, jj, ii] = vals[k]

    def vloc_G(self, G2):
        """PsPot_GTH.jl:164-189."""
        rl, z = self.rlocal, self.zval
        c1, c2, c3, c4 = self.c
        Gr = np.sqrt(G2) * rl
        e = np.exp(-0.5 * Gr * Gr)
        with np.errstate(divide="ignore", invalid="ignore"):
            v = (-4 * np.pi * z) / G2 * e + math.sqrt(8 * np.pi ** 3) * rl ** 3 * e * (
                c1 + c2 * (3.0 - Gr ** 2) + c3 * (15.0 - 10.0 * Gr ** 2 + Gr ** 4)
                + c4 * (105.0 - 105.0 * Gr ** 2 + 21.0 * Gr ** 4 - Gr ** 6))
        v0 = 2 * np.pi * z * rl ** 2 + (2 * np.pi) ** 1.5 * rl ** 3 * (c1 + 3.0 * c2 + 15.0 * c3 + 105.0 * c4)
        return np.where(np.sqrt(np.sqrt(G2)) > 1e-8, v, v0)

    def proj_G(self, l, i, Gm, Omega):
        """PsPot_GTH.jl:338-391 (i is 1-based)."""
        r = self.rc[l]
        x = (Gm * r) ** 2
        e = np.exp(-0.5 * x)
        poly = {
            (0, 1): e, (0, 2): 2.0 / math.sqrt(15.0) * e * (3.0 - x),
            (0, 3): (4.0 / 3.0) / math.sqrt(105.0) * e * (15.0 - 10.0 * x + x * x),
            (1, 1): e * Gm / math.sqrt(3.0), (1, 2): 2.0 / math.sqrt(105.0) * e * Gm * (5.0 - x),
            (1, 3): (4.0 / 3.0) / math.sqrt(1155.0) * e * Gm * (35.0 - 14.0 * x + x * x),
            (2, 1): e * Gm ** 2 / math.sqrt(15.0), (2, 2): (2.0 / 3.0) / math.sqrt(105.0) * e * Gm ** 2 * (7.0 - x),
            (3, 1): Gm ** 3 * e / math.sqrt(105.0),
        }[(l, i)]
        return 4.0 * np.pi ** 1.25 * math.sqrt(2.0 ** (l + 1) * r ** (2 * l + 3) / Omega) * poly


def ylm_real(l, m, g):
    """Ylm_real.jl:5-107 (g: (n, 3))."""
    x, y, z = g[:, 0], g[:, 1], g[:, 2]
    rr = np.sqrt(x * x + y * y + z * z)
    with np.errstate(divide="ignore", invalid="ignore"):
        ct = np.where(rr < 1e-9, 0.0, z / rr)
        at = np.arctan(y / x)
    phi = np.where(x > 1e-9, at, np.where(x < -1e-9, at + np.pi, np.where(y >= 0, np.pi / 2, -np.pi / 2)))
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    s, c = np.sin, np.cos
    table = {
        (0, 0): lambda: np.full_like(x, 0.5 * math.sqrt(1.0 / np.pi)),
        (1, -1): lambda: 0.5 * math.sqrt(3.0 / np.pi) * st * s(phi),
        (1, 0): lambda: 0.5 * math.sqrt(3.0 / np.pi) * ct,
        (1, 1): lambda: 0.5 * math.sqrt(3.0 / np.pi) * st * c(phi),
        (2, -2): lambda: math.sqrt(15.0 / 16.0 / np.pi) * st ** 2 * s(2 * phi),
        (2, -1): lambda: math.sqrt(15.0 / 4.0 / np.pi) * ct * st * s(phi),
        (2, 0): lambda: 0.25 * math.sqrt(5.0 / np.pi) * (3.0 * ct ** 2 - 1.0),
        (2, 1): lambda: math.sqrt(15.0 / 4.0 / np.pi) * ct * st * c(phi),
        (2, 2): lambda: math.sqrt(15.0 / 16.0 / np.pi) * st ** 2 * c(2 * phi),
        (3, -3): lambda: 0.25 * math.sqrt(35.0 / 2.0 / np.pi) * st ** 3 * s(3 * phi),
        (3, -2): lambda: 0.25 * math.sqrt(105.0 / np.pi) * st ** 2 * ct * s(2 * phi),
        (3, -1): lambda: 0.25 * math.sqrt(21.0 / 2.0 / np.pi) * st * (5.0 * ct ** 2 - 1.0) * s(phi),
        (3, 0): lambda: 0.25 * math.sqrt(7.0 / np.pi) * (5.0 * ct ** 3 - 3.0 * ct),
        (3, 1): lambda: 0.25 * math.sqrt(21.0 / 2.0 / np.pi) * st * (5.0 * ct ** 2 - 1.0) * c(phi),
        (3, 2): lambda: 0.25 * math.sqrt(105.0 / np.pi) * st ** 2 * ct * c(2 * phi),
        (3, 3): lambda: 0.25 * math.sqrt(35.0 / 2.0 / np.pi) * st ** 3 * c(3 * phi),
    }
    return table[(l, m)]()


# ------------------------------------------------------------- Hamiltonian
class System:
    """Atoms (Cartesian bohr, (3, Natoms)) + species + lattice."""

    def __init__(self, symbols, positions, LatVecs):
        self.symbols = list(symbols)
        self.positions = np.array(positions, dtype=np.float64)
        self.LatVecs = np.array(LatVecs, dtype=np.float64)
        self.species = []
        for s in symbols:
            if s not in self.species:
                self.species.append(s)
        self.atm2species = np.array([self.species.index(s) for s in symbols])


def local_potential(system, basis, pspots):
    """V_Ps_loc(r) (Hamiltonian.jl:113-141)."""
    G = basis.G
    Vg = np.zeros(basis.Npoints, dtype=np.complex128)
    for isp in range(len(system.species)):
        Vgl = pspots[isp].vloc_G(basis.G2_shells)[basis.idx_g2shells]
        sf = np.zeros(basis.Ng, dtype=np.complex128)
        for ia in np.nonzero(system.atm2species == isp)[0]:
            GX = G @ system.positions[:, ia]
            sf += np.cos(GX) - 1j * np.sin(GX)
        Vg[basis.idx_g2r] += sf * Vgl / basis.CellVolume
    N1, N2, N3 = basis.Ns
    V = np.fft.ifftn(Vg.reshape(N3, N2, N1)).real.ravel() * basis.Npoints
    return V


def projector_table(system, basis, pspots):
    """The column table of betaNL in the reference's (atom, l, m, iprj) order
    (PsPotNL.jl:147-195) for pw_build_nonlocal: atom, l, m, iproj (1-based),
    r_l, and eval_proj_G's normalisation 4 pi^(5/4) sqrt(2^(l+1) r_l^(2l+3)
    / Omega); plus the (ibeta, jbeta, h_ij) list (op_V_Ps_nloc.jl:59-76)."""
    cols, trip = [], []
    for ia in range(system.positions.shape[1]):
        psp = pspots[system.atm2species[ia]]
        for l in range(psp.lmax + 1):
            r = psp.rc[l]
            pref = 4.0 * np.pi ** 1.25 * math.sqrt(2.0 ** (l + 1) * r ** (2 * l + 3) / basis.CellVolume)
            for m in range(-l, l + 1):
                first = len(cols)
                for i in range(psp.Nproj_l[l]):
                    cols.append((ia, l, m, i + 1, r, pref))
                for i in range(psp.Nproj_l[l]):
                    for j in range(psp.Nproj_l[l]):
                        trip.append((first + i, first + j, psp.h[l, i, j]))
    t = np.array(cols, dtype=object).reshape(-1, 6) if cols else np.zeros((0, 6), dtype=object)
    table = {"atom": t[:, 0].astype(np.int32), "l": t[:, 1].astype(np.int32), "m": t[:, 2].astype(np.int32),
             "iproj": t[:, 3].astype(np.int32), "rc": t[:, 4].astype(np.float64), "pref": t[:, 5].astype(np.float64)}
    return table, trip


def projectors(system, basis, pspots, ik):
    """betaNL[ik] (Ngw, NbetaNL) and the (ibeta, jbeta, h_ij) list
    (PsPotNL.jl:40-69, 147-195; op_V_Ps_nloc.jl:59-76)."""
    g = basis.G[basis.idx_gw2g[ik]] + basis.kpts[:, ik][None, :]
    Gm = np.sqrt((g * g).sum(axis=1))
    cols, trip = [], []
    nb = 0
    for ia in range(system.positions.shape[1]):
        psp = pspots[system.atm2species[ia]]
        GX = g @ system.positions[:, ia]
        sf = np.cos(GX) - 1j * np.sin(GX)
        for l in range(psp.lmax + 1):
            for m in range(-l, l + 1):
                y = ylm_real(l, m, g)
                first = nb
                for i in range(psp.Nproj_l[l]):
                    cols.append(((-1j) ** l) * y * psp.proj_G(l, i + 1, Gm, basis.CellVolume) * sf)
                    nb += 1
                for i in range(psp.Nproj_l[l]):
                    for j in range(psp.Nproj_l[l]):
                        trip.append((first + i, first + j, psp.h[l, i, j]))
    beta = np.stack(cols, axis=1) if cols else np.zeros((len(Gm), 0), dtype=np.complex128)
    return beta, trip


ZATOMS = {"H": 1, "He": 2, "Li": 3, "C": 6, "N": 7, "O": 8, "Na": 11, "Mg": 12, "Al": 13, "Si": 14, "P": 15,
          "S": 16, "Cl": 17, "Ga": 31, "Ge": 32, "Pt": 78}


def kpoint_grid(LatVecs, mesh, time_reversal=True):
    """Gamma-centred Monkhorst-Pack grid reduced by k ~ -k only
    (KPoints.jl:121-260 with the identity as the only rotation).
    Returns Cartesian k (3, Nk) and weights summing to one."""
    n1, n2, n3 = mesh
    frac = np.array([[i / n1, j / n2, k / n3] for i in range(n1) for j in range(n2) for k in range(n3)])
    frac = frac - np.round(frac)
    keys = {}
    order, weight = [], []
    for f in frac:
        key = tuple(np.round(f * np.array(mesh)).astype(int) % np.array(mesh))
        mkey = tuple((-np.array(key)) % np.array(mesh))
        if key in keys:
            weight[keys[key]] += 1.0
        elif time_reversal and mkey in keys:
            weight[keys[mkey]] += 1.0
        else:
            keys[key] = len(order)
            order.append(f)
            weight.append(1.0)
    RecVecs = 2 * np.pi * np.linalg.inv(np.ascontiguousarray(np.asarray(LatVecs).T))
    k = RecVecs @ np.array(order).T
    w = np.array(weight)
    return k, w / w.sum()


def atmlength(zion, znucl):
    """Default decay length of the Gaussian starting density (guess_rhoe.jl:208-308)."""
    coreel, nval = znucl - zion, int(round(zion))
    tables = [(0.5, [0.6, 0.4, 0.3, 0.25], 0.2), (2.5, [1.8, 1.4, 1.0, 0.7, 0.6, 0.5, 0.4, 0.35], 0.3),
              (10.5, [2.0, 1.6, 1.25, 1.1, 1.0, 0.9, 0.8, 0.7, 0.7, 0.7], 0.6),
              (12.5, [1.9, 1.5, 1.15, 1.0, 0.9, 0.8, 0.7, 0.6, 0.6, 0.6], 0.5),
              (18.5, [2.0, 1.8, 1.5, 1.2, 1.0, 0.9, 0.85, 0.8, 0.75, 0.7, 0.65, 0.65], 0.6),
              (28.5, [1.5, 1.25, 1.15, 1.05, 1.00, 0.95, 0.95, 0.9, 0.9, 0.85, 0.85, 0.80, 0.8, 0.75], 0.7),
              (36.5, [2.0, 2.00, 1.60, 1.40, 1.25, 1.10, 1.00, 0.95, 0.90, 0.85, 0.80, 0.75], 0.7),
              (1e9, [2.0, 2.00, 1.55, 1.25, 1.15, 1.10, 1.05, 1.0, 0.95, 0.9, 0.85, 0.85], 0.8)]
    if nval == 0:
        return 0.0
    for lim, tab, dflt in tables:
        if coreel < lim:
            return tab[nval - 1] if nval <= len(tab) else dflt


def guess_rhoe(system, basis, pspots, Nelectrons):
    """Superposition of atomic Gaussians, normalised to Nelectrons (guess_rhoe.jl:1-38)."""
    rhoG = np.zeros(basis.Npoints, dtype=np.complex128)
    for ia in range(system.positions.shape[1]):
        psp = pspots[system.atm2species[ia]]
        L = atmlength(float(psp.zval), float(ZATOMS[psp.atsymb]))
        GX = basis.G @ system.positions[:, ia]
        rhoG[basis.idx_g2r] += psp.zval * (np.cos(GX) - 1j * np.sin(GX)) * np.exp(-basis.G2 * L * L)
    N1, N2, N3 = basis.Ns
    rho = np.fft.ifftn(rhoG.reshape(N3, N2, N1)).real.ravel()
    return rho * Nelectrons / (rho.sum() * basis.CellVolume / basis.Npoints)


def ewald_energy(LatVecs, positions, Z):
    """Ion-ion (Ewald) energy in Hartree (calc_E_NN.jl:60-172)."""
    from scipy.special import erfc
    t = [LatVecs[:, i] for i in range(3)]
    Omega = abs(np.linalg.det(LatVecs))
    R = 2 * np.pi * np.linalg.inv(LatVecs.T)
    g = [R[:, i] for i in range(3)]
    gcut, ebsl = 2.0, 1e-8
    gexp = -math.log(ebsl)
    eta = math.sqrt(gcut * gcut / gexp) / 2
    e = -2 * eta * float(np.sum(Z ** 2)) / math.sqrt(math.pi) - math.pi * float(np.sum(Z)) ** 2 / (Omega * eta ** 2)
    tmax = math.sqrt(0.5 * gexp) / eta
    m = [int(round(tmax / np.linalg.norm(v) + 1.5)) for v in t]
    ii, jj, kk = [a.ravel() for a in np.meshgrid(*[np.arange(-q, q + 1) for q in m], indexing="ij")]
    T = np.outer(t[0], ii) + np.outer(t[1], jj) + np.outer(t[2], kk)
    origin = (np.abs(ii) + np.abs(jj) + np.abs(kk)) == 0
    nat = positions.shape[1]
    for a in range(nat):
        for b in range(nat):
            r = np.sqrt((((positions[:, a] - positions[:, b])[:, None] - T) ** 2).sum(axis=0))
            keep = ~origin if a == b else np.ones_like(origin)
            e += Z[a] * Z[b] * float(np.sum(erfc(eta * r[keep]) / r[keep]))
    m = [int(round(gcut / np.linalg.norm(v) + 1.5)) for v in g]
    ii, jj, kk = [a.ravel() for a in np.meshgrid(*[np.arange(-q, q + 1) for q in m], indexing="ij")]
    keep = (np.abs(ii) + np.abs(jj) + np.abs(kk)) != 0
    Gv = (np.outer(g[0], ii) + np.outer(g[1], jj) + np.outer(g[2], kk))[:, keep]
    G2 = (Gv ** 2).sum(axis=0)
    xg = 4 * np.pi / Omega * np.exp(-0.25 * G2 / eta ** 2) / G2
    for a in range(nat):
        for b in range(nat):
            e += float(np.sum(xg * Z[a] * Z[b] * np.cos((positions[:, a] - positions[:, b]) @ Gv)))
    return 0.5 * e


class Hamiltonian:
    """Device-resident operator data for one geometry (mirror of the parts
    of PWDFT.jl's Hamiltonian that op_H / calc_rhoe read), plus the hidden
    (ik, ispin) state of the reference (Hamiltonian.jl: Ham.ik, Ham.ispin)."""

    def __init__(self, system, pspfiles, ecutwfc, kpts=None, wk=None, device=0, Ns=None, V_loc=None,
                 xcfunc="VWN", meshk=None, use_symmetry=False, device_projectors=False):
        """kpts (3, Nk) Cartesian with weights wk, or meshk: a Gamma-centred
        Monkhorst-Pack mesh reduced by k ~ -k and, with use_symmetry, by the
        crystal's rotations (Hamiltonian.jl:53-85); symmetry also makes
        calc_rhoe symmetrise the density (calc_rhoe.jl:129-132).
        device_projectors: betaNL evaluated on the device (pw_build_nonlocal)
        instead of on the host."""
        if xcfunc not in ("VWN", "PBE"):
            raise ValueError("xcfunc must be 'VWN' or 'PBE'")
        self.xcfunc = xcfunc
        self.system = system
        self.sym = None
        if use_symmetry:
            from .symmetry import crystal_symmetry
            s, ft = crystal_symmetry(system.LatVecs, system.positions, system.atm2species)
            if s.shape[2] > 1:
                self.sym = (s, ft)
        if meshk is not None and kpts is None:
            if self.sym is not None:
                from .symmetry import kpoint_grid_sym
                kpts, wk = kpoint_grid_sym(system.LatVecs, meshk, self.sym[0])
            else:
                kpts, wk = kpoint_grid(system.LatVecs, meshk)
        self.pspots = [GTH(f) for f in pspfiles]
        self.basis = b = Basis(system.LatVecs, ecutwfc, kpts=kpts, Ns=Ns)
        self.wk = np.ones(b.Nkpt) / b.Nkpt if wk is None else np.asarray(wk, dtype=np.float64)
        self.ctx = Context(b.Ns, b.CellVolume, b.idx_gw2r, b.Gk2, device=device)
        self.V_Ps_loc = local_potential(system, b, self.pspots)
        self.V_Total = self.V_Ps_loc.copy() if V_loc is None else np.asarray(V_loc, dtype=np.float64)
        self.ctx.set_vloc(self.V_Total)
        self.NbetaNL = 0
        if device_projectors:
            table, trip = projector_table(system, b, self.pspots)
            if len(trip) > 0:
                for ik in range(b.Nkpt):
                    self.ctx.set_gkvec(ik, b.G[b.idx_gw2g[ik]] + b.kpts[:, ik][None, :])
                    self.ctx.build_nonlocal(ik, table, system.positions)
                self.NbetaNL = len(table["l"])
                self.nl_triplets = trip
        for ik in range(b.Nkpt if not device_projectors else 0):
            beta, trip = projectors(system, b, self.pspots, ik)
            if beta.shape[1] > 0:
                self.ctx.set_nonlocal(ik, beta)
                self.NbetaNL = beta.shape[1]
                self.nl_triplets = trip
        if self.NbetaNL > 0:
            self.ctx.set_nonlocal_coef(self.nl_triplets)
        self.Zvals = np.array([p.zval for p in self.pspots], dtype=np.float64)
        self.Nelectrons = float(sum(self.Zvals[system.atm2species]))
        self.ik = 0
        self.ispin = 0

    def setup_density(self):
        """Uploads, once, the density G-sphere that update!, the energies and
        the forces run on, and the exchange-correlation choice
        (Hamiltonian.jl:270-277: the internal VWN or PBE)."""
        if getattr(self, "_density_set", False):
            return
        b = self.basis
        self.ctx.set_density_sphere(b.idx_g2r, b.G2)
        if self.xcfunc == "PBE":
            from ._lib import PW_XC_PBE
            self.ctx.set_xc(PW_XC_PBE, b.G)
        if self.sym is not None:
            from .symmetry import symmetrizer_tables
            isg, ph = symmetrizer_tables(self.system.LatVecs, b.G, *self.sym)
            self.ctx.set_symmetry(isg, ph)
        self._density_set = True

    def update_vloc(self, V):
        """New V_loc(r) after update! (Hamiltonian.jl:510-545)."""
        self.V_Total = np.asarray(V, dtype=np.float64)
        self.ctx.set_vloc(self.V_Total)
