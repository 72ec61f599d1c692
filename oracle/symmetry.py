"""Crystal symmetry, symmetry-reduced k-points and density symmetrisation.

Oracle (test infrastructure only).  Restates PWDFT.jl (itself following
Quantum ESPRESSO's symm_base):
  find_symm_bravais_latt   SymmetryInfo.jl:125-216  point group of the lattice
  sgam_at!                 SymmetryInfo.jl:248-386  subgroup of the crystal, with
                                                    fractional translations
  checksym! / eqvect       SymmetryInfo.jl:501-556
  copy_sym!                SymmetryInfo.jl:562-611
  SymmetryInfo(atoms)      SymmetryInfo.jl:711-784  (Nsyms, s, inv_s, ft, non_symmorphic, irt)
  symmetrize_vector!       SymmetryInfo.jl:923-966  (forces)
  gen_kpoint_grid          KPoints.jl:121-260       with the crystal's rotations
  RhoeSymmetrizer          RhoeSymmetrizer.jl:14-110  G-vector orbits
  symmetrize_rhoe!         RhoeSymmetrizer.jl:114-236

Conventions as the reference: s[:, :, isym] acts on reciprocal crystal
coordinates (s^T on direct crystal coordinates of positions), and an
operation maps atom positions x -> s^T x - ft.

The lattice point group is found here by enumeration: the integer matrices
with entries in {-1, 0, 1} that preserve the metric A^T A (the reference
rotates the lattice with a fixed table of 32 Cartesian rotations and keeps
those that are integer in crystal coordinates; both give the same set for
the cells used here, ordered differently; the identity comes first, as the
reference's s[:,:,1]).
"""
import itertools

import numpy as np

EPS1 = 1.0e-6
EPS2 = 1.0e-5


def lattice_point_group(LatVecs):
    """Integer s (3, 3, nrot) of the lattice, identity first."""
    A = np.asarray(LatVecs, dtype=np.float64) / np.linalg.norm(LatVecs[:, 0])
    M = A.T @ A
    out = []
    for e in itertools.product((-1, 0, 1), repeat=9):
        W = np.array(e, dtype=np.int64).reshape(3, 3)
        if abs(abs(round(np.linalg.det(W))) - 1) > 0:
            continue
        if np.abs(W.T @ M @ W - M).max() < EPS1:
            out.append(W.T.copy())            # s = W^T
    out.sort(key=lambda s: 0 if np.array_equal(s, np.eye(3, dtype=np.int64)) else 1)
    return np.stack(out, axis=2)


def eqvect(x, y, f, accep):
    d = x - y - f
    return bool(np.all(np.abs(d - np.round(d)) < accep))


def checksym(irot, ityp, xau, rau, ft, irt):
    nat = xau.shape[1]
    for ia in range(nat):
        found = False
        for ib in range(nat):
            if ityp[ib] == ityp[ia] and eqvect(rau[:, ia], xau[:, ib], ft, 1e-5):
                irt[irot, ia] = ib
                found = True
                break
        if not found:
            return False
    return True


def sgam_at(LatVecs, positions, ityp, s, fractional_translations=True):
    """sym (nrot,), ft (3, nrot), irt (nrot, nat)."""
    nrot = s.shape[2]
    nat = positions.shape[1]
    bg = np.linalg.inv(np.asarray(LatVecs, dtype=np.float64).T)
    xau = bg.T @ positions
    sym = np.zeros(nrot, dtype=bool)
    ft = np.zeros((3, nrot))
    irt = np.zeros((nrot, nat), dtype=np.int64)
    if fractional_translations:
        for na in range(1, nat):
            if ityp[0] != ityp[na]:
                continue
            f = xau[:, na] - xau[:, 0] - np.round(xau[:, na] - xau[:, 0])
            if checksym(0, ityp, xau, xau, f, irt):
                fractional_translations = False       # a supercell
                break
    for irot in range(nrot):
        rau = s[:, :, irot].T @ xau
        ft[:, irot] = 0.0
        sym[irot] = checksym(irot, ityp, xau, rau, np.zeros(3), irt)
        if not sym[irot] and fractional_translations:
            for na in range(nat):
                if ityp[0] != ityp[na]:
                    continue
                f = rau[:, na] - xau[:, 0] - np.round(rau[:, na] - xau[:, 0])
                bad = False
                for i in range(3):
                    if abs(f[i]) > EPS2:
                        aux = abs(1.0 / f[i] - round(1.0 / f[i]))
                        nfrac = round(1.0 / abs(f[i]))
                        if aux < EPS2 and nfrac not in (2, 3, 4, 6):
                            aux = 2 * EPS2
                        bad = bad or aux > EPS2
                if bad:
                    continue
                if checksym(irot, ityp, xau, rau, f, irt):
                    sym[irot] = True
                    ft[:, irot] = f
                    break
    return sym, ft, irt


class SymmetryInfo:
    """SymmetryInfo.jl:711-784 (no magnetic symmetry)."""

    def __init__(self, LatVecs, positions, ityp):
        s_all = lattice_point_group(LatVecs)
        sym, ft_all, irt = sgam_at(LatVecs, positions, ityp, s_all)
        keep = [i for i in range(s_all.shape[2]) if sym[i]]        # copy_sym!: kept ones first, in order
        self.Nsyms = len(keep)
        self.s = s_all[:, :, keep]
        self.ft = ft_all[:, keep]
        self.irt = irt[keep]
        self.inv_s = np.stack([np.round(np.linalg.inv(self.s[:, :, i])).astype(np.int64)
                               for i in range(self.Nsyms)], axis=2)
        self.non_symmorphic = np.abs(self.ft).max(axis=0) >= 1e-10


def symmetrize_vector(LatVecs, sym, v):
    """SymmetryInfo.jl:923-966: v (3, Natoms) Cartesian, averaged over the
    operations (atom ia takes s applied to its image irt[isym, ia])."""
    if sym.Nsyms == 1:
        return v.copy()
    L = np.asarray(LatVecs, dtype=np.float64)
    L = L / np.linalg.norm(L[:, 0])
    R = np.linalg.inv(L.T)
    tmp = L.T @ v
    out = np.zeros_like(v)
    for i in range(v.shape[1]):
        for isym in range(sym.Nsyms):
            out[:, i] += sym.s[:, :, isym].astype(np.float64) @ tmp[:, sym.irt[isym, i]]
    return R @ (out / sym.Nsyms)


def gen_kpoint_grid(LatVecs, nk, s, shift=(0, 0, 0), time_reversal=True):
    """KPoints.jl:121-260: (Nkpt, xk Cartesian (3, Nkpt), wk)."""
    nk1, nk2, nk3 = nk
    k1, k2, k3 = shift
    SMALL = 1.0e-5
    nkr = nk1 * nk2 * nk3
    xkg = np.zeros((3, nkr))
    for i in range(nk1):
        for j in range(nk2):
            for k in range(nk3):
                ik = k + j * nk3 + i * nk2 * nk3
                xkg[:, ik] = [i / nk1 + k1 / 2.0 / nk1, j / nk2 + k2 / 2.0 / nk2, k / nk3 + k3 / 2.0 / nk3]
    equiv = np.arange(nkr)
    wkk = np.zeros(nkr)

    def locate(x):
        q = np.array([x[0] * nk1 - 0.5 * k1, x[1] * nk2 - 0.5 * k2, x[2] * nk3 - 0.5 * k3])
        if np.any(np.abs(q - np.round(q)) > SMALL):
            return None
        i = int(round(x[0] * nk1 - 0.5 * k1 + 2 * nk1)) % nk1
        j = int(round(x[1] * nk2 - 0.5 * k2 + 2 * nk2)) % nk2
        k = int(round(x[2] * nk3 - 0.5 * k3 + 2 * nk3)) % nk3
        return k + j * nk3 + i * nk2 * nk3

    for ik in range(nkr):
        if equiv[ik] != ik:
            continue
        wkk[ik] = 1.0
        for irot in range(s.shape[2]):
            xkr = s[:, :, irot] @ xkg[:, ik]
            xkr = xkr - np.round(xkr)
            for x in ((xkr, -xkr) if time_reversal else (xkr,)):
                n = locate(x)
                if n is None:
                    continue
                if n > ik and equiv[n] == n:
                    equiv[n] = ik
                    wkk[ik] += 1.0
                elif equiv[n] != ik or n < ik:
                    raise RuntimeError("gen_kpoint_grid: inconsistent equivalence")
    irr = [ik for ik in range(nkr) if equiv[ik] == ik]
    wk = np.array([wkk[ik] for ik in irr])
    xk = np.stack([xkg[:, ik] - np.round(xkg[:, ik]) for ik in irr], axis=1)
    RecVecs = 2 * np.pi * np.linalg.inv(np.asarray(LatVecs, dtype=np.float64).T)
    return len(irr), RecVecs @ xk, wk / wk.sum(), equiv


class RhoeSymmetrizer:
    """RhoeSymmetrizer.jl:14-110: orbits (shells) of the density sphere under
    the rotations, and the Cartesian fractional translations fts."""

    def __init__(self, LatVecs, G, sym):
        LatVecs = np.asarray(LatVecs, dtype=np.float64)
        Ng = G.shape[1]
        Gc = np.round(LatVecs.T @ G / (2 * np.pi)).astype(np.int64)     # (3, Ng) crystal
        lookup = {tuple(Gc[:, i]): i for i in range(Ng)}
        done = np.zeros(Ng, dtype=bool)
        shells = []
        for ig in range(Ng):
            if done[ig]:
                continue
            members = []
            seen = set()
            for isym in range(sym.Nsyms):
                sn = tuple(sym.s[:, :, isym] @ Gc[:, ig])
                if sn not in seen:
                    seen.add(sn)
                    members.append(sn)
            idx = []
            for sn in members:
                j = lookup.get(sn)
                if j is None or done[j] or j < ig:
                    raise RuntimeError("Lone G-vector")
                done[j] = True
                idx.append(j)
            shells.append(np.array(idx))
        self.shells = shells
        self.fts = np.zeros((3, sym.Nsyms))
        for isym in range(sym.Nsyms):
            if sym.non_symmorphic[isym]:
                self.fts[:, isym] = LatVecs @ sym.ft[:, isym]


def symmetrize_rhoe(pw, sym, symz, Rhoe):
    """RhoeSymmetrizer.jl:114-236 for one spin channel: returns the
    symmetrised density.  Components of the FFT grid outside the density
    sphere are kept, as the reference does."""
    from .ham import R_to_G, G_to_R
    G = pw.gvec.G
    RhoeG = R_to_G(pw.Ns, Rhoe.astype(np.complex128))
    trmat = np.asarray(pw.LatVecs).T / (2 * np.pi)
    for shell in symz.shells:
        ng = len(shell)
        g0 = trmat @ G[:, shell]                       # (3, ng) crystal
        done = np.zeros(ng, dtype=bool)
        for ig in range(ng):
            if done[ig]:
                continue
            irot = np.zeros(sym.Nsyms, dtype=np.int64)
            rhosum = 0.0 + 0.0j
            for isym in range(sym.Nsyms):
                sg = sym.inv_s[:, :, isym] @ g0[:, ig]
                hit = np.where(np.all(np.abs(g0 - sg[:, None]) < 1e-5, axis=0))[0]
                if len(hit) == 0:
                    raise RuntimeError("Error in determining irot")
                irot[isym] = hit[0]
                isg = shell[irot[isym]]
                ip = pw.gvec.idx_g2r[isg]
                if sym.non_symmorphic[isym]:
                    arg = G[:, isg] @ symz.fts[:, isym]
                    rhosum += RhoeG[ip] * (np.cos(arg) - 1j * np.sin(arg))
                else:
                    rhosum += RhoeG[ip]
            rhosum /= sym.Nsyms
            for isym in range(sym.Nsyms):
                isg = shell[irot[isym]]
                ip = pw.gvec.idx_g2r[isg]
                if sym.non_symmorphic[isym]:
                    arg = G[:, isg] @ symz.fts[:, isym]
                    RhoeG[ip] = rhosum * (np.cos(arg) + 1j * np.sin(arg))
                else:
                    RhoeG[ip] = rhosum
                done[irot[isym]] = True
    return np.real(G_to_R(pw.Ns, RhoeG))
