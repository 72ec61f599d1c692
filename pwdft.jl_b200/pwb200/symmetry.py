"""Crystal symmetry set-up for the device density symmetrisation and the
symmetry-reduced k-point mesh (host, once per geometry).

  crystal_symmetry   SymmetryInfo(atoms) (SymmetryInfo.jl:711-784, the QE
                     symm_base procedure): the lattice's point group, the
                     subgroup that maps the crystal onto itself, possibly with
                     a fractional translation (disabled for supercells), as
                     s (3, 3, Nsyms) acting on reciprocal crystal coordinates
                     and ft (3, Nsyms); an operation maps x -> s^T x - ft
  kpoint_grid_sym    gen_kpoint_grid (KPoints.jl:121-260) with those rotations
                     and k ~ -k
  symmetrizer_tables RhoeSymmetrizer (RhoeSymmetrizer.jl:14-110) flattened for
                     pw_set_symmetry: per orbit of the density sphere, the
                     sphere index and phase e^{i G.ft} of inv_s g0 for every
                     operation (g0 the orbit's first member), the order in
                     which symmetrize_rhoe! (:114-236) visits them
The lattice point group is taken as the integer matrices with entries in
{-1, 0, 1} that preserve the lattice metric.
"""
import itertools

import numpy as np


def lattice_point_group(LatVecs):
    A = np.asarray(LatVecs, dtype=np.float64)
    A = A / np.linalg.norm(A[:, 0])
    M = A.T @ A
    W = np.array(list(itertools.product((-1, 0, 1), repeat=9)), dtype=np.int64).reshape(-1, 3, 3)
    d = np.abs(np.einsum("nji,jk,nkl->nil", W, M, W) - M[None]).max(axis=(1, 2))
    W = W[(d < 1e-6) & (np.abs(np.round(np.linalg.det(W))) == 1)]
    s = np.transpose(W, (0, 2, 1))                     # s = W^T
    ident = np.all(s == np.eye(3, dtype=np.int64)[None], axis=(1, 2))
    return np.concatenate([s[ident], s[~ident]])       # identity first


def _maps(xa, rot, ft, ityp, tol=1e-5):
    """True when every rotated atom minus ft lands on a like atom (mod 1)."""
    d = rot[:, :, None] - xa[:, None, :] - ft[:, None, None]
    ok = np.all(np.abs(d - np.round(d)) < tol, axis=0) & (ityp[:, None] == ityp[None, :])
    return bool(np.all(ok.any(axis=1)))


def _valid_fraction(f, eps=1e-5):
    for x in f:
        if abs(x) > eps:
            aux = abs(1.0 / x - round(1.0 / x))
            if aux < eps and round(1.0 / abs(x)) not in (2, 3, 4, 6):
                return False
            if aux > eps:
                return False
    return True


def crystal_symmetry(LatVecs, positions, ityp):
    """(s (3, 3, Nsyms), ft (3, Nsyms)) of the crystal, identity first."""
    ityp = np.asarray(ityp)
    xa = np.linalg.inv(np.asarray(LatVecs, dtype=np.float64)) @ np.asarray(positions, dtype=np.float64)
    nat = xa.shape[1]
    frac_ok = True
    for na in range(1, nat):
        if ityp[na] != ityp[0]:
            continue
        f = xa[:, na] - xa[:, 0]
        f = f - np.round(f)
        if _maps(xa, xa, f, ityp):
            frac_ok = False                             # a supercell: no fractional translations
            break
    S, F = [], []
    for s in lattice_point_group(LatVecs):
        rot = s.T @ xa
        if _maps(xa, rot, np.zeros(3), ityp):
            S.append(s)
            F.append(np.zeros(3))
            continue
        if not frac_ok:
            continue
        for na in range(nat):
            if ityp[na] != ityp[0]:
                continue
            f = rot[:, na] - xa[:, 0]
            f = f - np.round(f)
            if _valid_fraction(f) and _maps(xa, rot, f, ityp):
                S.append(s)
                F.append(f)
                break
    return np.stack(S, axis=2), np.stack(F, axis=1)


def atom_map(LatVecs, positions, ityp, s, ft):
    """irt (nsym, nat): the like atom each atom lands on under x -> s^T x - ft."""
    ityp = np.asarray(ityp)
    xa = np.linalg.inv(np.asarray(LatVecs, dtype=np.float64)) @ np.asarray(positions, dtype=np.float64)
    irt = np.zeros((s.shape[2], xa.shape[1]), dtype=np.int64)
    for i in range(s.shape[2]):
        d = (s[:, :, i].T @ xa)[:, :, None] - xa[:, None, :] - ft[:, i][:, None, None]
        ok = np.all(np.abs(d - np.round(d)) < 1e-5, axis=0) & (ityp[:, None] == ityp[None, :])
        irt[i] = np.argmax(ok, axis=1)
    return irt


def symmetrize_vectors(LatVecs, s, irt, v):
    """symmetrize_vector! (SymmetryInfo.jl:923-966): per-atom Cartesian
    vectors v (3, nat) averaged over the operations, in crystal axes."""
    L = np.asarray(LatVecs, dtype=np.float64)
    L = L / np.linalg.norm(L[:, 0])
    t = L.T @ v
    acc = np.einsum("ijs,jsa->ia", s.astype(np.float64), t[:, irt])
    return np.linalg.inv(L.T) @ (acc / s.shape[2])


def kpoint_grid_sym(LatVecs, mesh, s, time_reversal=True):
    """Gamma-centred mesh reduced by the rotations s and k ~ -k (each class
    represented by its first mesh point, weight = class size); Cartesian k
    (3, Nk) and weights summing to one."""
    n = np.array(mesh)
    idx = np.stack(np.meshgrid(*[np.arange(m) for m in mesh], indexing="ij"), axis=-1).reshape(-1, 3)
    lin = lambda a: (a[..., 0] % n[0]) * n[1] * n[2] + (a[..., 1] % n[1]) * n[2] + (a[..., 2] % n[2])
    frac = idx / n
    ops = [s[:, :, i] for i in range(s.shape[2])]
    equiv = np.arange(len(idx))
    weight = np.zeros(len(idx))
    for ik in range(len(idx)):
        if equiv[ik] != ik:
            continue
        weight[ik] = 1.0
        for o in ops:
            xr = o @ frac[ik]
            xr = xr - np.round(xr)
            for x in ((xr, -xr) if time_reversal else (xr,)):
                q = x * n
                if np.any(np.abs(q - np.round(q)) > 1e-5):
                    continue
                m = int(lin(np.round(q).astype(np.int64)))
                if m > ik and equiv[m] == m:
                    equiv[m] = ik
                    weight[ik] += 1.0
    irr = np.where(equiv == np.arange(len(idx)))[0]
    xk = frac[irr] - np.round(frac[irr])
    RecVecs = 2 * np.pi * np.linalg.inv(np.asarray(LatVecs, dtype=np.float64).T)
    w = weight[irr]
    return RecVecs @ xk.T, w / w.sum()


def symmetrizer_tables(LatVecs, G, s, ft):
    """Flattened orbit tables for pw_set_symmetry: isg (nshell, nsym) int32
    sphere indices and phase (nshell, nsym, 2) = (cos, sin) of G_isg . ft_cart
    (1, 0 for symmorphic operations).  G: (Ng, 3) Cartesian, the density
    sphere in its order."""
    LatVecs = np.asarray(LatVecs, dtype=np.float64)
    G = np.asarray(G, dtype=np.float64)
    nsym = s.shape[2]
    Gc = np.round(G @ LatVecs / (2 * np.pi)).astype(np.int64)        # (Ng, 3) crystal
    lookup = {tuple(v): i for i, v in enumerate(Gc)}
    inv_s = np.stack([np.round(np.linalg.inv(s[:, :, i])).astype(np.int64) for i in range(nsym)])
    sym_ns = np.abs(ft).max(axis=0) >= 1e-10
    fts = (LatVecs @ ft) * sym_ns[None, :]                            # (3, nsym) Cartesian
    done = np.zeros(len(G), dtype=bool)
    isg_rows, ph_rows = [], []
    for ig in range(len(G)):
        if done[ig]:
            continue
        rot = inv_s @ Gc[ig]                                          # (nsym, 3): inv_s g0
        row = np.array([lookup[tuple(v)] for v in rot], dtype=np.int32)
        done[row] = True
        arg = np.einsum("si,is->s", G[row], fts)
        isg_rows.append(row)
        ph_rows.append(np.stack([np.cos(arg), np.sin(arg)], axis=1))
    return np.array(isg_rows, dtype=np.int32), np.array(ph_rows)
