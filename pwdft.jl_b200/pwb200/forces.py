"""Ionic forces (Hartree/bohr): calc_forces.jl:1-17 for GTH pseudopotentials
without symmetry, NLCC or SCF correction.

  F = F_NN + F_Ps_loc + F_Ps_nloc
  F_Ps_loc    calc_forces_Ps_loc.jl:13-71        device (pw_forces_local)
  F_Ps_nloc   calc_forces_Ps_nloc.jl:291-411     device (pw_forces_nonlocal, per k-point)
  F_NN        calc_forces_NN.jl:1-142            host (Ewald sum, set-up arithmetic)
With symmetry the nonlocal part is averaged over the crystal's operations
(calc_forces.jl:11, symmetrize_vector!), as the reference does.
"""
import numpy as np
from scipy.special import erfc


def setup_forces(Ham):
    """Uploads, once per geometry, what the device force kernels need: the
    density sphere with its G vectors and V_sp(G) per species, the G+k
    vectors of every k-point and the atom of every projector."""
    b = Ham.basis
    ctx = Ham.ctx
    Ham.setup_density()
    VlocG = np.stack([psp.vloc_G(b.G2) for psp in Ham.pspots], axis=1)     # (Ng, nspecies)
    ctx.set_force_tables(VlocG, b.G)
    for ik in range(b.Nkpt):
        ctx.set_gkvec(ik, b.G[b.idx_gw2g[ik]] + b.kpts[:, ik][None, :])
    if Ham.NbetaNL > 0:
        atoms = []
        for ia, isp in enumerate(Ham.system.atm2species):
            psp = Ham.pspots[isp]
            atoms += [ia] * sum((2 * l + 1) * psp.Nproj_l[l] for l in range(psp.lmax + 1))
        ctx.set_nonlocal_atoms(Ham.system.positions.shape[1], atoms)
    Ham._forces_set = True


def ewald_forces(LatVecs, positions, Z, G, G2, ecutrho):
    """calc_forces_NN.jl:1-142: reciprocal-space sum over the density sphere
    (G = 0 excluded) with the reference's choice of alpha (the largest
    alpha in steps of 0.1 below 1 whose tail bound is under 1e-6), and the
    real-space sum over lattice images out to erfc < 1e-10."""
    Omega = abs(np.linalg.det(LatVecs))
    Z = np.asarray(Z, dtype=np.float64)
    q = float(Z.sum())
    alpha = 1.0
    while q * q * np.sqrt(alpha / np.pi) * erfc(np.sqrt(ecutrho / 2.0 / alpha)) > 1e-6:
        alpha -= 0.1
        if alpha <= 0.0:
            raise ValueError("no Ewald splitting parameter found")
    Gn, G2n = G[1:], G2[1:]                                  # (Ng-1, 3), G = 0 first
    phase = positions.T @ Gn.T                               # (natoms, Ng-1)
    c, s = np.cos(phase), np.sin(phase)
    S = (Z[:, None] * c).sum(axis=0) + 1j * (Z[:, None] * s).sum(axis=0)
    S *= np.exp(-G2n / (4.0 * alpha)) / G2n
    F = ((c * S.imag[None, :] - s * S.real[None, :]) @ Gn).T * (-4.0 * np.pi * Z[None, :] / Omega)
    eta = np.sqrt(alpha)
    rmax = np.sqrt(0.5 * np.log(1e10)) / eta
    n = [int(round(rmax / np.linalg.norm(LatVecs[:, i]) + 1.5)) for i in range(3)]
    grid = np.stack(np.meshgrid(*[np.arange(-m, m + 1) for m in n], indexing="ij"), axis=0).reshape(3, -1)
    T = LatVecs @ grid                                       # (3, nimages)
    nat = positions.shape[1]
    for ia in range(nat):
        for ja in range(ia + 1, nat):
            D = (positions[:, ia] - positions[:, ja])[:, None] - T
            r2 = (D * D).sum(axis=0)
            r = np.sqrt(r2)
            x = eta * r
            h = -2.0 * np.exp(-x * x) / np.sqrt(np.pi) - erfc(x) / x
            f = (D * (eta * h * Z[ia] * Z[ja] / r2)[None, :]).sum(axis=1)
            F[:, ia] -= f
            F[:, ja] += f
    return F


def calc_forces(Ham, psiks, rho, Focc, parts=False):
    """Total force (3, natoms) from the converged wavefunctions psiks (device
    blocks (nb, Ngw) per k-point), the density rho (device, N) and the
    occupations Focc (nb, Nkpt).  parts=True also returns the three terms."""
    if not getattr(Ham, "_forces_set", False):
        setup_forces(Ham)
    b = Ham.basis
    sysm = Ham.system
    Z = Ham.Zvals[sysm.atm2species]
    F_nn = ewald_forces(b.LatVecs, sysm.positions, Z, b.G, b.G2, b.ecutrho)
    F_loc = Ham.ctx.forces_local(rho, sysm.positions, sysm.atm2species)
    F_nl = np.zeros_like(F_loc)
    if Ham.NbetaNL > 0:
        for ik in range(b.Nkpt):
            F_nl += Ham.ctx.forces_nonlocal(ik, psiks[ik], Ham.wk[ik] * Focc[:, ik])
    if getattr(Ham, "sym", None) is not None:
        from .symmetry import atom_map, symmetrize_vectors
        s, ft = Ham.sym
        F_nl = symmetrize_vectors(b.LatVecs, s, atom_map(b.LatVecs, sysm.positions, sysm.atm2species, s, ft), F_nl)
    F = F_nn + F_loc + F_nl
    if parts:
        return F, {"NN": F_nn, "Ps_loc": F_loc, "Ps_nloc": F_nl}
    return F
