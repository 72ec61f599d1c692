"""Crystal symmetry, symmetry-reduced k-points and symmetrize_rhoe!.

Oracle pins (test/test_spglib.jl:9-21, Si fcc a = 10.2631 bohr):
  48 operations; the 4x4x4 Gamma-centred mesh has 8 irreducible points whose
  equivalence classes are those of the test's ir_reciprocal_mesh mapping.
  Si fcc 3x3x3 -> 4 k-points, Al4 conventional 8x8x8 -> 35.
  The Si fcc SCF with symmetry (4 k-points, symmetrised density) reproduces
  the ABINIT total energy (test/validations_old/Si_fcc.jl:15).
Host set-up (pwb200.symmetry) against the oracle: same operations,
translations, k-points and weights.  symmetrize_rhoe! is a projection: it
keeps a symmetric density, is idempotent and keeps the electron count.
Device (pw_symmetrize_rhoe) against the oracle on a non-symmetric density
(Si fcc has non-symmorphic operations): 1e-12.  Device SCF with symmetry
against ABINIT and the oracle.
"""
import numpy as np
import pytest

from conftest import cuda_ok

SPGLIB_MAP_444 = [0, 1, 2, 1, 1, 5, 6, 7, 2, 6, 10, 6, 1, 7, 6, 5, 1, 5, 6, 7, 5, 1, 7, 6, 6, 7, 6, 27, 7, 6, 27, 6,
                  2, 6, 10, 6, 6, 7, 6, 27, 10, 6, 2, 6, 6, 27, 6, 7, 1, 7, 6, 5, 7, 6, 27, 6, 6, 27, 6, 7, 5, 6, 7, 1]


def _classes(labels):
    out = {}
    for i, l in enumerate(labels):
        out.setdefault(l, set()).add(i)
    return sorted(sorted(v) for v in out.values())


def test_oracle_symmetry_matches_spglib_goldens():
    from oracle import systems, symmetry
    at = systems.si_fcc_atoms()
    sym = symmetry.SymmetryInfo(at.LatVecs, at.positions, at.atm2species)
    assert sym.Nsyms == 48
    n, _, wk, equiv = symmetry.gen_kpoint_grid(at.LatVecs, (4, 4, 4), sym.s)
    assert n == 8
    # the test's mesh index is a + 4 b + 16 c, this one c + 4 b + 16 a
    ours = [int(equiv[c + 4 * b + 16 * a]) for c in range(4) for b in range(4) for a in range(4)]
    assert _classes(ours) == _classes(SPGLIB_MAP_444)
    assert symmetry.gen_kpoint_grid(at.LatVecs, (3, 3, 3), sym.s)[0] == 4
    al = systems.al4_atoms()
    sal = symmetry.SymmetryInfo(al.LatVecs, al.positions, al.atm2species)
    assert sal.Nsyms == 48 and not sal.non_symmorphic.any()      # a supercell: no fractional translations
    assert symmetry.gen_kpoint_grid(al.LatVecs, (8, 8, 8), sal.s)[0] == 35


@pytest.mark.parametrize("name,mesh", [("si", (3, 3, 3)), ("si", (4, 4, 4)), ("al", (8, 8, 8)), ("pt", (3, 3, 3))])
def test_host_symmetry_matches_oracle(name, mesh):
    from oracle import systems, symmetry
    from pwb200 import symmetry as ps
    at = {"si": systems.si_fcc_atoms, "al": systems.al4_atoms, "pt": systems.pt_fcc_atoms}[name]()
    o = symmetry.SymmetryInfo(at.LatVecs, at.positions, at.atm2species)
    s, ft = ps.crystal_symmetry(at.LatVecs, at.positions, at.atm2species)
    assert s.shape[2] == o.Nsyms
    assert np.array_equal(s, o.s)
    assert np.abs(ft - o.ft).max() < 1e-12
    n, xk, wk, _ = symmetry.gen_kpoint_grid(at.LatVecs, mesh, o.s)
    k2, w2 = ps.kpoint_grid_sym(at.LatVecs, mesh, s)
    assert k2.shape[1] == n
    assert np.abs(k2 - xk).max() < 1e-12 and np.abs(w2 - wk).max() < 1e-14


def test_oracle_symmetrize_rhoe_is_a_projection():
    from oracle import ham, systems, symmetry
    at = systems.si_fcc_atoms()
    H = ham.Hamiltonian(at, [systems.psp("Si-q4.gth")], 15.0, meshk=(3, 3, 3), use_symmetry=True)
    pw = H.pw
    rho0 = H.guess_rhoe()                                   # symmetric by construction
    assert np.abs(symmetry.symmetrize_rhoe(pw, H.sym, H.symz, rho0) - rho0).max() < 1e-12 * rho0.max()
    rng = np.random.default_rng(2)
    r = rho0 * (1.0 + 0.2 * rng.standard_normal(rho0.shape))
    s1 = symmetry.symmetrize_rhoe(pw, H.sym, H.symz, r)
    s2 = symmetry.symmetrize_rhoe(pw, H.sym, H.symz, s1)
    assert np.abs(s2 - s1).max() < 1e-12 * np.abs(s1).max()
    assert abs(s1.sum() - r.sum()) < 1e-10 * abs(r.sum())
    assert np.abs(s1 - r).max() > 1e-3 * np.abs(r).max()     # it did change the perturbed density


@pytest.mark.slow
def test_oracle_si_fcc_scf_with_symmetry():
    from oracle import ham, systems, scf
    H = ham.Hamiltonian(systems.si_fcc_atoms(), [systems.psp("Si-q4.gth")], 15.0, meshk=(3, 3, 3),
                        use_symmetry=True)
    assert H.pw.kpoints.Nkpt == 4
    E, _, _ = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8)
    assert abs(E["Total"] - (-7.9110087934)) < 1e-5


def _device_si(use_symmetry=True):
    import pwb200
    from oracle import systems
    at = systems.si_fcc_atoms()
    return pwb200.Hamiltonian(pwb200.System(["Si", "Si"], at.positions, at.LatVecs), [systems.psp("Si-q4.gth")],
                              15.0, meshk=(3, 3, 3), use_symmetry=use_symmetry)


@pytest.mark.gpu
def test_device_symmetrize_rhoe_vs_oracle():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import ham, systems, symmetry
    Ho = ham.Hamiltonian(systems.si_fcc_atoms(), [systems.psp("Si-q4.gth")], 15.0, meshk=(3, 3, 3),
                         use_symmetry=True)
    rng = np.random.default_rng(6)
    rho = Ho.guess_rhoe() * (1.0 + 0.3 * rng.standard_normal(Ho.pw.Npoints))
    ref = symmetry.symmetrize_rhoe(Ho.pw, Ho.sym, Ho.symz, rho)
    H = _device_si()
    H.setup_density()
    r = torch.from_numpy(rho.copy()).cuda()
    H.ctx.symmetrize_rhoe(r)
    assert np.abs(r.cpu().numpy() - ref).max() < 1e-12 * np.abs(ref).max()
    H.ctx.check_device()
    H.ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_scf_si_fcc_with_symmetry(precision):
    """4 irreducible k-points and the symmetrised density: ABINIT's Etot,
    and the FP64 run within 2e-7 of the time-reversal-only device SCF."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from pwb200 import scf
    H = _device_si()
    assert H.basis.Nkpt == 4
    res = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8, precision=precision)
    assert abs(res["energies"]["Total"] - (-7.9110087934)) < 1e-5, res["log"][-3:]
    if precision == "fp64":
        H2 = _device_si(use_symmetry=False)
        r2 = scf.KS_solve_SCF(H2, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8)
        assert abs(res["energies"]["Total"] - r2["energies"]["Total"]) < 2e-7
        H2.ctx.close()
    H.ctx.close()


def test_host_vector_symmetrisation_matches_oracle():
    from oracle import systems, symmetry
    from pwb200 import symmetry as ps
    at = systems.si_fcc_atoms()
    pos = at.positions.copy()
    pos[:, 1] += 0.03                     # along (1,1,1): C3v, 6 operations
    o = symmetry.SymmetryInfo(at.LatVecs, pos, at.atm2species)
    assert o.Nsyms == 6
    s, ft = ps.crystal_symmetry(at.LatVecs, pos, at.atm2species)
    irt = ps.atom_map(at.LatVecs, pos, at.atm2species, s, ft)
    assert np.array_equal(irt, o.irt)
    v = np.random.default_rng(1).standard_normal((3, 2))
    ref = symmetry.symmetrize_vector(at.LatVecs, o, v)
    got = ps.symmetrize_vectors(at.LatVecs, s, irt, v)
    assert np.abs(got - ref).max() < 1e-14
    assert np.abs(ref[:, 0] - ref[0, 0]).max() < 1e-14       # along (1,1,1)


@pytest.mark.gpu
def test_device_forces_with_symmetry_match_full_mesh():
    """Si fcc with the second atom moved along (1,1,1) (6 operations): the
    forces from the symmetry-reduced SCF (symmetrised density and nonlocal
    force) equal those of the time-reversal-only mesh."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from pwb200 import scf, forces
    from oracle import systems
    at = systems.si_fcc_atoms()
    pos = at.positions.copy()
    pos[:, 1] += 0.03
    out = []
    for use_sym in (True, False):
        H = pwb200.Hamiltonian(pwb200.System(["Si", "Si"], pos, at.LatVecs), [systems.psp("Si-q4.gth")], 15.0,
                               meshk=(3, 3, 3), use_symmetry=use_sym)
        res = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-11, ethr_evals_last=1e-11)
        out.append((H.basis.Nkpt, res["energies"]["Total"], forces.calc_forces(H, res["psiks"], res["rho"], res["Focc"])))
        H.ctx.close()
    (n1, e1, f1), (n2, e2, f2) = out
    assert n1 < n2
    assert abs(e1 - e2) < 1e-9
    assert np.abs(f1 - f2).max() < 1e-7, (f1, f2)
    assert np.abs(f1[:, 1]).max() > 1e-3
