"""Parity at the benchmarked shapes, against the FP64 oracle, through the C ABI.

The op_H bench runs Si64 (75^3 grid, Ngw 23,871) with 160 bands: two FP32 band
batches of the 48 MiB intermediate (83 + 77 bands; four FP64 batches of 41),
the 75-point plane kernel taking 3 bands per CTA with a 2-band remainder CTA
in each batch.  These tests run exactly those launches and the shapes around
them (nb in {1, 2, 4, 83, 160, 161}), every launch-parameter candidate of the
autotuner, the batched op_H of config C3 on its full 8x8x8 mesh (260 k-points
by time reversal), and the energy components of config C5 (Si216, 480 bands)
on one wavefunction set.  References: op_H.jl:53-63, op_V_loc.jl:33-92,
calc_rhoe.jl:9-135, calc_energies.jl:7-58,245-375.

Tolerances (max-abs error relative to the max-abs of the oracle result):
  FP64 path (complex128):            1e-11
  mixed path (complex64, FP32 FFTs): 2e-5
Energies: FP64 1e-9 Ha per component; mixed 2e-5 relative.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-11, "c64": 2e-5}
NB_MAX = 161


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def smooth_field(pw, rng):
    """Seeded field with Fourier components at |G|^2 <= 4 only, max |dV| = 1."""
    g = pw.gvec
    sel = g.G2 <= 4.0
    c = np.zeros(pw.Npoints, dtype=np.complex128)
    c[g.idx_g2r[sel]] = rng.standard_normal(sel.sum()) + 1j * rng.standard_normal(sel.sum())
    N1, N2, N3 = pw.Ns
    f = np.fft.ifftn(c.reshape(N3, N2, N1)).real.ravel()
    return f / np.abs(f).max()


@pytest.fixture(scope="module")
def si64():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems, ops
    H = systems.Ham_Si64(Nstates=160)
    pw = H.pw
    rng = np.random.default_rng(20261203)
    H.V_Total = H.V_Ps_loc + 0.01 * smooth_field(pw, rng)
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    ctx.set_vloc(H.V_Total)
    ctx.set_nonlocal(0, H.betaNL[0])
    ctx.set_nonlocal_coef(H.nl_triplets)
    ngw = pw.gvecw.Ngw[0]
    psi = (rng.standard_normal((ngw, NB_MAX)) + 1j * rng.standard_normal((ngw, NB_MAX))) / np.sqrt(ngw)
    ref = ops.op_H(H, psi, 0)
    yield H, ctx, psi, ref
    ctx.close()


def to_dev(psi, dt):
    import torch
    return torch.from_numpy(np.ascontiguousarray(psi.T)).to("cuda").to(dt).contiguous()


def to_host(t):
    return t.cpu().numpy().T.astype(np.complex128)


@pytest.mark.parametrize("prec", ["c128", "c64"])
@pytest.mark.parametrize("nb", [1, 2, 4, 83, 160, 161])
def test_si64_op_H_band_counts(si64, prec, nb):
    import torch
    import pwb200
    H, ctx, psi, ref = si64
    dt = torch.complex128 if prec == "c128" else torch.complex64
    x = to_dev(psi[:, :nb], dt)
    y = torch.empty_like(x)
    ctx.apply(0, 0, x, y, pwb200.PW_OP_H)
    assert rel_err(to_host(y), ref[:, :nb]) < TOL[prec]


@pytest.mark.parametrize("prec", ["c128", "c64"])
@pytest.mark.parametrize("nb", [1, 2, 83, 161])
def test_si64_calc_rhoe_band_counts(si64, prec, nb):
    import torch
    from oracle import ops
    H, ctx, psi, _ = si64
    dt = torch.complex128 if prec == "c128" else torch.complex64
    w = np.linspace(2.0, 0.1, nb)
    rho = torch.zeros(H.pw.Npoints, dtype=torch.float64, device="cuda")
    ctx.calc_rhoe(0, to_dev(psi[:, :nb], dt), w, rho)
    assert rel_err(rho.cpu().numpy(), ops.calc_rhoe(H, [psi[:, :nb]], Focc=w[:, None])) < TOL[prec]


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_si64_op_H_host_160(si64, prec):
    """The reference-facing host call at the bench shape (pipelined over band
    chunks of 32: 5 chunks, each its own FFT batches)."""
    import pwb200
    H, ctx, psi, ref = si64
    code = pwb200.PW_C128 if prec == "c128" else pwb200.PW_C64
    got = ctx.op_H_host(0, 0, psi[:, :160], dtype=code)
    assert rel_err(got, ref[:, :160]) < TOL[prec]


CANDIDATES = [dict(plane_bands=pb, band_chunk_bytes=ch << 20, z_columns=zc)
              for pb in (1, 2, 3) for ch in (5, 48) for zc in (32, 128)]


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_si64_every_tuning_candidate(si64, prec):
    """Every launch-parameter set the autotuner may pick gives the oracle's
    op_H on 161 bands (band batches of 5 MiB = 8 bands put a remainder batch
    and remainder CTAs everywhere)."""
    import torch
    import pwb200
    H, ctx, psi, ref = si64
    dt = torch.complex128 if prec == "c128" else torch.complex64
    x = to_dev(psi, dt)
    y = torch.empty_like(x)
    saved = ctx.get_tuning()
    try:
        for cand in CANDIDATES:
            ctx.set_tuning(**cand)
            y.zero_()
            ctx.apply(0, 0, x, y, pwb200.PW_OP_H)
            assert rel_err(to_host(y), ref) < TOL[prec], cand
    finally:
        ctx.set_tuning(**saved)


def test_si64_gram_splits_and_autotune(si64, tmp_path):
    """Split-K candidates of the tensor-core Gram give the same product; the
    autotuner applies a choice, writes it to its cache and reads it back
    (no timing on the second call), and op_H still matches the oracle."""
    import torch
    import pwb200
    H, ctx, psi, ref = si64
    x = to_dev(psi[:, :96], torch.complex64)
    exact = to_host(x).conj().T @ to_host(x)
    saved = ctx.get_tuning()
    try:
        for sp in (0, 1, 3, 16):
            ctx.set_tuning(gemm_splits=sp)
            G = torch.zeros((96, 96), dtype=torch.complex128, device="cuda")
            ctx.gram(x, x, G)
            assert np.abs(G.cpu().numpy().T - exact).max() < 2e-5 * np.abs(exact).max(), sp
        cache = tmp_path / "tune.txt"
        t1, ms1 = ctx.autotune(0, 160, pwb200.PW_C64, cache_path=cache)
        assert ms1["op_H_tuned_ms"] > 0 and ms1["op_H_tuned_ms"] <= ms1["op_H_default_ms"] * 1.01
        assert ms1["rr_tuned_ms"] > 0
        assert ctx.get_tuning() == t1
        ctx.set_tuning(**saved)
        t2, ms2 = ctx.autotune(0, 160, pwb200.PW_C64, cache_path=cache)
        assert t2 == t1 and ms2["op_H_tuned_ms"] < 0
        xx = to_dev(psi[:, :160], torch.complex64)
        yy = torch.empty_like(xx)
        ctx.apply(0, 0, xx, yy, pwb200.PW_OP_H)
        assert rel_err(to_host(yy), ref[:, :160]) < TOL["c64"]
    finally:
        ctx.set_tuning(**saved)


@pytest.fixture(scope="module")
def al4_888():
    """Config C3's system on its full mesh: Al4, 8x8x8 reduced by time
    reversal to 260 k-points (Ngw 1208-1260), 10 bands per k-point."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    Ho = systems.Ham_Al4(meshk=(8, 8, 8))
    pw = Ho.pw
    rng = np.random.default_rng(31)
    Ho.V_Total = Ho.V_Ps_loc + 0.01 * smooth_field(pw, rng)
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(k) for k in range(pw.kpoints.Nkpt)])
    ctx.set_vloc(Ho.V_Total)
    for ik in range(pw.kpoints.Nkpt):
        ctx.set_nonlocal(ik, Ho.betaNL[ik])
    ctx.set_nonlocal_coef(Ho.nl_triplets)
    psis = [(rng.standard_normal((pw.gvecw.Ngw[ik], 10)) + 1j * rng.standard_normal((pw.gvecw.Ngw[ik], 10)))
            / np.sqrt(pw.gvecw.Ngw[ik]) for ik in range(pw.kpoints.Nkpt)]
    yield Ho, ctx, psis
    ctx.close()


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_al4_888_batched_op_H_vs_oracle(al4_888, prec):
    import torch
    from oracle import ops
    Ho, ctx, psis = al4_888
    assert len(psis) == 260
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = [to_dev(p, dt) for p in psis]
    HX = [torch.empty_like(x) for x in X]
    ctx.apply_multi(list(range(len(X))), 0, X, HX, graph=True)
    worst = 0.0
    for ik in range(len(X)):
        worst = max(worst, rel_err(to_host(HX[ik]), ops.op_H(Ho, psis[ik], ik)))
    assert worst < TOL[prec], worst
    ctx.check_device()


def test_si216_energy_components_vs_oracle():
    """Config C5 (Si216 with the seeded +-0.02 bohr displacements, 480 bands,
    432 occupied): on one wavefunction set, the device density, update! sums
    and band energies against the oracle's calc_rhoe, update! and
    calc_energies, FP64 and mixed."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from oracle import systems, ops, energies
    at = systems.diamond_supercell(3, 10.2631, displace=0.02, seed=20261203)
    Ho = systems.Hamiltonian(at, [systems.psp("Si-q4.gth")], 15.0, Nstates=480)
    pw = Ho.pw
    H = pwb200.Hamiltonian(pwb200.System(["Si"] * at.positions.shape[1], at.positions, at.LatVecs),
                           [systems.psp("Si-q4.gth")], 15.0)
    H.setup_density()
    assert H.basis.Ngw[0] == pw.gvecw.Ngw[0] == 80797
    rng = np.random.default_rng(5)
    ngw, nb = pw.gvecw.Ngw[0], 480
    psi = (rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb))) / np.sqrt(2 * ngw)
    Focc = np.zeros(nb)
    Focc[:432] = 2.0
    Ho.Focc = Focc[:, None]
    rho_o = ops.calc_rhoe(Ho, [psi], Focc=Focc[:, None])
    Ho.update(rho_o)
    E_o = energies.calc_energies(Ho, [psi], rho_o)
    dVol = pw.CellVolume / pw.Npoints
    for prec, tol_rel in (("c128", None), ("c64", 2e-5)):
        dt = torch.complex128 if prec == "c128" else torch.complex64
        x = to_dev(psi, dt)
        rho = torch.zeros(pw.Npoints, dtype=torch.float64, device="cuda")
        H.ctx.calc_rhoe(0, x, Focc, rho)
        Vps = torch.from_numpy(H.V_Ps_loc).cuda()
        sums = H.ctx.update(rho, Vps)
        ekin, enl = H.ctx.band_energies(0, x, Focc)
        got = {"Kinetic": ekin, "Ps_nloc": enl, "Hartree": 0.5 * sums[0] * dVol, "Ps_loc": sums[1] * dVol,
               "XC": sums[2] * dVol}
        for k, v in got.items():
            err = abs(v - E_o[k])
            if tol_rel is None:
                assert err < 1e-9 * max(1.0, abs(E_o[k])), (prec, k, v, E_o[k])
            else:
                assert err < tol_rel * max(1.0, abs(E_o[k])), (prec, k, v, E_o[k])
        r = rho.cpu().numpy()
        assert rel_err(r, rho_o) < (1e-11 if prec == "c128" else 2e-5)
    H.ctx.close()
