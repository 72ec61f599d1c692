"""Errors of the device path against the FP64 oracle for the benchmark
configurations, as a table (run on a GPU: python tests/config_errors.py).

  C2  Si64 (75^3 grid, Ngw 23,871), 160 bands: op_H, calc_rhoe and the band
      energies <psi_b|H|psi_b> on one orthonormal psi
  C3  Al4 on the full 8x8x8 mesh (260 k-points, 10 bands): the batched op_H
      per k-point and its band energies
  C5  Si216 (120^3 grid), 480 bands: the energy components of update! and
      the band energies on one psi and its density

Both precisions of the same kernels: FP64 (complex128 blocks) and the mixed
path (complex64 blocks, tensor-core projections).  Not collected by pytest;
tests/test_bench_shapes_gpu.py asserts the tolerances at these shapes.
"""
import json
import os
import sys
import traceback

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "pwdft.jl_b200")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import pwb200  # noqa: E402
from oracle import energies, ops, systems  # noqa: E402

DTYPES = (("fp64", torch.complex128), ("mixed", torch.complex64))


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def smooth(pw, rng):
    """A smooth random perturbation of V_loc (|G|^2 <= 4), max 1."""
    g = pw.gvec
    sel = g.G2 <= 4.0
    c = np.zeros(pw.Npoints, dtype=np.complex128)
    c[g.idx_g2r[sel]] = rng.standard_normal(sel.sum()) + 1j * rng.standard_normal(sel.sum())
    N1, N2, N3 = pw.Ns
    f = np.fft.ifftn(c.reshape(N3, N2, N1)).real.ravel()
    return f / np.abs(f).max()


def orthonormal(rng, ngw, nb):
    return np.linalg.qr(rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb)))[0]


def dev(a, dt):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().to(dt).contiguous()


def c2(out):
    H = systems.Ham_Si64(Nstates=160)
    pw = H.pw
    rng = np.random.default_rng(20261203)
    H.V_Total = H.V_Ps_loc + 0.01 * smooth(pw, rng)
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    ctx.set_vloc(H.V_Total)
    ctx.set_nonlocal(0, H.betaNL[0])
    ctx.set_nonlocal_coef(H.nl_triplets)
    psi = orthonormal(rng, pw.gvecw.Ngw[0], 160)
    ref = ops.op_H(H, psi, 0)
    w = np.full(160, 2.0)
    rho_ref = ops.calc_rhoe(H, [psi], Focc=w[:, None])
    eb = np.real(np.sum(psi.conj() * ref, axis=0))
    for name, dt in DTYPES:
        x = dev(psi, dt)
        y = torch.empty_like(x)
        ctx.apply(0, 0, x, y, pwb200.PW_OP_H)
        r = torch.zeros(pw.Npoints, dtype=torch.float64, device="cuda")
        ctx.calc_rhoe(0, x, w, r)
        got = y.cpu().numpy().T.astype(np.complex128)
        ebd = np.real(np.sum(psi.conj() * got, axis=0))
        out["C2 Si64 160 bands " + name] = {"op_H max rel": rel(got, ref), "rho max rel": rel(r.cpu().numpy(), rho_ref),
                                           "band energy max |err| (Ha)": float(np.abs(ebd - eb).max())}
    ctx.close()


def c3(out):
    Ho = systems.Ham_Al4(meshk=(8, 8, 8))
    pw = Ho.pw
    rng = np.random.default_rng(31)
    Ho.V_Total = Ho.V_Ps_loc + 0.01 * smooth(pw, rng)
    nk = pw.kpoints.Nkpt
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(k) for k in range(nk)])
    ctx.set_vloc(Ho.V_Total)
    for ik in range(nk):
        ctx.set_nonlocal(ik, Ho.betaNL[ik])
    ctx.set_nonlocal_coef(Ho.nl_triplets)
    psis = [orthonormal(rng, pw.gvecw.Ngw[ik], 10) for ik in range(nk)]
    refs = [ops.op_H(Ho, psis[ik], ik) for ik in range(nk)]
    for name, dt in DTYPES:
        X = [dev(p, dt) for p in psis]
        HX = [torch.empty_like(x) for x in X]
        ctx.apply_multi(list(range(nk)), 0, X, HX)
        got = [HX[ik].cpu().numpy().T.astype(np.complex128) for ik in range(nk)]
        de = max(float(np.abs(np.real(np.sum(psis[ik].conj() * (got[ik] - refs[ik]), axis=0))).max()) for ik in range(nk))
        out["C3 Al4 8x8x8 (260 k) " + name] = {"op_H max rel over k": max(rel(got[ik], refs[ik]) for ik in range(nk)),
                                               "band energy max |err| (Ha)": de}
    ctx.close()


def c5(out):
    at = systems.diamond_supercell(3, 10.2631, displace=0.02, seed=20261203)
    psp = systems.psp("Si-q4.gth")
    Ho = systems.Hamiltonian(at, [psp], 15.0, Nstates=480)
    pw = Ho.pw
    H = pwb200.Hamiltonian(pwb200.System(["Si"] * at.positions.shape[1], at.positions, at.LatVecs), [psp], 15.0)
    H.setup_density()
    rng = np.random.default_rng(5)
    psi = orthonormal(rng, pw.gvecw.Ngw[0], 480)
    Focc = np.zeros(480)
    Focc[:432] = 2.0
    Ho.Focc = Focc[:, None]
    rho_o = ops.calc_rhoe(Ho, [psi], Focc=Focc[:, None])
    Ho.update(rho_o)
    Ho.E_NN = 0.0
    E_o = energies.calc_energies(Ho, [psi], rho_o)
    dVol = pw.CellVolume / pw.Npoints
    natoms = at.positions.shape[1]
    for name, dt in DTYPES:
        x = dev(psi, dt)
        rho = torch.zeros(pw.Npoints, dtype=torch.float64, device="cuda")
        H.ctx.calc_rhoe(0, x, Focc, rho)
        sums = H.ctx.update(rho, torch.from_numpy(H.V_Ps_loc).cuda())
        ekin, enl = H.ctx.band_energies(0, x, Focc)
        got = {"Kinetic": ekin, "Ps_nloc": enl, "Hartree": 0.5 * sums[0] * dVol, "Ps_loc": sums[1] * dVol,
               "XC": sums[2] * dVol}
        row = {k + " |err| (Ha)": abs(v - E_o[k]) for k, v in got.items()}
        row["sum |err| per atom (Ha)"] = abs(sum(got.values()) - sum(E_o[k] for k in got)) / natoms
        out["C5 Si216 480 bands " + name] = row


def main():
    out = {}
    for f in (c2, c3, c5):
        try:
            f(out)
        except Exception:
            traceback.print_exc()
        print(json.dumps(out), flush=True)
    for cfg, row in out.items():
        print("%-32s %s" % (cfg, ", ".join("%s %.2e" % kv for kv in row.items())))


if __name__ == "__main__":
    main()
