"""Wavefunction files in the reference's format (read_psiks.jl:1-21,
KS_solve_DCM.jl:295-300): host and device blocks written by pwb200.io read
back by the oracle's reader and the other way round, bit-exact; the byte
layout is the raw column-major ComplexF64 matrix; a wrong size is an error;
the device SCF writes them with savewfc."""
import numpy as np
import pytest

from conftest import cuda_ok


def _blocks(rng, Ngw=(37, 41, 29), Nstates=5):
    return [rng.standard_normal((n, Nstates)) + 1j * rng.standard_normal((n, Nstates)) for n in Ngw]


def test_host_round_trip_and_layout(tmp_path):
    from oracle import wfc_io
    from pwb200 import io
    rng = np.random.default_rng(0)
    ps = _blocks(rng)
    io.write_psiks(ps, str(tmp_path))
    back = wfc_io.read_wfc([p.shape[0] for p in ps], 5, str(tmp_path))
    assert all(np.array_equal(a, b) for a, b in zip(ps, back))
    raw = (tmp_path / "WFC_ikspin_2.data").read_bytes()
    assert len(raw) == 41 * 5 * 16
    v = np.frombuffer(raw, dtype="<f8")
    assert v[0] == ps[1][0, 0].real and v[1] == ps[1][0, 0].imag and v[2] == ps[1][1, 0].real  # column-major
    wfc_io.write_wfc(ps, str(tmp_path))
    back2 = io.read_psiks([p.shape[0] for p in ps], 5, directory=str(tmp_path))
    assert all(np.array_equal(a, b) for a, b in zip(ps, back2))
    with pytest.raises(ValueError):
        io.read_psiks([40, 41, 29], 5, directory=str(tmp_path))


@pytest.mark.gpu
def test_device_blocks_and_scf_savewfc(tmp_path):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from pwb200 import io, scf
    from oracle import wfc_io, systems
    rng = np.random.default_rng(1)
    ps = _blocks(rng)
    dev = [torch.from_numpy(np.ascontiguousarray(p.T)).cuda() for p in ps]
    io.write_psiks(dev, str(tmp_path))
    back = wfc_io.read_wfc([p.shape[0] for p in ps], 5, str(tmp_path))
    assert all(np.array_equal(a, b) for a, b in zip(ps, back))
    d2 = io.read_psiks([p.shape[0] for p in ps], 5, directory=str(tmp_path), device="cuda:0", dtype=torch.complex64)
    assert all(np.abs(a.cpu().numpy().T - b).max() < 1e-6 * np.abs(b).max() for a, b in zip(d2, ps))
    at = systems.si_fcc_atoms()
    H = pwb200.Hamiltonian(pwb200.System(["Si", "Si"], at.positions, at.LatVecs), [systems.psp("Si-q4.gth")], 15.0,
                           meshk=(2, 2, 2))
    d = tmp_path / "scf"
    d.mkdir()
    res = scf.KS_solve_SCF(H, etot_conv_thr=1e-6, savewfc=True, wfc_dir=str(d))
    got = io.read_psiks(H.basis.Ngw, res["psiks"][0].shape[0], directory=str(d))
    for ik in range(H.basis.Nkpt):
        assert np.array_equal(got[ik], res["psiks"][ik].cpu().numpy().T)
    H.ctx.close()
