"""Failure detection on the device, without faulting or hanging the GPU.

  - Bounded waits: the cooperative kernels of the FP64 eigensolver
    (pw_eigh: Cholesky, triangular inverse, tridiagonalisation) synchronise
    with a grid barrier whose waits give up after a poll limit, record an
    error word and let the kernel run to completion.  A test-only hook
    shortens the limit and makes one CTA withhold its arrivals: the others'
    waits run out, pw_eigh reports PW_ERR_TIMEOUT, and once the hook is
    cleared the same context solves the next problem correctly.
  - Non-finite values: a NaN in the density, the wavefunctions or a LOBPCG
    block is reported as PW_ERR_NAN by the FP64 reductions that meet it
    (pw_update, pw_band_energies; pw_lobpcg reports it from its Ritz values
    or from the Cholesky of an overlap it meets first), and the context
    stays usable.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fcc():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from pwb200.system import kpoint_grid
    from oracle import systems
    Ho = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    sysm = pwb200.System(["Si", "Si"], Ho.atoms.positions, Ho.atoms.LatVecs)
    H = pwb200.Hamiltonian(sysm, [systems.psp("Si-q4.gth")], 15.0)
    H.setup_density()
    yield H
    H.ctx.close()


def _hook(limit, withhold):
    import pwb200
    f = pwb200.lib().pwk_test_gsync
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_longlong, C.c_int]
    assert f(0, limit, withhold) == 0


def _pencil(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    T = A + A.conj().T
    B = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    G = B @ B.conj().T + np.eye(n)
    return T, G


def test_eigh_barrier_timeout_is_reported_and_context_recovers(fcc):
    import torch
    import pwb200
    import scipy.linalg as sla
    ctx = fcc.ctx
    n, k = 192, 40
    T, G = _pencil(n, 3)
    dev = lambda M: torch.from_numpy(np.ascontiguousarray(M.T)).cuda()
    try:
        _hook(1 << 14, 0)
        with pytest.raises(pwb200.PWError) as e:
            ctx.eigh(dev(T), dev(G), k=k)
        assert e.value.status == pwb200._lib.PW_ERR_TIMEOUT
    finally:
        _hook(0, -1)
    lam, S = ctx.eigh(dev(T), dev(G), k=k)
    ref = sla.eigh(T, G, eigvals_only=True)[:k]
    assert np.abs(lam.cpu().numpy() - ref).max() < 1e-10 * np.abs(ref).max()
    ctx.check_device()


def test_non_finite_values_are_reported(fcc):
    import torch
    import pwb200
    H = fcc
    ctx = H.ctx
    N = H.basis.Npoints
    rho = torch.full((N,), 0.01, dtype=torch.float64, device="cuda")
    Vps = torch.from_numpy(H.V_Ps_loc).cuda()
    rho[17] = float("nan")
    with pytest.raises(pwb200.PWError) as e:
        ctx.update(rho, Vps)
    assert e.value.status == pwb200._lib.PW_ERR_NAN
    rho[17] = 0.01
    ctx.update(rho, Vps)                      # usable again
    ngw = H.basis.Ngw[0]
    rng = np.random.default_rng(4)
    X = torch.from_numpy(np.ascontiguousarray(np.linalg.qr(
        rng.standard_normal((ngw, 4)) + 1j * rng.standard_normal((ngw, 4)))[0].T)).cuda()
    Xn = X.clone()
    Xn[1, 5] = complex("nan+0j")
    with pytest.raises(pwb200.PWError) as e:
        ctx.band_energies(0, Xn, np.full(4, 2.0))
    assert e.value.status == pwb200._lib.PW_ERR_NAN
    with pytest.raises(pwb200.PWError) as e:
        ctx.lobpcg(0, 0, Xn, tol=1e-8, nitermax=5)
    # the NaN reaches the Ritz values, or first the Cholesky of an overlap
    assert e.value.status in (pwb200._lib.PW_ERR_NAN, pwb200._lib.PW_ERR_NOT_POSDEF)
    ev, _ = ctx.lobpcg(0, 0, X, tol=1e-8, nitermax=200)
    assert np.all(np.isfinite(ev))
    ctx.check_device()
