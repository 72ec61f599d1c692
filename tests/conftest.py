import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "pwdft.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: multi-second CPU oracle runs")


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def si_fcc_scf():
    """Converged oracle SCF for the reference's Si fcc test system."""
    from oracle import systems, scf
    H = systems.Ham_Si_fcc()
    E, psiks, rho = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8)
    return H, E, psiks, rho
