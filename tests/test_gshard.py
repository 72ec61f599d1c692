"""Gamma-point sharding (pwb200.gshard): one k-point's op_H split by bands,
its Rayleigh-Ritz Grams and rotations by plane-wave rows, the small FP64
problems solved on rank 0 and broadcast.

CPU:
  - the slices cover the ranges exactly;
  - diag_LOBPCG_gamma on the NumPy stand-in, 1 process and 2 gloo ranks,
    against the oracle's diag_LOBPCG_k from the same start (Si fcc, Gamma,
    8 bands): the same iteration count and eigenvalues to 1e-9;
  - the SCF driver on 2 gloo ranks (Gamma sharding chosen for one k-point)
    against the single-process driver, step by step (1e-10 Ha).
GPU: the device SCF of Si fcc at Gamma on 2 gloo ranks sharing one GPU (the
exchange is host-side, no kernel of one rank waits for the other) against
the single-process SCF (1e-9 Ha).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import cuda_ok

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_split_covers_range():
    from pwb200.gshard import split
    for n in (0, 1, 7, 160, 80797):
        for w in (1, 2, 3, 8):
            sl = split(n, w)
            assert sl[0][0] == 0 and sl[-1][1] == n and len(sl) == w
            assert all(a <= b for a, b in sl) and all(sl[i][1] == sl[i + 1][0] for i in range(w - 1))
            assert max(b - a for a, b in sl) - min(b - a for a, b in sl) <= 1


def _lobpcg_case():
    from oracle import systems
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1), extra_states=4)
    H.V_Total = H.V_Ps_loc + 0.02 * np.cos(0.01 * np.arange(H.pw.Npoints))
    ngw = H.pw.gvecw.Ngw[0]
    rng = np.random.default_rng(13)
    X0 = np.linalg.qr(rng.standard_normal((ngw, 8)) + 1j * rng.standard_normal((ngw, 8)))[0]
    return H, X0


def _rank_lobpcg(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from numpy_ctx import NumpyCtx
    from pwb200.gshard import GammaShards, diag_LOBPCG_gamma
    H, X0 = _lobpcg_case()
    X = torch.from_numpy(np.ascontiguousarray(X0.T))
    ev, it = diag_LOBPCG_gamma(NumpyCtx(H), X, GammaShards(), tol=1e-9, NiterMax=200)
    np.save(out + ".%d.npy" % rank, np.concatenate([[it], ev, np.abs(X.numpy()).ravel()[:50]]))
    dist.destroy_process_group()


def test_gamma_lobpcg_matches_oracle_one_and_two_ranks(tmp_path):
    import torch
    import torch.multiprocessing as mp
    from numpy_ctx import NumpyCtx
    from oracle.lobpcg import diag_LOBPCG_k
    from pwb200.gshard import GammaShards, diag_LOBPCG_gamma
    H, X0 = _lobpcg_case()
    Xo = X0.copy()
    stats = []
    ev_o = diag_LOBPCG_k(H, Xo, 0, tol=1e-9, NiterMax=200, stats=stats)
    X = torch.from_numpy(np.ascontiguousarray(X0.T))
    ev1, it1 = diag_LOBPCG_gamma(NumpyCtx(H), X, GammaShards(), tol=1e-9, NiterMax=200)
    assert it1 == stats[0]
    assert np.abs(ev1 - ev_o).max() < 1e-9
    out = str(tmp_path / "lob")
    port = 29800 + os.getpid() % 100
    mp.start_processes(_rank_lobpcg, args=(2, port, out), nprocs=2, start_method="spawn")
    r0, r1 = [np.load(out + ".%d.npy" % r) for r in (0, 1)]
    assert np.array_equal(r0, r1)                      # the ranks hold identical blocks
    assert int(r0[0]) == it1
    assert np.abs(r0[1:9] - ev_o).max() < 1e-9


def _rank_scf(rank, world, port, out):
    import json
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from numpy_ctx import HostHam
    from oracle import systems, scf as oscf
    from pwb200 import scf
    Ho = systems.Ham_Si_fcc(meshk=(1, 1, 1), extra_states=2)
    start = oscf.rand_BlochWavefunc(Ho, seed=31)
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    res = scf.KS_solve_SCF(HostHam(Ho, (1, 1, 1)), Nstates=6, betamix=0.3, mix_method="pulay", etot_conv_thr=1e-8,
                           precision="fp64", psiks=ps)
    with open(out + ".%d" % rank, "w") as f:
        json.dump({"E": [r[1] for r in res["log"]], "evals": res["evals"].tolist()}, f)
    dist.destroy_process_group()


def test_two_rank_gamma_scf_matches_single(tmp_path):
    import json
    import torch
    import torch.multiprocessing as mp
    from numpy_ctx import HostHam
    from oracle import systems, scf as oscf
    from pwb200 import scf
    Ho = systems.Ham_Si_fcc(meshk=(1, 1, 1), extra_states=2)
    start = oscf.rand_BlochWavefunc(Ho, seed=31)
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    ref = scf.KS_solve_SCF(HostHam(Ho, (1, 1, 1)), Nstates=6, betamix=0.3, mix_method="pulay", etot_conv_thr=1e-8,
                           precision="fp64", psiks=ps)
    out = str(tmp_path / "scf")
    port = 29900 + os.getpid() % 100
    mp.start_processes(_rank_scf, args=(2, port, out), nprocs=2, start_method="spawn")
    E = [row[1] for row in ref["log"]]
    for r in (0, 1):
        got = json.load(open(out + ".%d" % r))
        assert len(got["E"]) == len(E)
        assert np.abs(np.array(got["E"]) - np.array(E)).max() < 1e-10
        assert np.abs(np.array(got["evals"]) - ref["evals"]).max() < 1e-9


SCF_SCRIPT = r'''
import os, sys, json
sys.path[:0] = [%r, %r]
import numpy as np, torch, torch.distributed as dist
import pwb200
from pwb200 import scf
from oracle import systems
if os.environ.get("WORLD_SIZE", "1") != "1":
    dist.init_process_group("gloo")
at = systems.si_fcc_atoms()
H = pwb200.Hamiltonian(pwb200.System(["Si", "Si"], at.positions, at.LatVecs), [systems.psp("Si-q4.gth")], 15.0)
res = scf.KS_solve_SCF(H, Nstates=8, betamix=0.3, mix_method="pulay", etot_conv_thr=1e-10, precision="fp64")
print("RESULT", json.dumps({"rank": int(os.environ.get("RANK", "0")), "E": res["energies"]["Total"],
                            "it": res["iterations"], "evals": res["evals"][:, 0].tolist()}), flush=True)
if dist.is_initialized():
    dist.destroy_process_group()
''' % (ROOT, os.path.join(ROOT, "pwdft.jl_b200"))


@pytest.mark.gpu
def test_gamma_sharded_device_scf_matches_single(tmp_path):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import json
    script = tmp_path / "scf_gamma.py"
    script.write_text(SCF_SCRIPT)

    def run(cmd):
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-3000:]
        return [json.loads(l.split("RESULT ", 1)[1]) for l in p.stdout.splitlines() if l.startswith("RESULT ")]
    single = run([sys.executable, str(script)])[0]
    port = str(29650 + os.getpid() % 100)
    multi = run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                 "--master-addr=127.0.0.1", "--master-port=" + port, str(script)])
    assert len(multi) == 2
    for m in multi:
        assert abs(m["E"] - single["E"]) < 1e-9, (m, single)
        assert np.abs(np.array(m["evals"][:4]) - np.array(single["evals"][:4])).max() < 1e-8
