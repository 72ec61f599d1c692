"""k-point sharding (pwb200.kshard): the partition, and the density of a
2-rank gloo group (each rank sums calc_rhoe over its own k-points, then
all-reduce) against the single-process sum, on CPU with the oracle's
calc_rhoe; the whole SCF driver on 2 gloo ranks with the NumPy stand-in
against the single-process driver, on CPU; and on one GPU, the device SCF sharded over 2 gloo ranks
against the unsharded SCF (the kernels of the two ranks do not wait on
each other: the exchange is host-side)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import cuda_ok

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_shard_kpoints_balanced_and_complete():
    from pwb200.kshard import shard_kpoints
    rng = np.random.default_rng(0)
    costs = list(rng.integers(1000, 1300, 35))
    for world in (1, 2, 3, 4, 8, 40):
        own = shard_kpoints(costs, world)
        allk = sorted(k for o in own for k in o)
        assert allk == list(range(35))
        loads = [sum(costs[k] for k in o) for o in own]
        if world <= 35:
            assert max(loads) - min(loads) <= max(costs)
    assert shard_kpoints([5.0, 5.0, 5.0], 2) == [[0, 2], [1]]


def _rank_density(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    from oracle import systems, ops
    from pwb200.kshard import KShards
    H = systems.Ham_Si_fcc(meshk=(2, 2, 2), extra_states=0)
    rng = np.random.default_rng(4)
    psiks = [rng.standard_normal((n, 4)) + 1j * rng.standard_normal((n, 4)) for n in H.pw.gvecw.Ngw]
    sh = KShards(H.pw.gvecw.Ngw, 4)
    part = np.zeros(H.pw.Npoints)
    if sh.mine:
        sub = [psiks[ik] if ik in sh.mine else np.zeros_like(psiks[ik]) for ik in range(len(psiks))]
        part = ops.calc_rhoe(H, sub)
    t = sh.sum_(torch.from_numpy(part))
    if rank == 0:
        np.save(out, np.stack([t.numpy(), ops.calc_rhoe(H, psiks)]))
    dist.destroy_process_group()


def test_two_rank_density_matches_single(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "rho.npy")
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_rank_density, args=(2, port, out), nprocs=2, start_method="spawn")
    a, b = np.load(out)
    assert np.abs(a - b).max() < 1e-12 * np.abs(b).max()


def _rank_scf(rank, world, port, out):
    """One rank of the SCF driver on the NumPy stand-in, k-points sharded
    over a gloo group."""
    import json
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from numpy_ctx import HostHam
    from oracle import systems, scf as oscf
    from pwb200 import scf
    Ho = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    start = oscf.rand_BlochWavefunc(Ho, seed=21)
    Hd = HostHam(Ho, (2, 2, 2))
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    res = scf.KS_solve_SCF(Hd, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-6, precision="fp64", psiks=ps)
    with open(out + ".%d" % rank, "w") as f:
        json.dump({"E": [r[1] for r in res["log"]], "k": res["kpoints_local"], "evals": res["evals"].tolist()}, f)
    dist.destroy_process_group()


def test_two_rank_scf_matches_single(tmp_path):
    """The SCF driver's exchange steps (density, band energies, eigenvalues
    all-reduced over the group; KS_solve_SCF's k loop over this rank's
    k-points) on 2 gloo ranks reproduce the single-process SCF step by step."""
    import json
    import torch
    import torch.multiprocessing as mp
    from numpy_ctx import HostHam
    from oracle import systems, scf as oscf
    from pwb200 import scf
    Ho = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    start = oscf.rand_BlochWavefunc(Ho, seed=21)
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    ref = scf.KS_solve_SCF(HostHam(Ho, (2, 2, 2)), betamix=0.2, mix_method="pulay", etot_conv_thr=1e-6,
                           precision="fp64", psiks=ps)
    out = str(tmp_path / "scf")
    port = 29700 + os.getpid() % 1000
    mp.start_processes(_rank_scf, args=(2, port, out), nprocs=2, start_method="spawn")
    r0, r1 = [json.load(open(out + ".%d" % r)) for r in (0, 1)]
    assert sorted(r0["k"] + r1["k"]) == list(range(Ho.pw.kpoints.Nkpt)) and r0["k"] and r1["k"]
    E = [row[1] for row in ref["log"]]
    for r in (r0, r1):
        assert len(r["E"]) == len(E)
        assert np.abs(np.array(r["E"]) - np.array(E)).max() < 1e-10
        assert np.abs(np.array(r["evals"]) - ref["evals"]).max() < 1e-9


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
H = pwb200.Hamiltonian(pwb200.System(["Si", "Si"], at.positions, at.LatVecs), [systems.psp("Si-q4.gth")], 15.0,
                       meshk=(3, 3, 3))
res = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-10, precision=sys.argv[1])
print("RESULT", json.dumps({"rank": int(os.environ.get("RANK", "0")), "E": res["energies"]["Total"],
                            "k": res["kpoints_local"], "it": res["iterations"]}), flush=True)
if dist.is_initialized():
    dist.destroy_process_group()
''' % (ROOT, os.path.join(ROOT, "pwdft.jl_b200"))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sharded_device_scf_matches_single(tmp_path, precision):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import json
    script = tmp_path / "scf_run.py"
    script.write_text(SCF_SCRIPT)
    def run(cmd):
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-3000:]
        return [json.loads(l.split("RESULT ", 1)[1]) for l in p.stdout.splitlines() if l.startswith("RESULT ")]
    single = run([sys.executable, str(script), precision])[0]
    port = str(29600 + os.getpid() % 1000)
    multi = run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                 "--master-addr=127.0.0.1", "--master-port=" + port, str(script), precision])
    assert len(multi) == 2
    assert sorted(multi[0]["k"] + multi[1]["k"]) == list(range(14))
    for m in multi:
        assert abs(m["E"] - single["E"]) < 1e-9, (m, single)
