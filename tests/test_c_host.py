"""A C host (pwdft.jl_b200/examples/op_h_from_c.c) built against
include/pwb200.h and libpwb200.so alone: it compiles as C99 and links;
the basis it builds with the library's host functions (grid size,
init_gvec, init_gvecw) has the oracle's grid and sphere sizes; without a
GPU pw_create fails with a status (exit 2), and on a GPU op_K + op_V_loc
with a constant potential matches 0.5|G|^2 psi + V0 psi (exit 0)."""
import os
import subprocess

import pytest

from conftest import cuda_ok

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pwdft.jl_b200")


@pytest.fixture(scope="module")
def c_host(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("c_host") / "op_h_from_c")
    libdir = os.path.join(PKG, "pwb200")
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(PKG, "examples", "op_h_from_c.c"), "-L", libdir, "-lpwb200",
                    "-Wl,-rpath," + libdir, "-lm", "-o", exe], check=True)
    return exe


def _basis_line(out):
    line = [l for l in out.splitlines() if l.startswith("basis:")][0]
    f = line.replace(",", " ").split()
    return (int(f[3]), int(f[4]), int(f[5])), int(f[8]), int(f[11])


def test_c_host_builds_and_basis_matches_oracle(c_host):
    from oracle import systems
    r = subprocess.run([c_host], capture_output=True, text=True, timeout=120)
    Ns, Ng, Ngw = _basis_line(r.stdout)
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    assert Ns == tuple(H.pw.Ns) and Ng == H.pw.gvec.Ng and Ngw == H.pw.gvecw.Ngw[0]
    if not cuda_ok():
        assert r.returncode == 2 and "pw_create failed" in r.stderr


@pytest.mark.gpu
def test_c_host_op_h_on_gpu(c_host):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    r = subprocess.run([c_host], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.stdout, r.stderr)
