#!/usr/bin/env python
"""op_H throughput of the B200 path on the Si64 microbenchmark.

Workload (the op_H + LOBPCG microbenchmark configuration): Si 64-atom cubic
supercell (2x2x2 conventional diamond cells, a = 20.5262 bohr), Gamma only,
GTH-Pade Si-q4, ecutwfc = 15 Ha -> 75^3 grid (the reference's grid rule),
Ngw = 23,871, 160 bands, NbetaNL = 320.  psi: seeded complex Gaussian,
Cholesky-orthonormalised; V_loc = V_Ps_loc + a seeded smooth random field
(|G|^2 <= 4, max 0.01 Ha).  Synthetic inputs, generated here.

One step = one full op_H (K + V_loc + V_Ps_nloc) over all 160 bands.
  value        mixed precision (complex64, FP32 FFTs) op_H, inputs resident
               in HBM, device time (CUDA events), L2 flushed between steps
  e2e          the reference-facing host call pw_op_H_host on pinned host
               ComplexF64 arrays: H2D copy + op_H + D2H copy every step
  fp64_*       the same step on the FP64 path (complex128)
  roofline     the pruned-FFT op_V_loc round trip (K-zinv + K-plane + K-zfwd),
               timed alone, against the HBM copy peak
Unit: GB/s of algorithmic bytes, the FP32 byte model of the op_V_loc round
trip, c*(3*Ngw + 4*P) + 4*N/Nb per band with c = 8 B and P = Nx_active*N2*N3,
applied to every arm so that ratios between arms are throughput ratios.

--impl reference times the reference algorithm on the host CPU: the FP64
NumPy/SciPy restatement of PWDFT.jl's op_H (the Julia reference cannot run
in this image), all host threads, a bounded sample of bands per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "pwdft.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np

METRIC = "SCF time-to-1e-6 Ha/atom & op_H GB/s: mixed-prec batched vs FP64 on 1 B200"
A_SI = 10.2631
NBANDS = 160
SEED = 20261203
PSP = os.path.join(ROOT, "tests", "golden", "psp", "Si-q4.gth")
PSP_AL = os.path.join(ROOT, "tests", "golden", "psp", "Al-q3.gth")
DIAMOND = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                    [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes (read + write) of one FP32 pruned-FFT round trip of the Si64
# op_H (160 bands: kf_zinv + kx_plane_vloc + kf_zfwd over both band batches),
# summed over the six launches of the first timed op_H:
#   PW_BENCH_NO_SCF=1 PW_BENCH_NO_CPU=1 PW_BENCH_NO_MULTIK=1 PW_BENCH_NO_AUTOTUNE=1 ncu --metrics
#     dram__bytes_read.sum,dram__bytes_write.sum --clock-control none
#     -k "regex:kf_zinv|kx_plane_vloc|kf_zfwd" -s 18 -c 6 python bench.py --steps 3 --warmup 3
FFT_TRAFFIC_BYTES = {"si64": 260.6e6}
FALLBACK_HBM_GBS = 6650.0


def si216_geometry(seed):
    """3x3x3 conventional diamond cells, a = 30.7893 bohr, every atom moved
    by seeded uniform noise in [-0.02, 0.02] bohr per component."""
    frac = np.array([(b + np.array([i, j, k])) / 3.0 for i in range(3) for j in range(3) for k in range(3)
                     for b in DIAMOND]).T
    LL = 3 * A_SI * np.eye(3)
    rng = np.random.default_rng(seed)
    return LL, LL @ frac + rng.uniform(-0.02, 0.02, frac.shape)


def scf_comparison(device, seed):
    """Si216 (480 bands, 432 occupied) KS_solve_SCF to |dEtot| < 1e-6 Ha/atom
    twice, mixed precision (FP64 switch at 1e-5 Ha/atom) and FP64, from the
    same start.  Times the SCF loop (set-up excluded: it is the same host
    code for both), after two untimed iterations of each path."""
    import torch
    import pwb200
    from pwb200 import scf
    LL, pos = si216_geometry(seed)
    H = pwb200.Hamiltonian(pwb200.System(["Si"] * pos.shape[1], pos, LL), [PSP], 15.0, device=device)
    nat = pos.shape[1]
    runs = {}
    # launch parameters tuned per precision by the library's autotuner, then
    # an untimed warm-up of both paths (first-use allocations and kernel
    # loads), so that neither timed run carries the other's one-time costs
    tunes = {prec: H.ctx.autotune(0, 480, pwb200.PW_C64 if prec == "mixed" else pwb200.PW_C128)
             for prec in ("mixed", "fp64")}
    for prec in ("mixed", "fp64"):
        H.ctx.set_tuning(**tunes[prec][0])
        scf.KS_solve_SCF(H, Nstates=480, betamix=0.2, mix_method="pulay", NiterMax=2, precision=prec, seed=seed)
    for prec in ("mixed", "fp64"):
        H.ctx.set_tuning(**tunes[prec][0])
        torch.cuda.synchronize()
        res = scf.KS_solve_SCF(H, Nstates=480, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-6 * nat,
                               fp64_switch=1e-5 * nat, precision=prec, seed=seed)
        runs[prec] = res
    rm, rd = runs["mixed"], runs["fp64"]
    nocc = 432
    out = {"system": "Si216 Gamma, a=30.7893 bohr, +-0.02 bohr seeded displacements, 480 bands (432 occupied), "
                     "LDA-VWN, Pulay beta 0.2, ecutwfc 15 Ha (120^3 grid, Ngw %d)" % H.basis.Ngw[0],
           "criterion": "|dEtot| < 1e-6 Ha/atom twice", "timed": "SCF loop (host set-up excluded)",
           "mixed_s": rm["time_s"], "fp64_s": rd["time_s"], "speedup": rd["time_s"] / rm["time_s"],
           "mixed_iterations": rm["iterations"], "fp64_iterations": rd["iterations"],
           "mixed_switched_to_fp64_at": rm["switched_to_fp64_at"],
           "mixed_diag_s": rm["time_diag_s"], "fp64_diag_s": rd["time_diag_s"],
           "Etot_mixed": rm["energies"]["Total"], "Etot_fp64": rd["energies"]["Total"],
           "dEtot_per_atom": abs(rm["energies"]["Total"] - rd["energies"]["Total"]) / nat,
           "max_devals_occupied": float(np.abs(rm["evals"][:nocc] - rd["evals"][:nocc]).max()),
           "lobpcg_iterations_per_step": {"mixed": [r[4] for r in rm["log"]], "fp64": [r[4] for r in rd["log"]]},
           "warmup": "2 untimed SCF iterations per precision first",
           "autotune": {p: {"chosen": t[0], **t[1]} for p, t in tunes.items()}}
    del H, runs, rm, rd
    torch.cuda.empty_cache()
    return out


def scf_al4(device, sharded=False):
    """Config C3's SCF: Al4 conventional fcc cell, GTH Al-q3, LDA-VWN,
    ecutwfc 15 Ha, 8x8x8 mesh reduced by symmetry (35 k-points), 10 states,
    Fermi-Dirac kT 0.01 Ha, Pulay 0.2, to |dE| < 1e-6 Ha/atom twice, with the
    LOBPCG of all k-points advanced together (pw_lobpcg_multi): mixed (FP64
    switch at 1e-5 Ha/atom) vs FP64, and the FP64 SCF with one LOBPCG per
    k-point for comparison; an untimed warm-up of each first."""
    import pwb200
    from pwb200 import scf
    LL = 7.6524 * np.eye(3)
    frac = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]]).T
    H = pwb200.Hamiltonian(pwb200.System(["Al"] * 4, LL @ frac, LL), [PSP_AL], 15.0, meshk=(8, 8, 8),
                           use_symmetry=True, device=device)
    kw = dict(Nstates=10, betamix=0.2, mix_method="pulay", use_smearing=True, kT=0.01, seed=SEED)
    arms = {"mixed": ("mixed", True), "fp64": ("fp64", True), "fp64_per_k": ("fp64", False)}
    for prec, batched in arms.values():
        scf.KS_solve_SCF(H, NiterMax=2, precision=prec, batched=batched, **kw)
    runs = {name: scf.KS_solve_SCF(H, etot_conv_thr=4e-6, fp64_switch=4e-5, precision=prec, batched=batched, **kw)
            for name, (prec, batched) in arms.items()}
    if sharded:
        import torch
        import torch.distributed as dist
        t = torch.tensor([runs[a]["time_s"] for a in arms], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        for a, v in zip(arms, t.tolist()):
            runs[a]["time_s"] = v
    rm, rd, rp = runs["mixed"], runs["fp64"], runs["fp64_per_k"]
    out = {"system": "Al4 fcc, 8x8x8 with symmetry (%d k-points, Ngw %d-%d), 10 states, kT 0.01, LDA-VWN" % (
               H.basis.Nkpt, min(H.basis.Ngw), max(H.basis.Ngw)),
           "mixed_s": rm["time_s"], "fp64_s": rd["time_s"], "speedup": rd["time_s"] / rm["time_s"],
           "fp64_per_k_lobpcg_s": rp["time_s"], "batched_vs_per_k_fp64": rp["time_s"] / rd["time_s"],
           "mixed_iterations": rm["iterations"], "fp64_iterations": rd["iterations"],
           "Etot_mixed": rm["energies"]["Total"], "Etot_fp64": rd["energies"]["Total"],
           "Etot_fp64_per_k": rp["energies"]["Total"],
           "dEtot_per_atom": abs(rm["energies"]["Total"] - rd["energies"]["Total"]) / 4}
    H.ctx.close()
    return out


def si64_geometry():
    frac = np.array([(b + np.array([i, j, k])) / 2.0 for i in range(2) for j in range(2) for k in range(2)
                     for b in DIAMOND]).T
    LL = 2 * A_SI * np.eye(3)
    return LL, LL @ frac


def smooth_field(Ns, G2, idx_g2r, rng):
    """Seeded random field with Fourier components only at |G|^2 <= 4,
    normalised to max |dV| = 1 (G2, idx_g2r: the density sphere)."""
    N1, N2, N3 = Ns
    sel = G2 <= 4.0
    c = np.zeros(N1 * N2 * N3, dtype=np.complex128)
    c[idx_g2r[sel]] = rng.standard_normal(sel.sum()) + 1j * rng.standard_normal(sel.sum())
    f = np.fft.ifftn(c.reshape(N3, N2, N1)).real.ravel()
    return f / np.abs(f).max()


def orthonormal_psi(ngw, nb, rng):
    psi = rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb))
    L = np.linalg.cholesky(psi.conj().T @ psi)
    return np.linalg.solve(L.conj(), psi.T).T  # psi * inv(L^H)


def byte_model(Ns, idx_gw2r, nb):
    """Algorithmic bytes per band of the op_V_loc round trip, FP32 (c = 8)."""
    N1, N2, N3 = Ns
    nxa = len(np.unique(np.asarray(idx_gw2r) % N1))
    P = nxa * N2 * N3
    return 8 * (3 * len(idx_gw2r) + 4 * P) + 4 * N1 * N2 * N3 / nb, nxa


def bf16_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[0]) for r in self.rows if num(r[0]) is not None]
        mx = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        busy = [num(r[0]) for r in self.rows if num(r[6]) is not None and num(r[6]) > 0]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[2 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(busy or sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


WORKLOADS = {"si64": 160, "si216": 480}   # bands of the op_H microbenchmark per system


def workload_name(workload, nbands, ns, ngw, nbeta):
    return "%s Gamma op_H (K+V_loc+V_Ps_nloc), %d bands, %d^3 grid, Ngw %d, NbetaNL %d" % (
        "Si64" if workload == "si64" else "Si216", nbands, ns, ngw, nbeta)


def build_workload(device, workload="si64"):
    """The op_H microbenchmark: Si64 (2x2x2 cells, 160 bands) or Si216 (3x3x3
    cells with seeded +-0.02 bohr displacements, 480 bands), Gamma,
    ecutwfc 15 Ha; V_loc = GTH local part + 0.01 Ha seeded smooth field;
    psi seeded complex Gaussian, orthonormalised."""
    import pwb200
    LL, pos = si64_geometry() if workload == "si64" else si216_geometry(SEED)
    sysm = pwb200.System(["Si"] * pos.shape[1], pos, LL)
    H = pwb200.Hamiltonian(sysm, [PSP], 15.0, device=device)
    rng = np.random.default_rng(SEED)
    b = H.basis
    H.update_vloc(H.V_Ps_loc + 0.01 * smooth_field(b.Ns, b.G2, b.idx_g2r, rng))
    psi = orthonormal_psi(H.basis.Ngw[0], WORKLOADS[workload], rng)
    return H, psi


def time_rayleigh_ritz(ctx, psi32, nb, steps, flush):
    """The LOBPCG contractions at this workload's size on the tensor cores:
    the Gram Q^H Q (3nb x 3nb over Ngw) and the rotation Q U (Ngw x 3nb ->
    nb), split-BF16x3; flops counted once per complex multiply-add (8)."""
    import torch
    ngw = psi32.shape[1]
    Q = torch.cat([psi32, psi32.roll(1, 0), psi32.roll(2, 0)]).contiguous()
    G = torch.zeros((3 * nb, 3 * nb), dtype=torch.complex128, device=psi32.device)
    g = torch.Generator(device=psi32.device).manual_seed(SEED)
    U = torch.randn((nb, 3 * nb), dtype=torch.complex128, device=psi32.device, generator=g)
    out = torch.empty((nb, ngw), dtype=torch.complex64, device=psi32.device)
    res = {}
    for name, fn, flops in (("gram", lambda: ctx.gram(Q, Q, G), 8.0 * (3 * nb) ** 2 * ngw),
                            ("rotate", lambda: ctx.rotate(Q, U, out), 8.0 * 3 * nb * nb * ngw)):
        # an NVTX range per product, so that a profiler can select its launches
        # (ncu --nvtx --nvtx-include "rr_gram/")
        torch.cuda.nvtx.range_push("rr_" + name)
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            flush.add_(1)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e))
        torch.cuda.nvtx.range_pop()
        ms = sum(ts) / len(ts)
        res[name] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
    return res


def time_eigh(ctx, nb, steps):
    """The FP64 generalized eigenproblem of every LOBPCG iteration at this
    workload's size (diag_LOBPCG.jl:185: eigen(Hermitian(T), Hermitian(G)),
    order 3nb, lowest nb pairs) on seeded Hermitian T and positive definite G."""
    import torch
    n = 3 * nb
    g = torch.Generator().manual_seed(SEED)
    A = torch.randn((n, n), dtype=torch.complex128, generator=g)
    T0 = (A + A.conj().T).cuda()
    B = torch.randn((n, n), dtype=torch.complex128, generator=g) / n ** 0.5
    G0 = (B @ B.conj().T + torch.eye(n, dtype=torch.complex128)).cuda()
    ts = []
    for i in range(steps + 2):
        T, G = T0.clone(), G0.clone()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        ctx.eigh(T, G, k=nb)
        e.record()
        torch.cuda.synchronize()
        if i >= 2:
            ts.append(s.elapsed_time(e))
    return {"n": n, "k": nb, "ms": sum(ts) / len(ts)}


def time_device(ctx, x, y, ops, steps, warmup, flush):
    import torch
    for _ in range(warmup):
        ctx.apply(0, 0, x, y, ops)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    stream = torch.cuda.current_stream()
    for s, e in ev:
        flush.add_(1)               # write 256 MB: evicts L2 between steps (untimed)
        s.record(stream)
        ctx.apply(0, 0, x, y, ops)
        e.record(stream)
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in ev]


def multik_comparison(device, steps, flush):
    """Batched op_H over uneven k-points: Al4 conventional fcc cell
    (a = 7.6524 bohr, GTH Al-q3, ecutwfc 15 Ha, 27^3 grid), 8x8x8 k-mesh
    reduced by time reversal, 10 bands per k-point, V_loc = V_Ps_loc + a
    seeded smooth field, psi seeded and orthonormal (FP32).  Three arms on
    the same blocks: a host loop of pw_apply per k-point, one pw_apply_multi
    (one launch per stage for all k-points), its CUDA-graph replay, and all
    stages in one persistent cooperative launch (PW_PERSISTENT);
    device time per full op_H, L2 flushed between steps."""
    import torch
    import pwb200
    from pwb200.system import kpoint_grid
    LL = 7.6524 * np.eye(3)
    frac = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]]).T
    k, w = kpoint_grid(LL, (8, 8, 8))
    H = pwb200.Hamiltonian(pwb200.System(["Al"] * 4, LL @ frac, LL), [PSP_AL], 15.0, kpts=k, wk=w, device=device)
    rng = np.random.default_rng(SEED + 3)
    b = H.basis
    H.update_vloc(H.V_Ps_loc + 0.01 * smooth_field(b.Ns, b.G2, b.idx_g2r, rng))
    nb = 10
    dev = f"cuda:{device}"
    X = [torch.from_numpy(np.ascontiguousarray(orthonormal_psi(b.Ngw[ik], nb, rng).T)).to(dev).to(torch.complex64)
         .contiguous() for ik in range(b.Nkpt)]
    Y = [torch.empty_like(x) for x in X]
    iks = list(range(b.Nkpt))
    nbytes = sum(nb * byte_model(b.Ns, b.idx_gw2r[ik], nb)[0] for ik in iks)
    ctx = H.ctx

    def loop():
        for ik in iks:
            ctx.apply(ik, 0, X[ik], Y[ik])

    arms = {"per_k_loop": loop, "batched": lambda: ctx.apply_multi(iks, 0, X, Y),
            "batched_graph": lambda: ctx.apply_multi(iks, 0, X, Y, graph=True),
            "batched_persistent": lambda: ctx.apply_multi(iks, 0, X, Y, persistent=True)}
    res = {}
    stream = torch.cuda.current_stream()
    for name, fn in arms.items():
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        n0 = ctx.launch_count()
        ts = []
        for _ in range(steps):
            flush.add_(1)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e))
        ms = sum(ts) / len(ts)
        res[name] = {"ms": ms, "GB_s": nbytes / (ms * 1e-3) / 1e9,
                     "launches_per_op_H": (ctx.launch_count() - n0) // steps}
    ctx.close()
    return {"workload": "Al4 fcc conventional, 8x8x8 k-mesh (time reversal: %d k-points, Ngw %d-%d), %d bands/k, "
                        "27^3 grid, NbetaNL %d, FP32" % (b.Nkpt, min(b.Ngw), max(b.Ngw), nb, H.NbetaNL),
            "bytes_per_op_H": nbytes, **res}


def reference_workload():
    """The op_H workload of the GPU arm rebuilt in the FP64 oracle: the same
    Si64 basis, the same V_loc (V_Ps_loc + the seeded smooth field drawn from
    the same generator) and the same orthonormal 160-band psi."""
    from oracle import systems
    H = systems.Ham_Si64(Nstates=NBANDS)
    rng = np.random.default_rng(SEED)
    g = H.pw.gvec
    H.V_Total = H.V_Ps_loc + 0.01 * smooth_field(H.pw.Ns, g.G2, g.idx_g2r, rng)
    psi = orthonormal_psi(H.pw.gvecw.Ngw[0], NBANDS, rng)
    return H, psi


def cpu_reference(H, psi, steps, warmup, budget_s=None):
    """The FP64 oracle op_H (the reference's per-band FFT loop restated in
    NumPy/SciPy) on the host cores, all 160 bands per step: `warmup` untimed
    steps, then `steps` timed ones (fewer if budget_s seconds run out).
    Returns (seconds per step, steps timed)."""
    from oracle import ops
    for _ in range(max(1, warmup)):
        ops.op_H(H, psi, 0)
    n = 0
    t0 = time.perf_counter()
    while n < steps:
        ops.op_H(H, psi, 0)
        n += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    return (time.perf_counter() - t0) / n, n


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--workload", default="si64", choices=sorted(WORKLOADS),
                    help="op_H microbenchmark system (si64: the headline configuration)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        H, psi = reference_workload()
        pw = H.pw
        bpb, _ = byte_model(pw.Ns, pw.gvecw.idx_gw2r[0], NBANDS)
        dt, reps = cpu_reference(H, psi, args.steps, args.warmup)
        val = NBANDS * bpb / dt / 1e9
        out = {"impl": "reference", "metric": METRIC, "value": val, "unit": "GB/s", "n_gpus": args.gpus,
               "steps": reps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
               "data": "synthetic",
               "config": {"workload": workload_name("si64", NBANDS, pw.Ns[0], pw.gvecw.Ngw[0], H.NbetaNL),
                          "global_batch": NBANDS, "seq_len": 0, "parallelism": "cpu"},
               "cpu_baseline": {"value": val, "unit": "GB/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": "all 160 bands per step, %d timed steps after %d warm-up steps, "
                                          "FP64 NumPy/SciPy, all host threads" % (reps, args.warmup)},
               "e2e": {"value": val, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return

    import torch
    import pwb200
    if os.environ.get("PW_BENCH_ONLY_MULTIK") == "1":
        # the batched-k op_H arms alone (a short command for profiling them)
        torch.cuda.set_device(local)
        flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")
        print(json.dumps({"multik": multik_comparison(local, max(5, args.steps // 20), flush)}))
        return
    if os.environ.get("PW_BENCH_ONLY_EIGH") == "1":
        # the FP64 generalized eigensolver alone at this workload's size (a
        # short command for profiling it)
        torch.cuda.set_device(local)
        H, _ = build_workload(local, args.workload)
        print(json.dumps({"eigh_fp64": time_eigh(H.ctx, WORKLOADS[args.workload], max(1, args.steps))}))
        return
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    H, psi = build_workload(local, args.workload)
    ctx = H.ctx
    nbands = WORKLOADS[args.workload]
    bpb, nxa = byte_model(H.basis.Ns, H.basis.idx_gw2r[0], nbands)
    step_bytes = bpb * nbands
    x32 = torch.from_numpy(np.ascontiguousarray(psi.T)).to(f"cuda:{local}").to(torch.complex64).contiguous()
    x64 = torch.from_numpy(np.ascontiguousarray(psi.T)).to(f"cuda:{local}").contiguous()
    y32, y64 = torch.empty_like(x32), torch.empty_like(x64)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")
    OPS = pwb200.PW_OP_H
    # launch parameters from the library's autotuner (timed candidates, no
    # cache file): the mixed-precision path is tuned before its timing, the
    # FP64 path before its own
    # (PW_BENCH_NO_AUTOTUNE=1 keeps the built-in defaults: profiling captures
    # of one kernel instantiation)
    no_tune = os.environ.get("PW_BENCH_NO_AUTOTUNE") == "1"
    notune = (ctx.get_tuning(), {})
    tune_mixed = notune if no_tune else ctx.autotune(0, nbands, pwb200.PW_C64)

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # clocks are sampled over every device-timed arm (op_H mixed, FFT round
    # trip, op_H FP64): the K-step op_H arm alone lasts only ~20 ms
    clk = ClockSampler(local)
    clk.__enter__()
    time.sleep(0.3)          # the sampler's first rows
    n0 = ctx._L.pw_launch_count(ctx.h)
    t_mixed = time_device(ctx, x32, y32, OPS, args.steps, args.warmup, flush)
    n1 = ctx._L.pw_launch_count(ctx.h)
    launches = (n1 - n0) * args.steps // (args.steps + args.warmup)
    t_fft = time_device(ctx, x32, y32, pwb200.PW_OP_VLOC, args.steps, args.warmup, flush)
    tune_fp64 = notune if no_tune else ctx.autotune(0, nbands, pwb200.PW_C128)
    t_fp64 = time_device(ctx, x64, y64, OPS, max(10, args.steps // 4), args.warmup, flush)
    for _ in range(max(1, int(0.5 / max(1e-4, sum(t_fp64) / len(t_fp64) * 1e-3 * 60)))):
        # keep the GPU busy on the timed arms long enough for the clock samples
        time_device(ctx, x64, y64, OPS, 60, 0, flush)
    torch.cuda.synchronize()
    clk.__exit__()
    ms = sum(t_mixed) / len(t_mixed)
    ms_fft = sum(t_fft) / len(t_fft)
    ms64 = sum(t_fp64) / len(t_fp64)
    if dist:
        t = torch.tensor([ms, ms_fft, ms64], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_fft, ms64 = [float(v) for v in t.tolist()]

    ctx.set_tuning(**tune_mixed[0])
    rr = time_rayleigh_ritz(ctx, x32, nbands, max(5, args.steps // 20), flush)
    rr["eigh"] = time_eigh(ctx, nbands, max(3, args.steps // 40))

    # SCF time to 1e-6 Ha/atom on Si216 (the large mixed-precision SCF
    # workload): mixed vs FP64 on this GPU, rank 0 of a single-process run
    scf_out = None
    if os.environ.get("PW_BENCH_NO_SCF") != "1" and world == 1:
        scf_out = scf_comparison(local, SEED)

    # end to end through the host drop-in, pinned host buffers
    pin_in = torch.from_numpy(np.ascontiguousarray(psi.T)).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    a_in = pin_in.numpy().T     # (Ngw, nb) Fortran view of the pinned buffer
    a_out = pin_out.numpy().T
    for _ in range(args.warmup):
        ctx.op_H_host(0, 0, a_in, a_out, OPS, pwb200.PW_C64)
    e2e_steps = max(5, args.steps // 10)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.op_H_host(0, 0, a_in, a_out, OPS, pwb200.PW_C64)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    # the same host call on the reference's precision (FP64 end to end)
    ctx.set_tuning(**tune_fp64[0])
    for _ in range(args.warmup):
        ctx.op_H_host(0, 0, a_in, a_out, OPS, pwb200.PW_C128)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.op_H_host(0, 0, a_in, a_out, OPS, pwb200.PW_C128)
    e2e64_s = (time.perf_counter() - t0) / e2e_steps
    ctx.set_tuning(**tune_mixed[0])
    if dist:
        t = torch.tensor([e2e_s, e2e64_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s, e2e64_s = [float(v) for v in t.tolist()]

    hbm, peak_kind = peaks()
    fft_gbs = step_bytes / (ms_fft * 1e-3) / 1e9
    out = {
        "metric": METRIC,
        "value": world * step_bytes / (ms * 1e-3) / 1e9,
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64",
        "data": "synthetic",
        "config": {"workload": workload_name(args.workload, nbands, H.basis.Ns[0], H.basis.Ngw[0], H.NbetaNL),
                   "global_batch": nbands * world, "seq_len": 0,
                   "parallelism": ("band shards: rank r applies op_H to its %d-band slice of a %d-band block "
                                   "(independent bands, no collective)" % (nbands, nbands * world)) if world > 1
                                  else "single",
                   "l2": "flushed between steps (256 MB write)", "bytes_per_band": bpb, "nx_active": nxa},
        "fp64_ms_per_step": ms64,
        "fp64_value": world * step_bytes / (ms64 * 1e-3) / 1e9,
        "gpu_launches": int(launches),
        "e2e": {"value": world * step_bytes / e2e_s / 1e9, "unit": "GB/s",
                "h2d_bytes_per_step": int(psi.size * 16), "d2h_bytes_per_step": int(psi.size * 16),
                "ms_per_step": e2e_s * 1e3},
        "e2e_fp64": {"value": world * step_bytes / e2e64_s / 1e9, "unit": "GB/s",
                     "h2d_bytes_per_step": int(psi.size * 16), "d2h_bytes_per_step": int(psi.size * 16),
                     "ms_per_step": e2e64_s * 1e3, "dtype": "c128",
                     "note": "pw_op_H_host computing in FP64, the reference's precision"},
        "autotune": {"mixed": {"chosen": tune_mixed[0], **tune_mixed[1]},
                     "fp64": {"chosen": tune_fp64[0], **tune_fp64[1]},
                     "note": "pw_autotune on this workload before the timed arms; ms of op_H and of the "
                             "Rayleigh-Ritz Gram + rotation with the default and the chosen parameters"},
        "roofline": {"bound": "hbm", "achieved": fft_gbs, "peak": hbm, "unit": "GB/s", "frac": fft_gbs / hbm,
                     "traffic": FFT_TRAFFIC_BYTES.get(args.workload), "peak_kind": peak_kind,
                     "kernel": "op_V_loc pruned-FFT round trip (K-zinv+K-plane+K-zfwd), %.4f ms" % ms_fft},
        "clocks": clk.summary(),
        "rayleigh_ritz": {"gram_3nb": rr["gram"], "rotate_3nb_to_nb": rr["rotate"], "unit": "TFLOP/s",
                          "peak_bf16_tflops": bf16_peak(), "gram_frac_of_bf16_peak": rr["gram"]["tflops"] / bf16_peak(),
                          "eigh_fp64": rr["eigh"],
                          "note": "split-BF16x3: three BF16 products per logical product, one counted"},
    }
    if scf_out is not None:
        out["scf"] = scf_out
        out["scf_al4"] = scf_al4(local)
    if world > 1 and os.environ.get("PW_BENCH_NO_SCF") != "1":
        # config C3's SCF with its k-points shared out over the ranks (density,
        # band energies and eigenvalues all-reduced): device time of the SCF
        # loop, max over ranks
        out["scf_al4_sharded"] = scf_al4(local, sharded=True)
    if os.environ.get("PW_BENCH_NO_MULTIK") != "1" and world == 1:
        out["multik"] = multik_comparison(local, max(5, args.steps // 20), flush)
    if rank == 0 and world == 1 and args.workload == "si64" and os.environ.get("PW_BENCH_NO_CPU") != "1":
        Hc, psic = reference_workload()
        dt, reps = cpu_reference(Hc, psic, 1000, 1, args.cpu_budget)
        v = NBANDS * bpb / dt / 1e9
        out["cpu_baseline"] = {"value": v, "unit": "GB/s", "cores": os.cpu_count(), "kind": "port",
                               "sample": "all 160 bands per op_H, %d repetitions (about %.0f s), FP64 NumPy/SciPy, "
                                         "all host threads" % (reps, args.cpu_budget)}
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
