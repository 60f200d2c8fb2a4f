"""Benchmark: fTWA trajectory-RK4-steps/s on the 10x10 grid (16384 trajectories).

Workload (one GPU): 10x10 square grid, t=1, on-site U=4, static random site
potential uniform in [-1, 1] (seed 0), domain-wall product state (both spins on
x < 5), dt = 0.005, stepsParTimePoints = 1, 16384 trajectories, rho 2 x 100 x 100
complex per trajectory.  Synthetic, seeded inputs; no dataset is involved.

One benchmark step = one fpsg_run of 100 snapshots: every trajectory advanced by
100 RK4 steps with the diagDMatrix and onSiteDoublons ensemble sums recorded at
every snapshot (stepsParTimePoints = 1, so every step is a snapshot), state
resident in HBM before the timed region (1.3 GB of packed FP32 state, larger
than the 126 MB L2).  value = trajectories x RK steps over all ranks / max-over-
ranks device time (CUDA events of the call).

e2e = the same metric through the public C ABI as a user calls it, per step:
fpsg_set_system (host matrices) + fpsg_sample (host occupations) + fpsg_run with
observables recorded every snapshot, results copied back to the host.

--impl reference: the reference has no GPU code and cannot be built here (it needs
Armadillo + BLAS/LAPACK); its CPU algorithm is timed through the FP64 restatement
oracle/fps_oracle.c (dense commutator, OpenMP over trajectories, all host threads),
recording the same observables at every step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STEP_RK = 100          # RK4 steps per benchmark step
E2E_SNAPSHOTS = 100    # one e2e step = the headline step's 100 snapshots (100 RK steps)
FP64_STEP_RK = 20
# observables recorded at every snapshot in every timed leg and in the reference arm
# (the reference's diagDMatrix + onSiteDoublons, src/FHfTWASolver.cpp:370-397)
BENCH_OBS = 1 | 4
METRIC = "fTWA trajectory-RK4-steps/s"
UNIT = "traj-steps/s"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


def stencil_roofline(n: int, nnz: int, c: int, units: int, ms: float, hbm_peak: float, peak_kind: str,
                     sm_mhz: float, traffic_key: str | None = None, fp64: bool = False) -> dict:
    """Roofline object of a stencil-path leg: algorithmic bytes 16 n^2 c per
    trajectory-RK4-step (4 stages x read + write x 2 spins x n^2 x c bytes) and
    flops 64 n nnz(H), times `units` trajectory-steps, over the leg's device time
    `ms`; HBM peak measured (or fallback), FP32/FP64 CUDA-core peak nominal at the
    sampled SM clock (148 SMs x 128 FP32 / 64 FP64 lanes x 2 flops)."""
    bytes_alg = 16.0 * n * n * c
    flops_alg = 64.0 * n * nnz
    gbs = bytes_alg * units / (ms / 1e3) / 1e9
    tflops = flops_alg * units / (ms / 1e3) / 1e12
    lanes = 64 if fp64 else 128
    cpeak = 148 * lanes * 2 * sm_mhz * 1e6 / 1e12
    traffic = None
    if traffic_key:
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            with open(tp) as fh:
                traffic = json.load(fh).get(traffic_key)
    return {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
            "traffic": traffic, "peak_source": f"{peak_kind} HBM copy bandwidth",
            "bytes_per_traj_step": bytes_alg, "traj_steps": units, "device_ms": ms,
            "compute": {"achieved": tflops, "peak": cpeak, "unit": "TFLOP/s", "frac": tflops / cpeak,
                        "flops_per_traj_step": flops_alg,
                        "peak_source": f"nominal {'FP64' if fp64 else 'FP32'} CUDA-core peak at the sampled SM clock"}}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during timing."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def host_cores() -> int:
    """Host threads this process can actually use: the CPU affinity mask, capped by
    a cgroup CPU quota when one is set (a container may report more cores than its
    quota lets it run)."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    for path in ("/sys/fs/cgroup/cpu.max", "/sys/fs/cgroup/cpu/cpu.cfs_quota_us"):
        try:
            with open(path) as fh:
                f = fh.read().split()
        except OSError:
            continue
        try:
            if path.endswith("cpu.max") and f[0] != "max":
                n = min(n, max(1, int(-(-int(f[0]) // int(f[1])))))
            elif path.endswith("cfs_quota_us") and int(f[0]) > 0:
                with open("/sys/fs/cgroup/cpu/cpu.cfs_period_us") as fh:
                    n = min(n, max(1, int(-(-int(f[0]) // int(fh.read().split()[0])))))
        except (ValueError, IndexError, OSError):
            pass
        break
    return max(1, n)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_sample_rate(w, budget_s: float = 12.0, nthreads: int = 0, method: int = 0, coulomb: int = 1):
    """Times the FP64 oracle (reference algorithm) on a bounded sample of workload
    w: one trajectory per host thread (one for HF), as many RK4 steps as fit the
    budget, the bench's observables recorded at every step.  Returns (rate,
    cores, sample text, sample dict)."""
    from oracle import oracle as O
    sysm = O.System(tM=w.tM, U=w.U, V=w.V, ext=w.ext, coulomb=coulomb, ext_null=w.ext is None)
    cores = nthreads or host_cores()
    nthreads = cores
    hf = method == O.METHOD_HF
    Bc = 1 if hf else cores

    def start(seed):
        if hf:
            N0 = np.zeros((1, 2, w.n, w.n), dtype=complex)
            N0[0, 0] = np.diag(w.occ_up)
            N0[0, 1] = np.diag(w.occ_dn)
            return N0
        return O.sample(w.n, Bc, seed, w.occ_up, w.occ_dn)

    # calibrate on two RK steps
    t0 = time.perf_counter()
    O.run(sysm, method, w.dt, 1, 3 if hf else 2, start(1), obs=BENCH_OBS, nthreads=nthreads, want_final=False)
    rate = Bc * 2 / (time.perf_counter() - t0)
    steps = max(2, int(budget_s * rate / Bc))
    t0 = time.perf_counter()
    # fTWA steps once per snapshot (Tp snapshots -> Tp steps); HF records t = 0 first (Tp - 1 steps)
    O.run(sysm, method, w.dt, 1, steps + 1 if hf else steps, start(2), obs=BENCH_OBS, nthreads=nthreads,
          want_final=False)
    el = time.perf_counter() - t0
    what = "HF trajectory" if hf else "trajectories"
    return (Bc * steps / el, 1 if hf else cores,
            f"{Bc} {what} x {steps} RK4 steps of {w.name} ({el:.1f} s), observables every step",
            {"n_traj": Bc, "rk_steps": steps, "seconds": el})


def adjoint_leg(dev: int, rank: int, precision: int):
    """grad/fwd cost on the adjoint workload: 8x8 grid, U=4, 50-bin site pulse,
    2048 trajectories, dt=0.01, t in [0, 10] (1000 RK4 steps), checkpoints every 16
    steps.  grad = one fpsg_grad call (forward sweeps with checkpoints, keeping the
    stage inputs of every segment that fits, in trajectory chunks when the whole
    ensemble's do not; then the reverse sweeps); fwd = one fpsg_run of the same
    trajectories recording the doublon occupancy (the loss's observable) at every
    snapshot.  Both per RK step (fpsg_run takes one extra snapshot's steps)."""
    from fermiphasespace_b200 import configs, engine as E
    w, pulse = configs.adjoint_8x8()
    Tp = w.n_snapshots
    eng = E.Engine(dev)
    eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    eng.set_pulse(pulse["amp"], pulse["bin_width"], pulse["t0"], pulse["td"], pulse["proj"])
    eng.sample(w.n_traj, 11 + rank, w.occ_up, w.occ_dn)
    s0 = eng.get_state()
    eng.grad(precision, w.dt, 1, Tp, 16)
    import torch
    free_b, total_b = torch.cuda.mem_get_info(dev)
    t0 = time.perf_counter()
    g = eng.grad(precision, w.dt, 1, Tp, 16)
    g_wall = (time.perf_counter() - t0) * 1e3
    eng.set_initial_samples(s0)
    eng.run(E.METHOD_FTWA, precision, w.dt, 1, Tp, obs=E.OBS_DOUBLONS)
    eng.set_initial_samples(s0)
    t0 = time.perf_counter()
    r = eng.run(E.METHOD_FTWA, precision, w.dt, 1, Tp, obs=E.OBS_DOUBLONS)
    r_wall = (time.perf_counter() - t0) * 1e3
    eng.close()
    grad_per_step = g["device_ms"] / ((Tp - 1) * w.S)
    fwd_per_step = r.device_ms / (Tp * w.S)
    return {"workload": w.name, "n_traj": w.n_traj, "rk_steps": (Tp - 1) * w.S, "checkpoint_every": 16,
            "precision": "fp32" if precision == E.PREC_FP32 else "fp64",
            "grad_ms": g["device_ms"], "fwd_ms": r.device_ms, "grad_over_fwd": grad_per_step / fwd_per_step,
            "grad_wall_ms": g_wall, "fwd_wall_ms": r_wall,
            "device_free_gb_at_grad": free_b / 1e9,
            "grad_over_own_forward_sweep": g["device_ms"] / g["forward_ms"], "loss": g["loss"],
            "plan": {"chunks": g["chunks"], "chunk_traj": g["chunk_traj"], "segments": g["segments"],
                     "kept_segments": g["kept_segments"]},
            "dL_dU": g["dU"], "dL_dt": g["dt"], "target": "<= 3"}


def gpsr_leg(dev: int, cpu: bool, B: int = 1024, calls: int = 5):
    """The GPSR drift (fpsg_gpsr_drift: one 3/8-rule drift step of general complex
    states, FP64) on the headline lattice: 1024 trajectories of random non-Hermitian
    states near the domain-wall occupations, d_t = 0.005; per call the host states in,
    four stage launches over all 2048 matrices, the drifts out (wall time, host
    buffers, as the GPSR caller uses it).  Beside it the oracle's restatement on the
    host cores for 16 trajectories."""
    from fermiphasespace_b200 import configs, engine as E
    w = configs.grid_10x10(U0=4.0, n_traj=B)
    n = w.n
    rng = np.random.default_rng(5)
    rho = 0.05 * (rng.normal(size=(B, 2, n, n)) + 1j * rng.normal(size=(B, 2, n, n)))
    rho[:, 0] += np.diag(w.occ_up)
    rho[:, 1] += np.diag(w.occ_dn)
    eng = E.Engine(dev)
    eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    eng.gpsr_drift(rho, 0.005)
    t0 = time.perf_counter()
    for _ in range(calls):
        d = eng.gpsr_drift(rho, 0.005)
    wall = (time.perf_counter() - t0) / calls
    eng.close()
    out = {"workload": "grid10x10_U4_W2 (random non-Hermitian states)", "n_traj": B, "precision": "fp64",
           "value": B / wall, "unit": "trajectory drift steps/s", "ms_per_call": wall * 1e3,
           "h2d_bytes": int(rho.nbytes), "d2h_bytes": int(d.nbytes),
           "note": "wall time per fpsg_gpsr_drift call with host buffers in and out"}
    if cpu:
        from oracle import oracle as O
        Bc = 16
        sysm = O.System(tM=w.tM, U=w.U, V=w.V, ext=w.ext, coulomb=O.COUL_ONSITE, ext_null=False)
        t0 = time.perf_counter()
        ref = O.gpsr_drift(sysm, rho[:Bc], 0.005, nthreads=host_cores())
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": Bc / tc, "unit": "trajectory drift steps/s", "cores": host_cores(),
                               "kind": "port", "sample": f"{Bc} trajectories ({tc:.2f} s)"}
        out["max_abs_diff_vs_oracle"] = float(np.abs(d[:Bc] - ref).max())
    return out


def accuracy_leg(dev: int, rank: int, B: int = 4096, t_max: float = 20.0):
    """Observable error of the FP32 path against the plain FP64 GPU path on the
    benchmark workload (same samples, every snapshot of t in [0, t_max]), beside
    the statistical error sqrt(var(n_i)/B) of the ensemble mean; for the FP32
    resident path as it runs by default (compensated state update) and with plain
    FP32 state updates (FPSG_FLAG_FP32_PLAIN_STATE)."""
    from fermiphasespace_b200 import configs, engine as E
    w = configs.grid_10x10(n_traj=B, t_max=t_max)
    Tp = w.n_snapshots
    obs = E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS
    runs = {}
    for name, prec, flags in (("fp64", E.PREC_FP64, 0), ("fp32", E.PREC_FP32, 0),
                              ("fp32_plain_state", E.PREC_FP32, E.FLAG_FP32_PLAIN_STATE)):
        eng = E.Engine(dev, flags=flags)
        eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
        eng.sample(B, 77, w.occ_up, w.occ_dn, first=rank * B)
        runs[name] = eng.run(E.METHOD_FTWA, prec, w.dt, 1, Tp, obs=obs)
        eng.close()
    r64 = runs["fp64"]
    t = r64.time
    var = np.maximum(r64.n2iiu - r64.niiu ** 2, 0.0)
    stat = np.sqrt(var / B).max(axis=0)
    late = t >= t_max / 2
    marks = [tm for tm in (0.5, 1, 2, 5, 10, 15, 20) if tm <= t_max]
    idx = [int(round(tm / w.dt)) for tm in marks]
    out = {"workload": w.name, "n_traj": B, "t_max": t_max, "compared": "fp32 resident vs fp64 GPU, same samples",
           "observables": "max over sites of |dNiiu|, |dNiid|, |dNuNd|",
           "stat_err_at_t": {f"{tm:g}": float(stat[i]) for tm, i in zip(marks, idx)}, "fp64_path": r64.path_used}
    for name in ("fp32", "fp32_plain_state"):
        r32 = runs[name]
        err = np.maximum(np.abs(r32.niiu - r64.niiu).max(axis=0),
                         np.maximum(np.abs(r32.niid - r64.niid).max(axis=0), np.abs(r32.nund - r64.nund).max(axis=0)))
        over = np.nonzero(err > 1e-6)[0]
        key = "" if name == "fp32" else "plain_state_"
        out[key + "err_le_1e-6_until_t"] = float(t[over[0]]) if over.size else float(t[-1])
        out[key + "max_err_at_t"] = {f"{tm:g}": float(err[i]) for tm, i in zip(marks, idx)}
        out[key + "max_err_over_stat_err_t_ge_half"] = float((err[late] / np.maximum(stat[late], 1e-300)).max())
        out[key + "fp32_path"] = r32.path_used
    return out


def u_sweep_leg(dev: int, rank: int, U0: float, hbm_peak: float, peak_kind: str, sm_mhz: float, cpu: bool,
                B: int = 16384):
    """The headline workload at another on-site U (10x10 grid, domain wall, static
    disorder W = 2, dt = 0.005, B trajectories): FP32 resident path over 100
    snapshots and the plain FP64 path over 20, each recording the bench
    observables every snapshot (median of three calls), and the FP64 oracle on
    host cores."""
    from fermiphasespace_b200 import configs, engine as E
    w = configs.grid_10x10(U0=U0, n_traj=B)
    n, nnz = w.n, w.nnz_offdiag + w.n
    eng = E.Engine(dev)
    eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    eng.sample(B, 3000 + int(U0), w.occ_up, w.occ_dn, first=rank * B)
    # each timing: a warm-up call of the same shape, then the median of three calls (the
    # first call after a change of shape runs a few per cent slow)
    eng.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, STEP_RK, obs=BENCH_OBS)
    rs = sorted((eng.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, STEP_RK, obs=BENCH_OBS) for _ in range(3)),
                key=lambda x: x.device_ms)
    r = rs[1]
    v32 = B * STEP_RK / (r.device_ms / 1e3)
    eng.sample(B, 4000 + int(U0), w.occ_up, w.occ_dn, first=rank * B)
    eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, FP64_STEP_RK, obs=BENCH_OBS)
    rs = sorted((eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, FP64_STEP_RK, obs=BENCH_OBS) for _ in range(3)),
                key=lambda x: x.device_ms)
    r64 = rs[1]
    v64 = B * FP64_STEP_RK / (r64.device_ms / 1e3)
    eng.close()
    out = {"workload": w.name, "U": U0, "n_traj": B, "value": v32, "unit": UNIT,
           "precision": "fp32 stages with compensated state update, fp64 ensemble reduction", "path": r.path_used,
           "roofline": stencil_roofline(n, nnz, 8, B * STEP_RK, r.device_ms, hbm_peak, peak_kind, sm_mhz),
           "fp64_gpu": {"value": v64, "unit": UNIT, "path": r64.path_used,
                        "roofline": stencil_roofline(n, nnz, 16, B * FP64_STEP_RK, r64.device_ms, hbm_peak,
                                                     peak_kind, sm_mhz, fp64=True)},
           "mixed_over_fp64": v32 / v64}
    if cpu:
        v, cores, sample, _ = cpu_sample_rate(w, budget_s=4.0)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    return out


def hf_leg(dev: int, U0: float, hbm_peak: float, peak_kind: str, sm_mhz: float, cpu: bool):
    """Time-dependent Hartree-Fock on the headline system (src/FHHFSolver.cpp:181-434):
    10x10 grid, on-site U, disorder W = 2, one deterministic density matrix started
    from the domain-wall product state N0 = diag(occ), dt = 0.005, t in [0, 20]
    (4001 snapshots, 4000 RK4 steps), the bench observables at every snapshot.
    Plain FP64 (bit-identical to the oracle) and FP32 on the GPU, the FP64 oracle's
    HF on one host thread (the reference's HF loop is serial)."""
    from fermiphasespace_b200 import configs, engine as E
    w = configs.grid_10x10(U0=U0, n_traj=1)
    n, nnz = w.n, w.nnz_offdiag + w.n
    Tp = w.n_snapshots
    N0 = np.zeros((1, 2, n, n), dtype=complex)
    N0[0, 0] = np.diag(w.occ_up)
    N0[0, 1] = np.diag(w.occ_dn)
    eng = E.Engine(dev)
    eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    out = {"workload": w.name + "_HF", "U": U0, "snapshots": Tp, "rk_steps": (Tp - 1) * w.S, "unit": "RK4-steps/s"}
    for name, prec in (("fp64", E.PREC_FP64), ("fp32", E.PREC_FP32)):
        eng.set_initial_samples(N0)
        eng.run(E.METHOD_HF, prec, w.dt, w.S, 11, obs=BENCH_OBS)
        eng.set_initial_samples(N0)
        r = eng.run(E.METHOD_HF, prec, w.dt, w.S, Tp, obs=BENCH_OBS)
        steps = (Tp - 1) * w.S
        out[name] = {"value": steps / (r.device_ms / 1e3), "whole_run_ms": r.device_ms,
                     "path": {1: "stream", 2: "resident"}.get(r.path_used, r.path_used),
                     "launches": r.launches,
                     "roofline": stencil_roofline(n, nnz, 16 if prec == E.PREC_FP64 else 8, steps, r.device_ms,
                                                  hbm_peak, peak_kind, sm_mhz, fp64=prec == E.PREC_FP64)}
        out[name]["roofline"]["note"] = ("one trajectory occupies one CTA cluster of 148 SMs: the run is bound by "
                                         "the latency of its 16000 dependent RK stages, not by a throughput roof")
        if name == "fp64":
            niiu64 = r.niiu
        else:
            out["fp32_max_err_niiu"] = float(np.abs(r.niiu - niiu64).max())
    eng.close()
    out["value"] = out["fp64"]["value"]
    if cpu:
        from oracle import oracle as O
        v, cores, sample, _ = cpu_sample_rate(w, budget_s=4.0, nthreads=1, method=O.METHOD_HF)
        out["cpu_baseline"] = {"value": v, "unit": "RK4-steps/s", "cores": cores, "kind": "port", "sample": sample,
                               "whole_run_s_extrapolated": (Tp - 1) * w.S / v}
    return out


def moire_leg(dev: int, rank: int, bf16_peak_tflops: float, cpu: bool):
    """The long-range-hopping workload on the dense tensor-core path: twisted
    bilayer honeycomb, 256 sites, t(r) = exp(-(r - a)/0.45) up to 4a, long-range
    Coulomb U/(1 + r), 2048 trajectories, dt = 0.005.  Split BF16x3 against the
    FP32 and FP64 CUDA-core stream paths (global-memory variant at this n) and
    the FP64 oracle on host cores; observable error of BF16x3 against FP64 on the
    same samples."""
    from fermiphasespace_b200 import configs, engine as E
    pos = configs.moire_positions()
    w = configs.moire_8x8(n_traj=2048, pos=pos)
    n, B = w.n, w.n_traj
    eng = E.Engine(dev)
    eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_DISTANCE)
    eng.sample(B, 21, w.occ_up, w.occ_dn, first=rank * B)
    eng.advance(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, w.dt, 1, 1)
    steps = 6
    ms, nl = eng.advance(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, w.dt, 1, steps)
    rate = B * steps / (ms / 1e3)
    launch_ms = ms / (4 * steps)
    flops_alg = 64.0 * n ** 3                 # per traj-step (one complex product per spin per stage)
    flops_mma = 192.0 * n ** 3                # issued: 2 planes x 2 products x 3 split terms
    peak_eff = bf16_peak_tflops / 3.0
    out = {"workload": w.name, "sites": n, "n_traj": B, "dt": w.dt, "precision": "split bf16x3, fp32 state",
           "value": rate, "unit": "traj-steps/s", "ms_per_rk_step": ms / steps, "launches": nl,
           "roofline": {"bound": "tensor", "achieved": flops_alg * rate / 1e12, "peak": peak_eff, "unit": "TFLOP/s",
                        "frac": flops_alg * rate / 1e12 / peak_eff,
                        "peak_source": "measured BF16 dense peak / 3 (three split products)",
                        "issued_tflops": flops_mma * rate / 1e12,
                        "issued_frac_of_bf16_peak": flops_mma * rate / 1e12 / bf16_peak_tflops,
                        "launch_ms": launch_ms}}
    comp = {}
    for name, prec in (("fp32", E.PREC_FP32), ("fp64", E.PREC_FP64)):
        Bc = 512
        eng.sample(Bc, 22, w.occ_up, w.occ_dn)
        eng.advance(E.METHOD_FTWA, prec, w.dt, 1, 1)
        m2, _ = eng.advance(E.METHOD_FTWA, prec, w.dt, 1, 1)
        comp[name] = {"value": Bc / (m2 / 1e3), "n_traj": Bc, "path": "stream, global-memory matrices (CUDA cores)"}
    out["cuda_core"] = comp
    # the same workload in split TF32x3 (kind::tf32: half the bf16 rate, ~21 significant bits)
    eng.sample(B, 21, w.occ_up, w.occ_dn, first=rank * B)
    eng.advance(E.METHOD_FTWA, E.PREC_SPLIT_TF32X3, w.dt, 1, 1)
    mt, _ = eng.advance(E.METHOD_FTWA, E.PREC_SPLIT_TF32X3, w.dt, 1, 4)
    out["tf32x3"] = {"value": B * 4 / (mt / 1e3), "unit": "traj-steps/s",
                     "frac_of_tf32_split_peak": flops_alg * (B * 4 / (mt / 1e3)) / 1e12 / (bf16_peak_tflops / 2.0 / 3.0),
                     "peak_source": "measured BF16 peak / 2 (tf32 rate) / 3 (split products)"}
    out["dense_over_fp64_gpu"] = rate / comp["fp64"]["value"]
    Ba, Tp = 64, 101
    obs = E.OBS_DIAG | E.OBS_DOUBLONS
    res = {}
    for name, prec in (("fp64", E.PREC_FP64), ("bf16x3", E.PREC_SPLIT_BF16X3), ("tf32x3", E.PREC_SPLIT_TF32X3)):
        eng.sample(Ba, 5, w.occ_up, w.occ_dn)
        r = eng.run(E.METHOD_FTWA, prec, w.dt, 1, Tp, obs=obs)
        res[name] = r
    out["accuracy"] = {"n_traj": Ba, "compared": "dense split products vs fp64 GPU, same samples"}
    for name in ("bf16x3", "tf32x3"):
        err = np.maximum(np.abs(res[name].niiu - res["fp64"].niiu).max(axis=0),
                         np.abs(res[name].nund - res["fp64"].nund).max(axis=0))
        out["accuracy"][name + "_max_err_niiu_nund_at_step"] = {str(k): float(err[k]) for k in (1, 10, 50, 100)}
    eng.close()
    if cpu:
        from oracle import oracle as O
        Bo = host_cores()
        rho0 = O.sample(n, Bo, 3, w.occ_up, w.occ_dn)
        sysm = O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_DISTANCE, ext_null=True)
        t0 = time.perf_counter()
        O.run(sysm, O.METHOD_FTWA, w.dt, 1, 2, rho0, obs=1, nthreads=Bo, want_final=False)
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": Bo * 2 / el, "unit": "traj-steps/s", "cores": Bo, "kind": "port",
                               "sample": f"{Bo} trajectories x 2 RK4 steps ({el:.1f} s)"}
    return out


def batch_leg(dev: int, rank: int):
    """The uneven batch (kagome 108, honeycomb 24, periodic fcc 108, grids 64 and
    144 sites; 8192 trajectories, dt = 0.01, t in [0, 2]) through fpsg_run_batch
    (one persistent launch per stage, graph replay per snapshot), FP32, against
    the same systems run one after another through fpsg_run."""
    from fermiphasespace_b200 import configs, engine as E
    ws = configs.uneven_batch()
    eng = E.Engine(dev)
    ds = [{"tM": w.tM, "U": w.U, "V": w.V, "ext": None, "coulomb": E.COUL_ONSITE, "n_traj": w.n_traj,
           "seed": 7 + k + 100 * rank, "occ_up": w.occ_up, "occ_dn": w.occ_dn} for k, w in enumerate(ws)]
    Tp = ws[0].n_snapshots
    obs = E.OBS_DIAG | E.OBS_DOUBLONS
    _, first = eng.run_batch(ds, E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, Tp, obs=obs)
    _, info = eng.run_batch(ds, E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, Tp, obs=obs)
    seq_ms, seq_steps = 0.0, 0
    for k, w in enumerate(ws):
        eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        eng.sample(w.n_traj, 7 + k, w.occ_up, w.occ_dn)
        r = eng.run(E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, Tp, obs=obs)
        seq_ms += r.device_ms
        seq_steps += r.traj_steps
    eng.close()
    v = info["traj_steps"] / (info["device_ms"] / 1e3)
    # algorithmic bytes: sum over systems of B_s x RK steps x 16 n_s^2 x 8 (FP32 complex)
    steps = Tp * ws[0].S
    bytes_alg = sum(w.n_traj * steps * 16.0 * w.n * w.n * 8 for w in ws)
    gbs = bytes_alg / (info["device_ms"] / 1e3) / 1e9
    hbm_peak, _bf, peak_kind = peaks()
    return {"roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                         "peak_source": f"{peak_kind} HBM copy bandwidth",
                         "bytes": "sum_s B_s x steps x 16 n_s^2 x 8", "device_ms": info["device_ms"]},
            "systems": [f"{w.name} n={w.n} B={w.n_traj}" for w in ws], "snapshots": Tp, "precision": "fp32",
            "value": v, "unit": "traj-steps/s", "device_ms": info["device_ms"],
            "autotuned": {"block_threads": first["block_threads"], "schedule": first["schedule"],
                          "grid": first["grid"], "tune_ms": first["tune_ms"]},
            "graph_nodes": info["graph_nodes"], "kernel_launches": info["kernel_launches"],
            "sequential_fpsg_run": {"value": seq_steps / (seq_ms / 1e3), "device_ms": seq_ms}}


def cpu_case_leg(dev: int, cpu: bool):
    """The reference's own CPU-runnable case: 3x2 grid, U = 4, Neel state, 1000
    trajectories, dt = 0.01, stepsParTimePoints = 10, t_max = 10 (1001 snapshots,
    10010 RK4 steps).  Plain FP64 on the GPU through fpsg_run against the FP64
    oracle on all host cores, same samples, whole window."""
    from fermiphasespace_b200 import configs, engine as E
    w = configs.grid_3x2(n_traj=1000)
    Tp = w.n_snapshots
    eng = E.Engine(dev)
    eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    eng.sample(w.n_traj, 0, w.occ_up, w.occ_dn)
    rho0 = eng.get_state()
    eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, w.S, Tp, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    eng.set_initial_samples(rho0)
    r = eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, w.S, Tp, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    eng.close()
    out = {"workload": w.name, "n_traj": w.n_traj, "rk_steps": Tp * w.S, "precision": "fp64",
           "gpu": {"value": r.traj_steps / (r.device_ms / 1e3), "unit": "traj-steps/s", "device_ms": r.device_ms,
                   "path": {1: "stream", 2: "resident"}.get(r.path_used, r.path_used)}}
    if cpu:
        from oracle import oracle as O
        t0 = time.perf_counter()
        ref = O.run(O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True), O.METHOD_FTWA,
                    w.dt, w.S, Tp, rho0, obs=O.OBS_DIAG | O.OBS_DOUB, nthreads=host_cores(), want_final=False)
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": w.n_traj * Tp * w.S / el, "unit": "traj-steps/s", "cores": host_cores(),
                               "kind": "port", "sample": f"the whole case ({el:.1f} s)"}
        out["max_abs_diff_niiu_nund"] = float(max(np.abs(r.niiu - ref["niiu"]).max(), np.abs(r.nund - ref["nund"]).max()))
    return out


def config_dict(w, extra=None):
    d = {"workload": w.name, "sites": w.n, "n_traj": w.n_traj, "dt": w.dt, "steps_per_snapshot": w.S,
         "rk_steps_per_bench_step": STEP_RK, "snapshots_per_bench_step": STEP_RK,
         "observables": "diagDMatrix + onSiteDoublons ensemble sums at every snapshot",
         "precision": "fp32 stages, fp64 ensemble reduction",
         "l2": "inputs larger than L2 (1.3 GB packed FP32 state per GPU)", "parallelism": "trajectory shards"}
    if extra:
        d.update(extra)
    return d


def run_reference(args):
    """The reference arm: the reference's algorithm (the FP64 restatement, dense
    commutator, OpenMP over trajectories, all host threads) on the headline
    workload.  Each step is a bounded sample (one trajectory per host thread, as
    many RK4 steps as fit about 6 s, observables recorded every step); the value
    is trajectory-steps per second of that sample, the unit the full workload
    (16384 trajectories x 100 steps per bench step) scales by linearly."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from fermiphasespace_b200 import configs
    w = configs.grid_10x10(n_traj=16384)
    vals, step_s = [], []
    cores = host_cores()
    sample, smp = "", {}
    for i in range(args.warmup + args.steps):
        v, cores, sample, smp = cpu_sample_rate(w, budget_s=6.0 if i >= args.warmup else 1.0)
        if i >= args.warmup:
            vals.append(v)
            step_s.append(smp["seconds"])
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(step_s),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config_dict(w, {"precision": "fp64 (reference algorithm)"}),
            "extrapolated_from": {"n_traj_per_step": smp.get("n_traj"), "rk_steps_per_step": smp.get("rk_steps"),
                                  "full_step": {"n_traj": w.n_traj, "rk_steps": STEP_RK},
                                  "full_step_ms": 1e3 * w.n_traj * STEP_RK / value,
                                  "note": "trajectories are independent and the work per trajectory-step is "
                                          "constant, so the sample's rate is the full workload's rate"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample + "; the reference cannot be built here (Armadillo/BLAS absent), "
                                                "its algorithm is timed through the FP64 restatement"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# the systems of the uneven batch, in configs.uneven_batch order (profile cases)
BATCH_SYSTEMS = ["kagome108", "honeycomb24", "fcc108", "grid64", "grid144"]


def run_profile_case(args):
    """A small case of one workload for ncu captures: --workload grid10x10 (the
    benchmark system), moire (n = 256, dense path), adjoint (fpsg_grad on the
    8x8 pulse workload over --rk-steps steps, checkpoints every 16) or one system of
    the uneven batch (kagome108, honeycomb24, fcc108, grid64, grid144), --traj
    trajectories, --rk-steps steps per call, two calls."""
    from fermiphasespace_b200 import configs, engine as E
    if args.workload == "adjoint":
        prec = E.PREC_FP64 if args.precision == "fp64" else E.PREC_FP32
        w, pulse = configs.adjoint_8x8(n_traj=args.traj, t_max=args.rk_steps * 0.01)
        eng = E.Engine(0)
        eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        eng.set_pulse(pulse["amp"], pulse["bin_width"], pulse["t0"], pulse["td"], pulse["proj"])
        eng.sample(args.traj, 1, w.occ_up, w.occ_dn)
        for rep in range(2):
            g = eng.grad(prec, w.dt, 1, w.n_snapshots, 16)
            print(json.dumps({"case": "profile", "workload": w.name, "traj": args.traj, "rk_steps": args.rk_steps,
                              "grad_ms": g["device_ms"], "forward_ms": g["forward_ms"]}), flush=True)
        eng.close()
        return 0
    if args.workload == "moire":
        w = configs.moire_8x8(n_traj=args.traj)
        coul = E.COUL_DISTANCE
    elif args.workload in BATCH_SYSTEMS:
        w = configs.uneven_batch()[BATCH_SYSTEMS.index(args.workload)]
        coul = E.COUL_ONSITE
    else:
        w = configs.grid_10x10(n_traj=args.traj)
        coul = E.COUL_ONSITE
    eng = E.Engine(0)
    eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=coul)
    eng.sample(args.traj, 1, w.occ_up, w.occ_dn)
    prec = {"fp32": E.PREC_FP32, "fp64": E.PREC_FP64, "bf16x3": E.PREC_SPLIT_BF16X3}[args.precision]
    path = {"auto": E.PATH_AUTO, "stream": E.PATH_STREAM, "resident": E.PATH_RESIDENT, "dense": E.PATH_DENSE}[args.path]
    for rep in range(2):
        ms, nl = eng.advance(E.METHOD_FTWA, prec, w.dt, 1, args.rk_steps, path=path)
        print(json.dumps({"case": "profile", "workload": w.name, "traj": args.traj, "rk_steps": args.rk_steps,
                          "precision": args.precision, "path": args.path, "device_ms": ms, "launches": nl,
                          "traj_steps_per_s": args.traj * args.rk_steps / (ms / 1e3)}), flush=True)
    eng.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--fp64", type=int, default=1, help="also time the plain FP64 GPU path")
    ap.add_argument("--adjoint", type=int, default=1, help="also time grad/fwd on the adjoint workload")
    ap.add_argument("--accuracy", type=int, default=1, help="also measure the FP32 observable error vs FP64")
    ap.add_argument("--cpu-case", type=int, default=1, help="also run the 3x2 CPU-runnable case on GPU and CPU")
    ap.add_argument("--moire", type=int, default=1, help="also time the dense tensor-core path on the moire lattice")
    ap.add_argument("--batch", type=int, default=1, help="also time the uneven batch (fpsg_run_batch)")
    ap.add_argument("--u-sweep", type=int, default=1, help="also time the headline workload at U = 2 and U = 8")
    ap.add_argument("--hf", type=int, default=1, help="also time Hartree-Fock on the headline system, U = 2, 4, 8")
    ap.add_argument("--gpsr", type=int, default=1, help="also time the GPSR drift on the headline lattice")
    ap.add_argument("--profile", action="store_true",
                    help="small case for profilers: --traj trajectories, --rk-steps steps per launch, "
                         "--precision, two launches, no CPU / e2e legs")
    ap.add_argument("--traj", type=int, default=296)
    ap.add_argument("--rk-steps", type=int, default=20)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "bf16x3"])
    ap.add_argument("--path", default="auto", choices=["auto", "stream", "resident", "dense"])
    ap.add_argument("--workload", default="grid10x10", choices=["grid10x10", "moire", "adjoint", *BATCH_SYSTEMS])
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile_case(args)

    ws, rank, local = dist_env()
    import torch
    dist = None
    if ws > 1 or "TORCHELASTIC_RUN_ID" in os.environ:     # launched by torchrun (any world size)
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local if dist is not None else 0
    torch.cuda.set_device(dev)

    from fermiphasespace_b200 import configs, engine as E, shards
    w = configs.grid_10x10(U0=4.0, W=2.0, seed=0, n_traj=16384)
    B = w.n_traj
    eng = E.Engine(dev)
    eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    eng.sample(B, 1000, w.occ_up, w.occ_dn, first=rank * B)   # this rank's shard of one ensemble

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------- value: FP32 resident path, every snapshot recorded (S = 1: one
    # snapshot per RK step, diagDMatrix + onSiteDoublons), state resident in HBM
    for _ in range(args.warmup):
        eng.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, STEP_RK, obs=BENCH_OBS)
    clk = ClockSampler(dev)
    clk.start()
    barrier()
    dev_ms, launches = 0.0, 0
    w0 = time.perf_counter()
    for _ in range(args.steps):
        r = eng.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, STEP_RK, obs=BENCH_OBS)
        dev_ms += r.device_ms
        launches += r.launches
    barrier()
    wall_ms = (time.perf_counter() - w0) * 1e3
    clocks = clk.stop()
    dev_ms = max_over_ranks(dev_ms)
    traj_steps = B * STEP_RK * args.steps * ws
    value = traj_steps / (dev_ms / 1e3)
    ms_per_step = dev_ms / args.steps

    # the same trajectories advanced without observables (one resident launch per call)
    adv_ms = 0.0
    for _ in range(3):
        ms, _nl = eng.advance(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, STEP_RK)
        adv_ms += ms
    advance_only = {"value": B * STEP_RK * 3 / (adv_ms / 1e3), "unit": UNIT, "ms_per_call": adv_ms / 3,
                    "note": "fpsg_advance: the same steps with no snapshot recorded"}
    # the same step with plain FP32 state updates (no compensation)
    engp = E.Engine(dev, flags=E.FLAG_FP32_PLAIN_STATE)
    engp.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    engp.sample(B, 1000, w.occ_up, w.occ_dn, first=rank * B)
    engp.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, STEP_RK, obs=BENCH_OBS)
    pl_ms = 0.0
    for _ in range(3):
        pl_ms += engp.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, STEP_RK, obs=BENCH_OBS).device_ms
    engp.close()
    plain_state = {"value": B * STEP_RK * 3 / (pl_ms / 1e3), "unit": UNIT, "ms_per_step": pl_ms / 3,
                   "note": "the headline step with FPSG_FLAG_FP32_PLAIN_STATE (no compensated state update)"}

    # roofline of the resident kernel: algorithmic bytes and flops of the step's
    # trajectory-steps over the step's own device time (CUDA events of fpsg_run,
    # which cover the one resident launch and the fixed-order snapshot reduction)
    hbm_peak, bf16_peak, peak_kind = peaks()
    n = w.n
    nnz = w.nnz_offdiag + n
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    roofline = stencil_roofline(n, nnz, 8, B * STEP_RK, ms_per_step, hbm_peak, peak_kind, sm_mhz,
                                traffic_key="k_resident_fp32_split_grid10x10_per_launch_bytes")

    # ---------------- plain FP64 GPU path (the comparator of the mixed path)
    fp64 = None
    if args.fp64:
        eng.sample(B, 2000, w.occ_up, w.occ_dn, first=rank * B)
        eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, FP64_STEP_RK, obs=BENCH_OBS)   # warm-up, same shape
        barrier()
        ms64 = 0.0
        for _ in range(3):
            r64 = eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, FP64_STEP_RK, obs=BENCH_OBS)
            ms64 += r64.device_ms
        barrier()
        ms64 = max_over_ranks(ms64)
        v64 = B * FP64_STEP_RK * 3 * ws / (ms64 / 1e3)
        fp64 = {"value": v64, "unit": UNIT, "path": {1: "stream", 2: "resident"}.get(r64.path_used, r64.path_used),
                "precision": "fp64, bit-identical to the FP64 oracle", "mixed_over_fp64": value / v64,
                "roofline": stencil_roofline(n, nnz, 16, B * FP64_STEP_RK, ms64 / 3, hbm_peak, peak_kind, sm_mhz,
                                             fp64=True)}

    # ---------------- e2e through the public ABI with host buffers
    e2e_steps = max(1, min(args.steps, 5))
    Tp = E2E_SNAPSHOTS
    h2d = (4 * n * n * 16) + 2 * n * 8          # tM, U, V, ext (complex col-major) + occupations
    d2h = Tp * (5 * n + 4) * 8                   # the snapshot record of ensemble sums the call copies back
    for _ in range(max(3, args.warmup)):
        eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
        eng.sample(B, 7, w.occ_up, w.occ_dn, first=rank * B)
        eng.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, Tp, obs=BENCH_OBS)
    barrier()
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
        eng.sample(B, 100 + s, w.occ_up, w.occ_dn, first=rank * B)
        res = eng.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, Tp, obs=BENCH_OBS)
        if dist is not None:
            # the one exchange step of the sharded ensemble: FP64 sum of the observables
            shards.combine(vars(res), B, shards.torch_all_reduce_sum("cuda"))
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = B * Tp * e2e_steps * ws / e2e_s

    cpu_ok = rank == 0 and ws == 1 and not args.no_cpu
    u_sweep = None
    if args.u_sweep:
        u_sweep = {f"U{u:g}": u_sweep_leg(dev, rank, u, hbm_peak, peak_kind, sm_mhz, cpu_ok) for u in (2.0, 8.0)}

    hf = None
    if args.hf:
        hf = {f"U{u:g}": hf_leg(dev, u, hbm_peak, peak_kind, sm_mhz, cpu_ok) for u in (2.0, 4.0, 8.0)}

    gpsr = None
    if args.gpsr:
        gpsr = gpsr_leg(dev, cpu=(rank == 0 and ws == 1 and not args.no_cpu))

    cpu_case = None
    if args.cpu_case:
        cpu_case = cpu_case_leg(dev, cpu=(rank == 0 and ws == 1 and not args.no_cpu))

    acc = None
    if args.accuracy:
        acc = accuracy_leg(dev, rank)

    moire = None
    if args.moire:
        moire = moire_leg(dev, rank, bf16_peak, cpu=(rank == 0 and ws == 1 and not args.no_cpu))

    batch = None
    if args.batch:
        batch = batch_leg(dev, rank)

    adj = None
    if args.adjoint:
        adj = adjoint_leg(dev, rank, E.PREC_FP32)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        v, cores, sample, _smp = cpu_sample_rate(w, budget_s=12.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": config_dict(w, {"global_traj": B * ws}),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "note": f"set_system + sample + run({Tp} snapshots, observables) per step"},
                "gpu_launches": launches, "wall_ms_timed": wall_ms, "clocks": clocks, "roofline": roofline,
                "cpu_baseline": cpu, "fp64_gpu": fp64, "advance_only": advance_only, "fp32_plain_state": plain_state,
                "ftwa_cfg2_U": u_sweep, "hf_cfg2": hf, "cpu_runnable_case": cpu_case, "accuracy": acc, "moire_dense": moire, "uneven_batch": batch, "adjoint": adj, "gpsr_drift": gpsr}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
