#!/usr/bin/env python
"""Benchmark: split-operator BM4 steps/s on H_2D 1024^2 (real time, length gauge, FP64).

Workload (one "step" = one BM4 time step with its observables):
  1024 x 1024 grid, DR = 0.2, dt = 0.05 a.u., V = -1/sqrt(x^2 + y^2 + 0.64); initial state
  from imaginary time; 800 nm, 1e14 W/cm^2, 8-cycle sin^2 pulse (cos2 envelope), linear
  polarisation along x, length gauge; cos^(1/8) absorbing mask over the outer 10% of each axis;
  observables norm, dipole (x, y) and dipole acceleration (x, y) at every step. Synthetic inputs
  only (no dataset).

Reported (one JSON line on rank 0):
  value      device-resident steps/s over all ranks: inputs already in HBM, steps timed in calls
             of 100 consecutive steps (one device-resident chain each, the state on chip between
             steps as in a long propagation), a 256 MB write flushing the L2 before every call,
             CUDA events per call, max over ranks
  flush_every_step  the same with one call per step and the L2 flushed before every step
  e2e        the same steps through the public C ABI with pinned host buffers: state upload,
             qnd_run_length (field H2D and observable D2H every step), state download
  roofline   the fused axis-pass kernel: algorithmic bytes per launch / its mean event time
  cpu_baseline  the reference's own C code for this loop on the host cores (N=1, rank 0)
  mixed      the same steps in mixed precision (complex64 bulk, FP64 reductions) and its
             observable error against the FP64 run
  cufft_yardstick  the same transform sequence with torch.fft (cuFFT), timed only

--impl reference runs the reference's CPU implementation instead (rank 0 only).
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
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

NR, DR, DT, INTEG = 1024, 0.2, 0.05, "BM4"
SOFT = 0.64
OBS = ["norm", "dipole_r", "accel"]
METRIC = "split-op steps/s (H_2D 1024^2, BM4, FP64, length gauge, obs every step)"
FLUSH_BYTES = 256 << 20


def workload_arrays():
    from tdse_nd_mpi_b200.field import Mode, field_samples

    x = -0.5 * DR * NR + np.arange(NR) * DR
    X, Y = np.meshgrid(x, x, indexing="ij")
    r2 = X * X + Y * Y
    V = -1.0 / np.sqrt(r2 + SOFT)
    grads = [X / (r2 + SOFT) ** 1.5, Y / (r2 + SOFT) ** 1.5]
    half = 0.5 * DR * NR
    edge = 0.9 * half
    ax = np.abs(x)
    mask = np.ones(NR)
    zone = ax > edge
    mask[zone] = np.cos(0.5 * np.pi * (ax[zone] - edge) / (half - edge)).clip(0.0) ** 0.125
    w = 45.5637639947958 / 800.0
    tau = 8 * 2 * np.pi / w
    E, A, t = field_samples(2, [Mode(1e14, 800.0, 0.0, 0.0, 0.0, tau, "cos2")], INTEG, DT, tau)
    return V, grads, mask, E, t


def gaussian_guess():
    x = -0.5 * DR * NR + np.arange(NR) * DR
    X, Y = np.meshgrid(x, x, indexing="ij")
    psi = np.exp(-(X * X + Y * Y) / 2.0).astype(np.complex128)
    return psi / np.sqrt(np.sum(np.abs(psi) ** 2) * DR * DR)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.idx)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [p.strip() for p in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    p = os.path.join(ROOT, "profiles", "pass_kernel_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("bytes_per_launch"), d
    return None, None


# ------------------------------------------------------------------ CPU side --

def cpu_reference_steps(max_steps, budget_s):
    """Time the reference's own length-gauge loop (QuantumND_real.c:195-223) on this workload."""
    from oracle import oracle as O

    V, grads, mask, E, t = workload_arrays()
    kind = "reference"
    fast = False
    try:
        flags = open("/proc/cpuinfo").read()
        fast = O.ref_available(fast=True) and (" avx2" in flags and " fma" in flags)
    except OSError:
        pass
    nthreads = os.cpu_count() or 1
    if O.ref_available(fast) or O.ref_available():
        ctx = O.RefCtx(2, (NR, NR), (DR, DR), INTEG, DT, "H_2D", (0.0, 0.0), nthreads=nthreads, fast=fast)
        ctx.set_vpot(V)
        build = "reference sources, -O3 -ffast-math (its Makefile flags)" if fast else "reference sources, -O2 IEEE"
        names = ["dipole_r"]
    else:
        kind = "port"
        ctx = O.OracleCtx(2, (NR, NR), (DR, DR), INTEG, DT, nthreads=nthreads)
        ctx.set_vpot(V)
        for j in range(2):
            ctx.set_gradv(j, grads[j])
            ctx.set_mask_axis(j, mask)
        build = "C restatement (oracle/qnd_oracle.c)"
        names = ["norm", "dipole_r", "accel"]
    psi = gaussian_guess()
    i0 = len(t) // 2
    # one call of k steps costs 2 representation changes + k loop bodies: time a 1-step call and a
    # k-step call and take the difference, so the per-step figure is exactly the loop body's.
    t_a = time.perf_counter()
    ctx.run_length(psi, E[i0:i0 + 1], names)
    t1 = time.perf_counter() - t_a
    k = int(max(3, min(max_steps, budget_s / max(t1, 1e-6))))
    t_a = time.perf_counter()
    ctx.run_length(psi, E[i0 + 1:i0 + 1 + k], names)
    tk = time.perf_counter() - t_a
    per_step = (tk - t1) / (k - 1)
    sample = (f"{k} + 1 BM4 length-gauge steps of the H_2D 1024^2 workload with per-step {'+'.join(names)} "
              f"(loop of QuantumND_real.c:195-223), {build}, FFTW-API shim FFT (radix-2, OpenMP over lines), "
              f"{nthreads} threads; per-step time = (t[{k} steps] - t[1 step]) / {k - 1}")
    return {"value": 1.0 / per_step, "unit": "steps/s", "cores": nthreads, "kind": kind, "sample": sample}


def max_over_ranks(torch, dist, value, device):
    """The largest of a per-rank float over all ranks (the slowest rank sets the job's time); the
    value itself when there is no process group."""
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, steps, ms):
    """Whole-job steps/s: every rank (replica) runs `steps` steps, the job takes `ms`."""
    return world * steps / (ms / 1000.0)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    budget = float(os.environ.get("QND_REF_BUDGET_S", "150"))
    res = cpu_reference_steps(args.steps, budget)
    line = {
        "metric": METRIC, "value": res["value"], "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 / res["value"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": "H_2D 1024x1024 real-time BM4 length gauge, dt=0.05, obs every step", "nr": [NR, NR],
                   "dr": DR, "dt": DT, "integrator": INTEG, "parallelism": "replicas only",
                   "l2": "state 16.8 MB; CPU run"},
        "cpu_baseline": res,
        "e2e": {"value": res["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU side --

def cufft_yardstick(torch, V, E, steps):
    """The same per-step transform sequence (14 full 2-D transforms) with torch.fft (cuFFT)."""
    dev = torch.device("cuda")
    from tdse_nd_mpi_b200.field import integrator_coeffs

    asc = integrator_coeffs(INTEG, DT)
    s = len(asc) // 2
    p = 2 * np.pi * np.fft.fftfreq(NR, d=DR)
    KX, KY = np.meshgrid(p, p, indexing="ij")
    kin = torch.tensor(0.5 * (KX ** 2 + KY ** 2), device=dev)
    x = -0.5 * DR * NR + np.arange(NR) * DR
    X, Y = np.meshgrid(x, x, indexing="ij")
    Xt, Yt = torch.tensor(X, device=dev), torch.tensor(Y, device=dev)
    Vt = torch.tensor(V, device=dev)
    psi = torch.tensor(gaussian_guess(), device=dev)
    kc = [asc[0]] + [asc[2 * i - 1] + asc[2 * i] for i in range(1, s)] + [asc[2 * s - 1]]
    kph = [torch.exp(-1j * c * kin) for c in kc]
    hs = [asc[2 * i] + asc[2 * i + 1] for i in range(s)]

    def step(k):
        nonlocal psi
        ph = torch.fft.fft2(psi)
        for i in range(s):
            psi_r = torch.fft.ifft2(kph[i] * ph)
            ex, ey = float(E[k, i, 0]), float(E[k, i, 1])
            psi_r = psi_r * torch.exp(-1j * hs[i] * (Vt + Xt * ex + Yt * ey))
            ph = torch.fft.fft2(psi_r)
        psi = torch.fft.ifft2(kph[s] * ph)
        return (psi.abs() ** 2).sum()

    for k in range(3):
        step(k)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for k in range(steps):
        step(k)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    return {"value": 1000.0 / ms, "unit": "steps/s", "ms_per_step": ms,
            "what": "torch.fft fft2/ifft2 (cuFFT) with torch elementwise phases: 14 transforms per BM4 step, "
                    "no mask, reduction only of the norm; timed only, not on any product path"}


def setup_grid(torch, precision, V, grads, mask, stream):
    from tdse_nd_mpi_b200 import Grid

    g = Grid(2, (NR, NR), (DR, DR), INTEG, DT, precision=precision)
    g.set_stream(stream.cuda_stream)
    g.set_potential(V)
    for j in range(2):
        g.set_gradv(j, grads[j])
        g.set_mask_axis(j, mask)
    return g


def ground_state(torch, V, stream, nsteps):
    """Initial state: imaginary-time BM4 steps (dt = 0.05) from a Gaussian, on the GPU."""
    from tdse_nd_mpi_b200 import Grid

    gi = Grid(2, (NR, NR), (DR, DR), INTEG, DT)
    gi.set_stream(stream.cuda_stream)
    gi.set_potential(V)
    st = gi.state(gaussian_guess())
    gi.imag_propagate([st], 0, nsteps)
    psi = st.download()
    st.free()
    gi.close()
    return psi


BLOCK = 100  # consecutive steps per timed call (one device-resident chain); the L2 is flushed between calls


def timed_steps(torch, grid, psi_t, E_dev, obs_dev, names, i0, steps, warmup, flush, block=BLOCK, graph=True):
    """Warm-up, then `steps` steps as calls of `block` consecutive steps (the last one shorter), each
    call bracketed by CUDA events and preceded by an untimed 256 MB write that flushes the L2. Within a
    call the state stays on chip between steps, as in a long propagation.

    Each call of `block` steps is one qnd_run_length_dev chain captured once in a CUDA graph (after
    a warm-up call has built the tables) and replayed; the timed region of a call holds the copy of
    its field samples into the graph's input buffer, the replay and the copy of its observable rows
    out, so that the measurement does not depend on how fast the host enqueues launches. With
    graph=False every call is enqueued directly (the per-launch profiling run)."""
    def calls(n, first):
        k = 0
        while k < n:
            b = min(block, n - k)
            yield first + k, b
            k += b
    for k, b in calls(warmup, 0):
        flush.zero_()
        grid.run_length_dev(psi_t, E_dev[i0 + k:i0 + k + b], b, names, obs_dev[k:k + b])
    torch.cuda.synchronize()
    if not graph:
        todo = list(calls(steps, warmup))
        starts = [torch.cuda.Event(enable_timing=True) for _ in todo]
        ends = [torch.cuda.Event(enable_timing=True) for _ in todo]
        for (k, b), st, en in zip(todo, starts, ends):
            flush.zero_()
            st.record()
            grid.run_length_dev(psi_t, E_dev[i0 + k:i0 + k + b], b, names, obs_dev[k:k + b])
            en.record()
        torch.cuda.synchronize()
        return sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    graphs = {}

    def graph_for(b):
        if b not in graphs:
            e_buf = torch.empty_like(E_dev[:b])
            o_buf = torch.empty_like(obs_dev[:b])
            e_buf.copy_(E_dev[i0:i0 + b])
            grid.run_length_dev(psi_t.clone(), e_buf, b, names, o_buf)   # tables for this shape
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=torch.cuda.current_stream()):
                grid.run_length_dev(psi_t, e_buf, b, names, o_buf)
            graphs[b] = (g, e_buf, o_buf)
        return graphs[b]

    todo = list(calls(steps, warmup))
    for _, b in todo:
        graph_for(b)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in todo]
    ends = [torch.cuda.Event(enable_timing=True) for _ in todo]
    for (k, b), st, en in zip(todo, starts, ends):
        g, e_buf, o_buf = graphs[b]
        flush.zero_()
        st.record()
        e_buf.copy_(E_dev[i0 + k:i0 + k + b])
        g.replay()
        obs_dev[k:k + b].copy_(o_buf)
        en.record()
    torch.cuda.synchronize()
    total = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    graphs.clear()
    return total


def timed_steps_single(torch, grid, psi_t, E_dev, obs_dev, names, i0, steps, flush):
    """`steps` single-step qnd_run_length_dev calls, each bracketed by CUDA events, the L2 flushed
    before every step (no on-chip state across steps; host enqueue included)."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    torch.cuda.synchronize()
    for k in range(steps):
        flush.zero_()
        starts[k].record()
        grid.run_length_dev(psi_t, E_dev[i0 + k:i0 + k + 1], 1, names, obs_dev[k:k + 1])
        ends[k].record()
    torch.cuda.synchronize()
    return sum(s.elapsed_time(e) for s, e in zip(starts, ends))


def sweep_leg(torch, steps):
    """The sweep configuration: 96 H_2D length-gauge members (32 x 256^2, 48 x 512^2, 16 x 1024^2,
    DR 0.2), BM4 and Verlet alternating, mixed precision, each with a seeded CEP in [0, 2 pi) and an
    intensity log-uniform in [5e13, 3e14] W/cm^2 of an 800 nm 4-cycle sin^2 pulse (field samples from
    qnd_field_samples), norm + dipole every step. `steps` steps from the pulse's middle, timed with
    CUDA events around whole-sweep calls, each after an untimed call of the same shape: one CUDA graph
    per chunk for all members (qnd_run_length_batch) and, for comparison, one stream per member."""
    from tdse_nd_mpi_b200 import Grid
    from tdse_nd_mpi_b200.batch import Member, launch, prepare, release

    rng = np.random.default_rng(2024)
    tau = 4 * 2 * np.pi / (45.5637639947958 / 800.0)
    total = int(tau / DT)
    i0 = max(0, total // 2 - steps // 2)
    members = []
    for k, n in enumerate([256] * 32 + [512] * 48 + [1024] * 16):
        integ = "BM4" if k % 2 == 0 else "Verlet"
        mode = {"intensity": float(np.exp(rng.uniform(np.log(5e13), np.log(3e14)))), "lambda": 800.0,
                "ellipticity": 0.0, "cep": float(rng.uniform(0.0, 2 * np.pi)), "delay": 0.0, "duration": tau,
                "envelope": "cos2"}
        g = Grid(2, (n, n), (DR, DR), integ, DT)
        E = g.field_samples([mode], i0 + steps)[0][i0:]
        g.close()
        x = -0.5 * n * DR + np.arange(n) * DR
        X, Y = np.meshgrid(x, x, indexing="ij")
        psi = np.exp(-(X * X + Y * Y) / 2.0).astype(np.complex128)
        psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * DR * DR)
        members.append(Member(shape=(n, n), dr=(DR, DR), integrator=integ, dt=DT, potential="H_2D", field=E,
                              psi0=psi, cap=(0.05, 5.0), names=("norm", "dipole_r"), precision="mixed"))
    runs = prepare(members)
    points = sum(n * n for n in [256] * 32 + [512] * 48 + [1024] * 16)
    out = {"members": len(members), "grid_points": points, "steps": steps, "precision": "mixed",
           "what": "whole-sweep calls, CUDA events around each (the call returns when all members are done)"}
    for label, one in (("one_graph", True), ("streams", False)):
        launch(runs, one)  # warm-up: tables, the chunk graphs of this shape
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        launch(runs, one)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        out[label] = {"ms": ms, "member_steps_per_s": len(members) * steps / (ms / 1e3),
                      "point_steps_per_s": points * steps / (ms / 1e3)}
    release(runs)
    return out


def ne2d_leg(torch, steps, imag_steps):
    """The Ne_2D-style configuration: 2048^2, DR 0.15, BM6, the Ne_2D potential. Imaginary time for 8
    states (imag_steps steps each, Gram-Schmidt every step, FP64), then `steps` real-time
    length-gauge steps from the ground state under two modes (800 nm at 2e14 W/cm^2 and 400 nm at
    2e13 W/cm^2 with a seeded relative phase, 8- and 16-cycle sin^2 envelopes, field samples from
    qnd_field_samples), norm + dipole every step, in FP64 and in mixed precision: steps/s of each and
    the mixed observables' error against the FP64 run. CUDA events around each whole call."""
    from tdse_nd_mpi_b200 import Grid

    n, dr, dt = 2048, 0.15, 0.05
    g = Grid(2, (n, n), (dr, dr), "BM6", dt)
    g.set_potential("Ne_2D")
    x = -0.5 * n * dr + np.arange(n) * dr
    X, Y = np.meshgrid(x, x, indexing="ij")
    rng = np.random.default_rng(11)
    states = []
    for k in range(8):
        guess = np.exp(-(X * X + Y * Y) / 4.0) * (X ** (k % 3)) * (Y ** (k // 3)) + 0.01 * rng.standard_normal(X.shape)
        states.append(g.state(guess.astype(np.complex128)))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for j in range(8):
        g.imag_propagate(states, j, imag_steps)
    b.record()
    torch.cuda.synchronize()
    imag_ms = a.elapsed_time(b)
    energies = [float(g.energies(st, 1)[0]) for st in states]
    psi0 = states[0].download()
    w800, w400 = 45.5637639947958 / 800.0, 45.5637639947958 / 400.0
    modes = [{"intensity": 2e14, "lambda": 800.0, "ellipticity": 0.0, "cep": 0.0, "delay": 0.0,
              "duration": 8 * 2 * np.pi / w800, "envelope": "cos2"},
             {"intensity": 2e13, "lambda": 400.0, "ellipticity": 0.0, "cep": float(rng.uniform(0, 2 * np.pi)),
              "delay": 0.0, "duration": 16 * 2 * np.pi / w400, "envelope": "cos2"}]
    total = int(modes[0]["duration"] / dt)
    i0 = max(0, total // 2 - steps // 2)
    E = g.field_samples(modes, i0 + steps)[0][i0:]
    out = {"grid": [n, n], "dr": dr, "dt": dt, "integrator": "BM6", "potential": "Ne_2D",
           "imag": {"states": 8, "steps_per_state": imag_steps, "ms": imag_ms, "energies": energies},
           "real_steps": steps, "what": "CUDA events around each whole call (host field, host observable rows)"}
    obs = {}
    for prec in ("fp64", "mixed"):
        gg = g if prec == "fp64" else Grid(2, (n, n), (dr, dr), "BM6", dt, precision="mixed")
        if prec == "mixed":
            gg.set_potential("Ne_2D")
        st = gg.state(psi0)
        gg.run_length(st, E[: min(steps, 256)], ["norm", "dipole_r"])  # warm-up: tables, chunk graphs
        st.upload(psi0)
        torch.cuda.synchronize()
        a.record()
        rows = gg.run_length(st, E, ["norm", "dipole_r"])
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        obs[prec] = rows
        out[prec] = {"steps_per_s": steps / (ms / 1e3), "ms": ms}
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    # per column (norm, x, y) relative to the column's magnitude over the run; a column that vanishes
    # by symmetry (the y dipole under x polarisation) is reported as an absolute error
    col_scale = np.max(np.abs(obs["fp64"]), axis=0)
    live = col_scale > 1e-8
    err = np.max(np.abs(obs["mixed"] - obs["fp64"]), axis=0)
    out["mixed"]["max_rel_obs_err_vs_fp64"] = float(np.max(err[live] / col_scale[live])) if live.any() else None
    out["mixed"]["max_abs_err_symmetry_zero_obs"] = float(np.max(err[~live])) if (~live).any() else None
    return out


def adjoint_leg(torch, steps, n_fd=4):
    """The H_3D adjoint configuration: 256^3, DR 0.3, dt 0.05, BM4, V = -1/sqrt(r^2 + 0.5), an 800 nm
    field sampled at the sub-step times with seeded 1e-3 relative perturbations, J = the norm beyond
    |r| > 25 a.u., checkpoints every 50 steps. Times the forward run (qnd_run_length) and the adjoint
    call (J and dJ/dE for every sample, qnd_adjoint_length) with CUDA events, and checks the gradient
    at n_fd seeded samples against central differences of the forward J."""
    from tdse_nd_mpi_b200 import Grid
    from tdse_nd_mpi_b200.adjoint import absorbed_weight

    n, dr, dt = 256, 0.3, 0.05
    g = Grid(3, (n, n, n), (dr, dr, dr), "BM4", dt)
    x = g.axis_r(0)
    X = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X[0] ** 2 + X[1] ** 2 + X[2] ** 2)
    g.set_potential(-1.0 / np.sqrt(r * r + 0.5))
    g.set_cap(0.05, 5.0)
    w = absorbed_weight(g, 25.0)
    psi0 = (np.exp(-(r ** 2) / 2) * np.exp(1j * 1.5 * X[0])).astype(np.complex128)
    psi0 /= np.sqrt(np.sum(np.abs(psi0) ** 2) * dr ** 3)
    del X, r
    rng = np.random.default_rng(5)
    w800 = 45.5637639947958 / 800.0
    t = np.arange(steps)[:, None] * dt + np.cumsum(np.r_[g.as_scaled[0], g.as_scaled[1:-1:2] + g.as_scaled[2::2]])
    E = np.zeros((steps, g.s, 3))
    E[:, :, 0] = 0.0533803 * np.sin(w800 * t) * np.sin(np.pi * t / (steps * dt)) ** 2 * (
        1.0 + 1e-3 * rng.standard_normal((steps, g.s)))
    st, work = g.state(psi0), g.state()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def forward(Ep):
        work.upload(psi0)
        g.run_length(work, Ep, [])
        return g.dNr * float(np.sum(w * np.abs(work.download()) ** 2))

    forward(E[:50])  # warm-up: tables, chunk graphs, staging measurement
    torch.cuda.synchronize()
    a.record()
    J_fwd = forward(E)
    b.record()
    torch.cuda.synchronize()
    fwd_ms = a.elapsed_time(b)
    a.record()
    J, grad = g.adjoint_length(st, E, w, checkpoint=50)
    b.record()
    torch.cuda.synchronize()
    adj_ms = a.elapsed_time(b)
    eps, checks = 1e-5, []
    for _ in range(n_fd):
        idx = (int(rng.integers(steps // 4, steps)), int(rng.integers(0, g.s)), 0)
        Ep, Em = E.copy(), E.copy()
        Ep[idx] += eps
        Em[idx] -= eps
        fd = (forward(Ep) - forward(Em)) / (2 * eps)
        checks.append({"sample": list(idx), "adjoint": float(grad[idx]), "central_difference": fd,
                       "rel_diff": abs(fd - float(grad[idx])) / max(abs(fd), 1e-300)})
    return {"grid": [n, n, n], "steps": steps, "checkpoint": 50, "J": J, "J_forward": J_fwd,
            "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms,
            "gradient_entries": int(grad.size), "fd_checks": checks,
            "what": "CUDA events around whole calls; the adjoint call runs the forward pass, the "
                    "checkpointed recomputation and the backward sweep"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip mixed / cuFFT / CPU legs")
    ap.add_argument("--imag-steps", type=int, default=100, help="imaginary-time steps for the initial state")
    ap.add_argument("--sweep", type=int, default=0, metavar="STEPS",
                    help="also time the 96-member sweep configuration for STEPS steps (key 'sweep')")
    ap.add_argument("--adjoint", type=int, default=0, metavar="STEPS",
                    help="also run the H_3D 256^3 adjoint configuration for STEPS steps (key 'adjoint')")
    ap.add_argument("--ne2d", type=int, default=0, metavar="STEPS",
                    help="also run the Ne_2D-style 2048^2 BM6 configuration: 8 imaginary-time states, then "
                         "STEPS real-time steps in FP64 and mixed precision (key 'ne2d')")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    V, grads, mask, E, t = workload_arrays()
    nsteps_avail = E.shape[0]
    i0 = nsteps_avail // 2 - (args.steps + args.warmup) // 2
    i0 = max(0, min(i0, nsteps_avail - args.steps - args.warmup))
    psi0 = ground_state(torch, V, stream, args.imag_steps)
    grid = setup_grid(torch, "fp64", V, grads, mask, stream)
    nv = grid.nvalues(OBS)
    dev = torch.device("cuda", local)
    E_dev = torch.tensor(E, device=dev).contiguous()
    obs_dev = torch.zeros((args.steps + args.warmup, nv), dtype=torch.float64, device=dev)
    psi_t = torch.tensor(psi0.view(np.float64), device=dev).contiguous()   # complex128 as interleaved doubles
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    # ---- timed region (value)
    grid.get_profile(reset=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms = timed_steps(torch, grid, psi_t, E_dev, obs_dev, OBS, i0, args.steps, args.warmup, flush)
    grid.get_profile(reset=True)
    total_ms = max_over_ranks(torch, dist, total_ms, dev)
    value = job_throughput(world, args.steps, total_ms)
    ms_step = total_ms / args.steps
    obs_fp64 = obs_dev[args.warmup:].cpu().numpy()

    # ---- roofline of the fused pass kernel (per-launch CUDA events, L2 flushed between steps)
    grid.set_profiling(True)
    prof_steps = min(args.steps, 100)
    psi_t2 = torch.tensor(psi0.view(np.float64), device=dev).contiguous()
    timed_steps(torch, grid, psi_t2, E_dev, obs_dev, OBS, i0, prof_steps, 0, flush, graph=False)
    prof_kernels, passes, pass_ms = grid.get_profile(reset=True)
    grid.set_profiling(False)
    # our kernels per step, counted on the plain-call run (graph replays launch the same kernels)
    gpu_launches = int(round(prof_kernels / prof_steps * args.steps))
    # the same steps one call per step with the L2 flushed before each (no on-chip state across steps)
    fs_steps = min(args.steps, 100)
    psi_t3 = torch.tensor(psi0.view(np.float64), device=dev).contiguous()
    ms_fs = timed_steps_single(torch, grid, psi_t3, E_dev, obs_dev, OBS, i0, fs_steps, flush) / fs_steps
    flush_every_step = {"value": 1000.0 / ms_fs, "unit": "steps/s", "ms_per_step": ms_fs, "steps": fs_steps,
                        "what": "rank-local: one qnd_run_length_dev call per step, 256 MB L2 flush before each step"}
    n = NR * NR
    # Algorithmic bytes (the metric's accounting): every full-grid N-D transform is one read and one
    # write of the state, 2*N*16 bytes; a BM4 length-gauge step is 2s = 12 transforms plus the 2 of
    # the per-step observable round trip, 14 in all. The engine does that work in fewer, fused passes
    # (two-sandwich passes), so the per-launch figure is the step's algorithmic bytes over its launches.
    s_int = grid.s
    step_alg_bytes = (2 * s_int + 2) * 2 * n * 16
    passes_per_step = passes / prof_steps
    avg_pass_s = pass_ms / passes / 1000.0
    bytes_per_launch = step_alg_bytes / passes_per_step
    peak, peak_src = measured_peak()
    achieved = bytes_per_launch / avg_pass_s / 1e9
    traffic, _ = committed_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic,
                "peak_source": ("measured: MEASURED_PEAKS.json hbm_gbs" if peak_src == "measured"
                                else "fallback 6650 GB/s"),
                "kernel": "qnd_pass_kernel<double,1024,*> (fused FFT/phase/iFFT axis passes; one and two "
                          "sandwiches per launch)",
                "algorithmic_bytes_per_launch": bytes_per_launch, "mean_launch_us": avg_pass_s * 1e6,
                "launches_per_step": passes_per_step, "step_algorithmic_bytes": step_alg_bytes,
                "step_frac_of_peak": (step_alg_bytes / (ms_step / 1000.0) / 1e9) / peak}

    # ---- e2e through the C ABI with pinned host buffers
    import ctypes as C

    from tdse_nd_mpi_b200 import _lib

    e2e_steps = args.steps
    E_host = torch.tensor(E[i0:i0 + e2e_steps]).contiguous().pin_memory()
    obs_host = torch.zeros((e2e_steps, nv), dtype=torch.float64).pin_memory()
    psi_host = torch.tensor(psi0.view(np.float64)).contiguous().pin_memory()
    psi_dev_e2e = torch.empty_like(psi_t)
    names_c = (C.c_char_p * len(OBS))(*[s.encode() for s in OBS])
    L = _lib.lib()
    dptr = lambda tns: C.cast(C.c_void_p(tns.data_ptr()), C.POINTER(C.c_double))  # noqa: E731
    # warm-up: two untimed calls of the same shape (the engine runs a chunk shape directly the first
    # time it sees it and captures its graph the second time; the last, shorter chunk is seen once
    # per call)
    for _ in range(2):
        _lib.check(L.qnd_state_upload(grid.h, C.c_void_p(psi_dev_e2e.data_ptr()), dptr(psi_host)))
        _lib.check(L.qnd_run_length(grid.h, C.c_void_p(psi_dev_e2e.data_ptr()), dptr(E_host), e2e_steps, len(OBS),
                                    names_c, dptr(obs_host)))
    flush.zero_()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    h0 = time.perf_counter()
    _lib.check(L.qnd_state_upload(grid.h, C.c_void_p(psi_dev_e2e.data_ptr()), dptr(psi_host)))
    h1 = time.perf_counter()
    _lib.check(L.qnd_run_length(grid.h, C.c_void_p(psi_dev_e2e.data_ptr()), dptr(E_host), e2e_steps, len(OBS),
                                names_c, dptr(obs_host)))
    h2 = time.perf_counter()
    _lib.check(L.qnd_state_download(grid.h, dptr(psi_host), C.c_void_p(psi_dev_e2e.data_ptr())))
    h3 = time.perf_counter()
    b.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(torch, dist, a.elapsed_time(b), dev)
    e2e = {"value": job_throughput(world, e2e_steps, e2e_ms), "unit": "steps/s",
           "h2d_bytes_per_step": (n * 16 + e2e_steps * grid.s * 2 * 8) / e2e_steps,
           "d2h_bytes_per_step": (n * 16 + e2e_steps * nv * 8) / e2e_steps,
           "what": "qnd_state_upload + qnd_run_length (host E, host observable rows) + qnd_state_download, "
                   "after two untimed calls of the same shape",
           "host_ms": {"upload": 1e3 * (h1 - h0), "run_length": 1e3 * (h2 - h1), "download": 1e3 * (h3 - h2)}}

    extras = {}
    if not args.no_extras:
        # ---- mixed precision on the same steps, error vs the FP64 run
        gm = setup_grid(torch, "mixed", V, grads, mask, stream)
        psi_m = torch.tensor(psi0.astype(np.complex64).view(np.float32), device=dev).contiguous()
        obs_m = torch.zeros_like(obs_dev)
        ms_m = max_over_ranks(torch, dist, timed_steps(torch, gm, psi_m, E_dev, obs_m, OBS, i0, args.steps,
                                                      args.warmup, flush), dev) / args.steps
        om = obs_m[args.warmup:].cpu().numpy()
        # error of each observable relative to its own magnitude over the run; observables that vanish
        # by symmetry (y-dipole, y-acceleration under x polarisation) are reported as absolute errors
        col_scale = np.max(np.abs(obs_fp64), axis=0)
        live = col_scale > 1e-8
        rel_err = float(np.max(np.max(np.abs(om - obs_fp64), axis=0)[live] / col_scale[live])) if live.any() else None
        abs_err_dead = float(np.max(np.abs(om - obs_fp64)[:, ~live])) if (~live).any() else None
        extras["mixed"] = {"value": world * 1000.0 / ms_m, "ms_per_step": ms_m, "speedup_vs_fp64": ms_step / ms_m,
                           "max_rel_obs_err_vs_fp64": rel_err, "max_abs_err_symmetry_zero_obs": abs_err_dead,
                           "obs_err_definition": "max over steps |mixed - fp64| / max over steps |fp64|, per "
                                                 "observable column (norm, x, y, ax, ay)",
                           "dtype": "f32 bulk, f64 reductions"}
        gm.close()
        if rank == 0:
            try:
                extras["cufft_yardstick"] = cufft_yardstick(torch, V, E[i0:], min(args.steps, 50))
            except Exception as exc:  # yardstick only
                extras["cufft_yardstick"] = {"error": str(exc)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_extras:
        try:
            cpu = cpu_reference_steps(40, float(os.environ.get("QND_CPU_BUDGET_S", "20")))
        except Exception as exc:
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": f"CPU baseline failed: {exc}"}

    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "H_2D 1024x1024 real-time BM4 length gauge, dt=0.05, 800nm 1e14 W/cm^2 8-cycle "
                               "sin^2, cos^(1/8) mask, norm+dipole+accel every step",
                   "nr": [NR, NR], "dr": DR, "dt": DT, "integrator": INTEG, "parallelism": f"replicas x{world}",
                   "l2": f"state 16.8 MB < L2; timed in calls of {BLOCK} consecutive steps with a 256 MB L2 flush before each call"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches,
        "flush_every_step": flush_every_step,
        "clocks": clk.summary(),
    }
    line.update(extras)
    if args.sweep > 0 and world == 1:
        line["sweep"] = sweep_leg(torch, args.sweep)
    if args.ne2d > 0 and world == 1:
        line["ne2d"] = ne2d_leg(torch, args.ne2d, max(20, args.imag_steps))
    if args.adjoint > 0 and world == 1:
        line["adjoint"] = adjoint_leg(torch, args.adjoint)
    if rank == 0:
        print(json.dumps(line), flush=True)
    grid.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
