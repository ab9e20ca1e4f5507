#!/usr/bin/env python
"""Benchmark: split-operator BM4 steps/s on H_2D 1024^2 (real time, length gauge, FP64).

Workload (one "step" = one BM4 time step with its observables), identical in both arms:
  1024 x 1024 grid, DR = 0.2, dt = 0.05 a.u., V = -1/sqrt(x^2 + y^2 + 0.64); initial state: 100
  imaginary-time BM4 steps (normalised every step) from a Gaussian; 800 nm, 1e14 W/cm^2, 8-cycle
  sin^2 pulse (cos2 envelope), linear polarisation along x, length gauge; cos^(1/8) absorbing mask
  over the outer 10% of each axis, applied through the reference's own CAP channel as
  Vcap = -ln(mask)/dt (the factors exp(-h Vcap) of a step multiply to the mask, the coefficients h
  of a step summing to dt); observables norm, dipole (x, y) and dipole acceleration (x, y) at every
  step. Synthetic inputs only (no dataset).

Reported (one JSON line on rank 0):
  value      device-resident steps/s over all ranks: inputs already in HBM, steps timed in calls
             of 100 consecutive steps (one device-resident chain each, replayed from a CUDA graph),
             a 256 MB write flushing the L2 before every call, CUDA events per call, max over ranks
  roofline   the fused axis-pass kernel, from the same timed run: the step's algorithmic bytes over
             its launches, per launch, over the device time per launch (the timed time over the
             launches; the pass kernel is 99% of the device time by the committed ncu launch list)
  e2e        the whole 8-cycle pulse (17,651 steps) through the public C ABI with pinned host
             buffers: state upload, qnd_run_length (field H2D and observable rows D2H every chunk),
             state download
  mixed      the same device-timed steps in mixed precision (complex64 bulk, FP64 reductions), and
             the whole pulse in mixed precision against the FP64 run, column by column
  cpu_baseline  the reference's own C code for this loop on the host cores (N=1, rank 0)
  cufft_yardstick  the same transform sequence with torch.fft (cuFFT), timed only
  h1d, ne2d, sweep, adjoint   short runs of the other configurations (N=1): the H_1D imaginary-time
             job, the Ne_2D-style 2048^2 BM6 run (imaginary and real time, FP64 and mixed), the
             96-member sweep, and the 256^3 adjoint with 16 finite-difference checks

--impl reference runs the reference's CPU implementation of the same workload instead (rank 0).
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
IMAG_STEPS = 100
OBS = ["norm", "dipole_r", "accel"]
METRIC = "split-op steps/s (H_2D 1024^2, BM4, FP64, length gauge, obs every step)"
FLUSH_BYTES = 256 << 20
CONFIG = {
    "workload": "H_2D 1024x1024 real-time BM4 length gauge, dt=0.05, V=-1/sqrt(r^2+0.64), 800nm 1e14 W/cm^2 "
                "8-cycle sin^2 along x, cos^(1/8) mask on the outer 10% as Vcap=-ln(mask)/dt, initial state "
                "from 100 imaginary-time steps, norm+dipole+accel every step",
    "nr": [NR, NR], "dr": DR, "dt": DT, "integrator": INTEG, "parallelism": "replicas",
    "l2": "state 16.8 MB < L2; device-timed calls of 100 consecutive steps, a 256 MB L2 flush before each call",
}


def workload_arrays():
    """V, dV/dx_j, Vcap (the mask), the field samples E [steps][s][2] of the whole pulse, and t."""
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
    # the grid's first point sits on the box edge, where cos(pi/2) rounds to 6e-17: mask >= 0.0088
    vcap1 = -np.log(mask) / DT
    vcap = vcap1[:, None] + vcap1[None, :]
    w = 45.5637639947958 / 800.0
    tau = 8 * 2 * np.pi / w
    E, A, t = field_samples(2, [Mode(1e14, 800.0, 0.0, 0.0, 0.0, tau, "cos2")], INTEG, DT, tau)
    return V, grads, vcap, E, t


def gaussian_guess():
    x = -0.5 * DR * NR + np.arange(NR) * DR
    X, Y = np.meshgrid(x, x, indexing="ij")
    psi = np.exp(-(X * X + Y * Y) / 2.0).astype(np.complex128)
    return psi / np.sqrt(np.sum(np.abs(psi) ** 2) * DR * DR)


def timed_window(nsteps_avail, steps, warmup):
    """First step of the timed window: the pulse's middle (the same steps in both arms)."""
    i0 = nsteps_avail // 2 - (steps + warmup) // 2
    return max(0, min(i0, nsteps_avail - steps - warmup))


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

def reference_ctx(V, vcap, nthreads):
    """The reference's own sources (oracle/_ref; its -O3 -ffast-math build where the host has AVX2 and
    FMA), else the C restatement ("port"), set up with the workload's V and Vcap."""
    from oracle import oracle as O

    fast = False
    try:
        flags = open("/proc/cpuinfo").read()
        fast = O.ref_available(fast=True) and (" avx2" in flags and " fma" in flags)
    except OSError:
        pass
    if O.ref_available(fast) or O.ref_available():
        ctx = O.RefCtx(2, (NR, NR), (DR, DR), INTEG, DT, "H_2D", (0.0, 0.0), nthreads=nthreads, fast=fast)
        build = "reference sources, -O3 -ffast-math (its Makefile flags)" if fast else "reference sources, -O2 IEEE"
        kind = "reference"
    else:
        ctx = O.OracleCtx(2, (NR, NR), (DR, DR), INTEG, DT, nthreads=nthreads)
        build = "C restatement (oracle/qnd_oracle.c)"
        kind = "port"
    ctx.set_vpot(V)
    ctx.set_vcap(vcap)
    return ctx, kind, build


def reference_ground_state(ctx, kind):
    """The initial state of the workload on the host: IMAG_STEPS imaginary-time steps with the
    normalisation of Gram_Schmidt_orthonormalization (QuantumND_imag.c:182-185) from the Gaussian."""
    psi = gaussian_guess()
    if kind == "reference":
        ctx.imag_state([psi], 0, IMAG_STEPS)
    else:
        for _ in range(IMAG_STEPS):
            ctx.step_imag(psi, 1)
            ctx.gram_schmidt(0, [psi])
    return psi


def cpu_reference_steps(ctx, kind, build, psi0, grads, E, i0, max_steps, budget_s, nthreads):
    """Time the reference's length-gauge loop (QuantumND_real.c:195-223) on the workload, from psi0 at
    step i0: the reference's dipole_r, plus norm and accel on the same states (ref_run_length_ext)."""
    def run(psi, Ew):
        if kind == "reference":
            return ctx.run_length_ext(psi, Ew, OBS, grads)
        return ctx.run_length(psi, Ew, OBS)

    if kind == "port":
        for j in range(2):
            ctx.set_gradv(j, grads[j])
    psi = psi0.copy()
    # one call of k steps costs 2 representation changes + k loop bodies: time a 1-step call and a
    # k-step call and take the difference, so the per-step figure is exactly the loop body's
    t_a = time.perf_counter()
    run(psi, E[i0:i0 + 1])
    t1 = time.perf_counter() - t_a
    k = int(max(3, min(max_steps, budget_s / max(t1, 1e-6))))
    t_a = time.perf_counter()
    run(psi, E[i0 + 1:i0 + 1 + k])
    tk = time.perf_counter() - t_a
    per_step = (tk - t1) / (k - 1)
    sample = (f"{k} + 1 BM4 length-gauge steps of the workload from the pulse's middle with per-step "
              f"{'+'.join(OBS)} (the loop of QuantumND_real.c:195-223: the reference's dipole_r and CAP, norm and "
              f"accel computed on the same states), {build}, FFTW-API shim FFT (radix-2, OpenMP over lines), "
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
    nthreads = os.cpu_count() or 1
    V, grads, vcap, E, t = workload_arrays()
    ctx, kind, build = reference_ctx(V, vcap, nthreads)
    psi0 = reference_ground_state(ctx, kind)
    i0 = timed_window(E.shape[0], args.steps, args.warmup) + args.warmup
    res = cpu_reference_steps(ctx, kind, build, psi0, grads, E, i0, args.steps, budget, nthreads)
    line = {
        "metric": METRIC, "value": res["value"], "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 / res["value"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": CONFIG,
        "cpu_baseline": res,
        "e2e": {"value": res["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU side --

def cufft_yardstick(torch, V, vcap, E, steps):
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
    Ct = torch.tensor(vcap, device=dev)
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
            psi_r = psi_r * torch.exp(-hs[i] * Ct - 1j * hs[i] * (Vt + Xt * ex + Yt * ey))
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
            "what": "torch.fft fft2/ifft2 (cuFFT) with torch elementwise phases and CAP: 14 transforms per BM4 "
                    "step, reduction only of the norm; timed only, not on any product path"}


def setup_grid(torch, precision, V, grads, vcap, stream):
    from tdse_nd_mpi_b200 import Grid

    g = Grid(2, (NR, NR), (DR, DR), INTEG, DT, precision=precision)
    g.set_stream(stream.cuda_stream)
    g.set_potential(V)
    g.set_vcap(vcap)
    for j in range(2):
        g.set_gradv(j, grads[j])
    return g


def ground_state(torch, V, stream, nsteps):
    """Initial state: imaginary-time BM4 steps (dt = 0.05) from a Gaussian, normalised every step
    (qnd_imag_propagate, the loop of QuantumND_imag.c:182-185), on the GPU."""
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


def timed_steps(torch, grid, psi_t, E_dev, obs_dev, names, i0, steps, warmup, flush, block=BLOCK):
    """Warm-up, then `steps` steps as calls of `block` consecutive steps (the last one shorter), each
    call bracketed by CUDA events and preceded by an untimed 256 MB write that flushes the L2. Within a
    call the state stays on chip between steps, as in a long propagation.

    Each call of `block` steps is one qnd_run_length_dev chain captured once in a CUDA graph (after
    a warm-up call has built the tables) and replayed; the timed region of a call holds the copy of
    its field samples into the graph's input buffer, the replay and the copy of its observable rows
    out, so that the measurement does not depend on how fast the host enqueues launches."""
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
    # one untimed replay of every graph (the first launch of a graph uploads it to the device), on a
    # copy of the state that is put back afterwards
    saved = psi_t.clone()
    for g, _, _ in graphs.values():
        g.replay()
    psi_t.copy_(saved)
    del saved
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


def launches_per_step(torch, grid, psi_t, E_dev, obs_dev, names, i0, steps):
    """Our kernels per step, counted on a direct call of `steps` steps (a graph replay launches the
    same kernels)."""
    grid.get_profile(reset=True)
    grid.run_length_dev(psi_t, E_dev[i0:i0 + steps], steps, names, obs_dev[:steps])
    torch.cuda.synchronize()
    kernels, _, _ = grid.get_profile(reset=True)
    return kernels / steps


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


def pulse_run_c_abi(torch, grid, stream, psi0, E, nv, dist, dev, elem_dtype):
    """The whole pulse through the C ABI with pinned host buffers: qnd_state_upload, qnd_run_length
    (host field samples in, host observable rows out), qnd_state_download, bracketed by CUDA events
    on the context's stream after two untimed calls that see every chunk shape of the run (the engine
    runs a chunk shape directly the first time and captures its graph the second time). Returns the
    time, the observable rows and the bytes copied."""
    import ctypes as C

    from tdse_nd_mpi_b200 import _lib

    nsteps = E.shape[0]
    E_host = torch.tensor(E).contiguous().pin_memory()
    obs_host = torch.zeros((nsteps, nv), dtype=torch.float64).pin_memory()
    psi_host = torch.tensor(psi0.view(np.float64)).contiguous().pin_memory()
    psi_dev = torch.empty(psi0.size * 2, dtype=elem_dtype, device=dev)
    names_c = (C.c_char_p * len(OBS))(*[s.encode() for s in OBS])
    L = _lib.lib()
    dptr = lambda tns: C.cast(C.c_void_p(tns.data_ptr()), C.POINTER(C.c_double))  # noqa: E731
    # warm-up calls: every full chunk has one shape, the tail another; two full chunks and the tail
    warm = min(nsteps, 2 * 128 + nsteps % 128)
    for _ in range(2):
        _lib.check(L.qnd_state_upload(grid.h, C.c_void_p(psi_dev.data_ptr()), dptr(psi_host)))
        _lib.check(L.qnd_run_length(grid.h, C.c_void_p(psi_dev.data_ptr()), dptr(E_host), warm, len(OBS),
                                    names_c, dptr(obs_host)))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)            # the context's stream (set_stream at set-up)
    _lib.check(L.qnd_state_upload(grid.h, C.c_void_p(psi_dev.data_ptr()), dptr(psi_host)))
    _lib.check(L.qnd_run_length(grid.h, C.c_void_p(psi_dev.data_ptr()), dptr(E_host), nsteps, len(OBS),
                                names_c, dptr(obs_host)))
    _lib.check(L.qnd_state_download(grid.h, dptr(psi_host), C.c_void_p(psi_dev.data_ptr())))
    ev[1].record(stream)
    ev[1].synchronize()
    ms = max_over_ranks(torch, dist, ev[0].elapsed_time(ev[1]), dev)
    h2d = psi0.size * 16 + E.size * 8
    d2h = psi0.size * 16 + nsteps * nv * 8
    return ms, obs_host.numpy().copy(), h2d, d2h


def column_errors(obs_ref, obs, labels, live_floor=1e-6):
    """Per observable column: the FP64 scale max_t |O|, max_t |O_mixed - O_fp64|, and their ratio.
    A column whose FP64 scale is below live_floor times that of the other columns of the same
    observable (the y components under x polarisation, zero by symmetry up to the grid's one-point
    asymmetry) is judged against the live column's scale instead of its own."""
    scale = np.max(np.abs(obs_ref), axis=0)
    err = np.max(np.abs(obs - obs_ref), axis=0)
    groups = {}
    for i, lab in enumerate(labels):
        groups.setdefault(lab.split("_")[0], []).append(i)
    out, worst = [], 0.0
    for i, lab in enumerate(labels):
        live = max(scale[j] for j in groups[lab.split("_")[0]])
        zero = scale[i] < live_floor * live
        den = live if zero else scale[i]
        rel = float(err[i] / den) if den > 0 else None
        out.append({"column": lab, "fp64_scale": float(scale[i]), "max_abs_err": float(err[i]), "rel_err": rel,
                    "judged_against": "live component" if zero else "own scale"})
        if rel is not None:
            worst = max(worst, rel)
    return out, worst


def h1d_leg(torch):
    """The H_1D imaginary-time configuration: 4096 points, DR 0.1, DT 0.05, BM4, 4 states x 2001 steps
    (the reference's loop count for T = 100) with Gram-Schmidt every step, V = -1/sqrt(x^2 + 2),
    seeded Gaussian-random complex initial guesses normalised to 1. The whole job (qnd_imag_propagate
    per state, then the energies) timed with CUDA events, in FP64 and in mixed precision."""
    from tdse_nd_mpi_b200 import Grid

    n, dr, dt, nstates, nsteps = 4096, 0.1, 0.05, 4, 2001
    out = {"grid": [n], "dr": dr, "dt": dt, "states": nstates, "steps_per_state": nsteps}
    energies = {}
    for prec in ("fp64", "mixed"):
        g = Grid(1, (n,), (dr,), "BM4", dt, precision=prec)
        g.set_potential("H_1D")
        rng = np.random.default_rng(1)
        guesses = [(rng.standard_normal(n) + 1j * rng.standard_normal(n)) for _ in range(nstates)]
        states = [g.state(v / np.sqrt(np.sum(np.abs(v) ** 2) * dr)) for v in guesses]
        g.imag_propagate(states, 0, 3)     # warm-up: tables, graphs
        for st, v in zip(states, guesses):
            st.upload(v / np.sqrt(np.sum(np.abs(v) ** 2) * dr))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a.record()
        for j in range(nstates):
            g.imag_propagate(states, j, nsteps)
        e = [g.energies(st, 2) for st in states]
        b.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        energies[prec] = np.array([x[0] for x in e])
        out[prec] = {"job_ms": a.elapsed_time(b), "wall_s": wall, "energies": energies[prec].tolist(),
                     "variance": [float(x[1] - x[0] ** 2) for x in e]}
        g.close()
    out["mixed"]["max_abs_energy_err_vs_fp64_ha"] = float(np.max(np.abs(energies["mixed"] - energies["fp64"])))
    return out


def ne2d_leg(torch, steps, imag_steps):
    """The Ne_2D-style configuration: 2048^2, DR 0.15, BM6, the Ne_2D potential. Imaginary time for 8
    states (imag_steps steps each, Gram-Schmidt every step) in FP64 and in mixed precision from the
    same seeded guesses (FP64 reductions and Gram-Schmidt in both), with the eigenenergy difference;
    then `steps` real-time length-gauge steps from the FP64 ground state under two modes (800 nm at
    2e14 W/cm^2 and 400 nm at 2e13 W/cm^2 with a seeded relative phase, 8- and 16-cycle sin^2
    envelopes), norm + dipole every step, in FP64 and mixed: steps/s of each and the mixed
    observables' error. CUDA events around each whole call."""
    from tdse_nd_mpi_b200 import Grid

    n, dr, dt = 2048, 0.15, 0.05
    x = -0.5 * n * dr + np.arange(n) * dr
    X, Y = np.meshgrid(x, x, indexing="ij")
    rng = np.random.default_rng(11)
    guesses = [(np.exp(-(X * X + Y * Y) / 4.0) * (X ** (k % 3)) * (Y ** (k // 3))
                + 0.01 * rng.standard_normal(X.shape)).astype(np.complex128) for k in range(8)]
    cep2 = float(rng.uniform(0, 2 * np.pi))
    del X, Y
    out = {"grid": [n, n], "dr": dr, "dt": dt, "integrator": "BM6", "potential": "Ne_2D", "real_steps": steps,
           "what": "CUDA events around each whole call (host field, host observable rows)"}
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    grids, energies, psi0 = {}, {}, None
    for prec in ("fp64", "mixed"):
        g = Grid(2, (n, n), (dr, dr), "BM6", dt, precision=prec)
        g.set_potential("Ne_2D")
        grids[prec] = g
        states = [g.state(v) for v in guesses]
        g.imag_propagate(states, 0, 2)     # warm-up: tables
        states[0].upload(guesses[0])
        torch.cuda.synchronize()
        a.record()
        for j in range(8):
            g.imag_propagate(states, j, imag_steps)
        b.record()
        torch.cuda.synchronize()
        energies[prec] = np.array([float(g.energies(st, 1)[0]) for st in states])
        out[prec] = {"imag_ms": a.elapsed_time(b), "imag_steps_per_state": imag_steps,
                     "energies": energies[prec].tolist()}
        if prec == "fp64":
            psi0 = states[0].download()
        for st in states:
            st.free()
    out["mixed"]["max_abs_energy_err_vs_fp64_ha"] = float(np.max(np.abs(energies["mixed"] - energies["fp64"])))
    w800, w400 = 45.5637639947958 / 800.0, 45.5637639947958 / 400.0
    modes = [{"intensity": 2e14, "lambda": 800.0, "ellipticity": 0.0, "cep": 0.0, "delay": 0.0,
              "duration": 8 * 2 * np.pi / w800, "envelope": "cos2"},
             {"intensity": 2e13, "lambda": 400.0, "ellipticity": 0.0, "cep": cep2,
              "delay": 0.0, "duration": 16 * 2 * np.pi / w400, "envelope": "cos2"}]
    total = int(modes[0]["duration"] / dt)
    i0 = max(0, total // 2 - steps // 2)
    E = grids["fp64"].field_samples(modes, i0 + steps)[0][i0:]
    obs = {}
    for prec in ("fp64", "mixed"):
        gg = grids[prec]
        st = gg.state(psi0)
        gg.run_length(st, E, ["norm", "dipole_r"])  # warm-up: tables, chunk graphs
        gg.run_length(st, E, ["norm", "dipole_r"])
        st.upload(psi0)
        torch.cuda.synchronize()
        a.record()
        rows = gg.run_length(st, E, ["norm", "dipole_r"])
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        obs[prec] = rows
        out[prec].update({"steps_per_s": steps / (ms / 1e3), "ms": ms})
        st.free()
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    cols, worst = column_errors(obs["fp64"], obs["mixed"], ["norm", "dipole_x", "dipole_y"])
    out["mixed"]["obs_err"] = cols
    out["mixed"]["max_rel_obs_err_vs_fp64"] = worst
    for g in grids.values():
        g.close()
    return out


def sweep_leg(torch, steps):
    """The sweep configuration: 96 H_2D length-gauge members (32 x 256^2, 48 x 512^2, 16 x 1024^2,
    DR 0.2), BM4 and Verlet alternating, mixed precision, each with a seeded CEP in [0, 2 pi) and an
    intensity log-uniform in [5e13, 3e14] W/cm^2 of an 800 nm 4-cycle sin^2 pulse (field samples from
    qnd_field_samples), norm + dipole every step. `steps` steps from the pulse's middle, timed with
    CUDA events around whole-sweep calls, each after an untimed call of the same shape: one CUDA graph
    per chunk for all members (qnd_run_length_batch), one persistent kernel for all members
    (qnd_run_length_sweep) and one stream per member."""
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
    for label, one in (("persistent", "persistent"), ("one_graph", True), ("streams", False)):
        launch(runs, one)  # warm-up: tables, the chunk graphs of this shape
        launch(runs, one)
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


def adjoint_leg(torch, steps, n_fd=16):
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

    forward(E)  # warm-up: tables, chunk graphs, staging measurement
    forward(E)
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
        idx = (int(rng.integers(0, steps)), int(rng.integers(0, g.s)), 0)
        Ep, Em = E.copy(), E.copy()
        Ep[idx] += eps
        Em[idx] -= eps
        fd = (forward(Ep) - forward(Em)) / (2 * eps)
        checks.append({"sample": list(idx), "adjoint": float(grad[idx]), "central_difference": fd,
                       "rel_diff": abs(fd - float(grad[idx])) / max(abs(fd), 1e-300)})
    g.close()
    return {"grid": [n, n, n], "steps": steps, "checkpoint": 50, "J": J, "J_forward": J_fwd,
            "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms,
            "gradient_entries": int(grad.size), "fd_checks": checks,
            "max_fd_rel_diff": max(c["rel_diff"] for c in checks),
            "what": "CUDA events around whole calls (forward: state upload, the steps, state download; the "
                    "adjoint call runs the forward pass, the checkpointed recomputation and the backward sweep)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed, cuFFT, CPU and other-configuration legs")
    ap.add_argument("--imag-steps", type=int, default=IMAG_STEPS, help="imaginary-time steps for the initial state")
    ap.add_argument("--pulse-steps", type=int, default=0,
                    help="steps of the e2e and mixed-accuracy runs (default: the whole 8-cycle pulse)")
    ap.add_argument("--sweep", type=int, default=40, metavar="STEPS", help="sweep leg steps (0: skip)")
    ap.add_argument("--adjoint", type=int, default=200, metavar="STEPS", help="adjoint leg steps (0: skip)")
    ap.add_argument("--ne2d", type=int, default=40, metavar="STEPS", help="Ne_2D leg real-time steps (0: skip)")
    ap.add_argument("--ne2d-imag", type=int, default=200, help="Ne_2D leg imaginary-time steps per state")
    ap.add_argument("--no-h1d", action="store_true", help="skip the H_1D imaginary-time leg")
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

    V, grads, vcap, E, t = workload_arrays()
    nsteps_avail = E.shape[0]
    i0 = timed_window(nsteps_avail, args.steps, args.warmup)
    psi0 = ground_state(torch, V, stream, args.imag_steps)
    grid = setup_grid(torch, "fp64", V, grads, vcap, stream)
    nv = grid.nvalues(OBS)
    labels = ["norm", "dipole_x", "dipole_y", "accel_x", "accel_y"]
    dev = torch.device("cuda", local)
    E_dev = torch.tensor(E, device=dev).contiguous()
    obs_dev = torch.zeros((args.steps + args.warmup, nv), dtype=torch.float64, device=dev)
    psi_t = torch.tensor(psi0.view(np.float64), device=dev).contiguous()   # complex128 as interleaved doubles
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    # ---- timed region (value)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms = timed_steps(torch, grid, psi_t, E_dev, obs_dev, OBS, i0, args.steps, args.warmup, flush)
    total_ms = max_over_ranks(torch, dist, total_ms, dev)
    value = job_throughput(world, args.steps, total_ms)
    ms_step = total_ms / args.steps

    # ---- roofline of the fused pass kernel, from the timed run
    psi_t2 = torch.tensor(psi0.view(np.float64), device=dev).contiguous()
    lps = launches_per_step(torch, grid, psi_t2, E_dev, obs_dev, OBS, i0, min(args.steps, BLOCK))
    gpu_launches = int(round(lps * args.steps))
    n = NR * NR
    # Algorithmic bytes (the metric's accounting): every full-grid N-D transform is one read and one
    # write of the state, 2*N*16 bytes; a BM4 length-gauge step is 2s = 12 transforms plus the 2 of
    # the per-step observable round trip, 14 in all. The engine does that work in fewer, fused passes
    # (two-sandwich passes), so the per-launch figure is the step's algorithmic bytes over its launches,
    # and the device time per launch is the timed time over the launches.
    s_int = grid.s
    step_alg_bytes = (2 * s_int + 2) * 2 * n * 16
    launch_us = ms_step * 1000.0 / lps
    bytes_per_launch = step_alg_bytes / lps
    peak, peak_src = measured_peak()
    achieved = bytes_per_launch / (launch_us * 1e-6) / 1e9
    traffic, _ = committed_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic,
                "peak_source": ("measured: MEASURED_PEAKS.json hbm_gbs" if peak_src == "measured"
                                else "fallback 6650 GB/s"),
                "kernel": "qnd_pass_kernel<double,1024,*> (fused FFT/phase/iFFT axis passes; one and two "
                          "sandwiches per launch)",
                "algorithmic_bytes_per_launch": bytes_per_launch, "device_us_per_launch": launch_us,
                "launches_per_step": lps, "step_algorithmic_bytes": step_alg_bytes,
                "how": "device time per launch = the timed region's time per step / launches per step (gaps "
                       "between launches included, so achieved is a lower bound for the kernel)"}
    # the same steps one call per step with the L2 flushed before each step
    fs_steps = min(args.steps, 100)
    psi_t3 = torch.tensor(psi0.view(np.float64), device=dev).contiguous()
    ms_fs = timed_steps_single(torch, grid, psi_t3, E_dev, obs_dev, OBS, i0, fs_steps, flush) / fs_steps
    flush_every_step = {"value": 1000.0 / ms_fs, "unit": "steps/s", "ms_per_step": ms_fs, "steps": fs_steps,
                        "what": "rank-local: one qnd_run_length_dev call per step, 256 MB L2 flush before each step"}

    # ---- e2e: the whole pulse through the C ABI with host buffers
    Ep = E[: args.pulse_steps] if args.pulse_steps > 0 else E
    e2e_ms, obs_pulse64, h2d, d2h = pulse_run_c_abi(torch, grid, stream, psi0, Ep, nv, dist, dev, torch.float64)
    e2e = {"value": job_throughput(world, Ep.shape[0], e2e_ms), "unit": "steps/s", "steps": int(Ep.shape[0]),
           "h2d_bytes_per_step": h2d / Ep.shape[0], "d2h_bytes_per_step": d2h / Ep.shape[0],
           "what": "the whole 8-cycle pulse from the ground state: qnd_state_upload + qnd_run_length (host E, "
                   "host observable rows) + qnd_state_download, CUDA events on the context's stream, after two "
                   "untimed calls that see every chunk shape"}

    extras = {}
    if not args.no_extras:
        # ---- mixed precision: the device-timed steps, and the whole pulse against the FP64 run
        gm = setup_grid(torch, "mixed", V, grads, vcap, stream)
        psi_m = torch.tensor(psi0.astype(np.complex64).view(np.float32), device=dev).contiguous()
        obs_m = torch.zeros_like(obs_dev)
        ms_m = max_over_ranks(torch, dist, timed_steps(torch, gm, psi_m, E_dev, obs_m, OBS, i0, args.steps,
                                                      args.warmup, flush), dev) / args.steps
        e2e_m_ms, obs_pulse_m, _, _ = pulse_run_c_abi(torch, gm, stream, psi0, Ep, nv, dist, dev, torch.float32)
        cols, worst = column_errors(obs_pulse64, obs_pulse_m, labels)
        horizon = {}
        for h in (200, 2000, Ep.shape[0]):
            if h <= Ep.shape[0]:
                horizon[str(h)] = column_errors(obs_pulse64[:h], obs_pulse_m[:h], labels)[1]
        extras["mixed"] = {"value": world * 1000.0 / ms_m, "ms_per_step": ms_m, "speedup_vs_fp64": ms_step / ms_m,
                           "e2e_pulse_steps_per_s": job_throughput(world, Ep.shape[0], e2e_m_ms),
                           "e2e_pulse_speedup_vs_fp64": e2e_ms / e2e_m_ms,
                           "max_rel_obs_err_vs_fp64": worst, "max_rel_obs_err_by_horizon": horizon,
                           "obs_err": cols,
                           "obs_err_definition": "over the whole pulse (steps 0..N of the e2e runs), per column "
                                                 "(norm, dipole x/y, accel x/y): max_t |mixed - fp64| / max_t |fp64|; a "
                                                 "column zero by symmetry is divided by its live component's scale",
                           "dtype": "f32 bulk, f64 reductions"}
        gm.close()
        if rank == 0:
            try:
                extras["cufft_yardstick"] = cufft_yardstick(torch, V, vcap, E[i0:], min(args.steps, 50))
            except Exception as exc:  # yardstick only
                extras["cufft_yardstick"] = {"error": str(exc)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_extras:
        try:
            nthreads = os.cpu_count() or 1
            ctx, kind, build = reference_ctx(V, vcap, nthreads)
            cpu = cpu_reference_steps(ctx, kind, build, psi0, grads, E, i0 + args.warmup, 40,
                                      float(os.environ.get("QND_CPU_BUDGET_S", "20")), nthreads)
            del ctx
        except Exception as exc:
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": f"CPU baseline failed: {exc}"}

    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": CONFIG,
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches,
        "flush_every_step": flush_every_step,
        "clocks": clk.summary(),
    }
    line.update(extras)
    grid.close()
    if world == 1 and not args.no_extras:
        if not args.no_h1d:
            line["h1d"] = h1d_leg(torch)
        if args.ne2d > 0:
            line["ne2d"] = ne2d_leg(torch, args.ne2d, args.ne2d_imag)
        if args.sweep > 0:
            line["sweep"] = sweep_leg(torch, args.sweep)
        if args.adjoint > 0:
            line["adjoint"] = adjoint_leg(torch, args.adjoint)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
