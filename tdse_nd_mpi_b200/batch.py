"""Independent propagations run together: the sweep configuration of many grids of different sizes
(members), each its own real-time length-gauge run.

- On one GPU every member has its own context and stream, so the small grids' passes overlap.
  One 256^2 pass fills a tenth of a B200. Each member's chunks of steps replay its own CUDA graphs.
  Alternatively (one_graph) the members' chains of each chunk are the parallel branches of one CUDA
  graph (qnd_run_length_batch): one graph launch per chunk for the whole sweep, but every member
  waits for the slowest at each chunk's end; on the 96-member sweep configuration that measured 6%
  slower than the free-running streams (34.2k against 36.3k member-steps/s, mixed precision).
- Across ranks the members are shared out by a balanced-bytes greedy, with no data exchange during
  the runs. The observables are gathered on rank 0 at the end.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .engine import Grid


@dataclasses.dataclass
class Member:
    """One propagation: grid, integrator, potential (a name or an array on the grid), CAP, the field
    samples E [nsteps][s][dim], the initial r-space state and the observables of every step."""

    shape: tuple
    dr: tuple
    integrator: str
    dt: float
    potential: object
    field: np.ndarray
    psi0: np.ndarray
    cap: tuple = (0.0, 0.0)
    names: tuple = ("norm", "dipole_r")
    precision: str = "fp64"

    @property
    def state_bytes(self) -> int:
        return int(np.prod(self.shape)) * (16 if self.precision == "fp64" else 8)


def partition(members, world: int) -> list[list[int]]:
    """Member indices per rank: the largest members first, each to the rank with the fewest bytes so
    far (ties to the lower rank). Deterministic, so every rank computes the same assignment."""
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(members)), key=lambda i: (-members[i].state_bytes, i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += members[i].state_bytes
    for p in parts:
        p.sort()
    return parts


def prepare(members) -> list:
    """One context, device state, device field and observable buffer per member (on this GPU)."""
    import torch

    runs = []
    for m in members:
        g = Grid(len(m.shape), m.shape, m.dr, m.integrator, m.dt, precision=m.precision)
        if isinstance(m.potential, str):
            g.set_potential(m.potential)
        else:
            g.set_potential(np.asarray(m.potential, dtype=np.float64))
        g.set_cap(*m.cap)
        st = g.state(m.psi0)
        E = torch.tensor(np.ascontiguousarray(m.field, dtype=np.float64), device="cuda")
        nv = g.nvalues(list(m.names))
        obs = torch.zeros((E.shape[0], max(nv, 1)), dtype=torch.float64, device="cuda")
        runs.append((g, st, E, obs, nv, list(m.names)))
    torch.cuda.synchronize()  # inputs on the device before the contexts' own streams read them
    return runs


def launch(runs, one_graph=False, nsteps: int | None = None) -> None:
    """Run every prepared member (nsteps of its field, default all); returns when all are done.
    one_graph: True or "graph" runs all members through qnd_run_length_batch (one CUDA graph per
    chunk); "persistent" through qnd_run_length_sweep (one persistent kernel per 512 steps); both need
    the same nsteps and observables for every member. Otherwise each member's own device loop runs on
    its own stream."""
    import ctypes as C

    from ._lib import check, lib

    n = [r[2].shape[0] if nsteps is None else nsteps for r in runs]
    same = len({(k, tuple(r[5])) for k, r in zip(n, runs)}) == 1
    if one_graph and same and runs:
        k = len(runs)
        names = runs[0][5]
        arr = lambda xs: (C.c_void_p * k)(*xs)  # noqa: E731
        cnames = (C.c_char_p * max(1, len(names)))(*[x.encode() for x in names])
        fn = lib().qnd_run_length_sweep if one_graph == "persistent" else lib().qnd_run_length_batch
        check(fn(k, arr([r[0].h for r in runs]), arr([r[1].ptr for r in runs]), arr([r[2].data_ptr() for r in runs]),
                 int(n[0]), len(names), cnames, arr([r[3].data_ptr() for r in runs])))
    else:
        for (g, st, E, obs, nv, names), k in zip(runs, n):
            g.run_length_dev(st, E, k, names, obs if nv else None)
        for r in runs:
            r[0].synchronize()


def release(runs) -> None:
    for g, st, *_ in runs:
        st.free()
        g.close()


def run_members(members, one_graph: bool = False) -> list[dict]:
    """Run the members on the current GPU, concurrently; returns per member the observable rows after
    every step ([nsteps][nvalues], as qnd_run_length_dev) and the final state."""
    runs = prepare(members)
    launch(runs, one_graph)
    out = [{"obs": obs[:, :nv].cpu().numpy(), "psi": st.download()} for g, st, E, obs, nv, _ in runs]
    release(runs)
    return out


def run_sharded(members, dist=None, runner=run_members):
    """This rank's share of the members (partition), then a gather of every member's result on rank 0
    in member order; other ranks get None. Without a process group, all members run here."""
    if dist is None or not dist.is_initialized():
        return runner(members)
    world, rank = dist.get_world_size(), dist.get_rank()
    mine = partition(members, world)[rank]
    res = runner([members[i] for i in mine])
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, res)), gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(members)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
