"""Sweeps of independent members (tdse_nd_mpi_b200/batch.py): the balanced partition and the
rank-0 gather on two gloo ranks on the CPU; on the GPU, concurrent members against one-by-one runs."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tdse_nd_mpi_b200.batch import Member, partition, run_sharded

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _member(shape, seed, integ="BM4", nsteps=4):
    rng = np.random.default_rng(seed)
    dim = len(shape)
    s = {"BM4": 6, "Verlet": 1}[integ]
    psi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return Member(shape=shape, dr=(0.3,) * dim, integrator=integ, dt=0.05, potential="H_2D" if dim == 2 else "H_1D",
                  field=rng.standard_normal((nsteps, s, dim)) * 0.05, psi0=psi / np.linalg.norm(psi), cap=(0.1, 2.0))


def test_partition_balances_bytes_and_covers_every_member():
    # the sweep configuration's mix: 32 x 256^2, 48 x 512^2, 16 x 1024^2
    members = [_member((256, 256), 0)] * 32 + [_member((512, 512), 0)] * 48 + [_member((1024, 1024), 0)] * 16
    for world in (1, 2, 4, 8):
        parts = partition(members, world)
        assert sorted(i for p in parts for i in p) == list(range(len(members)))
        loads = [sum(members[i].state_bytes for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(m.state_bytes for m in members)
        assert parts == partition(members, world)          # the same on every rank


def _fake_runner(ms):
    return [{"obs": np.full((1, 1), float(np.prod(m.shape))), "psi": None} for m in ms]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        members = [_member((n, n), i) for i, n in enumerate((8, 16, 32, 16, 8))]
        out = run_sharded(members, dist, runner=_fake_runner)
        q.put((rank, None if out is None else [float(r["obs"][0, 0]) for r in out]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_member_in_order():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    assert got[0] == [64.0, 256.0, 1024.0, 256.0, 64.0]


@pytest.mark.gpu
def test_concurrent_members_match_one_by_one(qnd_lib):
    from tdse_nd_mpi_b200 import Grid
    from tdse_nd_mpi_b200.batch import run_members
    import torch

    members = [_member((128, 128), 1), _member((256, 256), 2, "Verlet"), _member((64, 128), 3), _member((1024,), 4)]
    together = run_members(members)
    for m, r in zip(members, together):
        g = Grid(len(m.shape), m.shape, m.dr, m.integrator, m.dt)
        g.set_potential(m.potential)
        g.set_cap(*m.cap)
        st = g.state(m.psi0)
        E = torch.tensor(m.field, device="cuda")
        obs = torch.zeros((E.shape[0], g.nvalues(list(m.names))), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        g.run_length_dev(st, E, E.shape[0], list(m.names), obs)
        g.synchronize()
        np.testing.assert_array_equal(obs.cpu().numpy(), r["obs"])
        np.testing.assert_array_equal(st.download(), r["psi"])
        g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_graph_sweep_matches_members_alone(qnd_lib, precision, monkeypatch):
    """qnd_run_length_batch over uneven grids, Verlet and BM4 members, 1-D and 2-D, 434 steps
    (chunks: direct, captured, replayed, a shorter direct one): every member's rows and final state
    equal its own run_length_dev, bit for bit; and equal the batch run with the graph switched off."""
    import dataclasses

    from tdse_nd_mpi_b200.batch import run_members

    def long_member(shape, seed, integ="BM4"):
        m = _member(shape, seed, integ)
        rng = np.random.default_rng(100 + seed)
        s = 1 if integ == "Verlet" else 6
        return dataclasses.replace(m, field=rng.standard_normal((434, s, len(shape))) * 0.05, precision=precision)

    members = [long_member((64, 64), 11), long_member((128, 64), 12, "Verlet"), long_member((32, 32), 13),
               long_member((2048,), 14, "Verlet")]
    together = run_members(members, one_graph=True)
    alone = run_members(members, one_graph=False)
    for a, b in zip(together, alone):
        np.testing.assert_array_equal(a["obs"], b["obs"])
        np.testing.assert_array_equal(a["psi"], b["psi"])
    monkeypatch.setenv("QND_NO_GRAPH", "1")
    direct = run_members(members, one_graph=True)
    for a, b in zip(together, direct):
        np.testing.assert_array_equal(a["obs"], b["obs"])
        np.testing.assert_array_equal(a["psi"], b["psi"])


@pytest.mark.gpu
def test_contexts_on_several_host_threads_match_one_thread(qnd_lib):
    """Different contexts driven from different host threads at once (the C calls release the
    interpreter lock, so they overlap): the same results as one thread running them in turn."""
    import threading

    from tdse_nd_mpi_b200.batch import run_members

    members = [_member((128, 128), 21), _member((256,), 22, "Verlet"), _member((64, 64, 32), 23), _member((8192,), 24)]
    alone = run_members(members)
    got = [None] * len(members)

    def work(i):
        got[i] = run_members([members[i]])[0]

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(members))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    for a, b in zip(alone, got):
        np.testing.assert_array_equal(a["obs"], b["obs"])
        np.testing.assert_array_equal(a["psi"], b["psi"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_sweep_matches_members_alone(qnd_lib, precision, monkeypatch):
    """qnd_run_length_sweep (one persistent kernel over every member's passes) over uneven grids,
    square and not, BM4 and Verlet members, 300 steps (chunks of 128, 128 and 44 steps): every
    member's rows and final state equal its own run_length_dev with direct launches and the default
    tile shapes, bit for bit."""
    import dataclasses

    from tdse_nd_mpi_b200.batch import run_members

    def sweep_member(shape, seed, integ="BM4"):
        m = _member(shape, seed, integ)
        rng = np.random.default_rng(200 + seed)
        s = 1 if integ == "Verlet" else 6
        return dataclasses.replace(m, field=rng.standard_normal((300, s, len(shape))) * 0.05, precision=precision)

    members = [sweep_member((128, 128), 31), sweep_member((256, 128), 32, "Verlet"), sweep_member((256, 256), 33),
               sweep_member((128, 512), 34, "Verlet"), sweep_member((512, 512), 35)]
    together = run_members(members, one_graph="persistent")
    # the members alone with direct launches and the default tile shapes, which the sweep kernel holds
    # (a tuned shape groups a reduction's partial sums differently: the same values to rounding)
    monkeypatch.setenv("QND_NO_GRAPH", "1")
    monkeypatch.setenv("QND_SHAPE", "0")
    alone = run_members(members, one_graph=False)
    for a, b in zip(together, alone):
        np.testing.assert_array_equal(a["obs"], b["obs"])
        np.testing.assert_array_equal(a["psi"], b["psi"])


@pytest.mark.gpu
def test_persistent_sweep_refuses_what_it_does_not_hold(qnd_lib):
    """Axis lengths outside 128..1024 and mixed precisions give QND_EUNSUPPORTED (no launch)."""
    from tdse_nd_mpi_b200 import QndError
    from tdse_nd_mpi_b200.batch import launch, prepare, release

    for members in ([_member((64, 128), 41)], [_member((128, 128), 42), _member((128, 128), 43)]):
        if len(members) == 2:
            import dataclasses
            members[1] = dataclasses.replace(members[1], precision="mixed")
        runs = prepare(members)
        with pytest.raises(QndError) as ei:
            launch(runs, "persistent")
        assert ei.value.code == 5
        release(runs)
