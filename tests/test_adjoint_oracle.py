"""The FP64 CPU adjoint (oracle/adjoint.py), checked before it checks the GPU:

* its forward run equals the C oracle's length-gauge run (pinned to the reference's
  Integration_step_length) with a CAP and the step mask, to 1e-12;
* its gradient equals central finite differences of its own objective.
"""
import numpy as np
import pytest

from oracle import adjoint as A
from oracle import oracle as O


def _setup(shape, dr, integ, dt, seed, masked=True):
    o = O.OracleCtx(len(shape), shape, dr, integ, dt)
    rs, _ = O.grid_axes(shape, dr)
    X = np.meshgrid(*rs, indexing="ij")
    r2 = sum(x * x for x in X)
    V = -1.0 / np.sqrt(r2 + 0.64)
    o.set_vpot(V)
    o.set_cap(0.05, 2.0)
    vcap = o.tables()[3]
    masks = None
    if masked:
        masks = []
        for j, r in enumerate(rs):
            m = np.where(np.abs(r) > 0.8 * np.abs(r).max(), 0.97, 1.0)
            o.set_mask_axis(j, m)
            masks.append(m)
    run = A.LengthRun(shape, dr, integ, dt, V, vcap, masks)
    psi0 = O.smooth_state(shape, dr, seed)
    E = np.random.default_rng(seed + 1).standard_normal((5, run.s, len(shape))) * 0.05
    return o, run, psi0, E, X


@pytest.mark.parametrize("shape,dr,integ", [((64,), (0.3,), "BM4"), ((32, 32), (0.4, 0.4), "BM6"),
                                            ((8, 8, 16), (0.6, 0.6, 0.5), "Verlet")])
def test_adjoint_restatement_forward_matches_oracle(shape, dr, integ):
    o, run, psi0, E, _ = _setup(shape, dr, integ, 0.05, 3)
    a = psi0.copy()
    o.run_length(a, E, [])
    got = run.run(psi0, E)
    assert np.linalg.norm(got - a) / np.linalg.norm(a) < 1e-12


@pytest.mark.parametrize("shape,dr,integ", [((64,), (0.3,), "BM4"), ((16, 16), (0.5, 0.5), "RKN4")])
def test_adjoint_restatement_matches_finite_differences(shape, dr, integ):
    _, run, psi0, E, X = _setup(shape, dr, integ, 0.05, 5)
    w = (np.sqrt(sum(x * x for x in X)) > 3.0).astype(float)
    J, grad = run.adjoint(psi0, E, w)
    assert J == pytest.approx(run.objective(psi0, E, w), rel=1e-14)
    rng = np.random.default_rng(7)
    eps = 1e-4
    for _ in range(6):
        idx = tuple(int(rng.integers(0, n)) for n in E.shape)
        Ep, Em = E.copy(), E.copy()
        Ep[idx] += eps
        Em[idx] -= eps
        fd = (run.objective(psi0, Ep, w) - run.objective(psi0, Em, w)) / (2 * eps)
        assert abs(fd - grad[idx]) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(grad).max())


@pytest.mark.parametrize("shape,dr,integ", [((64,), (0.3,), "BM4"), ((32, 32), (0.4, 0.4), "BM6"),
                                            ((8, 8, 16), (0.6, 0.6, 0.5), "Verlet")])
def test_velocity_adjoint_restatement_forward_matches_oracle(shape, dr, integ):
    o, run, psi0, E, _ = _setup(shape, dr, integ, 0.05, 3, masked=False)
    vrun = A.VelocityRun(shape, dr, integ, 0.05, run.V, run.Vcap, None)
    Avec = np.random.default_rng(31).standard_normal((4, vrun.s, len(shape))) * 0.3
    a = psi0.copy()
    o.step_velocity(a, Avec, 4)
    got = vrun.run(psi0, Avec)
    assert np.linalg.norm(got - a) / np.linalg.norm(a) < 1e-12


@pytest.mark.parametrize("shape,dr,integ", [((64,), (0.3,), "BM4"), ((16, 16), (0.5, 0.5), "RKN4")])
def test_velocity_adjoint_restatement_matches_finite_differences(shape, dr, integ):
    _, run, psi0, _, X = _setup(shape, dr, integ, 0.05, 5)
    rs, _ = O.grid_axes(shape, dr)
    masks = [np.where(np.abs(r) > 0.8 * np.abs(r).max(), 0.97, 1.0) for r in rs]
    vrun = A.VelocityRun(shape, dr, integ, 0.05, run.V, run.Vcap, masks)
    w = (np.sqrt(sum(x * x for x in X)) > 3.0).astype(float)
    Avec = np.random.default_rng(32).standard_normal((4, vrun.s, len(shape))) * 0.3
    J, grad = vrun.adjoint(psi0, Avec, w)
    assert J == pytest.approx(vrun.objective(psi0, Avec, w), rel=1e-14)
    rng = np.random.default_rng(8)
    eps = 1e-4
    for _ in range(6):
        idx = tuple(int(rng.integers(0, n)) for n in Avec.shape)
        Ap, Am = Avec.copy(), Avec.copy()
        Ap[idx] += eps
        Am[idx] -= eps
        fd = (vrun.objective(psi0, Ap, w) - vrun.objective(psi0, Am, w)) / (2 * eps)
        assert abs(fd - grad[idx]) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(grad).max())
