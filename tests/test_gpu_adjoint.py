"""GPU checks of qnd_adjoint_length (the differentiation extension): the gradient of
J = dNr sum w |psi_T|^2 with respect to every field sample E[k][ia][j] of a length-gauge run.

* against the FP64 CPU adjoint (oracle/adjoint.py, itself pinned to the C oracle's forward run
  and to finite differences): J to 1e-12, the gradient to 5e-10 relative (the gradient sums terms
  that cancel, so it carries the transforms' few-ulp rounding amplified; measured up to 1.8e-10
  in 3-D with BM6), 1-D to 3-D, a long
  1-D axis, CAP and step mask, several checkpoint intervals;
* against central finite differences of the engine's own forward run on a 3-D soft-Coulomb
  case with checkpoints every 50 of 200 steps: 1e-5 relative on 16 random samples;
* through torch.autograd (tdse_nd_mpi_b200.adjoint).
"""
import numpy as np
import pytest

from oracle import adjoint as A
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Grid(qnd_lib):
    from tdse_nd_mpi_b200 import Grid

    return Grid


def _pair(Grid, shape, dr, integ, precision="fp64", masked=True):
    dim = len(shape)
    grid = Grid(dim, shape, dr, integ, 0.05, precision=precision)
    X = np.meshgrid(*[grid.axis_r(j) for j in range(dim)], indexing="ij")
    r2 = sum(x * x for x in X)
    V = -1.0 / np.sqrt(r2 + 0.64)
    rmax = np.sqrt(r2).max()
    Vcap = 0.05 * np.maximum(np.sqrt(r2) - 0.8 * rmax, 0.0) ** 2
    grid.set_potential(V)
    grid.set_vcap(Vcap)
    masks = None
    if masked:
        masks = []
        for j in range(dim):
            r = grid.axis_r(j)
            m = np.where(np.abs(r) > 0.85 * np.abs(r).max(), 0.98, 1.0)
            grid.set_mask_axis(j, m)
            masks.append(m)
    run = A.LengthRun(shape, dr, integ, 0.05, V, Vcap, masks)
    w = (np.sqrt(r2) > 0.5 * rmax).astype(float)
    return grid, run, w


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("shape,dr,integ", [((256,), (0.3,), "BM4"), ((64, 64), (0.4, 0.4), "BM4"),
                                            ((16, 16, 16), (0.6, 0.6, 0.6), "Verlet"), ((8192,), (0.1,), "BM6")])
def test_adjoint_matches_cpu_adjoint(Grid, shape, dr, integ):
    grid, run, w = _pair(Grid, shape, dr, integ)
    psi0 = O.smooth_state(shape, dr, 21)
    E = np.random.default_rng(22).standard_normal((7, grid.s, len(shape))) * 0.05
    J_ref, g_ref = run.adjoint(psi0, E, w)
    st = grid.state(psi0)
    out = grid.state()
    J, g = grid.adjoint_length(st, E, w, checkpoint=3, psiT=out)
    assert abs(J - J_ref) <= 1e-12 * abs(J_ref)
    assert _rel(g, g_ref) < 5e-10
    assert _rel(st.download(), psi0) == 0.0                       # psi0 untouched
    assert _rel(out.download(), run.run(psi0, E)) < 1e-12         # psi(T)


def test_checkpoint_interval_does_not_change_the_gradient(Grid):
    grid, _, w = _pair(Grid, (64, 32), (0.4, 0.5), "BM4")
    psi0 = O.smooth_state((64, 32), (0.4, 0.5), 23)
    E = np.random.default_rng(24).standard_normal((9, grid.s, 2)) * 0.05
    st = grid.state(psi0)
    J1, g1 = grid.adjoint_length(st, E, w, checkpoint=1)
    for K in (4, 9, 100):
        J, g = grid.adjoint_length(st, E, w, checkpoint=K)
        assert abs(J - J1) <= 1e-13 * abs(J1)
        assert _rel(g, g1) < 1e-12


def test_adjoint_matches_finite_differences_3d(Grid):
    """H_3D-style soft-Coulomb 64^3, BM4, 200 steps of an 800 nm field with seeded 1e-3 perturbations,
    J = the norm beyond |r| > 5, checkpoints every 50 steps: the gradient at 16 random samples
    against central differences of the engine's own forward J."""
    shape, dr = (64, 64, 64), (0.3, 0.3, 0.3)
    grid = Grid(3, shape, dr, "BM4", 0.05)
    X = np.meshgrid(*[grid.axis_r(j) for j in range(3)], indexing="ij")
    r = np.sqrt(sum(x * x for x in X))
    grid.set_potential(-1.0 / np.sqrt(r * r + 0.5))
    grid.set_cap(0.05, 1.5)
    w = (r > 5.0).astype(float)
    psi0 = O.smooth_state(shape, dr, 25)
    nsteps = 200
    sub = np.cumsum(np.r_[0.0, grid.as_scaled[1:-1:2] + grid.as_scaled[2::2]])   # sub-step offsets
    t = np.arange(nsteps)[:, None] * 0.05 + grid.as_scaled[0] + sub[None, :]
    base = 0.0534 * np.sin(0.057 * t) * np.sin(np.pi * t / (nsteps * 0.05)) ** 2
    rng = np.random.default_rng(26)
    E = np.zeros((nsteps, grid.s, 3))
    E[:, :, 0] = base * (1.0 + 1e-3 * rng.standard_normal(base.shape))
    st = grid.state(psi0)
    J, g = grid.adjoint_length(st, E, w, checkpoint=50)
    out = grid.state()

    def objective(Ep):
        out.upload(psi0)
        grid.run_length(out, Ep, [])
        return grid.dNr * float(np.sum(w * np.abs(out.download()) ** 2))

    assert objective(E) == pytest.approx(J, rel=1e-12)
    eps = 1e-5
    scale = np.abs(g).max()
    for _ in range(16):
        idx = (int(rng.integers(0, nsteps)), int(rng.integers(0, grid.s)), int(rng.integers(0, 3)))
        Ep, Em = E.copy(), E.copy()
        Ep[idx] += eps
        Em[idx] -= eps
        fd = (objective(Ep) - objective(Em)) / (2 * eps)
        assert abs(fd - g[idx]) <= 1e-5 * max(abs(fd), 1e-3 * scale), (idx, fd, g[idx])


def test_mixed_precision_adjoint_against_fp64(Grid):
    shape, dr = (128, 128), (0.3, 0.3)
    gm, _, w = _pair(Grid, shape, dr, "BM4", precision="mixed")
    gd, _, _ = _pair(Grid, shape, dr, "BM4")
    psi0 = O.smooth_state(shape, dr, 27)
    E = np.random.default_rng(28).standard_normal((20, gm.s, 2)) * 0.05
    Jm, gmix = gm.adjoint_length(gm.state(psi0), E, w, checkpoint=5)
    Jd, gdbl = gd.adjoint_length(gd.state(psi0), E, w, checkpoint=5)
    assert abs(Jm - Jd) <= 1e-5 * abs(Jd)
    assert _rel(gmix, gdbl) < 3e-3   # measured 1.0e-3: the gradient is a small difference of FP32 states


def test_autograd_bridge(Grid):
    import torch

    from tdse_nd_mpi_b200.adjoint import absorbed_weight, length_gauge_objective

    grid, _, _ = _pair(Grid, (64, 64), (0.4, 0.4), "BM4")
    w = absorbed_weight(grid, 6.0)
    psi0 = O.smooth_state((64, 64), (0.4, 0.4), 29)
    st = grid.state(psi0)
    E0 = np.random.default_rng(30).standard_normal((6, grid.s, 2)) * 0.05
    E = torch.tensor(E0, requires_grad=True)
    J = length_gauge_objective(grid, st, E, w, checkpoint=2)
    (2.0 * J).backward()
    J_ref, g_ref = grid.adjoint_length(st, E0, w, checkpoint=2)
    assert float(J.detach()) == J_ref
    np.testing.assert_array_equal(E.grad.numpy(), 2.0 * g_ref)


def _vpair(Grid, shape, dr, integ, precision="fp64", masked=True):
    grid, run, w = _pair(Grid, shape, dr, integ, precision, masked)
    masks = None
    if masked:
        masks = [np.where(np.abs(grid.axis_r(j)) > 0.85 * np.abs(grid.axis_r(j)).max(), 0.98, 1.0)
                 for j in range(len(shape))]
    return grid, A.VelocityRun(shape, dr, integ, 0.05, run.V, run.Vcap, masks), w


@pytest.mark.parametrize("shape,dr,integ", [((256,), (0.3,), "BM4"), ((64, 64), (0.4, 0.4), "BM4"),
                                            ((16, 16, 16), (0.6, 0.6, 0.6), "Verlet"), ((8192,), (0.1,), "BM6")])
def test_velocity_adjoint_matches_cpu_adjoint(Grid, shape, dr, integ):
    """qnd_adjoint_velocity (dJ/dA of a velocity-gauge run) against the FP64 CPU adjoint."""
    grid, run, w = _vpair(Grid, shape, dr, integ)
    psi0 = O.smooth_state(shape, dr, 31)
    Avec = np.random.default_rng(32).standard_normal((7, grid.s, len(shape))) * 0.3
    J_ref, g_ref = run.adjoint(psi0, Avec, w)
    st = grid.state(psi0)
    out = grid.state()
    J, g = grid.adjoint_velocity(st, Avec, w, checkpoint=3, psiT=out)
    assert abs(J - J_ref) <= 1e-11 * abs(J_ref)
    assert _rel(g, g_ref) < 5e-10
    assert _rel(out.download(), run.run(psi0, Avec)) < 1e-12


def test_velocity_adjoint_matches_finite_differences(Grid):
    """2-D 128^2 BM4 with the step mask, 60 steps, checkpoints every 16: dJ/dA at 12 random samples
    against central differences of the engine's own forward run (qnd_run_velocity)."""
    shape, dr = (128, 128), (0.3, 0.3)
    grid, _, w = _vpair(Grid, shape, dr, "BM4")
    psi0 = O.smooth_state(shape, dr, 33)
    rng = np.random.default_rng(34)
    Avec = rng.standard_normal((60, grid.s, 2)) * 0.3
    J, g = grid.adjoint_velocity(grid.state(psi0), Avec, w, checkpoint=16)
    out = grid.state()

    def objective(Ap):
        out.upload(psi0)
        grid.run_velocity(out, Ap)
        return grid.dNr * float(np.sum(w * np.abs(out.download()) ** 2))

    assert objective(Avec) == pytest.approx(J, rel=1e-12)
    eps = 1e-5
    scale = np.abs(g).max()
    for _ in range(12):
        idx = (int(rng.integers(0, 60)), int(rng.integers(0, grid.s)), int(rng.integers(0, 2)))
        Ap, Am = Avec.copy(), Avec.copy()
        Ap[idx] += eps
        Am[idx] -= eps
        fd = (objective(Ap) - objective(Am)) / (2 * eps)
        assert abs(fd - g[idx]) <= 1e-5 * max(abs(fd), 1e-3 * scale), (idx, fd, g[idx])


def test_velocity_autograd_bridge(Grid):
    import torch

    from tdse_nd_mpi_b200.adjoint import absorbed_weight, velocity_gauge_objective

    grid, _, _ = _vpair(Grid, (64, 64), (0.4, 0.4), "BM4")
    w = absorbed_weight(grid, 6.0)
    st = grid.state(O.smooth_state((64, 64), (0.4, 0.4), 35))
    A0 = np.random.default_rng(36).standard_normal((5, grid.s, 2)) * 0.3
    Avec = torch.tensor(A0, requires_grad=True)
    J = velocity_gauge_objective(grid, st, Avec, w, checkpoint=2)
    J.backward()
    J_ref, g_ref = grid.adjoint_velocity(st, A0, w, checkpoint=2)
    assert float(J.detach()) == J_ref
    np.testing.assert_array_equal(Avec.grad.numpy(), g_ref)
