"""GPU parity of 1-D axes longer than one pass handles (N > 4096, up to 2^24).

The engine transforms such an axis in four steps over a virtual n1 x 4096 grid: length-n1
passes along the strided virtual axis, the twiddles W_N^{k1 n2}, length-4096 passes along the
contiguous one, with the k-space tables stored in the resulting slot order. The reference's own
example params.real runs the 1-D grid at NR = 262144, which needs this path.

Checked against the C oracle (pinned to the reference): FP64 relative L2 <= 1e-12 on
wavefunctions, observables <= 1e-11 relative; mixed precision within the bounds of the 2-D test;
at 2^22 and 2^24 points through size-independent properties (unitarity, reversibility, exact
round trips).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12
LONG = [(8192, 0.1), (65536, 0.05), (262144, 0.05)]


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.fixture(scope="module")
def Grid(qnd_lib):
    from tdse_nd_mpi_b200 import Grid

    return Grid


def soft_coulomb(x, a):
    V = -1.0 / np.sqrt(x * x + a)
    return V, x / (x * x + a) ** 1.5


def cos8_mask(axis, frac=0.1):
    half = np.max(np.abs(axis))
    edge = (1.0 - frac) * half
    m = np.ones_like(axis)
    zone = np.abs(axis) > edge
    m[zone] = np.cos(0.5 * np.pi * (np.abs(axis[zone]) - edge) / (half - edge)).clip(0.0) ** 0.125
    return m


def _pair(Grid, n, dr, integ="BM4", masked=True, precision="fp64"):
    grid = Grid(1, (n,), (dr,), integ, 0.05, precision=precision)
    V, g = soft_coulomb(grid.axis_r(0), 2.0)
    o = O.OracleCtx(1, (n,), (dr,), integ, 0.05)
    grid.set_potential(V)
    o.set_vpot(V)
    for ctx in (grid, o):
        ctx.set_cap(0.05, 2.0)
        ctx.set_gradv(0, g)
        if masked:
            ctx.set_mask_axis(0, cos8_mask(grid.axis_r(0)))
    return grid, o


@pytest.mark.parametrize("n,dr", LONG)
def test_long_axis_masked_length_run_vs_oracle(Grid, n, dr):
    """Length gauge with CAP, step mask and observables each step: r-space observables in one
    chunk chain, then k-space observables (dipole_v, energy) evaluated per step."""
    grid, o = _pair(Grid, n, dr)
    psi0 = O.smooth_state((n,), (dr,), 1)
    E = np.random.default_rng(2).standard_normal((4, grid.s, 1)) * 0.05
    for names in (["norm", "dipole_r", "accel"], ["norm", "dipole_v", "energy", "accel"]):
        a = psi0.copy()
        ob_o = o.run_length(a, E, names)
        st = grid.state(psi0)
        ob_g = grid.run_length(st, E, names)
        assert rel(st.download(), a) < TOL
        np.testing.assert_allclose(ob_g, ob_o, rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("n,dr", LONG[:2])
def test_long_axis_imag_velocity_length_steps_vs_oracle(Grid, n, dr):
    """Multi-step imaginary-time, velocity-gauge (k-space field phases in slot order) and p-space
    length-gauge calls."""
    grid, o = _pair(Grid, n, dr, "BM6", masked=False)
    psi0 = O.smooth_state((n,), (dr,), 3)
    steps = 3
    F = np.random.default_rng(4).standard_normal((steps, grid.s, 1)) * 0.05
    a = psi0.copy()
    o.step_imag(a, steps)
    st = grid.state(psi0)
    grid.integration_step_imag(st, steps)
    assert rel(st.download(), a) < TOL
    a = psi0.copy()
    o.step_velocity(a, F * 5, steps)
    st.upload(psi0)
    grid.integration_step_velocity(st, F * 5)
    assert rel(st.download(), a) < TOL
    a = psi0.copy()
    o.to_p(a)
    o.step_length(a, F, steps)
    st.upload(psi0)
    grid.to_p(st)
    grid.integration_step_length(st, F)
    assert rel(st.download(), a) < TOL


@pytest.mark.parametrize("n,dr", LONG[:2])
def test_long_axis_velocity_run_with_observables_vs_oracle(Grid, n, dr):
    grid, o = _pair(Grid, n, dr)
    psi0 = O.smooth_state((n,), (dr,), 5)
    steps = 3
    A = np.random.default_rng(6).standard_normal((steps, grid.s, 1)) * 0.3
    alpha = np.random.default_rng(7).standard_normal((steps, 1)) * 0.2
    names = ["norm", "dipole_r", "dipole_v", "energy"]
    a = psi0.copy()
    ob_o = o.run_velocity(a, A, alpha, names)
    st = grid.state(psi0)
    ob_g = grid.run_velocity(st, A, alpha, names)
    assert rel(st.download(), a) < TOL
    np.testing.assert_allclose(ob_g, ob_o, rtol=1e-11, atol=1e-13)


def test_long_axis_unitary_conversions_and_observables(Grid):
    n, dr = 65536, 0.05
    grid, o = _pair(Grid, n, dr, masked=False)
    psi0 = O.seeded_state((n,), 8)
    a = psi0.copy()
    o.to_p(a)
    st = grid.state(psi0)
    grid.to_p(st)
    assert rel(st.download(), a) < TOL
    grid.to_r(st)
    assert rel(st.download(), psi0) < TOL
    psi = O.smooth_state((n,), (dr,), 9) * np.exp(0.3j * grid.axis_r(0))
    st.upload(psi)
    names = ["norm", "dipole_r", "accel", "dipole_v", "energy", "Lz"]
    alpha = np.array([0.37])
    np.testing.assert_allclose(grid.observables(st, names, alpha), o.observables(psi, names, alpha), rtol=1e-11,
                               atol=1e-13)
    np.testing.assert_allclose(grid.energies(st, 2), o.energies(psi, 2), rtol=1e-11, atol=1e-13)


def test_long_axis_gram_schmidt_states_vs_oracle(Grid):
    """The imaginary-time driver's state loop (propagate, project, normalise) on a long axis."""
    n, dr = 8192, 0.1
    grid, o = _pair(Grid, n, dr, masked=False)
    grid.set_cap(0.0, 0.0)
    o.set_cap(0.0, 0.0)
    seeds = [O.seeded_state((n,), 10 + k) for k in range(3)]
    ho = [s.copy() for s in seeds]
    states = [grid.state(s) for s in seeds]
    for j in range(3):
        o.imag_state(ho, j, 20)
        grid.imag_propagate(states, j, 20)
        assert rel(states[j].download(), ho[j]) < 1e-11


def test_long_axis_graph_replayed_chunks(Grid, monkeypatch):
    """300 steps (three chunks: direct, captured, replayed) equal the directly launched run and
    the oracle."""
    n, dr = 8192, 0.1
    grid, o = _pair(Grid, n, dr)
    psi0 = O.smooth_state((n,), (dr,), 13)
    E = np.random.default_rng(14).standard_normal((300, grid.s, 1)) * 0.05
    names = ["norm", "dipole_r", "accel"]
    st = grid.state(psi0)
    ob_graph = grid.run_length(st, E, names)
    psi_graph = st.download()
    monkeypatch.setenv("QND_NO_GRAPH", "1")
    st.upload(psi0)
    ob_direct = grid.run_length(st, E, names)
    np.testing.assert_array_equal(ob_graph, ob_direct)
    np.testing.assert_array_equal(psi_graph, st.download())
    monkeypatch.delenv("QND_NO_GRAPH")
    a = psi0.copy()
    ob_o = o.run_length(a, E, names)
    assert rel(psi_graph, a) < 1e-11
    np.testing.assert_allclose(ob_graph, ob_o, rtol=1e-10, atol=1e-13)


def test_long_axis_final_spectra_vs_reference(Grid):
    n, dr = 65536, 0.05
    grid = Grid(1, (n,), (dr,), "BM4", 0.05)
    grid.set_potential("H_1D")
    psi = O.smooth_state((n,), (dr,), 16) * np.exp(1j * 0.7 * O.seeded_state((n,), 17).real)
    rmask, prmax, de, ne = (100.0, 400.0), (3.0,), 0.02, 120
    if O.ref_available():
        out = O.RefCtx(1, (n,), (dr,), "BM4", 0.05, potential="H_1D").final_observables(psi, rmask, prmax, de, ne)
        ped_ref, (head, data) = out["PED"][:, 1], out["PMD"]
        counts_ref = [int(v) for v in head["NPR"]]
    else:
        ped_ref, counts_ref, data = O.final_spectra_numpy(psi, (dr,), rmask, prmax, de, ne)
    ped, counts, pmd = grid.final_spectra(grid.state(psi), rmask, prmax, de, ne)
    np.testing.assert_allclose(ped, ped_ref, rtol=0, atol=1e-11 * np.max(np.abs(ped_ref)))
    assert counts == list(counts_ref)
    dens = data[:, 0]
    np.testing.assert_allclose(pmd[:, 0], dens, rtol=0, atol=1e-12 * dens.max())
    live = dens > 1e-10 * dens.max()
    assert np.max(np.abs(np.angle(np.exp(1j * (pmd[live, 1] - data[live, 1]))))) < 1e-8


def test_long_axis_mixed_precision_error_bound(Grid):
    n, dr = 65536, 0.05
    gm, o = _pair(Grid, n, dr, masked=False, precision="mixed")
    gm.set_cap(0.0, 0.0)
    o.set_cap(0.0, 0.0)
    psi0 = O.smooth_state((n,), (dr,), 18)
    E = np.random.default_rng(19).standard_normal((10, gm.s, 1)) * 0.05
    names = ["norm", "dipole_r", "accel"]
    a = psi0.copy()
    ob_o = o.run_length(a, E, names)
    st = gm.state(psi0)
    ob_m = gm.run_length(st, E, names)
    assert rel(st.download(), a) < 2e-5
    scale = np.maximum(np.abs(ob_o), 1e-3)
    assert np.max(np.abs(ob_m - ob_o) / scale) < 5e-6


@pytest.mark.parametrize("n", [1 << 22, 1 << 24])
def test_long_axis_full_length_properties(Grid, n):
    """Beyond the oracle's quick sizes: the unitary round trip r -> p -> r is exact to rounding,
    and without a CAP the length-gauge steps conserve the norm and run backwards to the start."""
    dr = 0.02
    grid = Grid(1, (n,), (dr,), "BM4", 0.05)
    V, _ = soft_coulomb(grid.axis_r(0), 2.0)
    grid.set_potential(V)
    psi0 = O.smooth_state((n,), (dr,), 20)
    st = grid.state(psi0)
    grid.to_p(st)
    grid.to_r(st)
    assert rel(st.download(), psi0) < 1e-13
    if n > 1 << 22:
        return
    E = np.full((6, grid.s, 1), 0.02)
    obs = grid.run_length(st, E, ["norm"])
    assert np.max(np.abs(obs[:, 0] / obs[0, 0] - 1.0)) < 1e-12
    back = Grid(1, (n,), (dr,), "BM4", -0.05)
    back.set_potential(V)
    back.run_length(st.ptr, E[::-1], [])
    back.synchronize()
    assert rel(st.download(), psi0) < 1e-11
