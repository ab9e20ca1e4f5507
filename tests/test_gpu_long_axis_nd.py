"""GPU parity of axes longer than one pass handles (N > 4096) on grids of two and three dimensions.

The reference takes any NR per axis (parameters.c:72-76 asks only for powers of two) and hands the
grid to one fftw_mpi_plan_dft (meshgrid.c:166-167). The engine transforms such an axis in four steps
in natural order (length-n1 passes along the virtual axis of stride n2 S, the twiddles W_N^{k1 m},
length-n2 passes along stride S, a permutation to natural order) and emulates every pass mode along it
from those transforms and element-wise kernels. Checked against the C oracle (pinned to the
reference): FP64 relative L2 <= 1e-12 on wavefunctions, observables <= 1e-11 relative.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12
CASES = [((8192, 8), (0.1, 0.6)), ((16, 8192), (0.6, 0.1)), ((4, 8192, 4), (0.7, 0.1, 0.7))]


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def cos8_mask(axis, frac=0.1):
    half = np.max(np.abs(axis))
    edge = (1.0 - frac) * half
    m = np.ones_like(axis)
    zone = np.abs(axis) > edge
    m[zone] = np.cos(0.5 * np.pi * (np.abs(axis[zone]) - edge) / (half - edge)).clip(0.0) ** 0.125
    return m


def _pair(shape, dr, integ="BM4", precision="fp64", masked=True):
    from tdse_nd_mpi_b200 import Grid

    dim = len(shape)
    g = Grid(dim, shape, dr, integ, 0.05, precision=precision)
    o = O.OracleCtx(dim, shape, dr, integ, 0.05)
    long_ax = int(np.argmax(shape))
    for ctx in (g, o):
        ctx.set_potential("H_3D")
        ctx.set_cap(0.2, 0.8)
        if masked:
            ctx.set_mask_axis(long_ax, cos8_mask(g.axis_r(long_ax)))
    return g, o


@pytest.mark.parametrize("shape,dr", CASES)
def test_long_axis_nd_length_run_vs_oracle(qnd_lib, shape, dr):
    """Length gauge with CAP and step mask, r- and k-space observables after every step."""
    g, o = _pair(shape, dr)
    dim = len(shape)
    psi0 = O.smooth_state(shape, dr, 1)
    E = np.random.default_rng(2).standard_normal((4, g.s, dim)) * 0.05
    for names in (["norm", "dipole_r"], ["norm", "dipole_r", "dipole_v", "energy", "Lz"]):
        a = psi0.copy()
        want = o.run_length(a, E, names)
        st = g.state(psi0)
        got = g.run_length(st, E, names)
        assert rel(st.download(), a) < TOL
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-13)
    g.close()


@pytest.mark.parametrize("shape,dr", CASES)
def test_long_axis_nd_imag_velocity_transforms_vs_oracle(qnd_lib, shape, dr):
    """Imaginary-time steps, velocity-gauge steps (k-space field phases along the long axis), the
    momentum-space transform and its inverse, energies."""
    g, o = _pair(shape, dr, "BM6", masked=False)
    dim = len(shape)
    psi0 = O.smooth_state(shape, dr, 3)
    a = psi0.copy()
    o.step_imag(a, 3)
    st = g.state(psi0)
    g.integration_step_imag(st, 3)
    assert rel(st.download(), a) < TOL
    A = np.random.default_rng(4).standard_normal((3, g.s, dim)) * 0.25
    a = psi0.copy()
    o.step_velocity(a, A, 3)
    st.upload(psi0)
    g.integration_step_velocity(st, A)
    assert rel(st.download(), a) < TOL
    a = psi0.copy()
    o.to_p(a)
    st.upload(psi0)
    g.to_p(st)
    assert rel(st.download(), a) < TOL
    g.to_r(st)
    assert rel(st.download(), psi0) < TOL
    np.testing.assert_allclose(g.energies(st, 2), o.energies(psi0, 2), rtol=1e-11, atol=1e-13)
    g.close()


def test_long_axis_nd_gram_schmidt_states_vs_oracle(qnd_lib):
    """The imaginary-time driver's state loop (propagate, project, normalise) with a long axis."""
    shape, dr = (8192, 8), (0.1, 0.6)
    g, o = _pair(shape, dr, masked=False)
    for ctx in (g, o):
        ctx.set_cap(0.0, 0.0)
    seeds = [O.seeded_state(shape, 10 + k) for k in range(3)]
    ho = [s.copy() for s in seeds]
    states = [g.state(s) for s in seeds]
    for j in range(3):
        o.imag_state(ho, j, 10)
        g.imag_propagate(states, j, 10)
        assert rel(states[j].download(), ho[j]) < 1e-11
    g.close()


def test_long_axis_nd_graph_replayed_chunks(qnd_lib, monkeypatch):
    """400 steps (chunks of 128 steps: launched directly, captured into a CUDA graph, replayed, and a
    16-step tail) equal the directly launched run bit for bit, and the oracle."""
    shape, dr = (8, 8192), (0.6, 0.1)
    g, o = _pair(shape, dr)
    psi0 = O.smooth_state(shape, dr, 13)
    E = np.random.default_rng(14).standard_normal((400, g.s, 2)) * 0.05
    names = ["norm", "dipole_r"]
    st = g.state(psi0)
    ob_graph = g.run_length(st, E, names)
    psi_graph = st.download()
    monkeypatch.setenv("QND_NO_GRAPH", "1")
    st.upload(psi0)
    ob_direct = g.run_length(st, E, names)
    np.testing.assert_array_equal(ob_graph, ob_direct)
    np.testing.assert_array_equal(psi_graph, st.download())
    monkeypatch.delenv("QND_NO_GRAPH")
    a = psi0.copy()
    want = o.run_length(a, E, names)
    assert rel(psi_graph, a) < 1e-11
    np.testing.assert_allclose(ob_graph, want, rtol=1e-10, atol=1e-13)
    g.close()


def test_long_axis_nd_mixed_precision_tracks_fp64(qnd_lib):
    """Complex64 storage with the same emulated passes: 40 length-gauge steps within 1e-5 of FP64."""
    shape, dr = (8192, 8), (0.1, 0.6)
    psi0 = O.smooth_state(shape, dr, 21)
    E = np.random.default_rng(22).standard_normal((40, 6, 2)) * 0.05
    out = {}
    for prec in ("fp64", "mixed"):
        g, _ = _pair(shape, dr, precision=prec)
        st = g.state(psi0)
        rows = g.run_length(st, E, ["norm", "dipole_r"])
        out[prec] = (rows, st.download())
        g.close()
    assert rel(out["mixed"][1], out["fp64"][1]) < 1e-5
    scale = np.max(np.abs(out["fp64"][0]), axis=0)
    assert np.max(np.abs(out["mixed"][0] - out["fp64"][0]) / scale) < 1e-5
