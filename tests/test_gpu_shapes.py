"""Every compiled tile shape of the 1024-point passes against the oracle.

The tile-shape autotuner picks one of several compiled shapes per pass geometry (the default 2-line
CTAs, 1-line CTAs, 4-line CTAs, and 7-line CTAs with one CTA per SM). Each shape is forced here
(QND_SHAPE) on a 1024 x 1024 BM4 length-gauge run with CAP and r- and k-space observables every
step, and must match the oracle (the C restatement pinned to the reference) to 1e-12 on the state
and 1e-11 on the rows; the mixed-precision run of each shape must stay within 1e-5 of the oracle.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [0, 1, 2, 3]
N, DR, STEPS = 1024, 0.2, 4
NAMES = ["norm", "dipole_r", "dipole_v", "energy"]


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.fixture(scope="module")
def reference_run():
    o = O.OracleCtx(2, (N, N), (DR, DR), "BM4", 0.05)
    o.set_potential("H_2D")
    o.set_cap(0.05, 10.0)
    psi0 = O.smooth_state((N, N), (DR, DR), 31)
    E = np.random.default_rng(32).standard_normal((STEPS, 6, 2)) * 0.05
    a = psi0.copy()
    rows = o.run_length(a, E, NAMES)
    return psi0, E, rows, a


def _run(precision, psi0, E):
    from tdse_nd_mpi_b200 import Grid

    g = Grid(2, (N, N), (DR, DR), "BM4", 0.05, precision=precision)
    g.set_potential("H_2D")
    g.set_cap(0.05, 10.0)
    st = g.state(psi0)
    rows = g.run_length(st, E, NAMES)
    psi = st.download()
    g.close()
    return rows, psi


@pytest.mark.parametrize("shape", SHAPES)
def test_forced_shape_matches_oracle(qnd_lib, reference_run, monkeypatch, shape):
    psi0, E, want_rows, want_psi = reference_run
    monkeypatch.setenv("QND_SHAPE", str(shape))
    rows, psi = _run("fp64", psi0, E)
    assert rel(psi, want_psi) < 1e-12
    np.testing.assert_allclose(rows, want_rows, rtol=1e-11, atol=1e-13)
    rows_m, psi_m = _run("mixed", psi0, E)
    assert rel(psi_m, want_psi) < 1e-5
    scale = np.max(np.abs(want_rows), axis=0)
    assert np.max(np.abs(rows_m - want_rows) / scale) < 1e-5
