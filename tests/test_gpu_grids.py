"""Grids beyond three dimensions: the reference reads DIMENSION from its parameter file and
allocates per dimension (parameters.c:46-48), and fftw_mpi_plan_dft takes any rank
(meshgrid.c:166-167). The engine takes 1 to 6 dimensions; here 4-D and 5-D grids against the
oracle (itself pinned bit for bit to the reference in 4-D by tests/test_oracle.py): real-time steps
in both gauges with every observable, imaginary time with Gram-Schmidt, energies.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("shape,dr", [((4, 8, 8, 16), (0.6, 0.5, 0.45, 0.4)),
                                      ((4, 4, 8, 8, 8), (0.7, 0.6, 0.5, 0.5, 0.45))])
def test_high_dimension_runs_vs_oracle(qnd_lib, shape, dr):
    from tdse_nd_mpi_b200 import Grid

    dim = len(shape)
    g = Grid(dim, shape, dr, "BM4", 0.05)
    g.set_potential("H_3D")
    g.set_cap(0.2, 0.8)
    o = O.OracleCtx(dim, shape, dr, "BM4", 0.05)
    o.set_potential("H_3D")
    o.set_cap(0.2, 0.8)
    psi0 = O.seeded_state(shape, 3)
    E = np.random.default_rng(6).standard_normal((5, g.s, dim)) * 0.05
    names = ["norm", "dipole_r", "dipole_v", "energy", "Lz"]
    a = psi0.copy()
    want = o.run_length(a, E, names)
    st = g.state(psi0)
    got = g.run_length(st, E, names)
    assert rel(st.download(), a) < 1e-12
    np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-13)

    a = psi0.copy()
    o.step_velocity(a, E, 5)
    st = g.state(psi0)
    g.integration_step_velocity(st, E)
    assert rel(st.download(), a) < 1e-12

    states_o = [O.seeded_state(shape, 10 + k) for k in range(3)]
    states_g = [g.state(p) for p in states_o]
    for j in range(3):
        for _ in range(4):
            o.step_imag(states_o[j], 1)
            o.gram_schmidt(j, states_o)
        g.imag_propagate(states_g, j, 4)
    for sg, so in zip(states_g, states_o):
        assert rel(sg.download(), so) < 1e-12
        np.testing.assert_allclose(g.energies(sg, 2), o.energies(so, 2), rtol=1e-11)
