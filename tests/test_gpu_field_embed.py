"""GPU checks of the two set-up steps the engine runs on the device:

* qnd_field_samples: E and A at the integrator's sub-step times and A at the step starts
  (Initialize_field_vectors, integrators.c:74-101; Field_vectors, parameters.c:899-949),
  against the reference's own functions compiled from its sources (the restatement when the
  reference is not built), every envelope, 1-D to 3-D, several integrators;
* qnd_state_embed: the centring and superposition of Read_wavefunction_MPI
  (io_functions.c:292-459) onto larger and smaller grids, against numpy.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Grid(qnd_lib):
    from tdse_nd_mpi_b200 import Grid

    return Grid


MODES = [
    {"intensity": 1e14, "lambda": 800.0, "ellipticity": 0.0, "cep": 0.3, "delay": 0.0, "duration": 60.0,
     "envelope": "cos2"},
    {"intensity": 2e13, "lambda": 400.0, "ellipticity": 0.5, "cep": 1.1, "delay": 7.5, "duration": 45.0,
     "envelope": "trapz"},
    {"intensity": 5e12, "lambda": 1300.0, "ellipticity": -0.2, "cep": 2.0, "delay": 3.0, "duration": 50.0,
     "envelope": "cos4"},
    {"intensity": 1e12, "lambda": 600.0, "ellipticity": 1.0, "cep": 0.0, "delay": 0.0, "duration": 10.0,
     "envelope": "constant"},
]


@pytest.mark.parametrize("dim,integ", [(1, "BM4"), (2, "BM6"), (2, "Verlet"), (3, "RKN4")])
def test_field_samples_match_reference(Grid, dim, integ):
    dt, T = 0.1, 70.0
    E_ref, A_ref, t_ref = O.field(dim, MODES, integ, dt, T, use_ref=O.ref_available())
    nt = E_ref.shape[0]
    grid = Grid(dim, (8,) * dim, (0.5,) * dim, integ, dt)
    E, A, alpha = grid.field_samples(MODES, nt)
    for got, ref in ((E, E_ref), (A, A_ref)):
        np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-15 * np.abs(ref).max())
    al_ref = np.array([O.field_at(dim, MODES, i * dt)[0] for i in range(nt)])
    np.testing.assert_allclose(alpha, al_ref, rtol=1e-13, atol=1e-15 * np.abs(al_ref).max())


def test_field_samples_into_device_buffers(Grid):
    import torch

    dt, T = 0.05, 40.0
    E_ref, A_ref, _ = O.field(2, MODES[:2], "BM4", dt, T)
    nt = E_ref.shape[0]
    grid = Grid(2, (8, 8), (0.5, 0.5), "BM4", dt)
    E = torch.zeros((nt, grid.s, 2), dtype=torch.float64, device="cuda")
    A = torch.zeros_like(E)
    torch.cuda.synchronize()
    grid.field_samples_dev(MODES[:2], nt, E, A, None)
    grid.synchronize()
    np.testing.assert_allclose(E.cpu().numpy(), E_ref, rtol=1e-13, atol=1e-15 * np.abs(E_ref).max())
    np.testing.assert_allclose(A.cpu().numpy(), A_ref, rtol=1e-13, atol=1e-15 * np.abs(A_ref).max())


def test_field_samples_reject_unknown_envelope(Grid, qnd_lib):
    from tdse_nd_mpi_b200 import QndError

    grid = Grid(1, (8,), (0.5,), "BM4", 0.1)
    with pytest.raises(ValueError):
        grid.field_samples([dict(MODES[0], envelope="gauss")], 4)
    arr = grid._modes(MODES[:1])
    arr[0].envelope = 9
    E = np.zeros(4 * grid.s)
    rc = qnd_lib.qnd_field_samples(grid.h, 1, arr, 4, E.ctypes.data, None, None, 0)
    assert rc == 1 and b"envelope" in qnd_lib.qnd_last_error()
    with pytest.raises(QndError):
        grid.field_samples(MODES * 5, 4)  # 20 modes > 16


def _embed_numpy(shape, srcs, coeffs):
    out = np.zeros(shape, dtype=np.complex128)
    for src, c in zip(srcs, coeffs):
        dst_sl, src_sl = [], []
        for n, m in zip(shape, src.shape):
            off = int((n - m) / 2)  # C division toward zero (all sizes here are even)
            lo, hi = max(0, off), min(n, off + m)
            dst_sl.append(slice(lo, hi))
            src_sl.append(slice(lo - off, hi - off))
        out[tuple(dst_sl)] += c * src[tuple(src_sl)]
    return out


@pytest.mark.parametrize("shape,src_shape", [((256,), (64,)), ((32,), (128,)), ((64, 32), (32, 64)),
                                             ((16, 8, 32), (8, 16, 16))])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_state_embed_centres_and_superposes(Grid, shape, src_shape, precision):
    grid = Grid(len(shape), shape, (0.3,) * len(shape), "BM4", 0.05, precision=precision)
    srcs = [O.seeded_state(src_shape, 30 + k) for k in range(3)]
    coeffs = [0.6 + 0.1j, -0.3j, 0.25]
    st = grid.state(O.seeded_state(shape, 40))   # overwritten by the first (non-accumulating) call
    for k, (src, c) in enumerate(zip(srcs, coeffs)):
        grid.embed(st, src, c, accumulate=k > 0)
    ref = _embed_numpy(shape, srcs, coeffs)
    got = st.download()
    tol = 1e-15 if precision == "fp64" else 5e-7
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
