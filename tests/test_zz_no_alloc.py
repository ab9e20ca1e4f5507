"""GPU check of qnd_observables_rspace_noalloc through the C ABI.

The no-allocation entry point takes its reduction scratch from a fixed device array set up on
the first call on a device. Two calls in a row (the set-up call and a call on the ready array)
must match qnd_observables, the allocating entry point, within test tolerance. The file is
named to be collected last, so it also runs after every other GPU test has used the device in
the same process; alone, it runs in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

NAMES = ["norm", "dipole_r", "accel"]


def _soft_coulomb(grid, a):
    X = np.meshgrid(*[grid.axis_r(j) for j in range(grid.dim)], indexing="ij")
    r2 = sum(x * x for x in X)
    return -1.0 / np.sqrt(r2 + a), [x / (r2 + a) ** 1.5 for x in X]


def _grid(shape, dr, precision):
    from tdse_nd_mpi_b200 import Grid

    grid = Grid(len(shape), shape, dr, "BM4", 0.05, precision=precision)
    V, grads = _soft_coulomb(grid, 0.64)
    grid.set_potential(V)
    for j in range(grid.dim):
        grid.set_gradv(j, grads[j])
    return grid


def _names(names):
    arr = (C.c_char_p * max(1, len(names)))()
    for i, n in enumerate(names):
        arr[i] = n.encode()
    return arr


# More than 8 values (the accumulators of one reduction launch) in 3-D: the call splits them over
# several launches that reuse the shared partial sums and ticket counter back to back.
MANY = ["dipole_r", "accel", "norm", "dipole_r"]


@pytest.mark.parametrize("shape,dr,precision,names", [((1024, 1024), (0.2, 0.2), "fp64", NAMES),
                                                      ((256, 256), (0.2, 0.2), "mixed", NAMES),
                                                      ((16, 32, 64), (0.5, 0.4, 0.3), "fp64", NAMES),
                                                      ((4096,), (0.1,), "fp64", NAMES),
                                                      ((32, 64, 128), (0.4, 0.3, 0.2), "fp64", MANY)])
def test_noalloc_matches_qnd_observables_two_calls(qnd_lib, shape, dr, precision, names):
    import torch

    grid = _grid(shape, dr, precision)
    st = grid.state(O.smooth_state(shape, dr, 7))
    ref = grid.observables(st, names)          # the allocating entry point
    nv = len(ref)
    out = torch.full((2, nv), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()                   # the fill runs on torch's stream, the reductions on the context's
    for call in range(2):
        rc = qnd_lib.qnd_observables_rspace_noalloc(grid.h, C.c_void_p(st.ptr), len(names), _names(names),
                                                    C.c_void_p(out[call].data_ptr()))
        assert rc == 0, qnd_lib.qnd_last_error()
    assert qnd_lib.qnd_synchronize(grid.h) == 0
    got = out.cpu().numpy()
    for row in got:
        np.testing.assert_allclose(row, ref, rtol=1e-12, atol=1e-15)


def test_noalloc_rejects_what_it_cannot_do(qnd_lib):
    grid = _grid((64, 64), (0.3, 0.3), "fp64")
    st = grid.state(O.smooth_state((64, 64), (0.3, 0.3), 2))
    dummy = C.c_void_p(st.ptr)                 # never written: every call below fails before launching
    rc = qnd_lib.qnd_observables_rspace_noalloc(grid.h, C.c_void_p(st.ptr), 2, _names(["norm", "energy"]), dummy)
    assert rc == 5 and b"k-space" in qnd_lib.qnd_last_error()
    too_many = ["dipole_r"] * 33                # 66 values > 64
    rc = qnd_lib.qnd_observables_rspace_noalloc(grid.h, C.c_void_p(st.ptr), len(too_many), _names(too_many), dummy)
    assert rc == 1 and b"at most 64" in qnd_lib.qnd_last_error()
    rc = qnd_lib.qnd_observables_rspace_noalloc(grid.h, C.c_void_p(st.ptr), 1, _names(["norm"]), None)
    assert rc == 1
