"""Mixed precision (complex64 bulk; FFTs and phases in FP32; norms, Gram-Schmidt inner products and
every observable sum in FP64) against the FP64 engine, itself pinned to the oracle.

* Imaginary time with Gram-Schmidt (the loop of QuantumND_imag.c:182-185 and its
  Gram_Schmidt_orthonormalization, :265-311) for 8 states of a Ne_2D grid with BM6, the
  Ne_2D-style configuration at 256^2: eigenenergy error and orthonormality of the mixed states.
* The benchmark workload (H_2D 1024^2, BM4, length gauge, CAP mask, norm + dipole + acceleration
  every step) over 300 steps from the pulse's middle: per observable column, the largest error over
  the run relative to the column's largest FP64 value (the y components, zero by symmetry up to the
  grid's one-point asymmetry, relative to their x component's). The bounds are the measured ones:
  mixed precision does not reach 1e-6 relative over this run (a drift of about 1e-8 per step in the
  norm from the FP32 storage).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _guesses(n, dr, count, seed):
    x = -0.5 * n * dr + np.arange(n) * dr
    X, Y = np.meshgrid(x, x, indexing="ij")
    rng = np.random.default_rng(seed)
    return [(np.exp(-(X * X + Y * Y) / 4.0) * (X ** (k % 3)) * (Y ** (k // 3))
             + 0.01 * rng.standard_normal(X.shape)).astype(np.complex128) for k in range(count)]


def test_mixed_imaginary_time_eigenenergies(qnd_lib):
    from tdse_nd_mpi_b200 import Grid

    n, dr, steps, nst = 256, 0.3, 300, 8
    guesses = _guesses(n, dr, nst, 11)
    res = {}
    for prec in ("fp64", "mixed"):
        g = Grid(2, (n, n), (dr, dr), "BM6", 0.05, precision=prec)
        g.set_potential("Ne_2D")
        sts = [g.state(v) for v in guesses]
        for j in range(nst):
            g.imag_propagate(sts, j, steps)
        m = np.array([g.energies(s, 2) for s in sts])
        e = m[:, 0]
        psis = [s.download() for s in sts]
        ov = np.array([[np.vdot(a, b) * dr * dr for b in psis] for a in psis])
        res[prec] = (e, ov, m[:, 1] - e * e)
        g.close()
    de = np.abs(res["mixed"][0] - res["fp64"][0])
    orth = np.max(np.abs(res["mixed"][1] - np.eye(nst)))
    var = res["fp64"][2]
    print("eigenenergy |mixed - fp64| (Ha):", de, "variance:", var, "orthonormality:", orth)
    # states converged in the FP64 run (variance <H^2> - E^2 below 1e-6) agree to 1e-6 Ha; the rest
    # (a degenerate pair still mixing with higher states after 300 steps) follow slightly different
    # paths in FP32 and agree to 2e-4 Ha (measured 9.1e-5); Gram-Schmidt in FP64 keeps the FP32
    # states orthonormal to the storage rounding
    conv = var < 1e-6
    assert conv.sum() >= 2
    assert np.max(de[conv]) < 1e-6
    assert np.max(de) < 2e-4
    assert orth < 1e-6


def test_mixed_bench_workload_observables(qnd_lib):
    import bench
    from tdse_nd_mpi_b200 import Grid

    V, grads, vcap, E, _ = bench.workload_arrays()
    i0 = E.shape[0] // 2
    Ew = np.ascontiguousarray(E[i0:i0 + 300])
    shape, dr = (bench.NR, bench.NR), (bench.DR, bench.DR)
    gi = Grid(2, shape, dr, bench.INTEG, bench.DT)
    gi.set_potential(V)
    st0 = gi.state(bench.gaussian_guess())
    gi.imag_propagate([st0], 0, 20)
    psi0 = st0.download()
    gi.close()
    rows = {}
    for prec in ("fp64", "mixed"):
        g = Grid(2, shape, dr, bench.INTEG, bench.DT, precision=prec)
        g.set_potential(V)
        g.set_vcap(vcap)
        for j in range(2):
            g.set_gradv(j, grads[j])
        rows[prec] = g.run_length(g.state(psi0), Ew, bench.OBS)
        g.close()
    cols, worst = bench.column_errors(rows["fp64"], rows["mixed"], ["norm", "dipole_x", "dipole_y", "accel_x",
                                                                      "accel_y"])
    print(cols)
    # stated bounds after 300 steps (measured: norm 5.9e-6, dipole 5.1e-6, acceleration 1.3e-5; the
    # symmetry-zero y columns 7.7e-6 and 1.5e-5 of their x components). The FP32 storage leaves a
    # steady drift of about 1e-8 per step in the norm, so a 1e-6 bound holds only over the first
    # hundred steps or so.
    rel = {c["column"]: c["rel_err"] for c in cols}
    assert rel["norm"] < 1e-5 and rel["dipole_x"] < 1e-5
    assert worst < 3e-5
