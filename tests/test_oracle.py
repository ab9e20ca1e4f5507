"""CPU tests pinning the oracle (oracle/qnd_oracle.c) to the reference.

1. Against the committed golden vectors produced by the reference's own sources
   (tests/golden/make_golden.py).
2. Live against the reference compiled here (oracle/_ref), bit for bit, when it
   is present (it is where the reference sources were available).
3. The FFT (FFTW-API shim) against numpy.fft.
"""
import numpy as np
import pytest

from oracle import oracle as O

GRIDS = {
    "1d": (1, (64,), (0.4,)),
    "2d": (2, (8, 16), (0.5, 0.35)),
    "3d": (3, (4, 8, 8), (0.6, 0.5, 0.45)),
}
POT = {"1d": "H_1D", "2d": "Ne_2D", "3d": "H_3D"}
OBS = ["dipole_r", "dipole_v", "energy", "Lz"]


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


@pytest.mark.parametrize("key", list(GRIDS))
@pytest.mark.parametrize("integ", ["Verlet", "BM4", "BM6", "RKN4"])
def test_steps_match_golden(golden, key, integ):
    g = golden["steps"]
    dim, nr, dr = GRIDS[key]
    tag = f"{key}_{integ}"
    o = O.OracleCtx(dim, nr, dr, integ, 0.05, nthreads=1)
    o.set_potential(POT[key])
    o.set_cap(0.2, 0.8)
    np.testing.assert_array_equal(O.coeffs(integ, 0.05), g[f"{tag}_coeffs"])
    _, _, v, vc, k = o.tables()
    np.testing.assert_allclose(v, g[f"{tag}_vpot"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(vc, g[f"{tag}_vcap"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(k, g[f"{tag}_kin"], rtol=1e-15, atol=0)
    psi0, E = g[f"{tag}_psi0"], g[f"{tag}_E"]
    for kind in ("imag", "length", "velocity"):
        a = psi0.copy()
        if kind == "imag":
            o.step_imag(a, 2)
        elif kind == "length":
            o.step_length(a, E, 2)
        else:
            o.step_velocity(a, E, 2)
        assert rel(a, g[f"{tag}_{kind}"]) < 1e-14, (kind, rel(a, g[f"{tag}_{kind}"]))


@pytest.mark.parametrize("key", list(GRIDS))
def test_observables_gs_match_golden(golden, key):
    g = golden["observables"]
    dim, nr, dr = GRIDS[key]
    o = O.OracleCtx(dim, nr, dr, "BM4", 0.05, nthreads=1)
    o.set_potential(POT[key])
    psi, alpha = g[f"{key}_psi"], g[f"{key}_alpha"]
    np.testing.assert_allclose(o.observables(psi, OBS, alpha), g[f"{key}_obs"], rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(o.energies(psi, 3), g[f"{key}_energies"], rtol=1e-13)
    states = [s.copy() for s in g[f"{key}_gs_in"]]
    for j in range(len(states)):
        rc, _ = o.gram_schmidt(j, states)
        assert rc == 0
    assert rel(np.stack(states), g[f"{key}_gs_out"]) < 1e-14


@pytest.mark.parametrize("integ", ["BM4", "Verlet"])
def test_trajectories_match_golden(golden, integ):
    g = golden["trajectory"]
    tag = f"traj_{integ}"
    o = O.OracleCtx(2, (16, 16), (0.4, 0.4), integ, 0.05, nthreads=1)
    o.set_potential("H_2D")
    o.set_cap(0.3, 1.2)
    a = g[f"{tag}_psi0"].copy()
    obs = o.run_length(a, g[f"{tag}_E"], OBS)
    np.testing.assert_allclose(obs, g[f"{tag}_length_obs"], rtol=1e-12, atol=1e-13)
    assert rel(a, g[f"{tag}_length_psi"]) < 1e-13
    a = g[f"{tag}_psi0"].copy()
    obs = o.run_velocity(a, g[f"{tag}_A"], g[f"{tag}_alpha"], OBS)
    np.testing.assert_allclose(obs, g[f"{tag}_velocity_obs"], rtol=1e-12, atol=1e-13)
    assert rel(a, g[f"{tag}_velocity_psi"]) < 1e-13


def test_imag_eigenstates_match_golden(golden):
    g = golden["imag"]
    o = O.OracleCtx(1, (128,), (0.4,), "BM4", 0.1, nthreads=1)
    o.set_potential("H_1D")
    nsteps = int(g["nsteps"])
    assert nsteps == O.imag_loop_count(20.0, 0.1)
    assert O.imag_loop_count(100.0, 0.05) == 2001  # FP accumulation of time+=dt (QuantumND_imag.c:182)
    states = [np.ascontiguousarray(g["guess"].astype(np.complex128)) for _ in range(3)]
    for j in range(3):
        assert o.imag_state(states, j, nsteps) == 0
        np.testing.assert_allclose(o.energies(states[j], 2), g["energies"][j], rtol=1e-12)
    assert rel(np.stack(states), g["states"]) < 1e-12
    # the ground state of the soft-core H_1D potential is E = -0.5 (a known exact value)
    assert abs(g["energies"][0][0] + 0.5) < 1e-6


@pytest.mark.parametrize("env", ["constant", "trapz", "cos2", "cos4"])
@pytest.mark.parametrize("integ", ["BM4", "BM6"])
def test_field_matches_golden(golden, env, integ):
    g = golden["field"]
    modes = [dict(intensity=1e14, ellipticity=0.4, cep=0.2, delay=2.0, duration=60.0, envelope=env,
                  **{"lambda": 80.0}),
             dict(intensity=2e13, ellipticity=0.0, cep=1.1, delay=0.0, duration=40.0, envelope=env,
                  **{"lambda": 40.0})]
    E, A, _ = O.field(2, modes, integ, 0.5, 70.0)
    np.testing.assert_allclose(E, g[f"{env}_{integ}_E"], rtol=1e-14, atol=1e-17)
    np.testing.assert_allclose(A, g[f"{env}_{integ}_A"], rtol=1e-14, atol=1e-17)


@pytest.mark.parametrize("shape", [(32,), (8, 16), (4, 8, 16)])
def test_fft_shim_matches_numpy(golden, shape):
    g = golden["fft"]
    tag = "x".join(map(str, shape))
    x = g[f"{tag}_in"]
    assert rel(O.fft(x, -1), g[f"{tag}_fwd"]) < 1e-15
    assert rel(O.fft(x, +1), g[f"{tag}_bwd"]) < 1e-15


@pytest.mark.parametrize("shape", [(1024,), (64, 128), (16, 32, 8)])
def test_fft_shim_random_sizes(shape):
    x = O.seeded_state(shape, 99)
    assert rel(O.fft(x, -1, nthreads=4), np.fft.fftn(x)) < 1e-15 * np.log2(x.size) * 2


def test_gram_schmidt_collapse_reported():
    """The reference aborts when ||v||^2 dNr < 1e-12 (QuantumND_imag.c:297-304); the oracle returns 2."""
    o = O.OracleCtx(1, (32,), (0.5,), "BM4", 0.05, nthreads=1)
    s0 = O.seeded_state((32,), 1, 0.5)
    states = [s0, s0.copy()]
    assert o.gram_schmidt(0, states)[0] == 0
    rc, norm = o.gram_schmidt(1, states)
    assert rc == 2 and norm < 1e-12


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here (needs its sources)")
@pytest.mark.parametrize("integ", ["Verlet", "BM4", "BM6", "RKN4"])
@pytest.mark.parametrize("pot", ["H_2D", "Ne_2D", "Ar_2D", "Kr_2D", "Xe_2D", "Ne_short_2D"])
def test_oracle_bit_identical_to_reference(integ, pot):
    dim, nr, dr = 2, (16, 32), (0.3, 0.2)
    o = O.OracleCtx(dim, nr, dr, integ, 0.05, nthreads=2)
    o.set_potential(pot)
    o.set_cap(0.1, 1.0)
    r = O.RefCtx(dim, nr, dr, integ, 0.05, pot, (0.1, 1.0), nthreads=2)
    assert np.array_equal(o.tables()[2], r.tables()[0])
    psi = O.seeded_state(nr, 1)
    E = np.random.default_rng(2).standard_normal((3, o.s, dim)) * 0.05
    for step in ("step_imag", "step_length", "step_velocity"):
        a, b = psi.copy(), psi.copy()
        if step == "step_imag":
            o.step_imag(a, 3), r.step_imag(b, 3)
        else:
            getattr(o, step)(a, E, 3), getattr(r, step)(b, E, 3)
        assert np.array_equal(a, b), step
    al = np.array([0.1, -0.2])
    assert np.array_equal(o.observables(psi, OBS, al), r.observables(psi, OBS, al))
    assert np.array_equal(o.energies(psi, 2), r.energies(psi, 2))


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here (needs its sources)")
def test_oracle_3d_and_1d_bit_identical_to_reference():
    for dim, nr, dr, pot in ((1, (128,), (0.3,), "H_1D"), (3, (8, 8, 16), (0.4, 0.5, 0.3), "H_3D")):
        o = O.OracleCtx(dim, nr, dr, "BM4", 0.05, nthreads=2)
        o.set_potential(pot)
        o.set_cap(0.3, 0.7)
        r = O.RefCtx(dim, nr, dr, "BM4", 0.05, pot, (0.3, 0.7), nthreads=2)
        psi = O.seeded_state(nr, 7)
        E = np.random.default_rng(3).standard_normal((2, o.s, dim)) * 0.05
        names = ["dipole_r", "dipole_v", "energy", "Lz"]
        a, b = psi.copy(), psi.copy()
        assert np.array_equal(o.run_length(a, E, names), r.run_length(b, E, names))
        assert np.array_equal(a, b)


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here (needs its sources)")
@pytest.mark.parametrize("shape,dr,pot", [((256,), (0.2,), "H_1D"), ((32, 64), (0.3, 0.25), "H_2D")])
def test_final_spectra_restatement_matches_reference(shape, dr, pot):
    """The PED/PMD restatement used by the checks against Write_final_observables itself."""
    r = O.RefCtx(len(shape), shape, dr, "BM4", 0.05, potential=pot, nthreads=2)
    psi = O.smooth_state(shape, dr, 4) * np.exp(0.5j * O.seeded_state(shape, 5).real)
    rmask, prmax, de, ne = (2.0, 6.0), (3.0,) * len(shape), 0.03, 80
    out = r.final_observables(psi, rmask, prmax, de, ne)
    ped, counts, pmd = O.final_spectra_numpy(psi, dr, rmask, prmax, de, ne)
    np.testing.assert_allclose(ped, out["PED"][:, 1], rtol=0, atol=1e-12 * out["PED"][:, 1].max())
    head, data = out["PMD"]
    assert counts == [int(v) for v in head["NPR"]]
    np.testing.assert_allclose(pmd[:, 0], data[:, 0], rtol=0, atol=1e-13 * data[:, 0].max())
    live = data[:, 0] > 1e-10 * data[:, 0].max()
    assert np.max(np.abs(np.angle(np.exp(1j * (pmd[live, 1] - data[live, 1]))))) < 1e-9


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here (needs its sources)")
def test_reference_loop_with_extension_observables_matches_oracle():
    """ref_run_length_ext (the reference's own length-gauge loop with norm and accel computed on the
    same states, the CPU baseline's loop) against the oracle's run_length with the same observables,
    a custom potential and a CAP: identical states, observables within summation-order rounding."""
    dim, nr, dr = 2, (32, 64), (0.3, 0.25)
    x = [-0.5 * n * d + np.arange(n) * d for n, d in zip(nr, dr)]
    X, Y = np.meshgrid(*x, indexing="ij")
    r2 = X * X + Y * Y
    V = -1.0 / np.sqrt(r2 + 0.64)
    grads = [X / (r2 + 0.64) ** 1.5, Y / (r2 + 0.64) ** 1.5]
    vcap = 0.02 * (np.abs(X) > 3.5) + 0.01 * (np.abs(Y) > 6.0)
    o = O.OracleCtx(dim, nr, dr, "BM4", 0.05, nthreads=2)
    o.set_vpot(V)
    o.set_vcap(vcap)
    for j in range(dim):
        o.set_gradv(j, grads[j])
    r = O.RefCtx(dim, nr, dr, "BM4", 0.05, "H_2D", (0.0, 0.0), nthreads=2)
    r.set_vpot(V)
    r.set_vcap(vcap)
    psi = O.seeded_state(nr, 4)
    E = np.random.default_rng(9).standard_normal((4, o.s, dim)) * 0.05
    names = ["norm", "dipole_r", "accel"]
    a, b = psi.copy(), psi.copy()
    got = r.run_length_ext(b, E, names, grads)
    want = o.run_length(a, E, names)
    assert got.shape == (4, 5)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)
    assert np.array_equal(a, b)
    # the reference's own columns are the reference's values
    c = psi.copy()
    np.testing.assert_array_equal(got[:, 1:3], r.run_length(c, E, ["dipole_r"]))


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here (needs its sources)")
def test_oracle_4d_bit_identical_to_reference():
    """DIMENSION above 3: the reference allocates per dimension (parameters.c:46-48) and plans an
    N-D transform of any rank (meshgrid.c:166-167); the restatement follows it in 4-D."""
    dim, nr, dr = 4, (4, 4, 8, 8), (0.6, 0.5, 0.45, 0.4)
    o = O.OracleCtx(dim, nr, dr, "BM4", 0.05, nthreads=2)
    o.set_potential("H_3D")
    o.set_cap(0.3, 0.7)
    r = O.RefCtx(dim, nr, dr, "BM4", 0.05, "H_3D", (0.3, 0.7), nthreads=2)
    psi = O.seeded_state(nr, 5)
    E = np.random.default_rng(4).standard_normal((2, o.s, dim)) * 0.05
    names = ["dipole_r", "dipole_v", "energy", "Lz"]
    a, b = psi.copy(), psi.copy()
    assert np.array_equal(o.run_length(a, E, names), r.run_length(b, E, names))
    assert np.array_equal(a, b)
    a, b = psi.copy(), psi.copy()
    o.step_imag(a, 2), r.step_imag(b, 2)
    assert np.array_equal(a, b)
    a, b = psi.copy(), psi.copy()
    o.step_velocity(a, E, 2), r.step_velocity(b, E, 2)
    assert np.array_equal(a, b)
