"""GPU parity: the CUDA engine (through the C ABI) against the reference.

Two anchors:
* golden vectors written by the reference's own sources (tests/golden/);
* the CPU oracle restatement (oracle/), itself pinned bit-for-bit to the reference,
  at sizes where it finishes in seconds.

Tolerances: FP64 relative L2 <= 1e-12 on wavefunctions (the stated bar); observables
<= 1e-11 relative (they are sums of O(N) terms); mixed precision is held to bounds
stated per test.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GRIDS = {
    "1d": (1, (64,), (0.4,)),
    "2d": (2, (8, 16), (0.5, 0.35)),
    "3d": (3, (4, 8, 8), (0.6, 0.5, 0.45)),
}
POT = {"1d": "H_1D", "2d": "Ne_2D", "3d": "H_3D"}
OBS = ["dipole_r", "dipole_v", "energy", "Lz"]
TOL = 1e-12


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.fixture(scope="module")
def Grid(qnd_lib):
    from tdse_nd_mpi_b200 import Grid

    return Grid


@pytest.mark.parametrize("key", list(GRIDS))
@pytest.mark.parametrize("integ", ["Verlet", "BM4", "BM6", "RKN4"])
def test_steps_vs_golden(Grid, golden, key, integ):
    g = golden["steps"]
    dim, nr, dr = GRIDS[key]
    tag = f"{key}_{integ}"
    grid = Grid(dim, nr, dr, integ, 0.05)
    grid.set_potential(POT[key])
    grid.set_cap(0.2, 0.8)
    np.testing.assert_allclose(grid.as_scaled, g[f"{tag}_coeffs"], rtol=0, atol=0)
    psi0, E = g[f"{tag}_psi0"], g[f"{tag}_E"]
    st = grid.state(psi0)
    grid.integration_step_imag(st, 2)
    assert rel(st.download(), g[f"{tag}_imag"]) < TOL
    st.upload(psi0)
    grid.integration_step_length(st, E)
    assert rel(st.download(), g[f"{tag}_length"]) < TOL
    st.upload(psi0)
    grid.integration_step_velocity(st, E)
    assert rel(st.download(), g[f"{tag}_velocity"]) < TOL


@pytest.mark.parametrize("key", list(GRIDS))
def test_observables_energies_gs_vs_golden(Grid, golden, key):
    g = golden["observables"]
    dim, nr, dr = GRIDS[key]
    grid = Grid(dim, nr, dr, "BM4", 0.05)
    grid.set_potential(POT[key])
    psi, alpha = g[f"{key}_psi"], g[f"{key}_alpha"]
    st = grid.state(psi)
    np.testing.assert_allclose(grid.observables(st, OBS, alpha), g[f"{key}_obs"], rtol=1e-11, atol=1e-12)
    np.testing.assert_allclose(grid.energies(st, 3), g[f"{key}_energies"], rtol=1e-11)
    states = [grid.state(s) for s in g[f"{key}_gs_in"]]
    for j in range(len(states)):
        grid.gram_schmidt(states, j)
    out = np.stack([s.download() for s in states])
    assert rel(out, g[f"{key}_gs_out"]) < TOL


@pytest.mark.parametrize("integ", ["BM4", "Verlet"])
def test_driver_trajectories_vs_golden(Grid, golden, integ):
    """QuantumND_real.c loops with observables every step (length and velocity gauges)."""
    g = golden["trajectory"]
    tag = f"traj_{integ}"
    grid = Grid(2, (16, 16), (0.4, 0.4), integ, 0.05)
    grid.set_potential("H_2D")
    grid.set_cap(0.3, 1.2)
    st = grid.state(g[f"{tag}_psi0"])
    obs = grid.run_length(st, g[f"{tag}_E"], OBS)
    np.testing.assert_allclose(obs, g[f"{tag}_length_obs"], rtol=1e-11, atol=1e-12)
    assert rel(st.download(), g[f"{tag}_length_psi"]) < TOL
    st.upload(g[f"{tag}_psi0"])
    obs = grid.run_velocity(st, g[f"{tag}_A"], g[f"{tag}_alpha"], OBS)
    np.testing.assert_allclose(obs, g[f"{tag}_velocity_obs"], rtol=1e-11, atol=1e-12)
    assert rel(st.download(), g[f"{tag}_velocity_psi"]) < TOL


def test_imag_eigenstates_vs_golden(Grid, golden):
    """QuantumND_imag.c:169-188 on 1-D H: three eigenstates with Gram-Schmidt every step."""
    g = golden["imag"]
    grid = Grid(1, (128,), (0.4,), "BM4", 0.1)
    grid.set_potential("H_1D")
    states = [grid.state(g["guess"].astype(np.complex128)) for _ in range(3)]
    for j in range(3):
        grid.imag_propagate(states, j, int(g["nsteps"]))
        np.testing.assert_allclose(grid.energies(states[j], 2), g["energies"][j], rtol=1e-11)
    out = np.stack([s.download() for s in states])
    assert rel(out, g["states"]) < 1e-11


def soft_coulomb(grid, a):
    axes = [grid.axis_r(j) for j in range(grid.dim)]
    X = np.meshgrid(*axes, indexing="ij")
    r2 = sum(x * x for x in X)
    V = -1.0 / np.sqrt(r2 + a)
    grads = [x / (r2 + a) ** 1.5 for x in X]   # dV/dx_j
    return V, grads


@pytest.mark.parametrize("shape,dr", [((256, 256), (0.2, 0.2)), ((1024, 1024), (0.2, 0.2)), ((64, 2048), (0.4, 0.1)),
                                      ((4096,), (0.1,)), ((32, 16, 64), (0.5, 0.5, 0.3))])
def test_length_run_vs_oracle_custom_potential(Grid, shape, dr):
    """H_2D-style custom V = -1/sqrt(r^2+0.64) with CAP, BM4, observables every step."""
    dim = len(shape)
    grid = Grid(dim, shape, dr, "BM4", 0.05)
    V, grads = soft_coulomb(grid, 0.64)
    grid.set_potential(V)
    grid.set_cap(0.05, 2.0)
    for j in range(dim):
        grid.set_gradv(j, grads[j])
    o = O.OracleCtx(dim, shape, dr, "BM4", 0.05)
    o.set_vpot(V)
    o.set_cap(0.05, 2.0)
    for j in range(dim):
        o.set_gradv(j, grads[j])
    psi0 = O.smooth_state(shape, dr, 1)
    nsteps = 3
    E = np.random.default_rng(0).standard_normal((nsteps, grid.s, dim)) * 0.05
    names = ["norm", "dipole_r", "accel"]
    a = psi0.copy()
    ob_o = o.run_length(a, E, names)
    st = grid.state(psi0)
    ob_g = grid.run_length(st, E, names)
    assert rel(st.download(), a) < TOL
    np.testing.assert_allclose(ob_g, ob_o, rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("shape,dr", [((512, 512), (0.2, 0.2)), ((16, 32, 64), (0.5, 0.4, 0.3))])
def test_imag_and_velocity_vs_oracle(Grid, shape, dr):
    dim = len(shape)
    grid = Grid(dim, shape, dr, "BM6", 0.05)
    grid.set_potential("H_3D" if dim == 3 else "Ne_2D")
    grid.set_cap(0.1, 1.5)
    o = O.OracleCtx(dim, shape, dr, "BM6", 0.05)
    o.set_potential("H_3D" if dim == 3 else "Ne_2D")
    o.set_cap(0.1, 1.5)
    psi0 = O.smooth_state(shape, dr, 2)
    a = psi0.copy()
    o.step_imag(a, 2)
    st = grid.state(psi0)
    grid.integration_step_imag(st, 2)
    assert rel(st.download(), a) < TOL
    A = np.random.default_rng(1).standard_normal((2, grid.s, dim)) * 0.3
    a = psi0.copy()
    o.step_velocity(a, A, 2)
    st.upload(psi0)
    grid.integration_step_velocity(st, A)
    assert rel(st.download(), a) < TOL


def test_unitary_conversions_roundtrip(Grid):
    grid = Grid(2, (128, 256), (0.3, 0.2), "BM4", 0.05)
    psi0 = O.seeded_state((128, 256), 5)
    o = O.OracleCtx(2, (128, 256), (0.3, 0.2), "BM4", 0.05)
    a = psi0.copy()
    o.to_p(a)
    st = grid.state(psi0)
    grid.to_p(st)
    assert rel(st.download(), a) < TOL
    grid.to_r(st)
    assert rel(st.download(), psi0) < TOL


def test_norm_conserved_and_reversible_at_full_size(Grid):
    """Size-independent properties at the benchmark size (1024^2, BM4): without a CAP the
    length-gauge step is unitary, and stepping with dt then -dt returns the state."""
    shape, dr = (1024, 1024), (0.2, 0.2)
    grid = Grid(2, shape, dr, "BM4", 0.05)
    V, _ = soft_coulomb(grid, 0.64)
    grid.set_potential(V)
    psi0 = O.smooth_state(shape, dr, 3)
    st = grid.state(psi0)
    E = np.full((20, grid.s, 2), 0.03)
    obs = grid.run_length(st, E, ["norm"])
    assert np.max(np.abs(obs[:, 0] - 1.0)) < 1e-12
    back = Grid(2, shape, dr, "BM4", -0.05)
    back.set_potential(V)
    back.run_length(st.ptr, E[::-1], [])
    back.synchronize()  # the state was advanced on `back`'s stream; `st` downloads on `grid`'s
    assert rel(st.download(), psi0) < 1e-11


def test_gram_schmidt_norm_collapse_is_an_error(Grid):
    from tdse_nd_mpi_b200 import QndError

    grid = Grid(1, (64,), (0.3,), "BM4", 0.05)
    s0 = O.seeded_state((64,), 1, 0.3)
    states = [grid.state(s0), grid.state(s0)]
    grid.gram_schmidt(states, 0)
    with pytest.raises(QndError) as ei:
        grid.gram_schmidt(states, 1)
    assert ei.value.code == 4 and "norm" in str(ei.value)


@pytest.mark.parametrize("shape,dr", [((256, 256), (0.2, 0.2)), ((1024, 1024), (0.2, 0.2)), ((4096,), (0.1,)),
                                      ((32, 32, 64), (0.5, 0.5, 0.4))])
def test_mixed_precision_error_bound(Grid, shape, dr):
    """Complex64 bulk with FP64 reductions: stated bounds against the FP64 oracle after 10 steps:
    wavefunction relative L2 <= 2e-5, observables relative <= 5e-6 (the norm drifts by ~1e-7 per
    step from the rounding of the float twiddle and phase tables)."""
    dim = len(shape)
    gm = Grid(dim, shape, dr, "BM4", 0.05, precision="mixed")
    V, grads = soft_coulomb(gm, 0.64)
    gm.set_potential(V)
    for j in range(dim):
        gm.set_gradv(j, grads[j])
    o = O.OracleCtx(dim, shape, dr, "BM4", 0.05)
    o.set_vpot(V)
    for j in range(dim):
        o.set_gradv(j, grads[j])
    psi0 = O.smooth_state(shape, dr, 4)
    E = np.random.default_rng(5).standard_normal((10, gm.s, dim)) * 0.05
    names = ["norm", "dipole_r", "accel"]
    a = psi0.copy()
    ob_o = o.run_length(a, E, names)
    st = gm.state(psi0)
    ob_m = gm.run_length(st, E, names)
    assert rel(st.download(), a) < 2e-5
    scale = np.maximum(np.abs(ob_o), 1e-3)
    assert np.max(np.abs(ob_m - ob_o) / scale) < 5e-6


def cos8_mask(axis, frac=0.1):
    """cos^(1/8) absorbing mask over the outer `frac` of an axis (the benchmark's mask)."""
    half = np.max(np.abs(axis))
    edge = (1.0 - frac) * half
    m = np.ones_like(axis)
    zone = np.abs(axis) > edge
    m[zone] = np.cos(0.5 * np.pi * (np.abs(axis[zone]) - edge) / (half - edge)).clip(0.0) ** 0.125
    return m


def _masked_pair(Grid, shape, dr, integ="BM4"):
    dim = len(shape)
    grid = Grid(dim, shape, dr, integ, 0.05)
    V, grads = soft_coulomb(grid, 0.64)
    o = O.OracleCtx(dim, shape, dr, integ, 0.05)
    for ctx in (grid, o):
        if ctx is grid:
            ctx.set_potential(V)
        else:
            ctx.set_vpot(V)
        ctx.set_cap(0.05, 2.0)
        for j in range(dim):
            ctx.set_gradv(j, grads[j])
            ctx.set_mask_axis(j, cos8_mask(grid.axis_r(j)))
    return grid, o


@pytest.mark.parametrize("shape,dr", [((256, 256), (0.2, 0.2)), ((16, 32, 64), (0.5, 0.4, 0.3)), ((2048,), (0.1,)),
                                      ((64, 2048), (0.4, 0.1))])
def test_masked_run_with_observables_vs_oracle(Grid, shape, dr):
    """Several steps in one sandwich chain: the step mask and each step's observables are applied
    inside the pass that straddles the step boundary (2-D, 3-D); per-step chains in 1-D."""
    grid, o = _masked_pair(Grid, shape, dr)
    dim = len(shape)
    psi0 = O.smooth_state(shape, dr, 6)
    nsteps = 5
    E = np.random.default_rng(7).standard_normal((nsteps, grid.s, dim)) * 0.05
    names = ["norm", "dipole_r", "accel"]
    a = psi0.copy()
    ob_o = o.run_length(a, E, names)
    st = grid.state(psi0)
    ob_g = grid.run_length(st, E, names)
    assert rel(st.download(), a) < TOL
    np.testing.assert_allclose(ob_g, ob_o, rtol=1e-11, atol=1e-13)


def test_device_loop_matches_host_loop_masked(Grid):
    """qnd_run_length_dev (rows after each step, device buffers) against qnd_run_length (rows before
    each step) on the same masked run: row i of the first is row i+1 of the second."""
    import torch

    shape, dr = (512, 512), (0.2, 0.2)
    grid, _ = _masked_pair(Grid, shape, dr)
    psi0 = O.smooth_state(shape, dr, 8)
    nsteps = 6
    E = np.random.default_rng(9).standard_normal((nsteps + 1, grid.s, 2)) * 0.05
    names = ["norm", "dipole_r", "accel"]
    st = grid.state(psi0)
    ob_host = grid.run_length(st, E, names)
    psi_host = st.download()
    st2 = grid.state(psi0)
    E_dev = torch.tensor(E, device="cuda")
    obs_dev = torch.zeros((nsteps + 1, ob_host.shape[1]), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    grid.run_length_dev(st2, E_dev, nsteps + 1, names, obs_dev)
    grid.synchronize()
    np.testing.assert_allclose(obs_dev.cpu().numpy()[:nsteps], ob_host[1:], rtol=1e-12, atol=1e-15)
    assert rel(st2.download(), psi_host) < 1e-13


def test_many_observable_values_fall_back_per_step(Grid):
    """More reduction outputs than one fused descriptor holds (3-D: 10 values): per-step chains
    with an extra grid reduction, same results."""
    shape, dr = (16, 32, 32), (0.5, 0.4, 0.4)
    grid, o = _masked_pair(Grid, shape, dr)
    psi0 = O.smooth_state(shape, dr, 10)
    E = np.random.default_rng(11).standard_normal((3, grid.s, 3)) * 0.05
    names = ["norm", "dipole_r", "accel", "dipole_r"]
    a = psi0.copy()
    ob_o = o.run_length(a, E, names)
    st = grid.state(psi0)
    ob_g = grid.run_length(st, E, names)
    assert rel(st.download(), a) < TOL
    np.testing.assert_allclose(ob_g, ob_o, rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("shape,dr", [((128, 256), (0.3, 0.2)), ((1024,), (0.2,)), ((16, 16, 32), (0.5, 0.5, 0.4))])
def test_multistep_length_velocity_imag_vs_oracle(Grid, shape, dr):
    """Multi-step calls without observables or mask: consecutive steps merge K(a_2s-1) K(a_0) into one
    sandwich (length gauge) or V(a_2s-1) V(a_0) into one factor (velocity, imaginary time)."""
    dim = len(shape)
    grid = Grid(dim, shape, dr, "BM4", 0.05)
    grid.set_potential(POT[{1: "1d", 2: "2d", 3: "3d"}[dim]])
    grid.set_cap(0.1, 1.0)
    o = O.OracleCtx(dim, shape, dr, "BM4", 0.05)
    o.set_potential(POT[{1: "1d", 2: "2d", 3: "3d"}[dim]])
    o.set_cap(0.1, 1.0)
    psi0 = O.smooth_state(shape, dr, 12)
    n = 4
    F = np.random.default_rng(13).standard_normal((n, grid.s, dim)) * 0.05
    a = psi0.copy()
    o.to_p(a)
    o.step_length(a, F, n)
    st = grid.state(psi0)
    grid.to_p(st)
    grid.integration_step_length(st, F)
    assert rel(st.download(), a) < TOL
    a = psi0.copy()
    o.step_velocity(a, F * 5, n)
    st.upload(psi0)
    grid.integration_step_velocity(st, F * 5)
    assert rel(st.download(), a) < TOL
    a = psi0.copy()
    o.step_imag(a, n)
    st.upload(psi0)
    grid.integration_step_imag(st, n)
    assert rel(st.download(), a) < TOL


def test_graph_replayed_chunks_match_direct_launches(Grid, monkeypatch):
    """Runs longer than one chunk (128 steps): the first chunk runs directly, the second is
    captured into a CUDA graph and the later ones replay it. Same results as direct launches
    (QND_NO_GRAPH) and as the oracle."""
    shape, dr = (64, 128), (0.4, 0.3)
    grid, o = _masked_pair(Grid, shape, dr)
    psi0 = O.smooth_state(shape, dr, 14)
    nsteps = 300
    E = np.random.default_rng(15).standard_normal((nsteps, grid.s, 2)) * 0.05
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


@pytest.mark.parametrize("shape,dr,pot,rmask,prmax", [((512,), (0.2,), "H_1D", (10.0, 20.0), (3.0,)),
                                                      ((64, 64), (0.3, 0.3), "H_2D", (3.0, 8.0), (4.0, 2.5)),
                                                      ((16, 16, 32), (0.5, 0.5, 0.4), "H_3D", (2.0, 5.0), (3.0, 3.0, 5.0))])
def test_final_spectra_vs_reference(Grid, shape, dr, pot, rmask, prmax):
    """PED and PMD (Write_final_observables, io_functions.c:136-287) against the reference's own
    function compiled from its sources: the energy distribution, the kept-momentum counts and the
    packed (|psi~|^2, arg psi~) pairs."""
    grid = Grid(len(shape), shape, dr, "BM4", 0.05)
    grid.set_potential(pot)
    psi = O.smooth_state(shape, dr, 16) * np.exp(1j * 0.7 * O.seeded_state(shape, 17).real)
    de, ne = 0.02, 120
    if O.ref_available():
        out = O.RefCtx(len(shape), shape, dr, "BM4", 0.05, potential=pot).final_observables(psi, rmask, prmax, de, ne)
    else:  # the restatement, pinned to the reference by test_oracle
        p_, c_, d_ = O.final_spectra_numpy(psi, dr, rmask, prmax, de, ne)
        out = {"PED": np.stack([np.arange(ne) * de, p_], axis=1), "PMD": ({"NPR": c_}, d_)}
    ped, counts, pmd = grid.final_spectra(grid.state(psi), rmask, prmax, de, ne)
    np.testing.assert_allclose(out["PED"][:, 0], np.arange(ne) * de, rtol=0, atol=1e-15)
    np.testing.assert_allclose(ped, out["PED"][:, 1], rtol=0, atol=1e-11 * np.max(np.abs(out["PED"][:, 1])))
    head, data = out["PMD"]
    assert counts == [int(v) for v in head["NPR"]]
    assert pmd.shape == data.shape
    dens = data[:, 0]
    np.testing.assert_allclose(pmd[:, 0], dens, rtol=0, atol=1e-12 * dens.max())
    live = dens > 1e-10 * dens.max()
    dphi = np.angle(np.exp(1j * (pmd[live, 1] - data[live, 1])))
    assert np.max(np.abs(dphi)) < 1e-8


@pytest.mark.parametrize("shape,dr", [((128, 128), (0.3, 0.3)), ((16, 16, 32), (0.5, 0.5, 0.4)), ((4096,), (0.1,))])
def test_masked_velocity_run_with_all_observables_vs_oracle(Grid, shape, dr):
    """Velocity gauge with CAP, step mask and every observable (norm, dipole_r, dipole_v with the
    step's A(t) shift, energy, Lz, accel) each step, against the oracle."""
    grid, o = _masked_pair(Grid, shape, dr)
    dim = len(shape)
    psi0 = O.smooth_state(shape, dr, 18)
    nsteps = 4
    rng = np.random.default_rng(19)
    A = rng.standard_normal((nsteps, grid.s, dim)) * 0.3
    alpha = rng.standard_normal((nsteps, dim)) * 0.2
    names = ["norm", "dipole_r", "dipole_v", "energy", "Lz", "accel"]
    a = psi0.copy()
    ob_o = o.run_velocity(a, A, alpha, names)
    st = grid.state(psi0)
    ob_g = grid.run_velocity(st, A, alpha, names)
    assert rel(st.download(), a) < TOL
    np.testing.assert_allclose(ob_g, ob_o, rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("shape", [(2, 64), (64, 2), (2, 2, 2), (2, 8, 256), (4096, 16), (16, 4096), (2, 4096)])
def test_extreme_axis_lengths_vs_oracle(Grid, shape):
    """The shortest (2) and longest (4096) pass axes, strided and contiguous, in 2-D and 3-D: imaginary
    time and length-gauge steps with observables against the oracle."""
    dim = len(shape)
    dr = (0.3,) * dim
    grid = Grid(dim, shape, dr, "BM4", 0.05)
    grid.set_potential(POT[{1: "1d", 2: "2d", 3: "3d"}[dim]])
    grid.set_cap(0.1, 0.5)
    o = O.OracleCtx(dim, shape, dr, "BM4", 0.05)
    o.set_potential(POT[{1: "1d", 2: "2d", 3: "3d"}[dim]])
    o.set_cap(0.1, 0.5)
    psi0 = O.seeded_state(shape, 21, float(np.prod(dr)))
    a = psi0.copy()
    o.step_imag(a, 2)
    st = grid.state(psi0)
    grid.integration_step_imag(st, 2)
    assert rel(st.download(), a) < TOL
    E = np.random.default_rng(22).standard_normal((3, grid.s, dim)) * 0.05
    names = ["norm", "dipole_r", "dipole_v", "energy"]
    a = psi0.copy()
    ob_o = o.run_length(a, E, names)
    st.upload(psi0)
    ob_g = grid.run_length(st, E, names)
    assert rel(st.download(), a) < TOL
    np.testing.assert_allclose(ob_g, ob_o, rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shape,dr", [((1024, 1024), (0.2, 0.2)), ((64, 64, 64), (0.4, 0.4, 0.4)), ((65536,), (0.05,))])
def test_staging_choice_never_changes_results(Grid, monkeypatch, precision, shape, dr):
    """Strided passes stage their lines by TMA boxes or by per-thread copies, whichever the staging
    autotuner measured faster; both paths must give bit-identical states and observables."""
    dim = len(shape)

    def run():
        grid, _ = _masked_pair(Grid, shape, dr)
        gm = grid if precision == "fp64" else None
        if gm is None:
            gm = Grid(dim, shape, dr, "BM4", 0.05, precision="mixed")
            V, grads = soft_coulomb(gm, 0.64)
            gm.set_potential(V)
            gm.set_cap(0.05, 2.0)
            for j in range(dim):
                gm.set_gradv(j, grads[j])
                gm.set_mask_axis(j, cos8_mask(gm.axis_r(j)))
        st = gm.state(O.smooth_state(shape, dr, 23))
        E = np.random.default_rng(24).standard_normal((5, gm.s, dim)) * 0.05
        obs = gm.run_length(st, E, ["norm", "dipole_r", "accel"])
        return obs, st.download()

    tuned = run()
    monkeypatch.setenv("QND_NO_TMA", "1")
    copies = run()
    np.testing.assert_array_equal(tuned[0], copies[0])
    np.testing.assert_array_equal(tuned[1], copies[1])
