"""The package's host-side field generator against the reference's golden field samples."""
import numpy as np
import pytest

from tdse_nd_mpi_b200.field import Mode, field_samples, integrator_coeffs, time_vector


@pytest.mark.parametrize("env", ["constant", "trapz", "cos2", "cos4"])
@pytest.mark.parametrize("integ", ["BM4", "BM6"])
def test_field_samples_match_reference(golden, env, integ):
    g = golden["field"]
    modes = [Mode(1e14, 80.0, 0.4, 0.2, 2.0, 60.0, env), Mode(2e13, 40.0, 0.0, 1.1, 0.0, 40.0, env)]
    E, A, t = field_samples(2, modes, integ, 0.5, 70.0)
    np.testing.assert_allclose(E, g[f"{env}_{integ}_E"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(A, g[f"{env}_{integ}_A"], rtol=1e-12, atol=1e-15)


def test_coefficients_and_time_vector(golden):
    for integ in ("Verlet", "BM4", "BM6", "RKN4"):
        np.testing.assert_array_equal(integrator_coeffs(integ, 0.05), golden["steps"][f"2d_{integ}_coeffs"])
    assert time_vector(882.5516, 0.05).size == 17651   # 8 cycles of 800 nm at dt = 0.05
    with pytest.raises(ValueError):
        integrator_coeffs("Euler", 0.1)
