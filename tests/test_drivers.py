"""The drop-in QuantumND_imag driver (tdse_nd_mpi_b200/drivers/): parameter-file checks on the CPU
(they run before any GPU call), output.imag against the reference's own executable on the GPU."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tdse_nd_mpi_b200", "QuantumND_imag")
REF_IMAG = os.path.join(ROOT, "oracle", "_ref", "QuantumND_imag")

PARAMS = """OUTPUT_IMAG \toutput.imag

DIMENSION\t1
N_STATES \t3

POTENTIAL\tH_1D

DR\t\t.2
NR\t\t256

INTEGRATOR \tBM4
DT \t\t.1
TINTEGRATION \t30
"""


@pytest.fixture(scope="module")
def driver(qnd_lib):
    from tdse_nd_mpi_b200.build import build_drivers

    build_drivers()
    assert os.path.exists(DRIVER)
    return DRIVER


def run(exe, params, tmp_path, *extra):
    p = tmp_path / "params.imag"
    p.write_text(params)
    return subprocess.run([exe, str(p), *extra], cwd=tmp_path, capture_output=True, text=True, timeout=600)


@pytest.mark.parametrize("text,msg", [
    ("FOO 1\n" + PARAMS, "Unknown parameter: FOO"),
    (PARAMS + "FOO 1\n", "found extra, unrecognized token 'FOO'"),   # as the reference: the previous key sees it
    (PARAMS.replace("NR\t\t256", "NR\t\t256 512"), "expected exactly 1 argument(s), but found extra"),
    (PARAMS.replace("NR\t\t256", "NR\t\t300"), "must be a power of 2"),
    (PARAMS.replace("DIMENSION\t1", ""), "The dimension is not specified"),
])
def test_driver_rejects_bad_parameter_files(driver, tmp_path, text, msg):
    r = run(driver, text, tmp_path)
    assert r.returncode == 1
    assert msg in r.stdout + r.stderr


def test_driver_rejects_unknown_override(driver, tmp_path):
    r = run(driver, PARAMS, tmp_path, "NR", "512")
    assert r.returncode == 1 and "Unrecognized parameter key 'NR'" in r.stderr


def read_output_imag(path):
    raw = open(path, "rb").read()
    k = raw.index(b"PSI\n") + 4
    head = {}
    for line in raw[:k].decode().splitlines():
        parts = line.split("\t")
        head[parts[0]] = [x for x in parts[1:] if x != ""]
    return raw[:k].decode(), head, np.frombuffer(raw[k:], dtype=np.complex128)


@pytest.mark.gpu
def test_output_imag_matches_reference_executable(driver, tmp_path):
    if not os.path.exists(REF_IMAG):
        pytest.skip("reference executable not built")
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    r1 = run(driver, PARAMS, ours)
    assert r1.returncode == 0, r1.stderr
    r2 = run(REF_IMAG, PARAMS, ref)
    assert r2.returncode == 0, r2.stderr
    t1, h1, psi1 = read_output_imag(ours / "output.imag")
    t2, h2, psi2 = read_output_imag(ref / "output.imag")
    for key in ("DIMENSION", "N_STATES", "NR", "DR", "POTENTIAL"):
        assert h1[key] == h2[key], key
    np.testing.assert_allclose(np.array(h1["E"], float), np.array(h2["E"], float), rtol=1e-11)
    np.testing.assert_allclose(np.array(h1["DE"], float), np.array(h2["DE"], float), atol=1e-9)
    assert t1.count("\n") == t2.count("\n") and psi1.shape == psi2.shape
    assert np.linalg.norm(psi1 - psi2) / np.linalg.norm(psi2) < 1e-10
    for line in ("PROGRAM IMAGINARY-TIME PROPAGATION", "> eigenfunction 3:", "# The code ended successfully"):
        assert line in r1.stdout
