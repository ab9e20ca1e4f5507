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


REAL_DRIVER = os.path.join(ROOT, "tdse_nd_mpi_b200", "QuantumND_real")
REF_REAL = os.path.join(ROOT, "oracle", "_ref", "QuantumND_real")

PARAMS_REAL = """OUTPUT_IMAG\toutput.imag
NR\t\t512
N_STATES\t2
J_STATES\t1 2
COEFFS_STATES\t1. 0.5+0.5j
CAP\t\t.1 20.
GAUGE\t\t{gauge}
N_MODES\t\t2
INTENSITY\t1.e13 5.e12
LAMBDA\t\t800 400
ELLIPTICITY\t0. 0.
CEP\t\t0. 1.
DELAY\t\t0. 10.
ENVELOPE\tcos2 trapz
DURATION\t40. 30.
INTEGRATOR\tBM4
DT\t\t.1
TINTEGRATION\t50
DT_SAVE\t\t1.
N_OBSERVABLES\t6
OBSERVABLES\tdipole_r dipole_v energy PED PMD wavefunction
P_MAX\t\t3.
R_MASK\t\t5. 10.
DE\t\t.05
NE\t\t40
"""


def test_real_driver_rejects_bad_parameter_files(driver, tmp_path):
    from tdse_nd_mpi_b200.build import build_drivers

    build_drivers()
    (tmp_path / "output.imag").write_bytes(b"DIMENSION\t1\nN_STATES\t2\nNR\t256\nDR\t0.2\nPOTENTIAL\tH_1D\n"
                                            b"E\t\t-0.5\t-0.1\nDE\t0\t0\nPSI\n" + bytes(16 * 512))
    p = tmp_path / "params.real"
    p.write_text(PARAMS_REAL.format(gauge="length") + "FOO 1\n")
    r = subprocess.run([REAL_DRIVER, str(p)], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 1 and "Unknown parameter: FOO" in r.stdout
    p.write_text(PARAMS_REAL.format(gauge="length"))
    r = subprocess.run([REAL_DRIVER, str(p), "NR", "256"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 1 and "Unrecognized parameter key 'NR'" in r.stderr


def _text_table(path):
    rows = [line.split() for line in open(path).read().splitlines() if line.strip()]
    return rows[0], np.array(rows[1:], dtype=float)


@pytest.mark.gpu
@pytest.mark.parametrize("gauge,nr", [("length", 512), ("velocity", 512), ("length", 16384)])
def test_real_driver_outputs_match_reference_executable(driver, tmp_path, gauge, nr):
    """QuantumND_real end to end (two-state superposition read from output.imag onto a larger grid,
    two laser modes, CAP, observables every step, PED/PMD/wavefunction) against the reference's
    executable on the same inputs: every output file. NR 16384: a 1-D axis past one pass (the
    four-step transform)."""
    from oracle import oracle as O

    if not (os.path.exists(REF_IMAG) and os.path.exists(REF_REAL)):
        pytest.skip("reference executables not built")
    seed = tmp_path / "seed"
    seed.mkdir()
    assert run(REF_IMAG, PARAMS.replace("TINTEGRATION \t30", "TINTEGRATION \t20"), seed).returncode == 0
    out = {}
    for who, exe in (("ours", REAL_DRIVER), ("ref", REF_REAL)):
        d = tmp_path / who
        d.mkdir()
        (d / "output.imag").write_bytes((seed / "output.imag").read_bytes())
        (d / "params.real").write_text(PARAMS_REAL.format(gauge=gauge).replace("NR\t\t512", f"NR\t\t{nr}"))
        r = subprocess.run([exe, "params.real"], cwd=d, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, (who, r.stdout[-2000:], r.stderr[-2000:])
        out[who] = d
    h1, o1 = _text_table(out["ours"] / "observables.real")
    h2, o2 = _text_table(out["ref"] / "observables.real")
    assert h1 == h2 and o1.shape == o2.shape
    np.testing.assert_allclose(o1, o2, rtol=1e-9, atol=1e-12)
    for f in ("electric_field.real", "vector_potential.real"):
        a = np.loadtxt(out["ours"] / f)
        b = np.loadtxt(out["ref"] / f)
        np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-15)
    ped1, ped2 = np.loadtxt(out["ours"] / "PED.real"), np.loadtxt(out["ref"] / "PED.real")
    np.testing.assert_allclose(ped1, ped2, rtol=0, atol=1e-10 * np.abs(ped2[:, 1]).max())
    (hd1, d1), (hd2, d2) = O.read_pmd(out["ours"] / "PMD.real"), O.read_pmd(out["ref"] / "PMD.real")
    assert hd1 == hd2 and d1.shape == d2.shape
    np.testing.assert_allclose(d1[:, 0], d2[:, 0], rtol=0, atol=1e-10 * d2[:, 0].max())
    w1 = open(out["ours"] / "wavefunction.real", "rb").read()
    w2 = open(out["ref"] / "wavefunction.real", "rb").read()
    k1, k2 = w1.index(b"PSI_BINARY_START\n") + 17, w2.index(b"PSI_BINARY_START\n") + 17
    assert w1[:k1] == w2[:k2]
    p1, p2 = np.frombuffer(w1[k1:], np.complex128), np.frombuffer(w2[k2:], np.complex128)
    assert np.linalg.norm(p1 - p2) / np.linalg.norm(p2) < 1e-9


# The reference's example inputs (its params.imag and params.real), as a user would run them;
# TINTEGRATION is shortened through the drivers' own KEY VALUE overrides so that the reference
# executable finishes in seconds on the host.
EXAMPLE_IMAG = """OUTPUT_IMAG \toutput.imag

DIMENSION\t1
N_STATES \t4

POTENTIAL\tH_1D

DR\t\t.2
NR\t\t512

INTEGRATOR \tBM4
DT \t\t.1
TINTEGRATION \t1e3
"""

EXAMPLE_REAL = """OUTPUT_IMAG\toutput.imag

NR \t\t262144

N_STATES \t1
J_STATES \t1
COEFFS_STATES\t1.

CAP \t\t.1\t20.

GAUGE \t\tlength
N_MODES \t10
INTENSITY \t1.e11 1.e11 1.e11 1.e11 1.e11 1.e11 1.e11 1.e11 1.e11 1.e11
LAMBDA \t\t800 88.8888888888889 72.7272727272727 61.5384615384615 53.3333333333333 47.0588235294118 42.1052631578947 38.0952380952381 34.7826086956522 32
ELLIPTICITY \t0. 0. 0. 0. 0. 0. 0. 0. 0. 0.
CEP \t\t0. 0. 0. 0. 0. 0. 0. 0. 0. 0.
DELAY \t\t0. 0. 0. 0. 0. 0. 0. 0. 0. 0.
ENVELOPE \tcos2 cos2 cos2 cos2 cos2 cos2 cos2 cos2 cos2 cos2
DURATION \t10000. 10000. 10000. 10000. 10000. 10000. 10000. 10000. 10000. 10000.

INTEGRATOR \tBM4
DT \t\t.1
TINTEGRATION \t15000.

DT_SAVE \t1.
N_OBSERVABLES \t3
OBSERVABLES \tPED PMD wavefunction

P_MAX \t\t10.
R_MASK \t\t20. 30.
DE \t\t.01
NE \t\t200
"""


@pytest.mark.gpu
def test_reference_example_inputs_end_to_end(driver, tmp_path):
    """The reference's own example: imaginary time on 512 points (4 states), then the real-time run
    on NR 262144 (a four-step long axis) under a 10-mode field, writing PED, PMD and the
    wavefunction; both stages shortened by TINTEGRATION overrides. Every file against the
    reference's executables on the same inputs."""
    from oracle import oracle as O

    if not (os.path.exists(REF_IMAG) and os.path.exists(REF_REAL)):
        pytest.skip("reference executables not built")
    out = {}
    for who, imag, real in (("ours", DRIVER, REAL_DRIVER), ("ref", REF_IMAG, REF_REAL)):
        d = tmp_path / who
        d.mkdir()
        r = run(imag, EXAMPLE_IMAG, d, "TINTEGRATION", "20")
        assert r.returncode == 0, (who, r.stdout[-1500:], r.stderr[-1500:])
        (d / "params.real").write_text(EXAMPLE_REAL)
        r = subprocess.run([real, "params.real", "TINTEGRATION", "3"], cwd=d, capture_output=True, text=True,
                           timeout=900)
        assert r.returncode == 0, (who, r.stdout[-1500:], r.stderr[-1500:])
        out[who] = d
    t1, h1, psi1 = read_output_imag(out["ours"] / "output.imag")
    t2, h2, psi2 = read_output_imag(out["ref"] / "output.imag")
    np.testing.assert_allclose(np.array(h1["E"], float), np.array(h2["E"], float), rtol=1e-11)
    assert np.linalg.norm(psi1 - psi2) / np.linalg.norm(psi2) < 1e-10
    for f in ("electric_field.real", "vector_potential.real"):
        np.testing.assert_allclose(np.loadtxt(out["ours"] / f), np.loadtxt(out["ref"] / f), rtol=1e-12, atol=1e-15)
    ped1, ped2 = np.loadtxt(out["ours"] / "PED.real"), np.loadtxt(out["ref"] / "PED.real")
    np.testing.assert_allclose(ped1, ped2, rtol=0, atol=1e-10 * np.abs(ped2[:, 1]).max())
    (hd1, d1), (hd2, d2) = O.read_pmd(out["ours"] / "PMD.real"), O.read_pmd(out["ref"] / "PMD.real")
    assert hd1 == hd2 and d1.shape == d2.shape
    # after 3 a.u. nothing has reached R_MASK: the spectra are at the FP64 rounding floor of a
    # normalised state (|psi~|^2 ~ 1e-21), so compare the amplitudes to an absolute 1e-13
    np.testing.assert_allclose(np.sqrt(d1[:, 0]), np.sqrt(d2[:, 0]), rtol=0, atol=1e-13)
    w1 = open(out["ours"] / "wavefunction.real", "rb").read()
    w2 = open(out["ref"] / "wavefunction.real", "rb").read()
    k1, k2 = w1.index(b"PSI_BINARY_START\n") + 17, w2.index(b"PSI_BINARY_START\n") + 17
    assert w1[:k1] == w2[:k2]
    p1, p2 = np.frombuffer(w1[k1:], np.complex128), np.frombuffer(w2[k2:], np.complex128)
    assert p1.size == 262144 and np.linalg.norm(p1 - p2) / np.linalg.norm(p2) < 1e-9
