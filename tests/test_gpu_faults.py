"""Failure paths, with every fault made on the host (no GPU fault, trap or hang):

* a device allocation refused through the QND_FAIL_ALLOC_ABOVE hook: a QND_ENOMEM status with the
  request's size, and the context works again once allocations succeed;
* a zero initial state in imaginary time: the Gram-Schmidt norm collapse (QuantumND_imag.c:297-304)
  as QND_ENORM;
* a truncated OUTPUT_IMAG: the real-time driver stops with the reference's read error and exit 1;
* a NaN in the input state under the debug scan (QND_CHECK_FINITE=1): QND_ENONFINITE;
* the bounded wait of a strided pass for its TMA box loads running out (QND_TMA_WAIT_TRIES=0 makes
  the first wait give up at once, while the second, draining wait keeps its full limit so that every
  load lands before the CTA leaves): QND_ECUDA, and the CTAs concerned leave their lines untouched.
"""
import sys
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_refused_allocation_is_enomem_and_the_context_recovers(qnd_lib, monkeypatch):
    from tdse_nd_mpi_b200 import Grid, QndError

    shape, dr = (1024, 1024), (0.2, 0.2)
    grid = Grid(2, shape, dr, "BM4", 0.05)
    grid.set_potential("H_2D")
    st = grid.state(O.smooth_state(shape, dr, 1))
    monkeypatch.setenv("QND_FAIL_ALLOC_ABOVE", str(1 << 20))
    with pytest.raises(QndError) as ei:
        grid.energies(st, 2)             # needs two 16.8 MB scratch states
    assert ei.value.code == 3 and "QND_FAIL_ALLOC_ABOVE" in str(ei.value)
    monkeypatch.delenv("QND_FAIL_ALLOC_ABOVE")
    got = grid.energies(st, 2)
    fresh = Grid(2, shape, dr, "BM4", 0.05)
    fresh.set_potential("H_2D")
    np.testing.assert_array_equal(got, fresh.energies(fresh.state(O.smooth_state(shape, dr, 1)), 2))


def test_zero_initial_state_collapses_in_imaginary_time(qnd_lib):
    from tdse_nd_mpi_b200 import Grid, QndError

    grid = Grid(1, (256,), (0.2,), "BM4", 0.05)
    grid.set_potential("H_1D")
    states = [grid.state(np.zeros(256, dtype=np.complex128))]
    with pytest.raises(QndError) as ei:
        grid.imag_propagate(states, 0, 3)
    assert ei.value.code == 4 and "norm" in str(ei.value)


def test_truncated_output_imag_stops_the_real_driver(qnd_lib, tmp_path):
    from tdse_nd_mpi_b200.build import build_drivers

    build_drivers()
    exe = os.path.join(ROOT, "tdse_nd_mpi_b200", "QuantumND_real")
    head = b"DIMENSION\t1\nN_STATES\t2\nNR\t256\nDR\t0.2\nPOTENTIAL\tH_1D\nE\t\t-0.5\t-0.1\nDE\t0\t0\nPSI\n"
    (tmp_path / "output.imag").write_bytes(head + bytes(16 * 300))   # state 2 of 256 points is cut short
    params = ("OUTPUT_IMAG\toutput.imag\nNR\t\t512\nN_STATES\t2\nJ_STATES\t1 2\nCOEFFS_STATES\t1. 1.\nCAP\t\t.1 20.\n"
              "GAUGE\t\tlength\nN_MODES\t\t1\nINTENSITY\t1.e13\nLAMBDA\t\t800\nELLIPTICITY\t0.\nCEP\t\t0.\n"
              "DELAY\t\t0.\nENVELOPE\tcos2\nDURATION\t40.\nINTEGRATOR\tBM4\nDT\t\t.1\nTINTEGRATION\t2\n"
              "DT_SAVE\t\t1.\nN_OBSERVABLES\t1\nOBSERVABLES\tdipole_r\nP_MAX\t\t3.\nR_MASK\t\t5. 10.\nDE\t\t.05\n"
              "NE\t\t40\n")
    (tmp_path / "params.real").write_text(params)
    r = subprocess.run([exe, "params.real"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 1
    assert "MPI Read Error during chunking" in r.stdout + r.stderr


def test_nonfinite_state_is_reported_when_checking(qnd_lib, monkeypatch):
    """QND_CHECK_FINITE=1 (the debug scan): a NaN planted in the host input makes the stepping call
    return QND_ENONFINITE; a clean state passes; without the switch nothing is checked."""
    from tdse_nd_mpi_b200 import Grid, QndError

    shape, dr = (64, 64), (0.3, 0.3)
    grid = Grid(2, shape, dr, "BM4", 0.05)
    grid.set_potential("H_2D")
    clean = O.smooth_state(shape, dr, 3)
    bad = clean.copy()
    bad[10, 20] = complex(np.nan, 0.0)
    E = np.zeros((2, grid.s, 2))
    grid.run_length(grid.state(bad), E, ["norm"])   # unchecked: NaN propagates silently
    monkeypatch.setenv("QND_CHECK_FINITE", "1")
    grid.run_length(grid.state(clean), E, ["norm"])
    with pytest.raises(QndError) as ei:
        grid.run_length(grid.state(bad), E, ["norm"])
    assert ei.value.code == 6 and "NaN or Inf" in str(ei.value)
    with pytest.raises(QndError):
        grid.integration_step_imag(grid.state(bad), 1)


_TMA_SCRIPT = r"""
import os, sys
import numpy as np
sys.path.insert(0, {root!r})
from tdse_nd_mpi_b200 import Grid, QndError
from oracle import oracle as O
shape, dr = (1024, 1024), (0.2, 0.2)
g = Grid(2, shape, dr, "BM4", 0.05)
psi0 = O.smooth_state(shape, dr, 2)
st = g.state(psi0)
os.environ["QND_TMA_WAIT_TRIES"] = "0"
g.to_p(st)                       # contiguous pass, then the strided pass (TMA boxes) that gives up
try:
    g.synchronize()
    print("NO_ERROR")
except QndError as e:
    print("CODE", e.code, "ran out" in str(e))
got = st.download()              # the flag was cleared by the report
# only the contiguous axis was transformed: the strided CTAs stored nothing
want = np.fft.fft(psi0, axis=1) / np.sqrt(1024.0)
print("HALF_ERR", np.linalg.norm(got - want) / np.linalg.norm(want))
del os.environ["QND_TMA_WAIT_TRIES"]
st.upload(psi0)
g.to_p(st)
g.synchronize()
want = np.fft.fft2(psi0) / 1024.0
print("FULL_ERR", np.linalg.norm(st.download() - want) / np.linalg.norm(want))
"""


def test_tma_wait_that_runs_out_is_reported_and_leaves_the_lines(qnd_lib):
    """QND_TMA_WAIT_TRIES=0 (a host-side setting, read at each launch): every strided CTA of a 1024^2
    FP64 unitary transform gives up on its first wait, drains its loads with the second, raises the
    error flag and stores nothing. The next synchronising call returns QND_ECUDA ("ran out"); the
    state then holds the contiguous axis' transform alone; without the setting the same context
    transforms correctly. Run in a child process with the staging fixed to TMA boxes (QND_TUNE=0:
    1024-point strided lines use them), so that no staging measurement sees the setting."""
    env = dict(os.environ, QND_TUNE="0")
    env.pop("QND_NO_TMA", None)
    r = subprocess.run([sys.executable, "-c", _TMA_SCRIPT.format(root=ROOT)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())
    assert out.get("CODE") == "2 True", r.stdout
    assert float(out["HALF_ERR"]) < 1e-13, r.stdout
    assert float(out["FULL_ERR"]) < 1e-13, r.stdout
