"""CPU checks of the C ABI boundary (no compute calls that need a GPU)."""
import ctypes as C
import os
import re

import pytest

from tdse_nd_mpi_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "qnd.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qnd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(qnd_lib):
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(qnd_lib, s)]
    assert not missing, missing
    # the Python mirror binds exactly the declared surface
    assert set(syms) == set(_lib.SIGNATURES)


def test_library_is_sm100a_cuda_build(qnd_lib):
    assert b"sm_100a" in qnd_lib.qnd_version()
    nm = os.popen(f"nm -D --defined-only {_lib.LIB_PATH}").read()
    for s in declared_symbols():
        assert re.search(rf"\bT {s}\b", nm), s


def _create(dim, nr, dr, integ="BM4", dt=0.05, prec=0):
    h = C.c_void_p()
    rc = _lib.lib().qnd_ctx_create(dim, (C.c_int64 * dim)(*nr), (C.c_double * dim)(*dr), integ.encode(), dt, prec,
                                   C.byref(h))
    return rc, h


@pytest.mark.parametrize(
    "args, code",
    [
        ((1, (100,), (0.1,)), _lib.QND_EINVAL),            # not a power of two (parameters.c:72-76)
        ((1, (1 << 25,), (0.1,)), _lib.QND_EUNSUPPORTED),  # beyond the longest 1-D axis (2^24)
        ((2, (1 << 25, 2), (0.1, 0.1)), _lib.QND_EUNSUPPORTED),  # beyond the longest axis (2^24)
        ((7, (2,) * 7, (1,) * 7), _lib.QND_EINVAL),        # beyond the 6 dimensions built
        ((1, (64,), (-0.1,)), _lib.QND_EINVAL),
    ],
)
def test_ctx_create_rejects_bad_grids(qnd_lib, args, code):
    rc, h = _create(*args)
    assert rc == code
    assert not h.value
    assert qnd_lib.qnd_last_error()


def test_unknown_integrator_message_matches_reference(qnd_lib):
    rc, _ = _create(1, (64,), (0.1,), integ="Euler")
    assert rc == _lib.QND_EINVAL
    assert b"Unknown integrator: Euler" in qnd_lib.qnd_last_error()   # integrators.c:58


def test_null_arguments_are_errors_not_crashes(qnd_lib):
    assert qnd_lib.qnd_ctx_create(1, None, None, b"BM4", 0.1, 0, None) == _lib.QND_EINVAL
    assert qnd_lib.qnd_step_imag(None, None, 1) == _lib.QND_EINVAL
    assert qnd_lib.qnd_ctx_destroy(None) == _lib.QND_OK


def test_no_gpu_fails_loudly(qnd_lib):
    """On a machine without a GPU a valid context cannot be created: an error, never a CPU fallback."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    rc, h = _create(2, (16, 16), (0.2, 0.2))
    assert rc == _lib.QND_ECUDA
    assert b"cuda" in qnd_lib.qnd_last_error().lower()


def test_missing_library_raises(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()
