"""ctypes bindings for the CPU oracle — TEST INFRASTRUCTURE ONLY.

Two CPU implementations of QuantumND's hot path are exposed with one interface:

* ``OracleCtx``: our C restatement (``oracle/qnd_oracle.c`` -> ``oracle/libqnd_oracle.so``).
* ``RefCtx``: the reference's own unmodified sources compiled against the
  single-rank MPI / FFTW-API shims (``oracle/Makefile`` -> ``oracle/_ref/``).
  Only present where the reference was compiled; ``ref_available()`` says so.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the shipped package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libqnd_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqnd_ref.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "libqnd_ref_fast.so")

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
_ll = C.c_longlong

_lib_oracle = None
_lib_ref = {}


def build_oracle() -> str:
    """Compile the restatement (gcc only; no reference sources needed)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return ORACLE_SO


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def _dptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _cstrs(names):
    arr = (C.c_char_p * max(1, len(names)))()
    for i, n in enumerate(names):
        arr[i] = n.encode()
    return arr


def _c128(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def oracle_lib():
    global _lib_oracle
    if _lib_oracle is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        L.or_create.restype = _vp
        L.or_create.argtypes = [C.c_int, C.POINTER(_ll), _dp, C.c_char_p, C.c_double, C.c_int]
        L.or_destroy.argtypes = [_vp]
        L.or_coeffs.argtypes = [C.c_char_p, C.c_double, _dp]
        L.or_set_potential_named.argtypes = [_vp, C.c_char_p]
        L.or_set_cap.argtypes = [_vp, C.c_double, C.c_double]
        L.or_set_vpot.argtypes = [_vp, _dp]
        L.or_set_vcap.argtypes = [_vp, _dp]
        L.or_set_gradv.argtypes = [_vp, C.c_int, _dp]
        L.or_set_mask_axis.argtypes = [_vp, C.c_int, _dp]
        L.or_set_threads.argtypes = [_vp, C.c_int]
        L.or_tables.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp]
        for fn in ("or_step_imag",):
            getattr(L, fn).argtypes = [_vp, _vp, _ll]
        L.or_step_length.argtypes = [_vp, _vp, _dp, _ll]
        L.or_step_velocity.argtypes = [_vp, _vp, _dp, _ll]
        L.or_to_p.argtypes = [_vp, _vp]
        L.or_to_r.argtypes = [_vp, _vp]
        L.or_apply_mask.argtypes = [_vp, _vp]
        L.or_gram_schmidt.argtypes = [_vp, C.c_int, C.POINTER(_vp), _dp]
        L.or_imag_loop_count.restype = _ll
        L.or_imag_loop_count.argtypes = [C.c_double, C.c_double]
        L.or_imag_state.argtypes = [_vp, C.POINTER(_vp), C.c_int, _ll]
        L.or_observable_count.argtypes = [_vp, C.c_int, C.POINTER(C.c_char_p)]
        L.or_observables.argtypes = [_vp, _vp, C.c_int, C.POINTER(C.c_char_p), _dp, _dp]
        L.or_energies.argtypes = [_vp, _vp, C.c_int, _dp]
        L.or_run_length.argtypes = [_vp, _vp, _dp, _ll, C.c_int, C.POINTER(C.c_char_p), _dp]
        L.or_run_velocity.argtypes = [_vp, _vp, _dp, _dp, _ll, C.c_int, C.POINTER(C.c_char_p), _dp]
        L.or_field.restype = _ll
        L.or_field.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_char_p), C.c_char_p,
                               C.c_double, C.c_double, _dp, _dp, _dp]
        L.or_field_at.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_char_p),
                                  C.c_double, _dp, _dp]
        L.or_fft.argtypes = [C.c_int, C.POINTER(_ll), _vp, _vp, C.c_int, C.c_int]
        _lib_oracle = L
    return _lib_oracle


def ref_available(fast: bool = False) -> bool:
    return os.path.exists(REF_FAST_SO if fast else REF_SO)


def ref_lib(fast: bool = False):
    key = "fast" if fast else "ieee"
    if key not in _lib_ref:
        path = REF_FAST_SO if fast else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (needs the reference sources: make -C oracle ref REF=<reference root>)")
        L = C.CDLL(path)
        L.ref_create.restype = _vp
        L.ref_create.argtypes = [C.c_int, C.POINTER(_ll), _dp, C.c_char_p, C.c_double, C.c_double, C.c_char_p,
                                 C.c_double, C.c_int]
        L.ref_destroy.argtypes = [_vp]
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_dim_hs.restype = _ll
        L.ref_dim_hs.argtypes = [_vp]
        L.ref_s.argtypes = [_vp]
        L.ref_coeffs.argtypes = [_vp, _dp]
        L.ref_tables.argtypes = [_vp, _dp, _dp, _dp]
        L.ref_set_vpot.argtypes = [_vp, _dp]
        L.ref_set_vcap.argtypes = [_vp, _dp]
        L.ref_step_imag.argtypes = [_vp, _vp, _ll]
        L.ref_step_length.argtypes = [_vp, _vp, _dp, _ll]
        L.ref_step_velocity.argtypes = [_vp, _vp, _dp, _ll]
        L.ref_gram_schmidt.argtypes = [_vp, C.c_int, C.POINTER(_vp)]
        L.ref_imag_loop_count.restype = _ll
        L.ref_imag_loop_count.argtypes = [C.c_double, C.c_double]
        L.ref_imag_state.argtypes = [_vp, C.POINTER(_vp), C.c_int, _ll]
        L.ref_energies.argtypes = [_vp, _vp, C.c_int, _dp]
        L.ref_observables.argtypes = [_vp, _vp, C.c_int, C.POINTER(C.c_char_p), _dp, _dp]
        L.ref_run_length.argtypes = [_vp, _vp, _dp, _ll, C.c_int, C.POINTER(C.c_char_p), _dp]
        L.ref_run_velocity.argtypes = [_vp, _vp, _dp, _dp, _ll, C.c_int, C.POINTER(C.c_char_p), _dp]
        L.ref_run_length_ext.argtypes = [_vp, _vp, _dp, _ll, C.c_int, C.POINTER(C.c_char_p), C.POINTER(_dp), _dp]
        L.ref_to_p.argtypes = [_vp, _vp]
        L.ref_final_observables.argtypes = [_vp, _vp, C.c_double, C.c_double, _dp, C.c_double, C.c_int, C.c_int,
                                            C.POINTER(C.c_char_p)]
        L.ref_to_r.argtypes = [_vp, _vp]
        L.ref_field.restype = _ll
        L.ref_field.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_char_p), C.c_char_p,
                                C.c_double, C.c_double, _dp, _dp, _dp]
        _lib_ref[key] = L
    return _lib_ref[key]


def obs_width(name: str, dim: int) -> int:
    """Values per observable name (calculate_observables.c:48-56, plus norm/accel)."""
    if name in ("PMD", "PED", "wavefunction", "none"):
        return 0
    if name in ("Lz", "energy", "norm"):
        return 1
    if name in ("dipole_r", "dipole_v", "accel"):
        return dim
    return 0


def coeffs(integrator: str, dt: float) -> np.ndarray:
    out = np.zeros(20)
    s = oracle_lib().or_coeffs(integrator.encode(), dt, _dptr(out))
    if s == 0:
        raise ValueError(f"unknown integrator {integrator}")
    return out[: 2 * s].copy()


def fft(x: np.ndarray, sign: int, nthreads: int = 1) -> np.ndarray:
    x = _c128(x)
    out = np.empty_like(x)
    nr = (_ll * x.ndim)(*x.shape)
    oracle_lib().or_fft(x.ndim, nr, _ptr(x), _ptr(out), sign, nthreads)
    return out


def imag_loop_count(T: float, dt: float) -> int:
    return int(oracle_lib().or_imag_loop_count(T, dt))


def field(dim, modes, integrator, dt, T, use_ref=False):
    """Sub-step field samples E, A [N_time, s, dim] and the time vector.

    ``modes`` is a list of dicts with keys intensity, lambda, ellipticity, cep, delay, duration, envelope."""
    nm = len(modes)
    arr = {k: _f64([m[k] for m in modes]) for k in ("intensity", "lambda", "ellipticity", "cep", "delay", "duration")}
    env = _cstrs([m["envelope"] for m in modes])
    L = ref_lib() if use_ref else oracle_lib()
    fn = L.ref_field if use_ref else L.or_field
    args = (dim, nm, _dptr(arr["intensity"]), _dptr(arr["lambda"]), _dptr(arr["ellipticity"]), _dptr(arr["cep"]),
            _dptr(arr["delay"]), _dptr(arr["duration"]), env, integrator.encode(), dt, T)
    nt = fn(*args, None, None, None)
    if nt < 0:
        raise ValueError("bad field specification")
    s = len(coeffs(integrator, dt)) // 2
    E = np.zeros((nt, s, dim))
    A = np.zeros((nt, s, dim))
    t = np.zeros(nt)
    fn(*args, _dptr(E), _dptr(A), _dptr(t))
    return E, A, t


def field_at(dim, modes, t):
    nm = len(modes)
    arr = {k: _f64([m[k] for m in modes]) for k in ("intensity", "lambda", "ellipticity", "cep", "delay", "duration")}
    env = _cstrs([m["envelope"] for m in modes])
    A = np.zeros(dim)
    E = np.zeros(dim)
    rc = oracle_lib().or_field_at(dim, nm, _dptr(arr["intensity"]), _dptr(arr["lambda"]),
                                  _dptr(arr["ellipticity"]), _dptr(arr["cep"]), _dptr(arr["delay"]),
                                  _dptr(arr["duration"]), env, t, _dptr(A), _dptr(E))
    if rc:
        raise ValueError("unknown envelope")
    return A, E


class _Base:
    dim: int
    shape: tuple

    def _check(self, psi):
        if not (isinstance(psi, np.ndarray) and psi.dtype == np.complex128 and psi.flags.c_contiguous
                and psi.size == int(np.prod(self.shape))):
            raise TypeError("psi must be a C-contiguous complex128 array of the grid's size")
        return psi


class OracleCtx(_Base):
    """The C restatement (oracle/qnd_oracle.c)."""

    def __init__(self, dim, nr, dr, integrator="BM4", dt=0.05, nthreads=None):
        self.L = oracle_lib()
        self.dim = dim
        self.shape = tuple(int(n) for n in nr)
        self.dr = tuple(float(d) for d in dr)
        nt = nthreads or os.cpu_count() or 1
        h = self.L.or_create(dim, (_ll * dim)(*self.shape), (C.c_double * dim)(*self.dr), integrator.encode(), dt, nt)
        if not h:
            raise ValueError("bad grid or integrator")
        self.h = h
        self.integrator = integrator
        self.dt = dt
        self.s = len(coeffs(integrator, dt)) // 2

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_destroy(self.h)
            self.h = None

    def set_potential(self, name):
        if self.L.or_set_potential_named(self.h, name.encode()):
            raise ValueError(f"unknown potential {name}")

    def set_cap(self, strength, length):
        self.L.or_set_cap(self.h, strength, length)

    def set_vpot(self, v):
        v = _f64(v)
        self.L.or_set_vpot(self.h, _dptr(v))

    def set_vcap(self, v):
        v = _f64(v)
        self.L.or_set_vcap(self.h, _dptr(v))

    def set_gradv(self, axis, g):
        g = _f64(g)
        self.L.or_set_gradv(self.h, axis, _dptr(g))

    def set_mask_axis(self, axis, m):
        if m is None:
            self.L.or_set_mask_axis(self.h, axis, None)
        else:
            m = _f64(m)
            self.L.or_set_mask_axis(self.h, axis, _dptr(m))

    def set_threads(self, n):
        self.L.or_set_threads(self.h, n)

    def tables(self):
        n = int(np.prod(self.shape))
        r = np.zeros(sum(self.shape))
        p = np.zeros(sum(self.shape))
        v, vc, k = np.zeros(n), np.zeros(n), np.zeros(n)
        self.L.or_tables(self.h, _dptr(r), _dptr(p), _dptr(v), _dptr(vc), _dptr(k))
        return r, p, v.reshape(self.shape), vc.reshape(self.shape), k.reshape(self.shape)

    def step_imag(self, psi, n=1):
        self.L.or_step_imag(self.h, _ptr(self._check(psi)), n)

    def step_length(self, psi_p, E, n=1):
        E = _f64(E)
        self.L.or_step_length(self.h, _ptr(self._check(psi_p)), _dptr(E), n)

    def step_velocity(self, psi, A, n=1):
        A = _f64(A)
        self.L.or_step_velocity(self.h, _ptr(self._check(psi)), _dptr(A), n)

    def to_p(self, psi):
        self.L.or_to_p(self.h, _ptr(self._check(psi)))

    def to_r(self, psi):
        self.L.or_to_r(self.h, _ptr(self._check(psi)))

    def apply_mask(self, psi):
        self.L.or_apply_mask(self.h, _ptr(self._check(psi)))

    def gram_schmidt(self, j, psis):
        arr = (_vp * len(psis))(*[p.ctypes.data for p in psis])
        norm = C.c_double(0.0)
        rc = self.L.or_gram_schmidt(self.h, j, arr, C.byref(norm))
        return rc, norm.value

    def imag_state(self, psis, j, nsteps):
        arr = (_vp * len(psis))(*[p.ctypes.data for p in psis])
        return self.L.or_imag_state(self.h, arr, j, nsteps)

    def energies(self, psi, n=2):
        out = np.zeros(n)
        self.L.or_energies(self.h, _ptr(self._check(psi)), n, _dptr(out))
        return out

    def observables(self, psi, names, alpha=None):
        nv = sum(obs_width(n, self.dim) for n in names)
        out = np.zeros(max(1, nv))
        al = _f64(alpha if alpha is not None else np.zeros(self.dim))
        rc = self.L.or_observables(self.h, _ptr(self._check(psi)), len(names), _cstrs(names), _dptr(al), _dptr(out))
        if rc < 0:
            raise ValueError("observable needs data that was not set (accel needs set_gradv)")
        return out[:nv]

    def run_length(self, psi_r, E, names):
        E = _f64(E)
        nsteps = E.shape[0]
        nv = sum(obs_width(n, self.dim) for n in names)
        out = np.zeros((nsteps, max(1, nv)))
        rc = self.L.or_run_length(self.h, _ptr(self._check(psi_r)), _dptr(E), nsteps, len(names), _cstrs(names),
                                  _dptr(out))
        if rc < 0:
            raise ValueError("observable evaluation failed")
        return out[:, :nv]

    def run_velocity(self, psi_r, A, alpha_steps, names):
        A = _f64(A)
        al = _f64(alpha_steps)
        nsteps = A.shape[0]
        nv = sum(obs_width(n, self.dim) for n in names)
        out = np.zeros((nsteps, max(1, nv)))
        rc = self.L.or_run_velocity(self.h, _ptr(self._check(psi_r)), _dptr(A), _dptr(al), nsteps, len(names),
                                    _cstrs(names), _dptr(out))
        if rc < 0:
            raise ValueError("observable evaluation failed")
        return out[:, :nv]


class RefCtx(_Base):
    """The reference's own sources (oracle/_ref/libqnd_ref.so), driven through ref_harness.c."""

    def __init__(self, dim, nr, dr, integrator="BM4", dt=0.05, potential="H_1D", cap=(0.0, 0.0), nthreads=None,
                 fast=False):
        self.L = ref_lib(fast)
        self.dim = dim
        self.shape = tuple(int(n) for n in nr)
        nt = nthreads or os.cpu_count() or 1
        self.h = self.L.ref_create(dim, (_ll * dim)(*self.shape), (C.c_double * dim)(*[float(d) for d in dr]),
                                   potential.encode(), float(cap[0]), float(cap[1]), integrator.encode(), dt, nt)
        self.s = self.L.ref_s(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def set_threads(self, n):
        self.L.ref_set_threads(n)

    def coeffs(self):
        out = np.zeros(2 * self.s)
        self.L.ref_coeffs(self.h, _dptr(out))
        return out

    def tables(self):
        n = int(np.prod(self.shape))
        v, vc, k = np.zeros(n), np.zeros(n), np.zeros(n)
        self.L.ref_tables(self.h, _dptr(v), _dptr(vc), _dptr(k))
        return v.reshape(self.shape), vc.reshape(self.shape), k.reshape(self.shape)

    def set_vpot(self, v):
        v = _f64(v)
        self.L.ref_set_vpot(self.h, _dptr(v))

    def set_vcap(self, v):
        v = _f64(v)
        self.L.ref_set_vcap(self.h, _dptr(v))

    def step_imag(self, psi, n=1):
        self.L.ref_step_imag(self.h, _ptr(self._check(psi)), n)

    def step_length(self, psi_p, E, n=1):
        E = _f64(E)
        self.L.ref_step_length(self.h, _ptr(self._check(psi_p)), _dptr(E), n)

    def step_velocity(self, psi, A, n=1):
        A = _f64(A)
        self.L.ref_step_velocity(self.h, _ptr(self._check(psi)), _dptr(A), n)

    def to_p(self, psi):
        self.L.ref_to_p(self.h, _ptr(self._check(psi)))

    def to_r(self, psi):
        self.L.ref_to_r(self.h, _ptr(self._check(psi)))

    def gram_schmidt(self, j, psis):
        arr = (_vp * len(psis))(*[p.ctypes.data for p in psis])
        self.L.ref_gram_schmidt(self.h, j, arr)

    def imag_state(self, psis, j, nsteps):
        arr = (_vp * len(psis))(*[p.ctypes.data for p in psis])
        self.L.ref_imag_state(self.h, arr, j, nsteps)

    def energies(self, psi, n=2):
        out = np.zeros(n)
        self.L.ref_energies(self.h, _ptr(self._check(psi)), n, _dptr(out))
        return out

    def observables(self, psi, names, alpha=None):
        nv = sum(obs_width(n, self.dim) for n in names)
        out = np.zeros(max(1, nv))
        al = _f64(alpha if alpha is not None else np.zeros(self.dim))
        self.L.ref_observables(self.h, _ptr(self._check(psi)), len(names), _cstrs(names), _dptr(al), _dptr(out))
        return out[:nv]

    def run_length(self, psi_r, E, names):
        E = _f64(E)
        nsteps = E.shape[0]
        nv = sum(obs_width(n, self.dim) for n in names)
        out = np.zeros((nsteps, max(1, nv)))
        self.L.ref_run_length(self.h, _ptr(self._check(psi_r)), _dptr(E), nsteps, len(names), _cstrs(names),
                              _dptr(out))
        return out[:, :nv]

    def run_length_ext(self, psi_r, E, names, gradv=None):
        """ref_run_length with the "norm" and "accel" extensions computed on the same states
        (gradv: dim arrays dV/dx_j in natural order, needed for "accel")."""
        E = _f64(E)
        nsteps = E.shape[0]
        nv = sum(obs_width(n, self.dim) for n in names)
        out = np.zeros((nsteps, max(1, nv)))
        gv = [_f64(g) for g in gradv] if gradv is not None else []
        arr = (C.POINTER(C.c_double) * max(1, self.dim))(*[_dptr(g) for g in gv]) if gv else None
        self.L.ref_run_length_ext(self.h, _ptr(self._check(psi_r)), _dptr(E), nsteps, len(names), _cstrs(names),
                                  arr, _dptr(out))
        return out[:, :nv]

    def run_velocity(self, psi_r, A, alpha_steps, names):
        A = _f64(A)
        al = _f64(alpha_steps)
        nsteps = A.shape[0]
        nv = sum(obs_width(n, self.dim) for n in names)
        out = np.zeros((nsteps, max(1, nv)))
        self.L.ref_run_velocity(self.h, _ptr(self._check(psi_r)), _dptr(A), _dptr(al), nsteps, len(names),
                                _cstrs(names), _dptr(out))
        return out[:, :nv]

    def final_observables(self, psi_r, r_mask, pr_max, de, ne, names=("PED", "PMD")):
        """Write_final_observables (io_functions.c:136-287) run in a scratch directory; returns the
        files it wrote as {"PED": [ne, 2] array, "PMD": (header dict, [count, 2] array)}."""
        import tempfile

        psi = self._check(psi_r.copy())
        prm = _f64(pr_max)
        out = {}
        cwd = os.getcwd()
        with tempfile.TemporaryDirectory() as tmp:
            os.chdir(tmp)
            try:
                self.L.ref_final_observables(self.h, _ptr(psi), float(r_mask[0]), float(r_mask[1]), _dptr(prm),
                                             float(de), int(ne), len(names), _cstrs(list(names)))
                if os.path.exists("PED.real"):
                    out["PED"] = np.loadtxt("PED.real").reshape(-1, 2)
                if os.path.exists("PMD.real"):
                    out["PMD"] = read_pmd("PMD.real")
            finally:
                os.chdir(cwd)
        return out


def grid_axes(shape, dr):
    """r axes (-L/2 + i dr) and p axes in FFT order (meshgrid.c:75-89)."""
    rs, ps = [], []
    for n, d in zip(shape, dr):
        rs.append(-0.5 * n * d + np.arange(n) * d)
        dp = 2.0 * np.pi / (n * d)
        k = np.arange(n)
        ps.append(np.where(k < n // 2, k, k - n) * dp)
    return rs, ps


def final_spectra_numpy(psi_r, dr, r_mask, pr_max, de, ne):
    """Restatement of Write_final_observables (io_functions.c:136-287) for the checks: the sin^2
    R_MASK mask, the unitary forward FFT (numpy's sign convention is FFTW's forward), the PED over
    the momenta with every |p_j| <= pr_max_j, and the packed PMD (|psi~|^2, arg psi~)."""
    shape = psi_r.shape
    dim = len(shape)
    rs, ps = grid_axes(shape, dr)
    R = np.sqrt(sum(x * x for x in np.meshgrid(*rs, indexing="ij")))
    f = np.where(R > r_mask[1], 1.0, 0.0)
    zone = (R >= r_mask[0]) & (R <= r_mask[1])
    f[zone] = np.sin(0.5 * np.pi * (R[zone] - r_mask[0]) / (r_mask[1] - r_mask[0])) ** 2
    q = np.fft.fftn(f * psi_r) / np.sqrt(psi_r.size)
    P = np.meshgrid(*ps, indexing="ij")
    kin = sum(0.5 * p * p for p in P)
    keep_ax = [np.abs(p) <= m for p, m in zip(ps, pr_max)]
    keep = np.ones(shape, dtype=bool)
    for j, k in enumerate(keep_ax):
        sl = [None] * dim
        sl[j] = slice(None)
        keep &= k[tuple(sl)]
    w = np.abs(q[keep]) ** 2
    E = np.arange(ne) * de
    norm = 1.0 / (2.0 * np.pi * de * de) ** (0.5 * dim)
    ped = np.array([np.sum(w * np.exp(-0.5 * (kin[keep] - e) ** 2 / (de * de))) * norm for e in E])
    pmd = np.stack([np.abs(q[keep]) ** 2, np.angle(q[keep])], axis=1)
    return ped, [int(k.sum()) for k in keep_ax], pmd


def read_pmd(path):
    """PMD.real (io_functions.c:236-281): text header, DATA_START, then (|psi~|^2, arg) doubles."""
    raw = open(path, "rb").read()
    k = raw.index(b"DATA_START\n") + len(b"DATA_START\n")
    head = {}
    for line in raw[:k].decode().splitlines():
        parts = line.split("\t")
        if parts[0] in ("NPR", "DP", "DIMENSION"):
            head[parts[0]] = [float(x) for x in parts[1:]]
    data = np.frombuffer(raw[k:], dtype=np.float64).reshape(-1, 2)
    return head, data


def seeded_state(shape, seed, normalise_dnr=None):
    """Seeded complex Gaussian N(0,1) state; normalised so sum|psi|^2 * dNr == 1 when dNr is given."""
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    if normalise_dnr is not None:
        psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * normalise_dnr)
    return np.ascontiguousarray(psi, dtype=np.complex128)


def smooth_state(shape, dr, seed, width=None):
    """Seeded smooth state: a Gaussian packet with random centre/momentum (band-limited, so the
    split-operator steps are well resolved), normalised with dNr."""
    rng = np.random.default_rng(seed)
    axes = []
    for n, d in zip(shape, dr):
        L = n * d
        axes.append(-0.5 * L + np.arange(n) * d)
    grids = np.meshgrid(*axes, indexing="ij")
    psi = np.ones(shape, dtype=np.complex128)
    for g, n, d in zip(grids, shape, dr):
        L = n * d
        w = width or L / 10
        x0 = rng.uniform(-L / 8, L / 8)
        k0 = rng.uniform(-1.0, 1.0)
        psi = psi * np.exp(-((g - x0) ** 2) / (2 * w * w) + 1j * k0 * g)
    dnr = float(np.prod(dr))
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * dnr)
    return np.ascontiguousarray(psi)
