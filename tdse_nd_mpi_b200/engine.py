"""Python mirror of QuantumND's hot-path interface over the C ABI (include/qnd.h).

The reference's internal API is a set of C functions on host arrays
(integrators.h:26-28, calculate_observables.h:28-29, QuantumND_imag.c:49). Here the
same operations act on device-resident states owned by a :class:`Grid` (the
MeshGrid + Integrator pair of the reference, meshgrid.h:12-36, integrators.h:17-21):

=============================================  ==================================
reference                                      this module
=============================================  ==================================
Initialize_meshgrid + Initialize_integrator    ``Grid(dim, nr, dr, integrator, dt)``
Integration_step_imag(Psi, grid, Int)          ``grid.integration_step_imag(psi, n)``
Integration_step_length(Psi, Et, dim, ...)     ``grid.integration_step_length(psi_p, E)``
Integration_step_velocity(Psi, At, dim, ...)   ``grid.integration_step_velocity(psi, A)``
Gram_Schmidt_orthonormalization(N, Psi, ...)   ``grid.gram_schmidt(states, j)``
Calculation_global_observables(...)            ``grid.observables(psi, names, alpha)``
Calculation_global_energies(Ej, N, Psi, ...)   ``grid.energies(psi, n)``
QuantumND_real.c length/velocity loops         ``grid.run_length`` / ``grid.run_velocity``
QuantumND_imag.c:182-185 loop body             ``grid.imag_propagate(states, j, n)``
=============================================  ==================================

Errors raise :class:`QndError` where the reference calls MPI_Abort.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import QND_FP64, QND_MIXED, QndError, check, lib  # noqa: F401  (QndError re-exported)

__all__ = ["Grid", "DeviceState", "QndError", "obs_width"]


def obs_width(name: str, dim: int) -> int:
    """Values per observable (calculate_observables.c:48-56, plus norm/accel)."""
    if name in ("Lz", "energy", "norm"):
        return 1
    if name in ("dipole_r", "dipole_v", "accel"):
        return dim
    return 0


def _names(names):
    arr = (C.c_char_p * max(1, len(names)))()
    for i, n in enumerate(names):
        arr[i] = n.encode()
    return arr


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _dptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class DeviceState:
    """One or more wavefunctions in device memory (complex128, or complex64 in mixed precision)."""

    def __init__(self, grid: "Grid", count: int = 1):
        self.grid = grid
        self.count = count
        p = C.c_void_p()
        check(lib().qnd_state_alloc(grid.h, count, C.byref(p)))
        self.ptr = p.value
        self.nbytes = grid.state_bytes

    def at(self, k: int) -> int:
        if not 0 <= k < self.count:
            raise IndexError(k)
        return self.ptr + k * self.nbytes

    def upload(self, host: np.ndarray, k: int = 0) -> "DeviceState":
        h = np.ascontiguousarray(host, dtype=np.complex128)
        if h.size != self.grid.n:
            raise ValueError(f"state has {h.size} values, grid has {self.grid.n}")
        check(lib().qnd_state_upload(self.grid.h, C.c_void_p(self.at(k)), h.view(np.float64).ctypes.data_as(
            C.POINTER(C.c_double))))
        return self

    def download(self, k: int = 0) -> np.ndarray:
        out = np.empty(self.grid.shape, dtype=np.complex128)
        check(lib().qnd_state_download(self.grid.h, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                       C.c_void_p(self.at(k))))
        return out

    def free(self) -> None:
        if self.ptr:
            check(lib().qnd_state_free(self.grid.h, C.c_void_p(self.ptr)))
            self.ptr = 0

    def __del__(self):
        try:
            if self.ptr and self.grid.h:
                lib().qnd_state_free(self.grid.h, C.c_void_p(self.ptr))
        except Exception:
            pass


def _ptr_of(x) -> int:
    if isinstance(x, DeviceState):
        return x.ptr
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):  # a torch tensor on the GPU
        return int(x.data_ptr())
    raise TypeError(f"not a device state: {type(x)}")


class Grid:
    """Grid + integrator context on one GPU (MeshGrid and Integrator of the reference)."""

    def __init__(self, dim, nr, dr, integrator="BM4", dt=0.05, precision="fp64"):
        self.dim = int(dim)
        self.shape = tuple(int(n) for n in nr)
        self.dr = tuple(float(d) for d in dr)
        if len(self.shape) != self.dim or len(self.dr) != self.dim:
            raise ValueError("nr and dr need DIMENSION entries")
        prec = {"fp64": QND_FP64, "mixed": QND_MIXED}[precision]
        self.precision = precision
        h = C.c_void_p()
        check(lib().qnd_ctx_create(self.dim, (C.c_int64 * self.dim)(*self.shape), (C.c_double * self.dim)(*self.dr),
                                   integrator.encode(), float(dt), prec, C.byref(h)))
        self.h = h.value
        n = C.c_int64()
        s = C.c_int()
        asc = (C.c_double * 20)()
        dnr, dnp = C.c_double(), C.c_double()
        check(lib().qnd_ctx_info(self.h, C.byref(n), C.byref(s), asc, C.byref(dnr), C.byref(dnp)))
        self.n, self.s = n.value, s.value
        self.as_scaled = np.array(asc[: 2 * self.s])
        self.dNr, self.dNp = dnr.value, dnp.value
        b = C.c_int64()
        check(lib().qnd_state_bytes(self.h, C.byref(b)))
        self.state_bytes = b.value
        self.integrator, self.dt = integrator, float(dt)

    # -- lifetime
    def close(self):
        if getattr(self, "h", None):
            check(lib().qnd_ctx_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        check(lib().qnd_ctx_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def synchronize(self):
        check(lib().qnd_synchronize(self.h))

    # -- axes (meshgrid.c:75-89)
    def axis_r(self, j):
        N, d = self.shape[j], self.dr[j]
        return -0.5 * d * N + np.arange(N) * d

    def axis_p(self, j):
        N, d = self.shape[j], self.dr[j]
        dp = 2 * np.pi / (d * N)
        i = np.arange(N)
        return np.where(i < N // 2, i * dp, (i - N) * dp)

    # -- potentials
    def set_potential(self, name_or_array):
        if isinstance(name_or_array, str):
            check(lib().qnd_set_potential_named(self.h, name_or_array.encode()))
        else:
            v = _f64(name_or_array)
            if v.size != self.n:
                raise ValueError("potential array size mismatch")
            check(lib().qnd_set_potential(self.h, _dptr(v)))

    def set_cap(self, strength, length):
        check(lib().qnd_set_cap(self.h, float(strength), float(length)))

    def set_vcap(self, vcap):
        v = None if vcap is None else _f64(vcap)
        check(lib().qnd_set_vcap(self.h, _dptr(v)))

    def set_gradv(self, axis, g):
        v = None if g is None else _f64(g)
        check(lib().qnd_set_gradv(self.h, int(axis), _dptr(v)))

    def set_mask_axis(self, axis, m):
        v = None if m is None else _f64(m)
        check(lib().qnd_set_mask_axis(self.h, int(axis), _dptr(v)))

    # -- states
    def state(self, host=None, count=1) -> DeviceState:
        st = DeviceState(self, count)
        if host is not None:
            st.upload(host)
        return st

    # -- hot path
    def integration_step_imag(self, psi, nsteps=1):
        check(lib().qnd_step_imag(self.h, C.c_void_p(_ptr_of(psi)), int(nsteps)))

    def _field(self, F, nsteps):
        F = _f64(F)
        if F.size != nsteps * self.s * self.dim:
            raise ValueError(f"field needs [nsteps][s={self.s}][dim={self.dim}] values")
        return F

    def integration_step_length(self, psi_p, E, nsteps=None):
        E = _f64(E)
        n = E.shape[0] if nsteps is None else nsteps
        E = self._field(E, n)
        check(lib().qnd_step_length(self.h, C.c_void_p(_ptr_of(psi_p)), _dptr(E), int(n)))

    def integration_step_velocity(self, psi, A, nsteps=None):
        A = _f64(A)
        n = A.shape[0] if nsteps is None else nsteps
        A = self._field(A, n)
        check(lib().qnd_step_velocity(self.h, C.c_void_p(_ptr_of(psi)), _dptr(A), int(n)))

    def to_p(self, psi):
        check(lib().qnd_to_p(self.h, C.c_void_p(_ptr_of(psi))))

    def to_r(self, psi):
        check(lib().qnd_to_r(self.h, C.c_void_p(_ptr_of(psi))))

    def nvalues(self, names):
        return sum(obs_width(n, self.dim) for n in names)

    def run_length(self, psi_r, E, names=()):
        E = _f64(E)
        n = E.shape[0]
        E = self._field(E, n)
        nv = self.nvalues(names)
        out = np.zeros((n, max(nv, 1)))
        check(lib().qnd_run_length(self.h, C.c_void_p(_ptr_of(psi_r)), _dptr(E), n, len(names), _names(names),
                                   _dptr(out)))
        return out[:, :nv]

    def run_velocity(self, psi_r, A, alpha=None, names=()):
        A = _f64(A)
        n = A.shape[0]
        A = self._field(A, n)
        nv = self.nvalues(names)
        al = _f64(alpha if alpha is not None else np.zeros((n, self.dim)))
        out = np.zeros((n, max(nv, 1)))
        check(lib().qnd_run_velocity(self.h, C.c_void_p(_ptr_of(psi_r)), _dptr(A), _dptr(al), n, len(names),
                                     _names(names), _dptr(out)))
        return out[:, :nv]

    def run_length_dev(self, psi_r, E_dev, nsteps, names, obs_dev):
        """Device-resident loop: E_dev / obs_dev are device addresses (or torch CUDA tensors)."""
        check(lib().qnd_run_length_dev(self.h, C.c_void_p(_ptr_of(psi_r)), C.c_void_p(_ptr_of(E_dev)), int(nsteps),
                                       len(names), _names(names),
                                       C.c_void_p(_ptr_of(obs_dev)) if obs_dev is not None else None))

    def set_profiling(self, enable: bool):
        check(lib().qnd_ctx_set_profiling(self.h, 1 if enable else 0))

    def get_profile(self, reset: bool = True):
        """(kernels launched, pass launches timed, summed pass milliseconds); synchronises."""
        k, p, ms = C.c_int64(), C.c_int64(), C.c_double()
        check(lib().qnd_ctx_get_profile(self.h, C.byref(k), C.byref(p), C.byref(ms), 1 if reset else 0))
        return k.value, p.value, ms.value

    def _ptr_array(self, states):
        ptrs = [_ptr_of(s) for s in states]
        return (C.c_void_p * len(ptrs))(*ptrs)

    def gram_schmidt(self, states, j):
        """states: list of device states (or addresses); returns ||v||^2 dNr."""
        norm = C.c_double()
        check(lib().qnd_gram_schmidt(self.h, self._ptr_array(states), int(j), C.byref(norm)))
        return norm.value

    def imag_propagate(self, states, j, nsteps):
        check(lib().qnd_imag_propagate(self.h, self._ptr_array(states), int(j), int(nsteps)))

    def observables(self, psi_r, names, alpha=None):
        nv = self.nvalues(names)
        out = np.zeros(max(nv, 1))
        al = None if alpha is None else _f64(alpha)
        check(lib().qnd_observables(self.h, C.c_void_p(_ptr_of(psi_r)), len(names), _names(names), _dptr(al),
                                    _dptr(out)))
        return out[:nv]

    def final_spectra(self, psi_r, r_mask, pr_max, de, ne):
        """Write_final_observables (io_functions.c:136-287) on the device: returns (ped [ne], npr [dim],
        pmd [prod(npr), 2]) for the R_MASK r_mask, momentum limits pr_max and the PED grid j*de."""
        prm = _f64(np.broadcast_to(np.asarray(pr_max, dtype=np.float64), (self.dim,)).copy())
        npr = (C.c_int64 * self.dim)()
        check(lib().qnd_final_spectra(self.h, C.c_void_p(_ptr_of(psi_r)), float(r_mask[0]), float(r_mask[1]),
                                      _dptr(prm), float(de), int(ne), None, npr, None))
        counts = [int(v) for v in npr]
        ped = np.zeros(max(int(ne), 1))
        pmd = np.zeros((int(np.prod(counts)), 2))
        check(lib().qnd_final_spectra(self.h, C.c_void_p(_ptr_of(psi_r)), float(r_mask[0]), float(r_mask[1]),
                                      _dptr(prm), float(de), int(ne), _dptr(ped), npr, _dptr(pmd)))
        return ped[:int(ne)], counts, pmd

    def energies(self, psi_r, n=2):
        out = np.zeros(n)
        check(lib().qnd_energies(self.h, C.c_void_p(_ptr_of(psi_r)), int(n), _dptr(out)))
        return out

    # -- differentiation
    def adjoint_length(self, psi0, E, weight, checkpoint=50, psiT=None):
        """J = dNr sum w |psi_T|^2 after the length-gauge steps with field samples E [nsteps, s, dim]
        from psi0 (not modified), and dJ/dE [nsteps, s, dim] by the adjoint (qnd_adjoint_length)."""
        return self._adjoint(lib().qnd_adjoint_length, psi0, E, weight, checkpoint, psiT)

    def adjoint_velocity(self, psi0, A, weight, checkpoint=50, psiT=None):
        """The same for velocity-gauge steps with vector-potential samples A: J and dJ/dA
        (qnd_adjoint_velocity)."""
        return self._adjoint(lib().qnd_adjoint_velocity, psi0, A, weight, checkpoint, psiT)

    def _adjoint(self, fn, psi0, F, weight, checkpoint, psiT):
        F = _f64(F)
        n = F.shape[0]
        F = self._field(F, n)
        w = _f64(np.broadcast_to(np.asarray(weight, dtype=np.float64), self.shape).copy())
        grad = np.zeros((n, self.s, self.dim))
        J = C.c_double()
        check(fn(self.h, C.c_void_p(_ptr_of(psi0)), _dptr(F), int(n), _dptr(w), int(checkpoint), C.byref(J), _dptr(grad),
                 None if psiT is None else C.c_void_p(_ptr_of(psiT))))
        return J.value, grad

    # -- laser field and initial state on the device
    @staticmethod
    def _modes(modes):
        """Modes as the reference's params keys (intensity [W/cm^2], lambda [nm], ellipticity, cep,
        delay, duration, envelope), converted as parameters.c:805-810."""
        from ._lib import QND_ENV, LaserMode

        arr = (LaserMode * max(1, len(modes)))()
        for k, m in enumerate(modes):
            if m["envelope"] not in QND_ENV:
                raise ValueError(f"Unknown envelope: {m['envelope']}")
            arr[k] = LaserMode(45.5637639947958 / m["lambda"], 5.33803e-9 * np.sqrt(m["intensity"]),
                               m["ellipticity"], m["cep"], m["delay"], m["duration"], QND_ENV[m["envelope"]])
        return arr

    def field_samples(self, modes, nsteps):
        """E, A [nsteps, s, dim] at the sub-step times and alpha [nsteps, dim] = A(i dt), computed on
        the device (Initialize_field_vectors, integrators.c:74-101)."""
        E = np.zeros((nsteps, self.s, self.dim))
        A = np.zeros((nsteps, self.s, self.dim))
        al = np.zeros((nsteps, self.dim))
        check(lib().qnd_field_samples(self.h, len(modes), self._modes(modes), int(nsteps), E.ctypes.data,
                                      A.ctypes.data, al.ctypes.data, 0))
        return E, A, al

    def field_samples_dev(self, modes, nsteps, E_dev=None, A_dev=None, alpha_dev=None):
        """The same into device buffers (torch tensors or pointers), asynchronously on the stream."""
        ptr = lambda x: None if x is None else _ptr_of(x)
        check(lib().qnd_field_samples(self.h, len(modes), self._modes(modes), int(nsteps), ptr(E_dev), ptr(A_dev),
                                      ptr(alpha_dev), 1))

    def embed(self, psi, src, coeff=1.0, accumulate=False):
        """psi <- (psi if accumulate else 0) + coeff * src centred on this grid (Read_wavefunction_MPI's
        centring and superposition, io_functions.c:292-459); src is a host complex128 array."""
        src = np.ascontiguousarray(src, dtype=np.complex128)
        if src.ndim != self.dim:
            raise ValueError("src needs DIMENSION axes")
        nr = (C.c_int64 * self.dim)(*src.shape)
        c = complex(coeff)
        check(lib().qnd_state_embed(self.h, C.c_void_p(_ptr_of(psi)), src.ctypes.data_as(C.POINTER(C.c_double)), nr,
                                    c.real, c.imag, int(bool(accumulate))))
