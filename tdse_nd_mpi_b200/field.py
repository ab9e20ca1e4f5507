"""Laser field samples for the real-time steps (host side, vectorised numpy).

Mirrors QuantumND's field definition:
  * amplitude F0 = 5.33803e-9 sqrt(I[W/cm^2]) and frequency w = 45.5637639947958 / lambda[nm]
    (parameters.c:807-810);
  * the time vector t_i = i*dt, N_time = floor(T/dt) (parameters.c:886-895);
  * the sum over modes of A(t) = F0 f(t) (cos(w t' + phi), xi sin(w t' + phi)) / w and the analytic
    E = -dA/dt, t' = t - delay, with envelopes constant / trapz / cos2 / cos4 (parameters.c:899-949);
    only axes 0 and 1 carry a field;
  * the sub-step sampling of Initialize_field_vectors: the first sample at t_i + as_scaled[0], then
    advancing by as_scaled[2j+1] + as_scaled[2j+2] (integrators.c:94-101).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["Mode", "field_at", "field_samples", "time_vector", "integrator_coeffs"]

_BASE = {
    "Verlet": [.5],
    "BM4": [.0792036964311957, .1303114101821663, .2228614958676077, -.3667132690474257, .3246481886897062,
            .1096884778767498],
    "BM6": [.050262764400392, .098553683500650, .314960616927694, -.447346482695478, .492426372489876,
            -.425118767797691, .237063913978122, .195602488600053, .346358189850727, -.362762779254345],
    "RKN4": [.082984406417405, .162314550766866, .233995250731502, .370877414979578, -.409933719901926,
             .059762097006575],
}


def integrator_coeffs(name: str, dt: float) -> np.ndarray:
    """as_scaled[0..2s): palindrome of the base coefficients times dt (integrators.c:22-64)."""
    if name not in _BASE:
        raise ValueError(f"Unknown integrator: {name}")
    b = list(_BASE[name])
    return np.array(b + b[::-1]) * dt


@dataclass
class Mode:
    intensity: float = 1e14      # W/cm^2
    wavelength: float = 800.0    # nm (LAMBDA)
    ellipticity: float = 1.0
    cep: float = 0.0
    delay: float = 0.0
    duration: float = 220.6380
    envelope: str = "cos4"

    @property
    def amplitude(self) -> float:
        return 5.33803e-9 * np.sqrt(self.intensity)

    @property
    def frequency(self) -> float:
        return 45.5637639947958 / self.wavelength


def _envelope(name, ts, tau, w):
    on = ((ts >= 0.0) & (ts <= tau)).astype(float)
    if name == "constant":
        return np.ones_like(ts), np.zeros_like(ts)
    if name == "trapz":
        ramp = 2.0 * 2.0 * np.pi / w
        up = ((ts >= 0.0) & (ts <= ramp)).astype(float)
        flat = ((ts > ramp) & (ts < tau - ramp)).astype(float)
        down = ((ts >= tau - ramp) & (ts <= tau)).astype(float)
        s_up, s_dn = np.sin(.5 * np.pi * ts / ramp), np.sin(.5 * np.pi * (ts - tau) / ramp)
        f = s_up ** 4 * up + flat + s_dn ** 4 * down
        df = np.pi / ramp * (s_up ** 2 * np.sin(np.pi * ts / ramp) * up + s_dn ** 2 * np.sin(np.pi * (ts - tau) / ramp)
                             * down)
        return f, df
    if name == "cos2":
        return np.sin(np.pi * ts / tau) ** 2 * on, np.pi * np.sin(2.0 * np.pi * ts / tau) / tau * on
    if name == "cos4":
        s = np.sin(np.pi * ts / tau)
        return s ** 4 * on, 4.0 * np.pi * np.cos(np.pi * ts / tau) * s ** 3 / tau * on
    raise ValueError(f"Unknown envelope: {name}")


def field_at(dim: int, modes, t):
    """(A, E) with shape t.shape + (dim,) summed over modes (parameters.c:899-949)."""
    t = np.asarray(t, dtype=float)
    A = np.zeros(t.shape + (dim,))
    E = np.zeros(t.shape + (dim,))
    for m in modes:
        w, F0, xi = m.frequency, m.amplitude, m.ellipticity
        ts = t - m.delay
        f, df = _envelope(m.envelope, ts, m.duration, w)
        c, s = np.cos(w * ts + m.cep), np.sin(w * ts + m.cep)
        E[..., 0] += -F0 * (df * c - f * w * s) / w
        A[..., 0] += F0 * f * c / w
        if dim >= 2:
            E[..., 1] += -F0 * xi * (df * s + f * w * c) / w
            A[..., 1] += F0 * xi * f * s / w
    return A, E


def time_vector(T: float, dt: float) -> np.ndarray:
    return np.arange(int(T / dt)) * dt


def field_samples(dim: int, modes, integrator: str, dt: float, T: float):
    """E, A as [N_time][s][dim] at the sub-step times, and the time vector (integrators.c:94-101)."""
    asc = integrator_coeffs(integrator, dt)
    s = len(asc) // 2
    t = time_vector(T, dt)
    # the reference accumulates t += ... per step starting from t_i + as[0]; reproduce that order
    tt = np.empty((t.size, s))
    cur = t + asc[0]
    for j in range(s):
        tt[:, j] = cur
        if j < s - 1:
            cur = cur + (asc[2 * j + 1] + asc[2 * j + 2])
    A, E = field_at(dim, modes, tt)
    return E, A, t
