"""FP64 CPU adjoints of the split-operator runs (length and velocity gauge) — TEST INFRASTRUCTURE ONLY.

The reference has no adjoint; these are the CPU restatements the engine's qnd_adjoint_length and
qnd_adjoint_velocity are checked against (numpy FFTs, FP64), themselves checked two ways by the
tests: their forward runs against the C oracle's length- and velocity-gauge runs (pinned to the
reference's Integration_step_length / _velocity, integrators.c:170-232), and their gradients
against central finite differences of their own J.

A length-gauge step on the r-space state (integrators.c:170-194 with the unitary transforms at
either end folded away) is the operator product
    psi <- M K(a_{2s-1}) D_{s-1} K(c_{s-1}) ... D_1 K(c_1) D_0 K(c_0) psi,
    c_0 = a_0, c_i = a_{2i-1} + a_{2i}, h_i = a_{2i} + a_{2i+1},
    K(c) = F^-1 exp(-i c |p|^2/2) F,  D_i = exp(min(700, -h_i Vcap)) exp(-i h_i (V + x.E[k][i])),
with M the product of the per-axis step masks (an extension). For J = dNr sum_x w |psi_T|^2 the
adjoint state starts at lambda_T = dNr w psi_T and goes back through every operator's adjoint;
the factor D_i adds dJ/dE[k][i][j] = 2 h_i sum_x x_j Im(conj(lambda') psi') with psi', lambda'
taken just after D_i.

Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

from .oracle import coeffs, grid_axes

MAX_EXP_ARG = 700.0  # integrators.h:12


class LengthRun:
    def __init__(self, shape, dr, integrator, dt, V, Vcap=None, masks=None):
        self.shape = tuple(int(n) for n in shape)
        self.dim = len(self.shape)
        self.dr = tuple(float(d) for d in dr)
        self.a = coeffs(integrator, dt)
        self.s = len(self.a) // 2
        rs, ps = grid_axes(self.shape, self.dr)
        self.X = np.meshgrid(*rs, indexing="ij")
        P = np.meshgrid(*ps, indexing="ij")
        self.kin = sum(p * p for p in P) / 2.0
        self.V = np.asarray(V, dtype=np.float64).reshape(self.shape)
        self.Vcap = np.zeros(self.shape) if Vcap is None else np.asarray(Vcap, dtype=np.float64).reshape(self.shape)
        self.M = None
        if masks is not None:
            self.M = np.ones(self.shape)
            for j, m in enumerate(masks):
                if m is not None:
                    sh = [1] * self.dim
                    sh[j] = -1
                    self.M = self.M * np.asarray(m, dtype=np.float64).reshape(sh)
        self.dNr = float(np.prod(self.dr))

    def c(self, i):
        return self.a[0] if i == 0 else self.a[2 * i - 1] + self.a[2 * i]

    def h(self, i):
        return self.a[2 * i] + self.a[2 * i + 1]

    def K(self, psi, c):
        return np.fft.ifftn(np.exp(-1j * c * self.kin) * np.fft.fftn(psi))

    def D(self, i, Ek):
        h = self.h(i)
        phase = self.V + sum(self.X[j] * Ek[i][j] for j in range(self.dim))
        return np.exp(np.minimum(MAX_EXP_ARG, -h * self.Vcap)) * np.exp(-1j * h * phase)

    def step(self, psi, Ek, keep=None):
        psi = self.K(psi, self.c(0))
        for i in range(self.s):
            psi = self.D(i, Ek) * psi
            if keep is not None:
                keep.append(psi)
            psi = self.K(psi, self.c(i + 1) if i + 1 < self.s else self.a[2 * self.s - 1])
        if self.M is not None:
            psi = self.M * psi
        return psi

    def run(self, psi0, E):
        psi = np.asarray(psi0, dtype=np.complex128).reshape(self.shape)
        for k in range(E.shape[0]):
            psi = self.step(psi, E[k])
        return psi

    def objective(self, psi0, E, w):
        psi = self.run(psi0, E)
        return self.dNr * float(np.sum(w * np.abs(psi) ** 2))

    def adjoint(self, psi0, E, w):
        """J and dJ/dE [nsteps, s, dim]."""
        E = np.asarray(E, dtype=np.float64)
        n = E.shape[0]
        starts = [np.asarray(psi0, dtype=np.complex128).reshape(self.shape)]
        for k in range(n):
            starts.append(self.step(starts[-1], E[k]))
        psiT = starts[-1]
        J = self.dNr * float(np.sum(w * np.abs(psiT) ** 2))
        lam = self.dNr * w * psiT
        grad = np.zeros((n, self.s, self.dim))
        for k in range(n - 1, -1, -1):
            subs = []
            self.step(starts[k], E[k], keep=subs)
            if self.M is not None:
                lam = self.M * lam
            lam = self.K(lam, -self.a[2 * self.s - 1])
            for i in range(self.s - 1, -1, -1):
                cross = np.imag(np.conj(lam) * subs[i])
                for j in range(self.dim):
                    grad[k, i, j] = 2.0 * self.h(i) * float(np.sum(self.X[j] * cross))
                lam = np.conj(self.D(i, E[k])) * lam
                lam = self.K(lam, -self.c(i))
        return J, grad


class VelocityRun(LengthRun):
    """Velocity gauge (integrators.c:201-232 on the r-space state): per step
        psi <- M V(a_{2s-1}) P_{s-1} V(a_{2s-2}) V(a_{2s-3}) ... P_0 V(a_0) psi,
        V(a) = exp(min(700, -a Vcap)) exp(-i a V),
        P_i = F^-1 exp(-i h_i sum_j (p_j^2/2 + (p_j + A_j/2) A_j)) F,  A = A[k][i].
    For J = dNr sum_x w |psi_T|^2 the sample A[k][i][j] contributes
        dJ/dA[k][i][j] = 2 h_i sum_k (p_j + A_j) Im(conj(lam~') psi~')
    with unitary transforms of the state and the adjoint state just after P_i."""

    def __init__(self, *args, **kw):
        super().__init__(*args, **kw)
        _, ps = grid_axes(self.shape, self.dr)
        self.P = np.meshgrid(*ps, indexing="ij")

    def vfac(self, a):
        return np.exp(np.minimum(MAX_EXP_ARG, -a * self.Vcap)) * np.exp(-1j * a * self.V)

    def Pk(self, i, Ak):
        ph = self.kin + sum((self.P[j] + 0.5 * Ak[i][j]) * Ak[i][j] for j in range(self.dim))
        return np.exp(-1j * self.h(i) * ph)

    def step(self, psi, Ak, keep=None):
        for i in range(self.s):
            psi = self.vfac(self.a[2 * i]) * psi
            psi = np.fft.ifftn(self.Pk(i, Ak) * np.fft.fftn(psi))
            if keep is not None:
                keep.append(psi)
            psi = self.vfac(self.a[2 * i + 1]) * psi
        if self.M is not None:
            psi = self.M * psi
        return psi

    def adjoint(self, psi0, A, w):
        A = np.asarray(A, dtype=np.float64)
        n = A.shape[0]
        starts = [np.asarray(psi0, dtype=np.complex128).reshape(self.shape)]
        for k in range(n):
            starts.append(self.step(starts[-1], A[k]))
        psiT = starts[-1]
        J = self.dNr * float(np.sum(w * np.abs(psiT) ** 2))
        lam = self.dNr * w * psiT
        grad = np.zeros((n, self.s, self.dim))
        norm = "ortho"
        for k in range(n - 1, -1, -1):
            subs = []
            self.step(starts[k], A[k], keep=subs)
            if self.M is not None:
                lam = self.M * lam
            for i in range(self.s - 1, -1, -1):
                lam = np.conj(self.vfac(self.a[2 * i + 1])) * lam
                cross = np.imag(np.conj(np.fft.fftn(lam, norm=norm)) * np.fft.fftn(subs[i], norm=norm))
                for j in range(self.dim):
                    grad[k, i, j] = 2.0 * self.h(i) * float(np.sum((self.P[j] + A[k][i][j]) * cross))
                lam = np.fft.ifftn(np.conj(self.Pk(i, A[k])) * np.fft.fftn(lam))
                lam = np.conj(self.vfac(self.a[2 * i])) * lam
        return J, grad
