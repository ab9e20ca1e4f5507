"""Generate the golden vectors in tests/golden/ from the reference's OWN sources.

Runs the unmodified QuantumND C sources (compiled by ``make -C oracle ref REF=<reference root>`` against
the single-rank MPI / FFTW-API shims) on seeded inputs and stores inputs and
outputs as compressed .npz fixtures. The reference is only available where its
sources are (this script is not run by tests); the fixtures are committed so
parity tests work anywhere.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

OBS = ["dipole_r", "dipole_v", "energy", "Lz"]
GRIDS = {
    "1d": (1, (64,), (0.4,)),
    "2d": (2, (8, 16), (0.5, 0.35)),
    "3d": (3, (4, 8, 8), (0.6, 0.5, 0.45)),
}
POT = {"1d": "H_1D", "2d": "Ne_2D", "3d": "H_3D"}


def steps_fixture():
    out = {}
    for key, (dim, nr, dr) in GRIDS.items():
        for integ in ("Verlet", "BM4", "BM6", "RKN4"):
            ref = O.RefCtx(dim, nr, dr, integ, 0.05, POT[key], (0.2, 0.8), nthreads=1)
            s = ref.s
            psi0 = O.seeded_state(nr, 11, float(np.prod(dr)))
            rng = np.random.default_rng(5)
            E = rng.standard_normal((2, s, dim)) * 0.05
            tag = f"{key}_{integ}"
            out[f"{tag}_psi0"] = psi0
            out[f"{tag}_E"] = E
            a = psi0.copy(); ref.step_imag(a, 2); out[f"{tag}_imag"] = a
            a = psi0.copy(); ref.step_length(a, E, 2); out[f"{tag}_length"] = a
            a = psi0.copy(); ref.step_velocity(a, E, 2); out[f"{tag}_velocity"] = a
            out[f"{tag}_coeffs"] = ref.coeffs()
            v, vc, k = ref.tables()
            out[f"{tag}_vpot"], out[f"{tag}_vcap"], out[f"{tag}_kin"] = v, vc, k
    np.savez_compressed(os.path.join(HERE, "steps.npz"), **out)


def observables_fixture():
    out = {}
    for key, (dim, nr, dr) in GRIDS.items():
        ref = O.RefCtx(dim, nr, dr, "BM4", 0.05, POT[key], (0.0, 0.0), nthreads=1)
        psi = O.seeded_state(nr, 21, float(np.prod(dr)))
        alpha = np.linspace(-0.2, 0.3, dim)
        out[f"{key}_psi"] = psi
        out[f"{key}_alpha"] = alpha
        out[f"{key}_obs"] = ref.observables(psi, OBS, alpha)
        out[f"{key}_energies"] = ref.energies(psi, 3)
        states = [O.seeded_state(nr, 30 + k) for k in range(4)]
        out[f"{key}_gs_in"] = np.stack(states)
        for j in range(4):
            ref.gram_schmidt(j, states)
        out[f"{key}_gs_out"] = np.stack(states)
    np.savez_compressed(os.path.join(HERE, "observables.npz"), **out)


def trajectory_fixture():
    """Driver-loop trajectories (QuantumND_real.c:168-229) with observables every step."""
    out = {}
    dim, nr, dr = 2, (16, 16), (0.4, 0.4)
    modes = [dict(intensity=1e14, ellipticity=0.2, cep=0.3, delay=0.0, duration=20.0, envelope="cos2",
                  **{"lambda": 800.0})]
    for integ in ("BM4", "Verlet"):
        ref = O.RefCtx(dim, nr, dr, integ, 0.05, "H_2D", (0.3, 1.2), nthreads=1)
        E, A, t = O.field(dim, modes, integ, 0.05, 0.4, use_ref=True)
        alpha = np.stack([O.field_at(dim, modes, ti)[0] for ti in t])
        psi0 = O.smooth_state(nr, dr, 4)
        tag = f"traj_{integ}"
        out[f"{tag}_psi0"], out[f"{tag}_E"], out[f"{tag}_A"], out[f"{tag}_alpha"] = psi0, E, A, alpha
        a = psi0.copy(); out[f"{tag}_length_obs"] = ref.run_length(a, E, OBS); out[f"{tag}_length_psi"] = a
        a = psi0.copy(); out[f"{tag}_velocity_obs"] = ref.run_velocity(a, A, alpha, OBS)
        out[f"{tag}_velocity_psi"] = a
    np.savez_compressed(os.path.join(HERE, "trajectory.npz"), **out)


def imag_fixture():
    """Imaginary-time eigenstates (QuantumND_imag.c:169-188) from the reference's deterministic guess."""
    dim, nr, dr = 1, (128,), (0.4,)
    ref = O.RefCtx(dim, nr, dr, "BM4", 0.1, "H_1D", (0.0, 0.0), nthreads=1)
    r = -0.5 * nr[0] * dr[0] + np.arange(nr[0]) * dr[0]
    guess = (np.abs(r) + (np.arange(nr[0]) % 3)) * np.exp(-np.abs(r))
    nsteps = O.imag_loop_count(20.0, 0.1)
    states = [np.ascontiguousarray(guess.astype(np.complex128)) for _ in range(3)]
    energies = []
    for j in range(3):
        ref.imag_state(states, j, nsteps)
        energies.append(ref.energies(states[j], 2))
    np.savez_compressed(os.path.join(HERE, "imag.npz"), guess=guess, nsteps=nsteps, states=np.stack(states),
                        energies=np.array(energies))


def field_fixture():
    out = {}
    for env in ("constant", "trapz", "cos2", "cos4"):
        # short wavelengths so the trapz ramps (4*pi/w) fall inside the sampled window
        modes = [dict(intensity=1e14, ellipticity=0.4, cep=0.2, delay=2.0, duration=60.0, envelope=env,
                      **{"lambda": 80.0}),
                 dict(intensity=2e13, ellipticity=0.0, cep=1.1, delay=0.0, duration=40.0, envelope=env,
                      **{"lambda": 40.0})]
        for integ in ("BM4", "BM6"):
            E, A, t = O.field(2, modes, integ, 0.5, 70.0, use_ref=True)
            out[f"{env}_{integ}_E"], out[f"{env}_{integ}_A"] = E, A
    np.savez_compressed(os.path.join(HERE, "field.npz"), **out)


def fft_fixture():
    out = {}
    for shape in ((32,), (8, 16), (4, 8, 16)):
        x = O.seeded_state(shape, 7)
        tag = "x".join(map(str, shape))
        out[f"{tag}_in"] = x
        out[f"{tag}_fwd"] = np.fft.fftn(x)
        out[f"{tag}_bwd"] = np.fft.ifftn(x) * x.size
    np.savez_compressed(os.path.join(HERE, "fft.npz"), **out)


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref/libqnd_ref.so missing: run `make -C oracle ref REF=<reference root>` where the reference sources exist")
    steps_fixture()
    observables_fixture()
    trajectory_fixture()
    imag_fixture()
    field_fixture()
    fft_fixture()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
