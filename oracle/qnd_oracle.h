/*
 * qnd_oracle.h — CPU restatement of QuantumND's split-operator hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker that the CUDA library is
 * compared against (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline
 * leg). Nothing in the shipped library links or calls it.
 *
 * Pinning: every function here is checked in tests/ against the reference's
 * own sources compiled by oracle/Makefile (oracle/_ref/) and against the
 * committed golden vectors in tests/golden/ that those sources produced.
 *
 * Arrays are row-major, axis 0 slowest (meshgrid.c:205-211); complex values are
 * C99 double complex (interleaved re, im). Functions return 0 on success and a
 * non-zero code on failure (the reference aborts instead).
 */
#ifndef QND_ORACLE_H
#define QND_ORACLE_H

#include <complex.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_ctx or_ctx;

/* Integrator coefficients as_scaled[0..2s) (integrators.c:13-71); returns s or 0 for an unknown name. */
int or_coeffs(const char *integrator, double dt, double *as_scaled);

or_ctx *or_create(int dim, const long long *nr, const double *dr, const char *integrator, double dt, int nthreads);
void or_destroy(or_ctx *c);
int or_set_potential_named(or_ctx *c, const char *name);          /* meshgrid.c:140-153 */
void or_set_cap(or_ctx *c, double strength, double length);        /* meshgrid.c:133-135 */
void or_set_vpot(or_ctx *c, const double *v);
void or_set_vcap(or_ctx *c, const double *v);
void or_set_gradv(or_ctx *c, int axis, const double *g);           /* dV/dx_axis, for the "accel" extension */
void or_set_mask_axis(or_ctx *c, int axis, const double *m);       /* extension: per-axis step mask, NULL clears */
void or_set_threads(or_ctx *c, int nthreads);
void or_tables(const or_ctx *c, double *r_axes, double *p_axes, double *vpot, double *vcap, double *kin);

void or_step_imag(or_ctx *c, double complex *psi, long long nsteps);                    /* integrators.c:135-163 */
void or_step_length(or_ctx *c, double complex *psi_p, const double *E, long long nsteps); /* integrators.c:170-194 */
void or_step_velocity(or_ctx *c, double complex *psi, const double *A, long long nsteps);/* integrators.c:201-232 */
void or_to_p(or_ctx *c, double complex *psi);  /* unitary r->p, QuantumND_real.c:190-192 */
void or_to_r(or_ctx *c, double complex *psi);  /* unitary p->r, QuantumND_real.c:200-202 */
void or_apply_mask(or_ctx *c, double complex *psi_r);

/* Modified Gram-Schmidt of psis[j] against psis[0..j) (QuantumND_imag.c:265-311); norm2_out gets ||v||^2 dNr. */
int or_gram_schmidt(or_ctx *c, int j, double complex **psis, double *norm2_out);
long long or_imag_loop_count(double T, double dt);                                     /* QuantumND_imag.c:182 */
int or_imag_state(or_ctx *c, double complex **psis, int j, long long nsteps);         /* QuantumND_imag.c:182-185 */

/* Observable values by name: PMD/PED/wavefunction/none -> 0 values, Lz/energy/norm -> 1, dipole_r/dipole_v/accel -> dim
 * (calculate_observables.c:48-56 plus the norm/accel extensions). Returns the value count, or -1 on error. */
int or_observable_count(const or_ctx *c, int nobs, const char *const *names);
int or_observables(or_ctx *c, const double complex *psi_r, int nobs, const char *const *names, const double *alpha,
                   double *out);
void or_energies(or_ctx *c, const double complex *psi_r, int n, double *out); /* calculate_observables.c:89-116 */

/* Real-time loops (QuantumND_real.c:168-229), psi in r-space in and out, obs_out [nsteps][count]. */
int or_run_length(or_ctx *c, double complex *psi_r, const double *E, long long nsteps, int nobs,
                  const char *const *names, double *obs_out);
int or_run_velocity(or_ctx *c, double complex *psi_r, const double *A, const double *alpha_steps, long long nsteps,
                    int nobs, const char *const *names, double *obs_out);

/* Laser field (parameters.c:807-810, 886-949; integrators.c:94-101). envelope names: constant, trapz, cos2, cos4.
 * E/A are [N_time][s][dim]; returns N_time, or -1 for an unknown envelope or integrator. */
long long or_field(int dim, int nmodes, const double *intensity, const double *lambda, const double *ellipticity,
                   const double *cep, const double *delay, const double *duration, const char *const *envelope,
                   const char *integrator, double dt, double T, double *E, double *A, double *times);
int or_field_at(int dim, int nmodes, const double *intensity, const double *lambda, const double *ellipticity,
                const double *cep, const double *delay, const double *duration, const char *const *envelope, double t,
                double *A, double *E);

/* Unnormalised N-D DFT with FFTW's sign convention (sign -1 forward, +1 backward). */
void or_fft(int dim, const long long *nr, const double complex *in, double complex *out, int sign, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
