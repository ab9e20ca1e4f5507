/*
 * ref_harness.c — TEST INFRASTRUCTURE ONLY.
 *
 * A thin C entry layer, linked against the reference's own unmodified sources
 * (QuantumND src/*.c compiled by oracle/Makefile into oracle/_ref/), so that
 * tests and the CPU baseline can call the reference's hot-path functions
 * directly on seeded inputs:
 *   Initialize_integrator        integrators.c:13-71
 *   Integration_step_imag        integrators.c:135-163
 *   Integration_step_length      integrators.c:170-194
 *   Integration_step_velocity    integrators.c:201-232
 *   Initialize_meshgrid          meshgrid.c:17-179
 *   Gram_Schmidt_orthonormalization  QuantumND_imag.c:265-311
 *   Calculation_global_energies / _observables  calculate_observables.c:89-140
 *   Field_vectors                parameters.c:899-949
 *   Write_final_observables      io_functions.c:136-287
 * The driver loops (QuantumND_imag.c:182-185, QuantumND_real.c:168-229) are
 * replayed here call for call so trajectories match the executables.
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "calculate_observables.h"
#include "integrators.h"
#include "io_functions.h"
#include "meshgrid.h"
#include "parameters.h"

void Gram_Schmidt_orthonormalization(const int N, double complex **Psi, const MeshGrid *grid, MPI_Comm comm);

typedef struct {
    Parameters P;
    MeshGrid grid;
    Integrator Int;
    ptrdiff_t local_n[8], local_start[8];
} RefCtx;

RefCtx *ref_create(int dim, const long long *nr, const double *dr, const char *potential, double cap_strength,
                   double cap_length, const char *integrator, double dt, int nthreads) {
    RefCtx *c = (RefCtx *)calloc(1, sizeof(RefCtx));
    c->P.dim = dim;
    c->P.Nr_global = (ptrdiff_t *)malloc(dim * sizeof(ptrdiff_t));
    c->P.dr = (double *)malloc(dim * sizeof(double));
    c->P.pr_max = (double *)malloc(dim * sizeof(double));
    for (int j = 0; j < dim; ++j) {
        c->P.Nr_global[j] = (ptrdiff_t)nr[j];
        c->P.dr[j] = dr[j];
        c->P.pr_max[j] = 1.0;
    }
    snprintf(c->P.potential, MAX_POTENTIAL_CHAR, "%s", potential);
    snprintf(c->P.integrator, MAX_INTEGRATOR_CHAR, "%s", integrator);
    c->P.cap[0] = cap_strength;
    c->P.cap[1] = cap_length;
    c->P.dt = dt;
    Initialize_integrator(integrator, dt, &c->Int, MPI_COMM_WORLD);
    for (int j = 0; j < dim; ++j) { c->local_n[j] = nr[j]; c->local_start[j] = 0; }
    ptrdiff_t alloc = 1;
    for (int j = 0; j < dim; ++j) alloc *= nr[j];
    Initialize_meshgrid(&c->P, &c->grid, c->local_n, c->local_start, alloc, MPI_COMM_WORLD);
    fftw_plan_with_nthreads(nthreads);
    return c;
}

void ref_set_threads(int nthreads) { fftw_plan_with_nthreads(nthreads); }

void ref_destroy(RefCtx *c) {
    if (!c) return;
    Finalize_meshgrid(&c->grid);
    free(c->P.Nr_global);
    free(c->P.dr);
    free(c->P.pr_max);
    free(c);
}

long long ref_dim_hs(const RefCtx *c) { return (long long)c->grid.dim_HS; }
int ref_s(const RefCtx *c) { return c->Int.s_integrator; }
void ref_coeffs(const RefCtx *c, double *as_scaled) {
    for (int j = 0; j < 2 * c->Int.s_integrator; ++j) as_scaled[j] = c->Int.as_scaled[j];
}
void ref_tables(const RefCtx *c, double *vpot, double *vcap, double *kin) {
    size_t n = (size_t)c->grid.dim_HS;
    if (vpot) memcpy(vpot, c->grid.Vpot, n * sizeof(double));
    if (vcap) memcpy(vcap, c->grid.Vcap, n * sizeof(double));
    if (kin) memcpy(kin, c->grid.Kin, n * sizeof(double));
}
void ref_set_vpot(RefCtx *c, const double *v) { memcpy(c->grid.Vpot, v, (size_t)c->grid.dim_HS * sizeof(double)); }
void ref_set_vcap(RefCtx *c, const double *v) { memcpy(c->grid.Vcap, v, (size_t)c->grid.dim_HS * sizeof(double)); }

void ref_step_imag(RefCtx *c, double complex *psi, long long nsteps) {
    for (long long k = 0; k < nsteps; ++k) Integration_step_imag(psi, &c->grid, &c->Int);
}

/* E is laid out [nsteps][s][dim] like F.E (integrators.c:81, QuantumND_real.c:216). */
void ref_step_length(RefCtx *c, double complex *psi_p, const double *E, long long nsteps) {
    int sd = c->Int.s_integrator * c->P.dim;
    for (long long k = 0; k < nsteps; ++k) Integration_step_length(psi_p, E + k * sd, c->P.dim, &c->grid, &c->Int);
}

void ref_step_velocity(RefCtx *c, double complex *psi, const double *A, long long nsteps) {
    int sd = c->Int.s_integrator * c->P.dim;
    for (long long k = 0; k < nsteps; ++k) Integration_step_velocity(psi, A + k * sd, c->P.dim, &c->grid, &c->Int);
}

void ref_gram_schmidt(RefCtx *c, int j, double complex **psis) {
    Gram_Schmidt_orthonormalization(j, psis, &c->grid, MPI_COMM_WORLD);
}

/* Number of passes of `for(time=0.;time<T;time+=dt)` (QuantumND_imag.c:182). */
long long ref_imag_loop_count(double T, double dt) {
    long long n = 0;
    for (double time = 0.; time < T; time += dt) ++n;
    return n;
}

/* Imaginary-time loop for state j: step + Gram-Schmidt, nsteps times (QuantumND_imag.c:182-185). */
void ref_imag_state(RefCtx *c, double complex **psis, int j, long long nsteps) {
    for (long long k = 0; k < nsteps; ++k) {
        Integration_step_imag(psis[j], &c->grid, &c->Int);
        Gram_Schmidt_orthonormalization(j, psis, &c->grid, MPI_COMM_WORLD);
    }
}

void ref_energies(RefCtx *c, const double complex *psi, int n, double *out) {
    Calculation_global_energies(out, n, psi, &c->grid, MPI_COMM_WORLD);
}

/* Evaluate observables by name (calculate_observables.c:119-140); returns the value count. */
int ref_observables(RefCtx *c, const double complex *psi, int nobs, char **names, double *alpha, double *out) {
    Observables Obs;
    memset(&Obs, 0, sizeof Obs);
    Initialize_observables(&Obs, names, nobs, c->P.dim, MPI_COMM_WORLD);
    int nv = Obs.total_values;
    if (nv > 0) {
        Calculation_global_observables(psi, c->P.dim, &c->grid, &Obs, alpha, MPI_COMM_WORLD);
        memcpy(out, Obs.values, (size_t)nv * sizeof(double));
    }
    Finalize_observables(&Obs);
    return nv;
}

/*
 * Length-gauge real-time loop exactly as QuantumND_real.c:188-229: psi (r-space)
 * goes to the unitary p-representation, then every step converts back to r,
 * evaluates the observables (alpha = 0), converts to p and integrates; at the
 * end psi returns to r. obs_out is [nsteps][total_values].
 */
int ref_run_length(RefCtx *c, double complex *psi, const double *E, long long nsteps, int nobs, char **names,
                   double *obs_out) {
    MeshGrid *g = &c->grid;
    ptrdiff_t n = g->dim_HS;
    int sd = c->Int.s_integrator * c->P.dim;
    double alpha[8] = {0};
    Observables Obs;
    memset(&Obs, 0, sizeof Obs);
    Initialize_observables(&Obs, names, nobs, c->P.dim, MPI_COMM_WORLD);
    int nv = Obs.total_values;
    for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
    fftw_execute(g->plan_forward);
    for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
    for (long long it = 0; it < nsteps; ++it) {
        if (nv > 0) {
            for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
            fftw_execute(g->plan_backward);
            for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
            for (int j = 0; j < c->P.dim; j++) alpha[j] = 0.;
            Calculation_global_observables(psi, c->P.dim, g, &Obs, alpha, MPI_COMM_WORLD);
            memcpy(obs_out + it * nv, Obs.values, (size_t)nv * sizeof(double));
            for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
            fftw_execute(g->plan_forward);
            for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
        }
        Integration_step_length(psi, E + it * sd, c->P.dim, g, &c->Int);
    }
    for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
    fftw_execute(g->plan_backward);
    for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
    Finalize_observables(&Obs);
    return nv;
}

/*
 * The loop of ref_run_length with the two observable extensions of this project (the reference
 * has neither) evaluated on the same r-space state at the same point of each step:
 *   "norm"  = sum |psi|^2 dNr                        (1 value)
 *   "accel" = -sum |psi|^2 dV/dx_j dNr, j < dim       (dim values; gradv[j] in natural order)
 * Every other name goes to the reference's own Calculation_global_observables. Output columns
 * follow the order of names. Used for the CPU baseline, where both sides must compute the same
 * observables of the same run.
 */
int ref_run_length_ext(RefCtx *c, double complex *psi, const double *E, long long nsteps, int nobs, char **names,
                       const double *const *gradv, double *obs_out) {
    MeshGrid *g = &c->grid;
    ptrdiff_t n = g->dim_HS;
    int dim = c->P.dim, sd = c->Int.s_integrator * dim;
    double alpha[8] = {0};
    char *rnames[32];
    int nref = 0, width = 0, kind[32], wref[32];
    for (int k = 0; k < nobs && k < 32; ++k) {
        if (strcmp(names[k], "norm") == 0) {
            kind[k] = 1;
            width += 1;
        } else if (strcmp(names[k], "accel") == 0) {
            kind[k] = 2;
            width += dim;
        } else {
            kind[k] = 0;
            rnames[nref++] = names[k];
        }
    }
    Observables Obs;
    memset(&Obs, 0, sizeof Obs);
    Initialize_observables(&Obs, rnames, nref, dim, MPI_COMM_WORLD);
    for (int k = 0, q = 0; k < nobs && k < 32; ++k)
        if (kind[k] == 0) wref[k] = Obs.dimensions[q++];
    width += Obs.total_values;
    for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
    fftw_execute(g->plan_forward);
    for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
    for (long long it = 0; it < nsteps; ++it) {
        if (width > 0) {
            for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
            fftw_execute(g->plan_backward);
            for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
            for (int j = 0; j < dim; j++) alpha[j] = 0.;
            if (Obs.total_values > 0) Calculation_global_observables(psi, dim, g, &Obs, alpha, MPI_COMM_WORLD);
            double nrm = 0.0, acc[8] = {0};
#pragma omp parallel for reduction(+ : nrm)
            for (ptrdiff_t i = 0; i < n; i++) nrm += creal(psi[i] * conj(psi[i]));
            for (int j = 0; j < dim && gradv; j++) {
                double a = 0.0;
                const double *gv = gradv[j];
                if (!gv) continue;
#pragma omp parallel for reduction(+ : a)
                for (ptrdiff_t i = 0; i < n; i++) a += creal(psi[i] * conj(psi[i])) * gv[i];
                acc[j] = -a * g->dNr;
            }
            double *row = obs_out + it * width;
            for (int k = 0, col = 0, off = 0; k < nobs && k < 32; ++k) {
                if (kind[k] == 1) {
                    row[col++] = nrm * g->dNr;
                } else if (kind[k] == 2) {
                    for (int j = 0; j < dim; j++) row[col++] = acc[j];
                } else {
                    for (int j = 0; j < wref[k]; j++) row[col++] = Obs.values[off + j];
                    off += wref[k];
                }
            }
            for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
            fftw_execute(g->plan_forward);
            for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
        }
        Integration_step_length(psi, E + it * sd, dim, g, &c->Int);
    }
    for (ptrdiff_t i = 0; i < n; i++) g->in[i] = psi[i];
    fftw_execute(g->plan_backward);
    for (ptrdiff_t i = 0; i < n; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
    Finalize_observables(&Obs);
    return width;
}

/*
 * Velocity-gauge loop as QuantumND_real.c:168-187. alpha_steps[it*dim..] is
 * A(t_it) for the observables (Field_vectors at P.time[itime]); A holds the
 * sub-step samples [nsteps][s][dim].
 */
int ref_run_velocity(RefCtx *c, double complex *psi, const double *A, const double *alpha_steps, long long nsteps,
                     int nobs, char **names, double *obs_out) {
    int sd = c->Int.s_integrator * c->P.dim;
    double alpha[8] = {0};
    Observables Obs;
    memset(&Obs, 0, sizeof Obs);
    Initialize_observables(&Obs, names, nobs, c->P.dim, MPI_COMM_WORLD);
    int nv = Obs.total_values;
    for (long long it = 0; it < nsteps; ++it) {
        if (nv > 0) {
            for (int j = 0; j < c->P.dim; j++) alpha[j] = alpha_steps[it * c->P.dim + j];
            Calculation_global_observables(psi, c->P.dim, &c->grid, &Obs, alpha, MPI_COMM_WORLD);
            memcpy(obs_out + it * nv, Obs.values, (size_t)nv * sizeof(double));
        }
        Integration_step_velocity(psi, A + it * sd, c->P.dim, &c->grid, &c->Int);
    }
    Finalize_observables(&Obs);
    return nv;
}

/* Unitary transforms used by the length-gauge driver (QuantumND_real.c:190-192, 200-202). */
void ref_to_p(RefCtx *c, double complex *psi) {
    MeshGrid *g = &c->grid;
    for (ptrdiff_t i = 0; i < g->dim_HS; i++) g->in[i] = psi[i];
    fftw_execute(g->plan_forward);
    for (ptrdiff_t i = 0; i < g->dim_HS; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
}
void ref_to_r(RefCtx *c, double complex *psi) {
    MeshGrid *g = &c->grid;
    for (ptrdiff_t i = 0; i < g->dim_HS; i++) g->in[i] = psi[i];
    fftw_execute(g->plan_backward);
    for (ptrdiff_t i = 0; i < g->dim_HS; i++) psi[i] = g->out[i] * sqrt(g->fft_scaling);
}

/*
 * Field samples exactly as Initialize_field_vectors (integrators.c:94-101) with
 * amplitude/frequency from parameters.c:807-810; the time vector as
 * parameters.c:886-895. E and A are [N_time][s][dim]; returns N_time.
 */
long long ref_field(int dim, int nmodes, const double *intensity, const double *lambda, const double *ellipticity,
                    const double *cep, const double *delay, const double *duration, char **envelope,
                    const char *integrator, double dt, double T, double *E, double *A, double *times) {
    Parameters P;
    Field F;
    Integrator Int;
    memset(&P, 0, sizeof P);
    memset(&F, 0, sizeof F);
    memset(&Int, 0, sizeof Int);
    P.dim = dim;
    Initialize_integrator(integrator, dt, &Int, MPI_COMM_WORLD);
    F.N_modes = nmodes;
    F.intensity = (double *)intensity;
    F.lambda = (double *)lambda;
    F.ellipticity = (double *)ellipticity;
    F.cep = (double *)cep;
    F.delay = (double *)delay;
    F.duration = (double *)duration;
    F.envelope = envelope;
    F.amplitude = (double *)malloc(nmodes * sizeof(double));
    F.frequency = (double *)malloc(nmodes * sizeof(double));
    for (int j = 0; j < nmodes; j++) {
        F.amplitude[j] = 5.33803e-9 * sqrt(F.intensity[j]);
        F.frequency[j] = 45.5637639947958 / (double)F.lambda[j];
    }
    long long N_time = (long long)(T / (double)dt);
    if (E == NULL) { free(F.amplitude); free(F.frequency); return N_time; }
    for (long long i = 0; i < N_time; i++) {
        double time_i = i * dt;
        if (times) times[i] = time_i;
        double t = time_i + Int.as_scaled[0];
        long long ind = i * dim * Int.s_integrator;
        for (int j = 0; j < Int.s_integrator; j++) {
            Field_vectors(&P, &F, t, &A[ind + j * dim], &E[ind + j * dim], MPI_COMM_WORLD);
            if (j < Int.s_integrator - 1) t += Int.as_scaled[2 * j + 1] + Int.as_scaled[2 * j + 2];
        }
    }
    free(F.amplitude);
    free(F.frequency);
    return N_time;
}

/* One Field_vectors evaluation at time t (parameters.c:899-949). */
void ref_field_at(int dim, int nmodes, const double *intensity, const double *lambda, const double *ellipticity,
                  const double *cep, const double *delay, const double *duration, char **envelope, double t, double *A,
                  double *E) {
    Parameters P;
    Field F;
    memset(&P, 0, sizeof P);
    memset(&F, 0, sizeof F);
    P.dim = dim;
    F.N_modes = nmodes;
    F.intensity = (double *)intensity;
    F.lambda = (double *)lambda;
    F.ellipticity = (double *)ellipticity;
    F.cep = (double *)cep;
    F.delay = (double *)delay;
    F.duration = (double *)duration;
    F.envelope = envelope;
    F.amplitude = (double *)malloc(nmodes * sizeof(double));
    F.frequency = (double *)malloc(nmodes * sizeof(double));
    for (int j = 0; j < nmodes; j++) {
        F.amplitude[j] = 5.33803e-9 * sqrt(F.intensity[j]);
        F.frequency[j] = 45.5637639947958 / (double)F.lambda[j];
    }
    Field_vectors(&P, &F, t, A, E, MPI_COMM_WORLD);
    free(F.amplitude);
    free(F.frequency);
}

/*
 * Write_final_observables (io_functions.c:136-287) on psi (r-space; masked and transformed in
 * place, as the reference does at the end of QuantumND_real): writes PED.real, PMD.real and
 * wavefunction.real into the current directory.
 */
void ref_final_observables(RefCtx *c, double complex *psi, double rmin, double rmax, const double *pr_max, double de,
                           int ne, int nobs, char **names) {
    for (int j = 0; j < c->P.dim; ++j) c->P.pr_max[j] = pr_max[j];
    c->P.R_mask[0] = rmin;
    c->P.R_mask[1] = rmax;
    c->P.de = de;
    c->P.Ne = ne;
    Observables Obs;
    memset(&Obs, 0, sizeof Obs);
    Initialize_observables(&Obs, names, nobs, c->P.dim, MPI_COMM_WORLD);
    Write_final_observables(psi, &c->P, &c->grid, &Obs, c->local_start, MPI_COMM_WORLD);
    Finalize_observables(&Obs);
}
