/*
 * qnd_oracle.c — CPU restatement of QuantumND's split-operator hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see qnd_oracle.h). Each function names the
 * reference lines it restates. Floating-point expressions keep the
 * reference's evaluation order so that, built without -ffast-math and with the
 * same FFT (shim/shim.c), results agree bit for bit with the reference's own
 * sources compiled by oracle/Makefile; tests/ check that.
 *
 * Extensions that the reference does not have (marked EXT): the per-axis step
 * mask, the "norm" and "accel" observables, and caller-supplied dV/dx arrays.
 */
#include "qnd_oracle.h"

#include "shim/fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAX_DIM 6
#define OR_MAX_EXP_ARG 700.   /* integrators.h:12 */
#define OR_MAX_STAGES 10      /* integrators.h:13 */

struct or_ctx {
    int dim;
    ptrdiff_t nr[OR_MAX_DIM];
    double dr[OR_MAX_DIM];
    ptrdiff_t n;                       /* dim_HS */
    int s;                             /* integrator stages */
    double as[2 * OR_MAX_STAGES];      /* as_scaled */
    double *r[OR_MAX_DIM], *p[OR_MAX_DIM];
    double *vpot, *vcap, *kin;
    double *gradv[OR_MAX_DIM];         /* EXT */
    double *mask[OR_MAX_DIM];          /* EXT */
    double fft_scaling, dNr, dNp;
    double complex *in, *out;
    int nthreads;
};

/* integrators.c:13-71: base coefficients, mirrored into a palindrome, scaled by dt. */
int or_coeffs(const char *integrator, double dt, double *as_scaled) {
    static const double verlet[] = {.5};
    static const double bm4[] = {.0792036964311957, .1303114101821663, .2228614958676077,
                                 -.3667132690474257, .3246481886897062, .1096884778767498};
    static const double bm6[] = {.050262764400392, .098553683500650, .314960616927694, -.447346482695478,
                                 .492426372489876, -.425118767797691, .237063913978122, .195602488600053,
                                 .346358189850727, -.362762779254345};
    static const double rkn4[] = {.082984406417405, .162314550766866, .233995250731502,
                                  .370877414979578, -.409933719901926, .059762097006575};
    const double *base;
    int s;
    if (strcmp(integrator, "Verlet") == 0) { base = verlet; s = 1; }
    else if (strcmp(integrator, "BM4") == 0) { base = bm4; s = 6; }
    else if (strcmp(integrator, "BM6") == 0) { base = bm6; s = 10; }
    else if (strcmp(integrator, "RKN4") == 0) { base = rkn4; s = 6; }
    else return 0;
    double as[2 * OR_MAX_STAGES];
    for (int j = 0; j < s; ++j) as[j] = base[j];
    for (int j = 0; j < s; ++j) as[s + j] = as[s - 1 - j];
    for (int j = 0; j < 2 * s; ++j) as_scaled[j] = as[j] * dt;
    return s;
}

void or_fft(int dim, const long long *nr, const double complex *in, double complex *out, int sign, int nthreads) {
    ptrdiff_t n[OR_MAX_DIM];
    for (int j = 0; j < dim; ++j) n[j] = (ptrdiff_t)nr[j];
    qnd_shim_fft_nd(dim, n, in, out, sign, nthreads);
}

static void fwd(or_ctx *c) { qnd_shim_fft_nd(c->dim, c->nr, c->in, c->out, FFTW_FORWARD, c->nthreads); }
static void bwd(or_ctx *c) { qnd_shim_fft_nd(c->dim, c->nr, c->in, c->out, FFTW_BACKWARD, c->nthreads); }

/* Row-major multi-index of flat i (meshgrid.c:205-211). */
static void unflatten(const or_ctx *c, ptrdiff_t i, ptrdiff_t *idx) {
    for (int j = c->dim - 1; j >= 0; --j) { idx[j] = i % c->nr[j]; i /= c->nr[j]; }
}

/* meshgrid.c:22-28, 75-89, 123-136, 162-163 */
or_ctx *or_create(int dim, const long long *nr, const double *dr, const char *integrator, double dt, int nthreads) {
    if (dim < 1 || dim > OR_MAX_DIM) return NULL;
    or_ctx *c = (or_ctx *)calloc(1, sizeof *c);
    c->dim = dim;
    c->nthreads = nthreads < 1 ? 1 : nthreads;
    c->s = or_coeffs(integrator, dt, c->as);
    if (c->s == 0) { free(c); return NULL; }
    c->n = 1;
    c->dNr = 1.;
    c->dNp = 1.;
    c->fft_scaling = 1.;
    for (int j = 0; j < dim; ++j) {
        c->nr[j] = (ptrdiff_t)nr[j];
        c->dr[j] = dr[j];
        c->n *= c->nr[j];
        c->dNr *= dr[j];
        c->dNp *= 2. * M_PI / (double)(dr[j] * c->nr[j]);
    }
    for (int j = 0; j < dim; ++j) c->fft_scaling /= (double)c->nr[j];
    for (int j = 0; j < dim; ++j) {
        ptrdiff_t N = c->nr[j];
        double L = c->dr[j] * N, dp = 2. * M_PI / L;
        c->r[j] = (double *)malloc(N * sizeof(double));
        c->p[j] = (double *)malloc(N * sizeof(double));
        for (ptrdiff_t i = 0; i < N; ++i) {
            c->r[j][i] = -.5 * L + i * c->dr[j];
            c->p[j][i] = i < N / 2 ? i * dp : (i - N) * dp;
        }
    }
    c->vpot = (double *)calloc(c->n, sizeof(double));
    c->vcap = (double *)calloc(c->n, sizeof(double));
    c->kin = (double *)calloc(c->n, sizeof(double));
    c->in = (double complex *)calloc(c->n, sizeof(double complex));
    c->out = (double complex *)calloc(c->n, sizeof(double complex));
    ptrdiff_t idx[OR_MAX_DIM];
    for (ptrdiff_t i = 0; i < c->n; ++i) {
        unflatten(c, i, idx);
        double k = 0.;
        for (int j = 0; j < dim; ++j) {
            double pj = c->p[j][idx[j]];
            k += .5 * pj * pj;
        }
        c->kin[i] = k;
    }
    return c;
}

void or_destroy(or_ctx *c) {
    if (!c) return;
    for (int j = 0; j < c->dim; ++j) { free(c->r[j]); free(c->p[j]); free(c->gradv[j]); free(c->mask[j]); }
    free(c->vpot); free(c->vcap); free(c->kin); free(c->in); free(c->out);
    free(c);
}

void or_set_threads(or_ctx *c, int nthreads) { c->nthreads = nthreads < 1 ? 1 : nthreads; }

/* meshgrid.c:137-153: the named potentials as functions of |r|. */
int or_set_potential_named(or_ctx *c, const char *name) {
    ptrdiff_t idx[OR_MAX_DIM];
    int kind;
    if (!strcmp(name, "H_1D")) kind = 0;
    else if (!strcmp(name, "H_3D")) kind = 1;
    else if (!strcmp(name, "H_2D")) kind = 2;
    else if (!strcmp(name, "Ne_2D")) kind = 3;
    else if (!strcmp(name, "Ar_2D")) kind = 4;
    else if (!strcmp(name, "Kr_2D")) kind = 5;
    else if (!strcmp(name, "Xe_2D")) kind = 6;
    else if (!strcmp(name, "Ne_short_2D")) kind = 7;
    else return 1;
    for (ptrdiff_t i = 0; i < c->n; ++i) {
        unflatten(c, i, idx);
        double r = 0.;
        for (int j = 0; j < c->dim; ++j) { double x = c->r[j][idx[j]]; r += x * x; }
        r = sqrt(r);
        double v;
        switch (kind) {
        case 0: v = -1. / (double)sqrt(r * r + 2.); break;
        case 1: v = -1. / (double)sqrt(r * r + 1e-4); break;
        case 2: v = -1. / (double)sqrt(r * r + .7396); break;
        case 3: v = -(1. + 9. * exp(-r * r)) / (double)sqrt(r * r + 2.88172); break;
        case 4: v = -(1. + 17. * exp(-r * r)) / (double)sqrt(r * r + .91205); break;
        case 5: v = -(1. + 35. * exp(-r * r)) / (double)sqrt(r * r + .7875); break;
        case 6: v = -(1. + 53. * exp(-r * r)) / (double)sqrt(r * r + .52592); break;
        default: v = -2.7459 * exp(-.5 * r * r / 1.96); break;
        }
        c->vpot[i] = v;
    }
    return 0;
}

/* meshgrid.c:133-135: per-axis quadratic CAP beyond half-box minus `length`. */
void or_set_cap(or_ctx *c, double strength, double length) {
    ptrdiff_t idx[OR_MAX_DIM];
    for (ptrdiff_t i = 0; i < c->n; ++i) {
        unflatten(c, i, idx);
        double v = 0.;
        for (int j = 0; j < c->dim; ++j) {
            double x = c->r[j][idx[j]];
            double L = .5 * c->nr[j] * c->dr[j] - length;
            if (fabs(x) >= L) v += strength * (fabs(x) - L) * (fabs(x) - L);
        }
        c->vcap[i] = v;
    }
}

void or_set_vpot(or_ctx *c, const double *v) { memcpy(c->vpot, v, c->n * sizeof(double)); }
void or_set_vcap(or_ctx *c, const double *v) { memcpy(c->vcap, v, c->n * sizeof(double)); }

void or_set_gradv(or_ctx *c, int axis, const double *g) {
    if (axis < 0 || axis >= c->dim) return;
    if (!c->gradv[axis]) c->gradv[axis] = (double *)malloc(c->n * sizeof(double));
    memcpy(c->gradv[axis], g, c->n * sizeof(double));
}

void or_set_mask_axis(or_ctx *c, int axis, const double *m) {
    if (axis < 0 || axis >= c->dim) return;
    if (!m) { free(c->mask[axis]); c->mask[axis] = NULL; return; }
    if (!c->mask[axis]) c->mask[axis] = (double *)malloc(c->nr[axis] * sizeof(double));
    memcpy(c->mask[axis], m, c->nr[axis] * sizeof(double));
}

void or_tables(const or_ctx *c, double *r_axes, double *p_axes, double *vpot, double *vcap, double *kin) {
    ptrdiff_t off = 0;
    for (int j = 0; j < c->dim; ++j) {
        if (r_axes) memcpy(r_axes + off, c->r[j], c->nr[j] * sizeof(double));
        if (p_axes) memcpy(p_axes + off, c->p[j], c->nr[j] * sizeof(double));
        off += c->nr[j];
    }
    if (vpot) memcpy(vpot, c->vpot, c->n * sizeof(double));
    if (vcap) memcpy(vcap, c->vcap, c->n * sizeof(double));
    if (kin) memcpy(kin, c->kin, c->n * sizeof(double));
}

/* integrators.c:135-163 */
void or_step_imag(or_ctx *c, double complex *psi, long long nsteps) {
    for (long long step = 0; step < nsteps; ++step) {
        for (int ia = 0; ia < c->s; ++ia) {
            double a = c->as[2 * ia], b = c->as[2 * ia + 1];
            for (ptrdiff_t i = 0; i < c->n; ++i) {
                double arg = -a * c->vpot[i];
                if (arg > OR_MAX_EXP_ARG) arg = OR_MAX_EXP_ARG;
                c->in[i] = exp(arg) * psi[i];
            }
            fwd(c);
            for (ptrdiff_t i = 0; i < c->n; ++i) {
                double arg = -(a + b) * c->kin[i];
                if (arg > OR_MAX_EXP_ARG) arg = OR_MAX_EXP_ARG;
                c->in[i] = exp(arg) * c->out[i];
            }
            bwd(c);
            for (ptrdiff_t i = 0; i < c->n; ++i) {
                double arg = -b * c->vpot[i];
                if (arg > OR_MAX_EXP_ARG) arg = OR_MAX_EXP_ARG;
                psi[i] = exp(arg) * c->out[i] * c->fft_scaling;
            }
        }
    }
}

/* integrators.c:170-194 (psi in the p-representation; E is [nsteps][s][dim]). */
void or_step_length(or_ctx *c, double complex *psi, const double *E, long long nsteps) {
    ptrdiff_t idx[OR_MAX_DIM];
    for (long long step = 0; step < nsteps; ++step) {
        const double *Et = E + step * c->s * c->dim;
        for (int ia = 0; ia < c->s; ++ia) {
            double a = c->as[2 * ia], b = c->as[2 * ia + 1];
            for (ptrdiff_t i = 0; i < c->n; ++i) c->in[i] = cexp(-I * a * c->kin[i]) * psi[i];
            bwd(c);
            for (ptrdiff_t i = 0; i < c->n; ++i) {
                unflatten(c, i, idx);
                double w = 0.;
                for (int j = 0; j < c->dim; ++j) w += c->r[j][idx[j]] * Et[ia * c->dim + j];
                double arg = -(a + b) * c->vcap[i];
                if (arg > OR_MAX_EXP_ARG) arg = OR_MAX_EXP_ARG;
                c->in[i] = cexp(arg - I * (a + b) * (c->vpot[i] + w)) * c->out[i];
            }
            fwd(c);
            for (ptrdiff_t i = 0; i < c->n; ++i) psi[i] = cexp(-I * b * c->kin[i]) * c->out[i] * c->fft_scaling;
        }
    }
}

/* integrators.c:201-232 (psi in the r-representation; A is [nsteps][s][dim]). */
void or_step_velocity(or_ctx *c, double complex *psi, const double *A, long long nsteps) {
    ptrdiff_t idx[OR_MAX_DIM];
    for (long long step = 0; step < nsteps; ++step) {
        const double *At = A + step * c->s * c->dim;
        for (int ia = 0; ia < c->s; ++ia) {
            double a = c->as[2 * ia], b = c->as[2 * ia + 1];
            for (ptrdiff_t i = 0; i < c->n; ++i) {
                double arg = -a * c->vcap[i];
                if (arg > OR_MAX_EXP_ARG) arg = OR_MAX_EXP_ARG;
                c->in[i] = cexp(arg - I * a * c->vpot[i]) * psi[i];
            }
            fwd(c);
            for (ptrdiff_t i = 0; i < c->n; ++i) {
                unflatten(c, i, idx);
                double w = 0.;
                for (int j = 0; j < c->dim; ++j) {
                    double Aj = At[ia * c->dim + j];
                    w += (c->p[j][idx[j]] + .5 * Aj) * Aj;
                }
                c->in[i] = cexp(-I * (a + b) * (c->kin[i] + w)) * c->out[i];
            }
            bwd(c);
            for (ptrdiff_t i = 0; i < c->n; ++i) {
                double arg = -b * c->vcap[i];
                if (arg > OR_MAX_EXP_ARG) arg = OR_MAX_EXP_ARG;
                psi[i] = cexp(arg - I * b * c->vpot[i]) * c->out[i] * c->fft_scaling;
            }
        }
    }
}

void or_to_p(or_ctx *c, double complex *psi) {
    memcpy(c->in, psi, c->n * sizeof(double complex));
    fwd(c);
    for (ptrdiff_t i = 0; i < c->n; ++i) psi[i] = c->out[i] * sqrt(c->fft_scaling);
}

void or_to_r(or_ctx *c, double complex *psi) {
    memcpy(c->in, psi, c->n * sizeof(double complex));
    bwd(c);
    for (ptrdiff_t i = 0; i < c->n; ++i) psi[i] = c->out[i] * sqrt(c->fft_scaling);
}

/* EXT: multiply by prod_j mask_j(x_j) over the axes that have a mask. */
void or_apply_mask(or_ctx *c, double complex *psi) {
    int any = 0;
    for (int j = 0; j < c->dim; ++j) any |= c->mask[j] != NULL;
    if (!any) return;
    ptrdiff_t idx[OR_MAX_DIM];
    for (ptrdiff_t i = 0; i < c->n; ++i) {
        unflatten(c, i, idx);
        double m = 1.;
        for (int j = 0; j < c->dim; ++j)
            if (c->mask[j]) m *= c->mask[j][idx[j]];
        psi[i] *= m;
    }
}

/* QuantumND_imag.c:265-311 */
int or_gram_schmidt(or_ctx *c, int j, double complex **psis, double *norm2_out) {
    double complex *v = (double complex *)malloc(c->n * sizeof(double complex));
    memcpy(v, psis[j], c->n * sizeof(double complex));
    for (int k = 0; k < j; ++k) {
        double complex s = 0.;
        for (ptrdiff_t i = 0; i < c->n; ++i) s += conj(psis[k][i]) * v[i] * c->dNr;
        for (ptrdiff_t i = 0; i < c->n; ++i) v[i] -= s * psis[k][i];
    }
    double norm = 0.;
    for (ptrdiff_t i = 0; i < c->n; ++i) norm += cabs(v[i]) * cabs(v[i]) * c->dNr;
    if (norm2_out) *norm2_out = norm;
    if (norm < 1.e-12) { free(v); return 2; }
    double inv = 1. / (double)sqrt(norm);
    for (ptrdiff_t i = 0; i < c->n; ++i) psis[j][i] = v[i] * inv;
    free(v);
    return 0;
}

long long or_imag_loop_count(double T, double dt) {
    long long count = 0;
    for (double t = 0.; t < T; t += dt) ++count;
    return count;
}

int or_imag_state(or_ctx *c, double complex **psis, int j, long long nsteps) {
    for (long long k = 0; k < nsteps; ++k) {
        or_step_imag(c, psis[j], 1);
        int rc = or_gram_schmidt(c, j, psis, NULL);
        if (rc) return rc;
    }
    return 0;
}

/* calculate_observables.c:146-175 */
static void energies_local(or_ctx *c, const double complex *psi, int nmom, double complex *e) {
    double complex *h = (double complex *)malloc(c->n * sizeof(double complex));
    memcpy(h, psi, c->n * sizeof(double complex));
    for (int m = 0; m < nmom; ++m) {
        e[m] = 0.;
        memcpy(c->in, h, c->n * sizeof(double complex));
        fwd(c);
        for (ptrdiff_t i = 0; i < c->n; ++i) c->in[i] = c->kin[i] * c->out[i];
        bwd(c);
        for (ptrdiff_t i = 0; i < c->n; ++i) {
            h[i] = c->out[i] * c->fft_scaling + c->vpot[i] * h[i];
            e[m] += conj(psi[i]) * h[i] * c->dNr;
        }
    }
    free(h);
}

void or_energies(or_ctx *c, const double complex *psi, int n, double *out) {
    if (n <= 0) return;
    double complex e[16];
    energies_local(c, psi, n > 16 ? 16 : n, e);
    for (int m = 0; m < n && m < 16; ++m) out[m] = creal(e[m]);
}

/* calculate_observables.c:178-230 (dim >= 2; 0 otherwise, :129) */
static double complex lz_local(or_ctx *c, const double complex *psi, const double *alpha) {
    if (c->dim <= 1) return 0.;
    ptrdiff_t idx[OR_MAX_DIM];
    double complex *pp = (double complex *)malloc(c->n * sizeof(double complex));
    double complex lz = 0.;
    memcpy(c->in, psi, c->n * sizeof(double complex));
    fwd(c);
    memcpy(pp, c->out, c->n * sizeof(double complex));
    for (ptrdiff_t i = 0; i < c->n; ++i) { unflatten(c, i, idx); c->in[i] = (c->p[1][idx[1]] + alpha[1]) * pp[i]; }
    bwd(c);
    for (ptrdiff_t i = 0; i < c->n; ++i) { unflatten(c, i, idx); lz += conj(psi[i]) * c->r[0][idx[0]] * c->out[i]; }
    for (ptrdiff_t i = 0; i < c->n; ++i) { unflatten(c, i, idx); c->in[i] = (c->p[0][idx[0]] + alpha[0]) * pp[i]; }
    bwd(c);
    for (ptrdiff_t i = 0; i < c->n; ++i) { unflatten(c, i, idx); lz -= conj(psi[i]) * c->r[1][idx[1]] * c->out[i]; }
    lz *= c->fft_scaling * c->dNr;
    free(pp);
    return lz;
}

static int obs_width(const or_ctx *c, const char *name) {
    if (!strcmp(name, "PMD") || !strcmp(name, "PED") || !strcmp(name, "wavefunction") || !strcmp(name, "none")) return 0;
    if (!strcmp(name, "Lz") || !strcmp(name, "energy") || !strcmp(name, "norm")) return 1;
    if (!strcmp(name, "dipole_r") || !strcmp(name, "dipole_v") || !strcmp(name, "accel")) return c->dim;
    return 0; /* unknown names take no room (calculate_observables.c:52-55) */
}

int or_observable_count(const or_ctx *c, int nobs, const char *const *names) {
    int total = 0;
    for (int k = 0; k < nobs; ++k) total += obs_width(c, names[k]);
    return total;
}

/* calculate_observables.c:119-140, 233-266, plus EXT norm/accel (r-space reductions). */
int or_observables(or_ctx *c, const double complex *psi, int nobs, const char *const *names, const double *alpha,
                   double *out) {
    ptrdiff_t idx[OR_MAX_DIM];
    int off = 0;
    for (int k = 0; k < nobs; ++k) {
        const char *nm = names[k];
        double complex acc[OR_MAX_DIM];
        if (!strcmp(nm, "Lz")) {
            out[off++] = creal(lz_local(c, psi, alpha));
        } else if (!strcmp(nm, "energy")) {
            double complex e;
            energies_local(c, psi, 1, &e);
            out[off++] = creal(e);
        } else if (!strcmp(nm, "dipole_r")) {
            for (int j = 0; j < c->dim; ++j) {
                acc[j] = 0.;
                for (ptrdiff_t i = 0; i < c->n; ++i) {
                    unflatten(c, i, idx);
                    acc[j] += conj(psi[i]) * c->r[j][idx[j]] * psi[i] * c->dNr;
                }
                out[off++] = creal(acc[j]);
            }
        } else if (!strcmp(nm, "dipole_v")) {
            memcpy(c->in, psi, c->n * sizeof(double complex));
            fwd(c);
            for (int j = 0; j < c->dim; ++j) {
                acc[j] = 0.;
                for (ptrdiff_t i = 0; i < c->n; ++i) {
                    unflatten(c, i, idx);
                    acc[j] += conj(c->out[i]) * (c->p[j][idx[j]] + alpha[j]) * c->out[i] * c->dNp * c->fft_scaling;
                }
                out[off++] = creal(acc[j]);
            }
        } else if (!strcmp(nm, "norm")) {
            double s = 0.;
            for (ptrdiff_t i = 0; i < c->n; ++i) s += cabs(psi[i]) * cabs(psi[i]) * c->dNr;
            out[off++] = s;
        } else if (!strcmp(nm, "accel")) {
            for (int j = 0; j < c->dim; ++j) {
                if (!c->gradv[j]) return -1;
                double s = 0.;
                for (ptrdiff_t i = 0; i < c->n; ++i) s -= cabs(psi[i]) * cabs(psi[i]) * c->gradv[j][i] * c->dNr;
                out[off++] = s;
            }
        } else {
            off += obs_width(c, nm);
        }
    }
    return off;
}

/* QuantumND_real.c:188-229 with psi in r-space on entry and exit; EXT: the mask after each step. */
int or_run_length(or_ctx *c, double complex *psi, const double *E, long long nsteps, int nobs,
                  const char *const *names, double *obs_out) {
    int nv = or_observable_count(c, nobs, names);
    double alpha[OR_MAX_DIM] = {0};
    int masked = 0;
    for (int j = 0; j < c->dim; ++j) masked |= c->mask[j] != NULL;
    or_to_p(c, psi);
    for (long long it = 0; it < nsteps; ++it) {
        if (nv > 0) {
            or_to_r(c, psi);
            if (or_observables(c, psi, nobs, names, alpha, obs_out + it * nv) < 0) return -1;
            or_to_p(c, psi);
        }
        or_step_length(c, psi, E + it * c->s * c->dim, 1);
        if (masked) { or_to_r(c, psi); or_apply_mask(c, psi); or_to_p(c, psi); }
    }
    or_to_r(c, psi);
    return nv;
}

/* QuantumND_real.c:168-187; alpha_steps[it*dim+j] = A_j(t_it); EXT: the mask after each step. */
int or_run_velocity(or_ctx *c, double complex *psi, const double *A, const double *alpha_steps, long long nsteps,
                    int nobs, const char *const *names, double *obs_out) {
    int nv = or_observable_count(c, nobs, names);
    for (long long it = 0; it < nsteps; ++it) {
        if (nv > 0 && or_observables(c, psi, nobs, names, alpha_steps + it * c->dim, obs_out + it * nv) < 0) return -1;
        or_step_velocity(c, psi, A + it * c->s * c->dim, 1);
        or_apply_mask(c, psi);
    }
    return nv;
}

/* parameters.c:899-949: sum of modes, analytic E = -dA/dt, components for axes 0 and 1 only. */
int or_field_at(int dim, int nmodes, const double *intensity, const double *lambda, const double *ellipticity,
                const double *cep, const double *delay, const double *duration, const char *const *envelope, double t,
                double *A, double *E) {
    for (int j = 0; j < dim; ++j) { E[j] = 0.; A[j] = 0.; }
    for (int m = 0; m < nmodes; ++m) {
        double w = 45.5637639947958 / (double)lambda[m];         /* parameters.c:809 */
        double F0 = 5.33803e-9 * sqrt(intensity[m]);             /* parameters.c:808 */
        double xi = ellipticity[m], tau = duration[m], phase = cep[m];
        double ts = t - delay[m];
        double f, df;
        const char *env = envelope[m];
        if (!strcmp(env, "constant")) {
            f = 1.;
            df = 0.;
        } else if (!strcmp(env, "trapz")) {
            double ramp = 2. * 2. * M_PI / w;
            double up = (ts >= 0. && ts <= ramp), flat = (ts > ramp && ts < (tau - ramp)),
                   down = (ts >= tau - ramp && ts <= tau);
            f = pow(sin(.5 * M_PI * ts / (double)ramp), 4) * up + flat +
                pow(sin(.5 * M_PI * (ts - tau) / (double)ramp), 4) * down;
            df = M_PI / (double)ramp *
                 (pow(sin(.5 * M_PI * ts / (double)ramp), 2) * sin(M_PI * ts / (double)ramp) * up +
                  pow(sin(.5 * M_PI * (ts - tau) / (double)ramp), 2) * sin(M_PI * (ts - tau) / (double)ramp) * down);
        } else if (!strcmp(env, "cos2")) {
            double on = (ts >= 0. && ts <= tau);
            f = pow(sin(M_PI * ts / (double)tau), 2) * on;
            df = M_PI * sin(2. * M_PI * ts / (double)tau) / (double)tau * on;
        } else if (!strcmp(env, "cos4")) {
            double on = (ts >= 0. && ts <= tau);
            f = pow(sin(M_PI * ts / (double)tau), 4) * on;
            df = 4. * M_PI * cos(M_PI * ts / (double)tau) * pow(sin(M_PI * ts / (double)tau), 3) / (double)tau * on;
        } else {
            return 1;
        }
        E[0] += -F0 * (df * cos(w * ts + phase) - f * w * sin(w * ts + phase)) / (double)w;
        if (dim >= 2) E[1] += -F0 * xi * (df * sin(w * ts + phase) + f * w * cos(w * ts + phase)) / (double)w;
        A[0] += F0 * f * cos(w * ts + phase) / (double)w;
        if (dim >= 2) A[1] += F0 * xi * f * sin(w * ts + phase) / (double)w;
    }
    return 0;
}

/* parameters.c:886-895 (time vector) and integrators.c:94-101 (sub-step sampling). */
long long or_field(int dim, int nmodes, const double *intensity, const double *lambda, const double *ellipticity,
                   const double *cep, const double *delay, const double *duration, const char *const *envelope,
                   const char *integrator, double dt, double T, double *E, double *A, double *times) {
    double as[2 * OR_MAX_STAGES];
    int s = or_coeffs(integrator, dt, as);
    if (s == 0) return -1;
    long long nt = (long long)(T / (double)dt);
    if (!E) return nt;
    for (long long i = 0; i < nt; ++i) {
        double ti = i * dt;
        if (times) times[i] = ti;
        double t = ti + as[0];
        long long base = i * dim * s;
        for (int j = 0; j < s; ++j) {
            if (or_field_at(dim, nmodes, intensity, lambda, ellipticity, cep, delay, duration, envelope, t,
                            &A[base + j * dim], &E[base + j * dim]))
                return -1;
            if (j < s - 1) t += as[2 * j + 1] + as[2 * j + 2];
        }
    }
    return nt;
}
