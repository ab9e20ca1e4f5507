/*
 * quantumnd_real.c — drop-in QuantumND_real (QuantumND_real.c:56-264) over the C ABI of
 * libqnd_b200.so: the same params.real keys and `KEY VALUE` overrides (parameters.c:215-800), the
 * same initial state read from OUTPUT_IMAG (centred, superposed: io_functions.c:292-459), the same
 * laser field (parameters.c:899-949, integrators.c:74-129) and the same files: observables.real,
 * electric_field.real, vector_potential.real, PED.real, PMD.real, wavefunction.real
 * (io_functions.c:11-287). The propagation, the observables and the final spectra run on the GPU.
 *
 *     QuantumND_real <params.real> [KEY VALUE ...]
 *
 * Grids are limited to what the engine builds: powers of two up to 2^24 points per axis.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/qnd.h"
#include "params.h"

#define CK(x)                                                   \
    do {                                                        \
        int rc_ = (x);                                          \
        if (rc_ != QND_OK) {                                    \
            fprintf(stderr, "ERROR: %s\n", qnd_last_error());   \
            exit(1);                                            \
        }                                                       \
    } while (0)

static const char *const KEYS_REAL[] = {"OUTPUT_IMAG", "NR", "N_STATES", "J_STATES", "COEFFS_STATES", "CAP", "GAUGE",
                                        "N_MODES", "INTENSITY", "LAMBDA", "ELLIPTICITY", "CEP", "ENVELOPE", "DURATION",
                                        "DELAY", "INTEGRATOR", "DT", "TINTEGRATION", "DT_SAVE", "N_OBSERVABLES",
                                        "OBSERVABLES", "P_MAX", "R_MASK", "DE", "NE", NULL};

typedef struct {
    int dim;
    int64_t nr[QND_DRV_MAX_DIM], nr_imag[QND_DRV_MAX_DIM];
    double dr[QND_DRV_MAX_DIM];
    char potential[64], integrator[64], output_imag[256], gauge[32];
    int nstates, nstates_imag, nobs, nmodes, ne;
    int *j_states;
    double complex *coeffs;
    char (*obs)[64];
    double cap[2], dt, T, dt_save, pr_max[QND_DRV_MAX_DIM], r_mask[2], de;
    char (*envelope)[32];
    double *intensity, *lambda, *ellipticity, *cep, *delay, *duration, *amplitude, *frequency;
} RealParams;

static void fail(const char *msg) {
    fprintf(stderr, "%s\n", msg);
    exit(1);
}

static int read_d(const char *s, double *x) { return sscanf(s, "%lf", x) == 1; }
static int read_i(const char *s, int *x) { return sscanf(s, "%d", x) == 1; }

/* "a+bj", "a-bj", "bj" or "a" (parameters.c parse_complex) */
static double complex parse_complex(const char *s) {
    double re = 0., im = 0.;
    const char *plus = strchr(s, '+'), *minus = strrchr(s, '-'), *j = strchr(s, 'j');
    if (plus && j) sscanf(s, "%lf+%lfj", &re, &im);
    else if (minus && minus != s && j) {
        sscanf(s, "%lf-%lfj", &re, &im);
        im = -im;
    } else if (j) sscanf(s, "%lfj", &im);
    else sscanf(s, "%lf", &re);
    return re + im * I;
}

/* the token after index i, or exit with the reference's message */
static const char *value(const qnd_tokens *t, int i, const char *what) {
    if (i >= t->ntok) fail(what);
    return t->tok[i];
}

static void read_params(const char *file, int argc, char **argv, RealParams *P) {
    qnd_tokens t;
    qnd_read_tokens(file, &t);
    memset(P, 0, sizeof *P);
    P->nstates = 1;
    snprintf(P->integrator, sizeof P->integrator, "BM4");
    P->dt = .1;
    P->T = 220.6380;
    P->nmodes = 1;
    snprintf(P->gauge, sizeof P->gauge, "velocity");
    P->dt_save = 1.;
    P->r_mask[0] = 20.;
    P->r_mask[1] = 30.;
    P->ne = 100;
    P->de = .01;
    /* first pass: the sizes (parameters.c:260-318) */
    int found_out = 0, found_ns = 0, found_no = 0, found_nm = 0;
    for (int i = 0; i < t.ntok; ++i) {
        const char *k = t.tok[i];
        if (!strcmp(k, "OUTPUT_IMAG")) {
            qnd_expect(&t, i, 1, KEYS_REAL);
            snprintf(P->output_imag, sizeof P->output_imag, "%s", t.tok[i + 1]);
            found_out = 1;
        } else if (!strcmp(k, "N_STATES")) {
            qnd_expect(&t, i, 1, KEYS_REAL);
            if (!read_i(t.tok[i + 1], &P->nstates)) fail("The number of states is undetermined");
            found_ns = 1;
        } else if (!strcmp(k, "N_OBSERVABLES")) {
            qnd_expect(&t, i, 1, KEYS_REAL);
            if (!read_i(t.tok[i + 1], &P->nobs)) fail("The number of observables is undetermined");
            found_no = 1;
        } else if (!strcmp(k, "N_MODES")) {
            qnd_expect(&t, i, 1, KEYS_REAL);
            if (!read_i(t.tok[i + 1], &P->nmodes)) fail("The number of field modes is undetermined");
            found_nm = 1;
        }
        if (found_out && found_ns && found_no && found_nm) break;
    }
    if (!found_out) fail("The output file is not specified\n\n FATAL ERROR: Critical parameters missing. Aborting.");
    if (!found_ns) printf("WARNING: The number of states is not specified\nDefault value: N_STATES=1\n");
    if (!found_no) printf("WARNING: The number of observables is not specified\nDefault value: N_OBSERVABLES=0\n");
    if (!found_nm) printf("WARNING: The number of field modes is not specified\nDefault value: N_MODES=1\n");
    if (P->nstates < 1 || P->nobs < 0 || P->nmodes < 1) fail("ERROR: N_STATES, N_OBSERVABLES or N_MODES out of range");
    P->j_states = calloc((size_t)P->nstates, sizeof(int));
    P->coeffs = calloc((size_t)P->nstates, sizeof(double complex));
    P->obs = calloc((size_t)P->nobs + 1, sizeof *P->obs);
    P->envelope = calloc((size_t)P->nmodes, sizeof *P->envelope);
    double **mode_arrays[] = {&P->intensity, &P->lambda, &P->ellipticity, &P->cep, &P->delay, &P->duration,
                              &P->amplitude, &P->frequency};
    for (size_t a = 0; a < sizeof mode_arrays / sizeof mode_arrays[0]; ++a)
        *mode_arrays[a] = calloc((size_t)P->nmodes, sizeof(double));
    for (int j = 0; j < P->nstates; ++j) {
        P->j_states[j] = 1;
        P->coeffs[j] = 1.;
    }
    for (int j = 0; j < P->nobs; ++j) snprintf(P->obs[j], sizeof P->obs[j], "none");
    for (int j = 0; j < P->nmodes; ++j) {
        snprintf(P->envelope[j], sizeof P->envelope[j], "cos4");
        P->intensity[j] = 1.e14;
        P->lambda[j] = 800.;
        P->ellipticity[j] = 1.;
        P->cep[j] = 0.;
        P->delay[j] = 0.;
        P->duration[j] = 220.6380;
    }
    /* the dimension and the grid of OUTPUT_IMAG (parameters.c:404-466) */
    qnd_tokens ti;
    {
        FILE *f = fopen(P->output_imag, "rb");
        if (!f) fail("Rank 0 Error: Failed to open imaginary output file for parameter read.");
        char buf[512];
        ti.ntok = 0;
        while (fscanf(f, "%511s", buf) == 1 && ti.ntok < QND_MAX_TOKENS) {
            ti.tok[ti.ntok++] = strdup(buf);
            if (!strcmp(buf, "PSI")) break;
        }
        fclose(f);
    }
    P->dim = qnd_find_dimension(&ti);
    if (P->dim < 1 || P->dim > QND_DRV_MAX_DIM) fail("ERROR: DIMENSION out of range (1 to 6)");
    for (int j = 0; j < P->dim; ++j) {
        P->nr[j] = 256;
        P->dr[j] = .1;
        P->pr_max[j] = 1.;
    }
    int bad = 0;
    for (int i = 0; i < ti.ntok; ++i) {
        const char *k = ti.tok[i];
        if (!strcmp(k, "PSI")) break;
        else if (!strcmp(k, "DIMENSION")) ++i;
        else if (!strcmp(k, "N_STATES")) {
            if (!read_i(value(&ti, ++i, "The number of states of OUTPUT_IMAG is undetermined"), &P->nstates_imag)) bad = 1;
            if (P->nstates > P->nstates_imag)
                printf("WARNING: The number of states for the superposition of the initial wave function is larger than the number of states computed in OUTPUT_IMAG");
        } else if (!strcmp(k, "E") || !strcmp(k, "DE")) i += P->nstates_imag;
        else if (!strcmp(k, "NR")) {
            for (int j = 0; j < P->dim; ++j) {
                long long x;
                if (sscanf(value(&ti, ++i, "NR of OUTPUT_IMAG"), "%lld", &x) != 1) bad = 1;
                P->nr_imag[j] = x;
            }
        } else if (!strcmp(k, "DR")) {
            for (int j = 0; j < P->dim; ++j)
                if (!read_d(value(&ti, ++i, "DR of OUTPUT_IMAG"), &P->dr[j])) bad = 1;
        } else if (!strcmp(k, "POTENTIAL")) {
            snprintf(P->potential, sizeof P->potential, "%s", value(&ti, ++i, "The potential name of OUPUT_IMAG is undetermined"));
        } else {
            printf("\nUnknown parameter: %s\n", k);
            bad = 1;
        }
    }
    /* second pass: every parameter (parameters.c:468-700) */
    for (int i = 0; i < t.ntok && !bad; ++i) {
        const char *k = t.tok[i];
#define NEXT() value(&t, ++i, "The value of a parameter is undetermined")
        if (!strcmp(k, "OUTPUT_IMAG") || !strcmp(k, "N_STATES") || !strcmp(k, "N_OBSERVABLES") || !strcmp(k, "N_MODES")) {
            ++i;
        } else if (!strcmp(k, "NR")) {
            for (int j = 0; j < P->dim; ++j) {
                long long x;
                if (sscanf(NEXT(), "%lld", &x) != 1) bad = 1;
                if (x != 0 && (x & (x - 1)) != 0) {
                    printf("\nThe number of points on the grid must be a power of 2\n");
                    bad = 1;
                }
                if (x < P->nr_imag[j]) printf("WARNING: The number of points on the grid is smaller than for the imaginary time propagation\n");
                P->nr[j] = x;
            }
        } else if (!strcmp(k, "J_STATES")) {
            for (int j = 0; j < P->nstates; ++j) {
                if (!read_i(NEXT(), &P->j_states[j])) bad = 1;
                if (P->j_states[j] > P->nstates_imag) {
                    printf("\nAn initial eigenstate is not computed in the imaginary time propagation\n");
                    bad = 1;
                }
            }
        } else if (!strcmp(k, "COEFFS_STATES")) {
            for (int j = 0; j < P->nstates; ++j) P->coeffs[j] = parse_complex(NEXT());
        } else if (!strcmp(k, "CAP")) {
            if (!read_d(NEXT(), &P->cap[0]) || !read_d(NEXT(), &P->cap[1])) bad = 1;
            P->cap[0] = fabs(P->cap[0]);
            P->cap[1] = fabs(P->cap[1]);
        } else if (!strcmp(k, "DT_SAVE")) {
            if (!read_d(NEXT(), &P->dt_save)) bad = 1;
        } else if (!strcmp(k, "P_MAX")) {
            for (int j = 0; j < P->dim; ++j)
                if (!read_d(NEXT(), &P->pr_max[j])) bad = 1;
        } else if (!strcmp(k, "R_MASK")) {
            if (!read_d(NEXT(), &P->r_mask[0]) || !read_d(NEXT(), &P->r_mask[1])) bad = 1;
        } else if (!strcmp(k, "DE")) {
            if (!read_d(NEXT(), &P->de)) bad = 1;
        } else if (!strcmp(k, "NE")) {
            if (!read_i(NEXT(), &P->ne)) bad = 1;
        } else if (!strcmp(k, "OBSERVABLES")) {
            for (int j = 0; j < P->nobs; ++j) snprintf(P->obs[j], sizeof P->obs[j], "%s", NEXT());
        } else if (!strcmp(k, "DT")) {
            if (!read_d(NEXT(), &P->dt)) bad = 1;
        } else if (!strcmp(k, "TINTEGRATION")) {
            if (!read_d(NEXT(), &P->T)) bad = 1;
        } else if (!strcmp(k, "INTEGRATOR")) {
            snprintf(P->integrator, sizeof P->integrator, "%s", NEXT());
        } else if (!strcmp(k, "GAUGE")) {
            snprintf(P->gauge, sizeof P->gauge, "%s", NEXT());
        } else if (!strcmp(k, "ENVELOPE")) {
            for (int j = 0; j < P->nmodes; ++j) snprintf(P->envelope[j], sizeof P->envelope[j], "%s", NEXT());
        } else if (!strcmp(k, "INTENSITY") || !strcmp(k, "LAMBDA") || !strcmp(k, "ELLIPTICITY") || !strcmp(k, "CEP") ||
                   !strcmp(k, "DELAY") || !strcmp(k, "DURATION")) {
            double *arr = !strcmp(k, "INTENSITY") ? P->intensity : !strcmp(k, "LAMBDA") ? P->lambda
                        : !strcmp(k, "ELLIPTICITY") ? P->ellipticity : !strcmp(k, "CEP") ? P->cep
                        : !strcmp(k, "DELAY") ? P->delay : P->duration;
            for (int j = 0; j < P->nmodes; ++j) {
                if (!read_d(NEXT(), &arr[j])) bad = 1;
                if (arr == P->delay && arr[j] < 0) bad = 1;
            }
        } else {
            printf("\nUnknown parameter: %s\n", k);
            bad = 1;
        }
#undef NEXT
    }
    if (bad) fail("\n FATAL ERROR: Data arrays or complex fields failed to read. Aborting.");
    /* command-line overrides (parameters.c:716-770): scalars, the first laser mode */
    for (int a = 2; a < argc; a += 2) {
        if (a + 1 >= argc) {
            fprintf(stderr, "Rank 0 ERROR: Parameter key '%s' found without a corresponding value.\n", argv[a]);
            exit(1);
        }
        const char *k = argv[a];
        const double v = atof(argv[a + 1]);
        if (!strcmp(k, "DT")) P->dt = v;
        else if (!strcmp(k, "TINTEGRATION")) P->T = v;
        else if (!strcmp(k, "NE")) P->ne = atoi(argv[a + 1]);
        else if (!strcmp(k, "DE")) P->de = v;
        else if (!strcmp(k, "INTENSITY")) P->intensity[0] = v;
        else if (!strcmp(k, "ELLIPTICITY")) P->ellipticity[0] = v;
        else if (!strcmp(k, "LAMBDA")) P->lambda[0] = v;
        else if (!strcmp(k, "CEP")) P->cep[0] = v;
        else if (!strcmp(k, "DELAY")) P->delay[0] = v;
        else if (!strcmp(k, "DURATION")) P->duration[0] = v;
        else {
            fprintf(stderr, "Rank 0 ERROR: Unrecognized parameter key '%s'. Check spelling.\n", k);
            exit(1);
        }
    }
    /* normalised superposition coefficients, laser amplitude and frequency (parameters.c:803-812) */
    double norm2 = 0.;
    for (int j = 0; j < P->nstates; ++j) norm2 += cabs(P->coeffs[j]) * cabs(P->coeffs[j]);
    for (int j = 0; j < P->nstates; ++j) P->coeffs[j] /= sqrt(norm2);
    for (int j = 0; j < P->nmodes; ++j) {
        P->amplitude[j] = 5.33803e-9 * sqrt(P->intensity[j]);
        P->frequency[j] = 45.5637639947958 / P->lambda[j];
    }
}

static void print_params(const RealParams *P) {
    int j;
    printf("> For real-time propagation:\n");
    printf("  DIMENSION\t\t%d\n", P->dim);
    printf("  NR\t\t");
    for (j = 0; j < P->dim; j++) printf("\t%lld", (long long)P->nr[j]);
    printf("\n  DR\t\t");
    for (j = 0; j < P->dim; j++) printf("\t%16.15f", P->dr[j]);
    printf("\n  N_STATES\t\t%d\n", P->nstates);
    printf("  J_STATES\t");
    for (j = 0; j < P->nstates; j++) printf("\t%d", P->j_states[j]);
    printf("\n  COEFFS_STATES\t");
    for (j = 0; j < P->nstates; j++) printf("\t%16.15f+I*%16.15f", creal(P->coeffs[j]), cimag(P->coeffs[j]));
    printf("\n  POTENTIAL\t\t%s\n", P->potential);
    printf("  CAP\t\t\t%16.15f\t%16.15f\n", P->cap[0], P->cap[1]);
    printf("  INTEGRATOR\t\t%s\n", P->integrator);
    printf("  DT\t\t\t%16.15f\n", P->dt);
    printf("  TINTEGRATION\t\t%16.15f\n\n", P->T);
    printf("> Field parameters:\n");
    printf("  GAUGE\t\t\t%s\n", P->gauge);
    printf("  N_MODES\t\t%d\n", P->nmodes);
    printf("  ENVELOPE\t");
    for (j = 0; j < P->nmodes; j++) printf("\t%s", P->envelope[j]);
    printf("\n  DURATION\t");
    for (j = 0; j < P->nmodes; j++) printf("\t%16.15f", P->duration[j]);
    printf("\n  INTENSITY\t");
    for (j = 0; j < P->nmodes; j++) printf("\t%6.5e", P->intensity[j]);
    printf("\n  LAMBDA\t");
    for (j = 0; j < P->nmodes; j++) printf("\t%16.15f", P->lambda[j]);
    printf("\n  ELLIPTICITY\t");
    for (j = 0; j < P->nmodes; j++) printf("\t%16.15f", P->ellipticity[j]);
    printf("\n  CEP\t\t");
    for (j = 0; j < P->nmodes; j++) printf("\t%16.15f", P->cep[j]);
    printf("\n  DELAY\t\t");
    for (j = 0; j < P->nmodes; j++) printf("\t%16.15f", P->delay[j]);
    printf("\n\n> Observables:\n");
    printf("  N_OBSERVABLES\t\t%d\n", P->nobs);
    printf("  OBSERVABLES\t");
    for (j = 0; j < P->nobs; j++) printf("\t%s", P->obs[j]);
    printf("\n  DT_SAVE\t\t%16.15f\n", P->dt_save);
    printf("  P_MAX\t\t");
    for (j = 0; j < P->dim; j++) printf("\t%16.15f", P->pr_max[j]);
    printf("\n  R_MASK\t\t%16.15f\t%16.15f\n", P->r_mask[0], P->r_mask[1]);
    printf("  DE\t\t\t%16.15f\n", P->de);
    printf("  NE\t\t\t%d\n\n", P->ne);
    printf("> For the imaginary-time propagation's data taken from '%s':\n", P->output_imag);
    printf("  OUTPUT_IMAG\t\t%s\n", P->output_imag);
    printf("  DIMENSION\t\t%d\n", P->dim);
    printf("  NR\t\t");
    for (j = 0; j < P->dim; j++) printf("\t%lld", (long long)P->nr_imag[j]);
    printf("\n  N_STATES\t\t%d\n", P->nstates_imag);
    fflush(stdout);
}

/* The field modes for qnd_field_samples, which evaluates Field_vectors (parameters.c:899-949) on the
 * device; an unknown envelope name stops the run as Field_vectors does. */
static qnd_laser_mode *laser_modes(const RealParams *P) {
    qnd_laser_mode *m = calloc((size_t)P->nmodes + 1, sizeof(qnd_laser_mode));
    static const char *const env[] = {"constant", "trapz", "cos2", "cos4"};
    for (int k = 0; k < P->nmodes; ++k) {
        m[k].frequency = P->frequency[k];
        m[k].amplitude = P->amplitude[k];
        m[k].ellipticity = P->ellipticity[k];
        m[k].cep = P->cep[k];
        m[k].delay = P->delay[k];
        m[k].duration = P->duration[k];
        m[k].envelope = -1;
        for (int e = 0; e < 4; ++e)
            if (!strcmp(P->envelope[k], env[e])) m[k].envelope = e;
        if (m[k].envelope < 0) {
            printf("\nUnknown envelope: %s\n", P->envelope[k]);
            fail("Error with the envelope name");
        }
    }
    return m;
}

/* Read_wavefunction_MPI (io_functions.c:292-459): the chosen OUTPUT_IMAG states are read here and
 * centred on the (possibly larger or smaller) real-time grid and superposed with the normalised
 * coefficients on the device (qnd_state_embed). */
static void read_initial_state(const RealParams *P, qnd_ctx *q, void *psi_dev) {
    FILE *f = fopen(P->output_imag, "rb");
    if (!f) fail("Rank 0: Error opening the output of the imaginary time propagation");
    char key[64];
    long off = 0;
    while (fscanf(f, "%63s", key) == 1) {
        if (!strcmp(key, "PSI")) {
            int c;
            while ((c = fgetc(f)) != '\n' && c != EOF) {
            }
            off = ftell(f);
            break;
        }
    }
    if (off == 0) fail("Rank 0: Error: Could not find 'PSI' marker in file.");
    int64_t n_imag = 1;
    for (int j = 0; j < P->dim; ++j) n_imag *= P->nr_imag[j];
    double complex *buf = calloc((size_t)n_imag, sizeof(double complex));
    if (P->nstates < 1) CK(qnd_state_embed(q, psi_dev, (const double *)buf, P->nr_imag, 0., 0., 0));  /* zero state */
    for (int k = 0; k < P->nstates; ++k) {
        if (fseek(f, off + (long)(P->j_states[k] - 1) * (long)n_imag * (long)sizeof(double complex), SEEK_SET) != 0 ||
            fread(buf, sizeof(double complex), (size_t)n_imag, f) != (size_t)n_imag)
            fail("Rank 0: MPI Read Error during chunking");
        CK(qnd_state_embed(q, psi_dev, (const double *)buf, P->nr_imag, creal(P->coeffs[k]), cimag(P->coeffs[k]), k > 0));
    }
    free(buf);
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "Usage: %s <param_file> [KEY VALUE ...]\n", argv[0]);
        return 1;
    }
    printf("\n##############################################\n");
    printf("\n##      PROGRAM REAL-TIME PROPAGATION       ##\n");
    printf("\n##############################################\n");
    printf("\n# Parameters read and broadcasted to all ranks\n\n");
    RealParams P;
    read_params(argv[1], argc, argv, &P);
    print_params(&P);

    /* integrator, time grid, field samples at the sub-step times (integrators.c:74-129) */
    qnd_ctx *q = NULL;
    CK(qnd_ctx_create(P.dim, P.nr, P.dr, P.integrator, P.dt, QND_FP64, &q));
    int64_t n = 0;
    int s = 0;
    double as[64];
    CK(qnd_ctx_info(q, &n, &s, as, NULL, NULL));
    const int64_t nt = (int64_t)(P.T / P.dt);
    double *E = calloc((size_t)(nt * s * P.dim) + 1, sizeof(double));
    double *A = calloc((size_t)(nt * s * P.dim) + 1, sizeof(double));
    FILE *fe = fopen("electric_field.real", "w"), *fa = fopen("vector_potential.real", "w");
    if (!fe || !fa) fail("Error opening the files of the vector potential and the laser electric field.");
    double *alpha = calloc((size_t)(nt * P.dim) + 1, sizeof(double));
    qnd_laser_mode *modes = laser_modes(&P);
    CK(qnd_field_samples(q, P.nmodes, modes, nt, E, A, alpha, 0));
    free(modes);
    for (int64_t i = 0; i < nt; ++i) {
        double t = (double)i * P.dt + as[0];
        const int64_t ind = i * P.dim * s;
        for (int j = 0; j < s; ++j) {
            fprintf(fe, "%16.15f ", t);
            fprintf(fa, "%16.15f ", t);
            for (int k = 0; k < P.dim; ++k) {
                fprintf(fe, "%16.15f ", E[ind + j * P.dim + k]);
                fprintf(fa, "%16.15f ", A[ind + j * P.dim + k]);
            }
            fprintf(fe, "\n");
            fprintf(fa, "\n");
            if (j < s - 1) t += as[2 * j + 1] + as[2 * j + 2];
        }
    }
    fclose(fe);
    fclose(fa);

    /* observables.real header (QuantumND_real.c:88-95; the column test reads dimensions[k], as there) */
    if (P.nobs > 64) fail("ERROR: at most 64 observables");
    const char **names = malloc(sizeof(char *) * (size_t)(P.nobs + 1));
    int width[64] = {0};
    for (int j = 0; j < P.nobs; ++j) {
        names[j] = P.obs[j];
        if (!strcmp(names[j], "Lz") || !strcmp(names[j], "energy")) width[j] = 1;
        else if (!strcmp(names[j], "dipole_r") || !strcmp(names[j], "dipole_v")) width[j] = P.dim;
        else if (strcmp(names[j], "PMD") && strcmp(names[j], "PED") && strcmp(names[j], "wavefunction") &&
                 strcmp(names[j], "none")) {
            printf("Unknown observable: %s. Skipping.\n", names[j]);
            names[j] = "none";
        }
    }
    FILE *fo = fopen("observables.real", "w");
    if (!fo) fail("Error opening the file of the observables");
    fprintf(fo, "time");
    for (int j = 0; j < P.nobs; ++j)
        for (int k = 0; k < width[j]; ++k)
            if (k >= P.nobs || width[k] != 0) fprintf(fo, "\t%s", names[j]);
    fprintf(fo, "\n");

    CK(qnd_set_potential_named(q, P.potential));
    CK(qnd_set_cap(q, P.cap[0], P.cap[1]));
    printf("\n# Initialization of the wave function\n");
    double complex *psi = malloc(sizeof(double complex) * (size_t)n);
    void *psi_dev = NULL;
    CK(qnd_state_alloc(q, 1, &psi_dev));
    read_initial_state(&P, q, psi_dev);

    printf("\n# Real-time propagation\n");
    clock_t c0 = clock();
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    int nv = 0;
    CK(qnd_observable_count(q, P.nobs, names, &nv));
    double *rows = calloc((size_t)(nt * (nv > 0 ? nv : 1)), sizeof(double));
    if (!strcmp(P.gauge, "velocity")) {
        CK(qnd_run_velocity(q, psi_dev, A, alpha, nt, P.nobs, names, rows));
    } else if (!strcmp(P.gauge, "length")) {
        CK(qnd_run_length(q, psi_dev, E, nt, P.nobs, names, rows));
    } else {
        fail("ERROR: unknown GAUGE (velocity or length)");
    }
    /* advancement report of the loop (printed as the reference would, once the run is done) */
    for (int64_t i = 0, percent = 0; i < nt; ++i)
        if (percent < 100 * i / nt) {
            printf("> %d%%\n", (int)percent);
            percent += 10;
        }
    if (P.nobs > 0)
        for (int64_t i = 0; i < nt; ++i) {
            fprintf(fo, "%16.15f", (double)i * P.dt);
            for (int v = 0; v < nv; ++v) fprintf(fo, "\t%16.15f", rows[i * nv + v]);
            fprintf(fo, "\n");
        }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    printf("  Elapsed time\t\t%16.15f seconds\n", (double)(clock() - c0) / CLOCKS_PER_SEC);
    printf("  Elapsed real time\t%16.15f seconds\n",
           (double)(t1.tv_sec - t0.tv_sec) + (double)(t1.tv_nsec - t0.tv_nsec) / 1e9);
    fclose(fo);

    /* final observables (io_functions.c:136-287) */
    printf("\n# Calculation of the final observables\n");
    int want_ped = 0, want_pmd = 0;
    for (int j = 0; j < P.nobs; ++j) {
        if (!strcmp(names[j], "PED")) want_ped = 1;
        else if (!strcmp(names[j], "PMD")) want_pmd = 1;
        else if (!strcmp(names[j], "wavefunction")) {
            CK(qnd_state_download(q, (double *)psi, psi_dev));
            FILE *fw = fopen("wavefunction.real", "w");
            if (!fw) fail("Error opening the file in write_wavefunction_imag_to_file");
            fprintf(fw, "DIMENSION\t%d\nNR", P.dim);
            for (int k = 0; k < P.dim; ++k) fprintf(fw, "\t%lld", (long long)P.nr[k]);
            fprintf(fw, "\nDR");
            for (int k = 0; k < P.dim; ++k) fprintf(fw, "\t%16.15f", P.dr[k]);
            fprintf(fw, "\nPSI_BINARY_START\n");
            fclose(fw);
            fw = fopen("wavefunction.real", "ab");
            if (!fw || fwrite(psi, sizeof(double complex), (size_t)n, fw) != (size_t)n) fail("Error writing Psi array to binary file");
            fclose(fw);
        }
    }
    if (want_ped || want_pmd) {
        int64_t npr[QND_DRV_MAX_DIM] = {1, 1, 1, 1, 1, 1};
        CK(qnd_final_spectra(q, psi_dev, P.r_mask[0], P.r_mask[1], P.pr_max, P.de, P.ne, NULL, npr, NULL));
        int64_t cnt = 1;
        for (int k = 0; k < P.dim; ++k) cnt *= npr[k];
        double *ped = want_ped ? calloc((size_t)P.ne + 1, sizeof(double)) : NULL;
        double *pmd = want_pmd ? calloc((size_t)(2 * cnt) + 1, sizeof(double)) : NULL;
        CK(qnd_final_spectra(q, psi_dev, P.r_mask[0], P.r_mask[1], P.pr_max, P.de, P.ne, ped, npr, pmd));
        if (want_ped) {
            printf("> Calculation of the photoelectron energy distribution\n");
            FILE *fp = fopen("PED.real", "w");
            if (!fp) fail("Error opening the file in write_output_imag");
            for (int j = 0; j < P.ne; ++j) fprintf(fp, "%16.15f\t%16.15f\n", j * P.de, ped[j]);
            fclose(fp);
        }
        if (want_pmd) {
            printf("> Calculation of the photoelectron momentum distribution\n");
            FILE *fp = fopen("PMD.real", "w");
            if (!fp) fail("Error opening the PMD.real file");
            fprintf(fp, "DIMENSION\t%d\nNPR", P.dim);
            for (int k = 0; k < P.dim; ++k) fprintf(fp, "\t%lld", (long long)npr[k]);
            fprintf(fp, "\nDP");
            for (int k = 0; k < P.dim; ++k) fprintf(fp, "\t%16.15f", 2. * M_PI / (double)(P.dr[k] * (double)P.nr[k]));
            fprintf(fp, "\nDATA_START\n");
            fclose(fp);
            fp = fopen("PMD.real", "ab");
            if (!fp || fwrite(pmd, sizeof(double), (size_t)(2 * cnt), fp) != (size_t)(2 * cnt))
                fprintf(stderr, "Rank 0 ERROR: Failed to write complete PMD record.\n");
            if (fp) fclose(fp);
        }
        free(ped);
        free(pmd);
    }
    printf("\n# The code ended successfully\n\n");
    CK(qnd_state_free(q, psi_dev));
    CK(qnd_ctx_destroy(q));
    free(psi);
    free(rows);
    free(E);
    free(A);
    free(alpha);
    free(names);
    return 0;
}
