/*
 * quantumnd_imag.c — drop-in QuantumND_imag (QuantumND_imag.c:56-264) over the C ABI of
 * libqnd_b200.so: the same parameter file and `KEY VALUE` overrides, the same console report and
 * the same output.imag (text header, then the complex128 states, io_functions.c:56-105). The
 * imaginary-time loop, Gram-Schmidt and the energies run on the GPU (include/qnd.h).
 *
 *     QuantumND_imag <params.imag> [DT v] [TINTEGRATION v] [OUTPUT_IMAG name]
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

static const char *const KEYS_IMAG[] = {"OUTPUT_IMAG", "DIMENSION", "DR", "NR", "N_STATES", "POTENTIAL",
                                        "INTEGRATOR", "DT", "TINTEGRATION", NULL};

typedef struct {
    int dim;
    int64_t nr[QND_DRV_MAX_DIM];
    double dr[QND_DRV_MAX_DIM];
    int nstates;
    char potential[64], integrator[64], output[256];
    double dt, T;
} ImagParams;

/* Initialize_parameters_imag (parameters.c:11-212): defaults, file, command-line overrides. */
static void read_params(const char *file, int argc, char **argv, ImagParams *P) {
    qnd_tokens t;
    qnd_read_tokens(file, &t);
    memset(P, 0, sizeof *P);
    snprintf(P->output, sizeof P->output, "output.imag");
    P->nstates = 1;
    snprintf(P->potential, sizeof P->potential, "H_3D");
    snprintf(P->integrator, sizeof P->integrator, "BM4");
    P->dt = .1;
    P->T = 100.;
    P->dim = qnd_find_dimension(&t);
    if (P->dim < 1 || P->dim > QND_DRV_MAX_DIM) {
        fprintf(stderr, "ERROR: DIMENSION %d is not supported (1 to %d)\n", P->dim, QND_DRV_MAX_DIM);
        exit(1);
    }
    for (int j = 0; j < P->dim; ++j) {
        P->nr[j] = 256;
        P->dr[j] = .1;
    }
    for (int i = 0; i < t.ntok;) {
        const char *k = t.tok[i];
        int n;
        if (!strcmp(k, "DIMENSION")) n = 1;
        else if (!strcmp(k, "NR") || !strcmp(k, "DR")) n = P->dim;
        else if (!strcmp(k, "N_STATES") || !strcmp(k, "DT") || !strcmp(k, "TINTEGRATION") || !strcmp(k, "POTENTIAL") ||
                 !strcmp(k, "INTEGRATOR") || !strcmp(k, "OUTPUT_IMAG"))
            n = 1;
        else {
            printf("\nUnknown parameter: %s\n", k);
            fprintf(stderr, "Error with params.txt\n");
            exit(1);
        }
        qnd_expect(&t, i, n, KEYS_IMAG);
        const char *v = t.tok[i + 1];
        if (!strcmp(k, "NR")) {
            for (int j = 0; j < P->dim; ++j) {
                long long x;
                if (sscanf(t.tok[i + 1 + j], "%lld", &x) != 1) {
                    perror("The number of grid points is not completely determined");
                    exit(1);
                }
                if (x != 0 && (x & (x - 1)) != 0) {
                    printf("\nThe number of points on the grid must be a power of 2\n");
                    fprintf(stderr, "Error with grid points number\n");
                    exit(1);
                }
                P->nr[j] = x;
            }
        } else if (!strcmp(k, "DR")) {
            for (int j = 0; j < P->dim; ++j)
                if (sscanf(t.tok[i + 1 + j], "%lf", &P->dr[j]) != 1) {
                    perror("The grid spacing is not completely determined");
                    exit(1);
                }
        } else if (!strcmp(k, "N_STATES")) {
            if (sscanf(v, "%d", &P->nstates) != 1) {
                perror("The number of states is undetermined");
                exit(1);
            }
        } else if (!strcmp(k, "DT")) {
            if (sscanf(v, "%lf", &P->dt) != 1) {
                perror("The time step is undetermined");
                exit(1);
            }
        } else if (!strcmp(k, "TINTEGRATION")) {
            if (sscanf(v, "%lf", &P->T) != 1) {
                perror("The time integration is undetermined");
                exit(1);
            }
        } else if (!strcmp(k, "POTENTIAL")) {
            snprintf(P->potential, sizeof P->potential, "%s", v);
        } else if (!strcmp(k, "INTEGRATOR")) {
            snprintf(P->integrator, sizeof P->integrator, "%s", v);
        } else if (!strcmp(k, "OUTPUT_IMAG")) {
            snprintf(P->output, sizeof P->output, "%s", v);
        }
        i += 1 + n;
    }
    if (P->dim == 0 || P->nr[0] <= 0 || P->nstates <= 0) {
        fprintf(stderr, "ERROR: Could not read or interpret the file %s properly.\n", file);
        fprintf(stderr, "\n--- FATAL ERROR: Parameter file processing failed. Aborting job. ---\n");
        exit(1);
    }
    for (int a = 2; a < argc; a += 2) {
        if (a + 1 >= argc) {
            fprintf(stderr, "Rank 0 ERROR: Parameter key '%s' found without a corresponding value.\n", argv[a]);
            exit(1);
        }
        if (!strcmp(argv[a], "DT")) P->dt = atof(argv[a + 1]);
        else if (!strcmp(argv[a], "TINTEGRATION")) P->T = atof(argv[a + 1]);
        else if (!strcmp(argv[a], "OUTPUT_IMAG")) snprintf(P->output, sizeof P->output, "%s", argv[a + 1]);
        else {
            fprintf(stderr, "Rank 0 ERROR: Unrecognized parameter key '%s'. Check spelling.\n", argv[a]);
            exit(1);
        }
    }
    printf("  DIMENSION\t\t%d\n", P->dim);
    printf("  NR\t\t");
    for (int j = 0; j < P->dim; ++j) printf("\t%lld", (long long)P->nr[j]);
    printf("\n  DR\t\t");
    for (int j = 0; j < P->dim; ++j) printf("\t%16.15f", P->dr[j]);
    printf("\n");
    printf("  N_STATES\t\t%d\n", P->nstates);
    printf("  POTENTIAL\t\t%s\n", P->potential);
    printf("  INTEGRATOR\t\t%s\n", P->integrator);
    printf("  DT\t\t\t%16.15f\n", P->dt);
    printf("  TINTEGRATION\t\t%16.15f\n", P->T);
    printf("  OUTPUT_IMAG\t\t%s\n", P->output);
    fflush(stdout);
}

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "Usage: %s <param_file> [KEY VALUE ...]\n", argv[0]);
        return 1;
    }
    printf("\n##############################################\n");
    printf("\n##    PROGRAM IMAGINARY-TIME PROPAGATION    ##\n");
    printf("\n##############################################\n");
    ImagParams P;
    read_params(argv[1], argc, argv, &P);

    qnd_ctx *q = NULL;
    CK(qnd_ctx_create(P.dim, P.nr, P.dr, P.integrator, P.dt, QND_FP64, &q));
    CK(qnd_set_potential_named(q, P.potential));
    int64_t n = 0;
    double dNr = 0;
    CK(qnd_ctx_info(q, &n, NULL, NULL, &dNr, NULL));
    int64_t bytes = 0;
    CK(qnd_state_bytes(q, &bytes));
    void *base = NULL;
    CK(qnd_state_alloc(q, P.nstates, &base));
    void **states = malloc(sizeof(void *) * (size_t)P.nstates);
    for (int j = 0; j < P.nstates; ++j) states[j] = (char *)base + (size_t)j * (size_t)bytes;

    /* grid axes (meshgrid.c:75-89): r = -L/2 + i dr */
    double complex *psi = malloc(sizeof(double complex) * (size_t)n);
    double complex *all = malloc(sizeof(double complex) * (size_t)n * (size_t)P.nstates);
    double (*E)[2] = malloc(sizeof(double[2]) * (size_t)P.nstates);
    /* the imaginary-time loop count of `for (time = 0; time < T; time += dt)` (QuantumND_imag.c:182) */
    int64_t nsteps = 0;
    for (double time = 0.; time < P.T; time += P.dt) ++nsteps;

    printf("\n# Imaginary-time propagation\n");
    for (int j = 0; j < P.nstates; ++j) {
        clock_t c0 = clock();
        struct timespec t0, t1;
        clock_gettime(CLOCK_MONOTONIC, &t0);
        /* initial state (QuantumND_imag.c:171-177): (|r| + (i % 3)) exp(-|r|) */
        for (int64_t i = 0; i < n; ++i) {
            int64_t ik[QND_DRV_MAX_DIM] = {0}, idx = i;
            for (int k = P.dim - 1; k >= 0; --k) {
                ik[k] = idx % P.nr[k];
                idx /= P.nr[k];
            }
            double r2 = 0;
            for (int k = 0; k < P.dim; ++k) {
                const double x = -.5 * ((double)P.nr[k] * P.dr[k]) + (double)ik[k] * P.dr[k];
                r2 += x * x;
            }
            const double radius = sqrt(r2);
            psi[i] = (radius + (double)(i % 3)) * exp(-radius) + I * 0.;
        }
        CK(qnd_state_upload(q, states[j], (const double *)psi));
        CK(qnd_imag_propagate(q, states, j, nsteps));
        CK(qnd_energies(q, states[j], 2, E[j]));
        clock_gettime(CLOCK_MONOTONIC, &t1);
        const char *lz = "Lz";
        double Lz = 0;
        CK(qnd_observables(q, states[j], 1, &lz, NULL, &Lz));
        printf("\n> eigenfunction %d:\n", j + 1);
        printf("  E\t\t\t%16.15f\n", E[j][0]);
        printf("  DE\t\t\t%5.4e \n", E[j][1] - E[j][0] * E[j][0]);
        printf("  Lz\t\t\t%5.4e \n", Lz);
        printf("  Elapsed CPU time\t%16.15f seconds\n", (double)(clock() - c0) / CLOCKS_PER_SEC);
        printf("  Elapsed real time\t%16.15f seconds\n",
               (double)(t1.tv_sec - t0.tv_sec) + (double)(t1.tv_nsec - t0.tv_nsec) / 1e9);
    }
    printf("\n");

    /* remove each state's global phase: the phase at its largest |psi| (QuantumND_imag.c:213-243) */
    for (int j = 0; j < P.nstates; ++j) {
        double complex *s = all + (size_t)j * (size_t)n;
        CK(qnd_state_download(q, (double *)s, states[j]));
        double best = 0., ph = 0.;
        for (int64_t i = 0; i < n; ++i) {
            const double m = cabs(s[i]);
            if (m > best) {
                best = m;
                ph = carg(s[i]);
            }
        }
        const double complex f = cexp(-I * ph);
        for (int64_t i = 0; i < n; ++i) s[i] *= f;
    }

    /* output.imag (io_functions.c:56-105) */
    FILE *f = fopen(P.output, "w");
    if (!f) {
        perror("Error opening the file in write_output_imag");
        return 1;
    }
    fprintf(f, "DIMENSION\t%d\n", P.dim);
    fprintf(f, "N_STATES\t%d\n", P.nstates);
    fprintf(f, "NR");
    for (int j = 0; j < P.dim; ++j) fprintf(f, "\t%lld", (long long)P.nr[j]);
    fprintf(f, "\nDR");
    for (int j = 0; j < P.dim; ++j) fprintf(f, "\t%16.15f", P.dr[j]);
    fprintf(f, "\nPOTENTIAL\t%s\n", P.potential);
    fprintf(f, "E\t");
    for (int j = 0; j < P.nstates; ++j) fprintf(f, "\t%16.15f", E[j][0]);
    fprintf(f, "\nDE");
    for (int j = 0; j < P.nstates; ++j) fprintf(f, "\t%16.15f", E[j][1] - E[j][0] * E[j][0]);
    fprintf(f, "\nPSI\n");
    fclose(f);
    f = fopen(P.output, "ab");
    if (!f) {
        perror("Error opening the appended file in write_output_imag");
        return 1;
    }
    if (fwrite(all, sizeof(double complex), (size_t)n * (size_t)P.nstates, f) != (size_t)n * (size_t)P.nstates) {
        fprintf(stderr, "Rank 0 ERROR: Failed to write all elements to binary file.\n");
        return 1;
    }
    fclose(f);
    printf("# The code ended successfully\n\n");
    CK(qnd_state_free(q, base));
    CK(qnd_ctx_destroy(q));
    free(states);
    free(psi);
    free(all);
    free(E);
    return 0;
}
