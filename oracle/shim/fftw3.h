/*
 * FFTW3-API shim — TEST INFRASTRUCTURE ONLY.
 *
 * The reference (QuantumND) links FFTW3 + FFTW3-MPI (Makefile:7), whose version
 * is unpinned and which is not installed here. This header declares the subset
 * of the FFTW API the reference calls (meshgrid.c:159-167, every fftw_execute
 * site) and the implementation in fft_shim.c computes the same mathematical
 * object: the unnormalised complex DFT with FFTW's sign convention,
 * FORWARD = exp(-2*pi*i*k*n/N), BACKWARD = exp(+2*pi*i*k*n/N), over all axes of
 * a row-major array, out of place. Our FFT is an independent FP64 radix-2
 * implementation validated against numpy.fft (pocketfft).
 */
#ifndef QND_SHIM_FFTW3_H
#define QND_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* With <complex.h> included first (as the reference does) FFTW uses the C99 type. */
typedef double _Complex fftw_complex;
typedef struct qnd_shim_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
fftw_complex *fftw_alloc_complex(size_t n);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup(void);
void fftw_cleanup_threads(void);

/* Not part of FFTW: direct entry used by the oracle restatement and tests. */
void qnd_shim_fft_nd(int rank, const ptrdiff_t *n, const fftw_complex *in, fftw_complex *out, int sign, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
