/*
 * Implementation of the single-rank MPI shim and the FFTW3-API shim —
 * TEST INFRASTRUCTURE ONLY (the oracle and the CPU baseline link it; the CUDA
 * library never does).
 *
 * The FFT is an iterative radix-2 decimation-in-time transform on contiguous
 * lines (power-of-two lengths only: the reference rejects other NR,
 * parameters.c:72-76). Multi-dimensional transforms are done axis by axis;
 * strided axes are gathered into contiguous blocks of lines first. Twiddles
 * are evaluated in long double and rounded once. OpenMP spreads lines over
 * threads (the reference hands FFTW omp_get_max_threads() threads,
 * meshgrid.c:159-161).
 */
#include "fftw3-mpi.h"

#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ MPI -- */

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; fflush(stdout); fflush(stderr); exit(code); }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm) {
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return MPI_SUCCESS;
}

static size_t shim_type_size(MPI_Datatype t) {
    switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_LONG_LONG_INT: return 8;
    case MPI_OFFSET: return 8;
    case MPI_C_DOUBLE_COMPLEX: return 16;
    case MPI_DOUBLE_INT: return 16;
    default: fprintf(stderr, "mpi shim: unknown datatype %d\n", t); exit(2);
    }
}

int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
    (void)op; (void)comm;
    if (in != MPI_IN_PLACE && in != out) memmove(out, in, (size_t)count * shim_type_size(type));
    return MPI_SUCCESS;
}

struct shim_file { int fd; };

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh) {
    (void)comm; (void)amode; (void)info;
    int fd = open(name, O_RDONLY);
    if (fd < 0) return 1;
    struct shim_file *f = (struct shim_file *)malloc(sizeof *f);
    f->fd = fd;
    *fh = (MPI_File)f;
    return MPI_SUCCESS;
}

int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype type, MPI_Status *st) {
    (void)st;
    struct shim_file *f = (struct shim_file *)fh;
    size_t want = (size_t)count * shim_type_size(type), got = 0;
    while (got < want) {
        ssize_t r = pread(f->fd, (char *)buf + got, want - got, (off_t)(offset + (MPI_Offset)got));
        if (r <= 0) break;
        got += (size_t)r;
    }
    if (got < want) memset((char *)buf + got, 0, want - got); /* short file: zero-fill, like a failed read */
    return got == want ? MPI_SUCCESS : 1;
}

int MPI_File_close(MPI_File *fh) {
    struct shim_file *f = (struct shim_file *)*fh;
    if (f) { close(f->fd); free(f); }
    *fh = NULL;
    return MPI_SUCCESS;
}

int MPI_Error_string(int code, char *str, int *len) {
    *len = snprintf(str, MPI_MAX_ERROR_STRING, "mpi shim error %d", code);
    return MPI_SUCCESS;
}

/* ------------------------------------------------------------------ FFT -- */

typedef struct { double re, im; } shim_c;

static int g_nthreads = 1;

/* Twiddles w[k] = exp(sign * 2*pi*i*k/n), k < n/2, evaluated in long double. */
static shim_c *make_twiddles(ptrdiff_t n, int sign) {
    ptrdiff_t h = n / 2 > 0 ? n / 2 : 1;
    shim_c *w = (shim_c *)malloc((size_t)h * sizeof(shim_c));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (ptrdiff_t k = 0; k < h; ++k) {
        long double a = two_pi * (long double)k / (long double)n;
        w[k].re = (double)cosl(a);
        w[k].im = (double)(sign * sinl(a));
    }
    return w;
}

/* In-place radix-2 DIT FFT of one contiguous line. */
static void fft_line(shim_c *a, ptrdiff_t n, const shim_c *w) {
    for (ptrdiff_t i = 1, j = 0; i < n; ++i) {
        ptrdiff_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { shim_c t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (ptrdiff_t len = 2; len <= n; len <<= 1) {
        ptrdiff_t half = len >> 1, step = n / len;
        for (ptrdiff_t i = 0; i < n; i += len) {
            for (ptrdiff_t k = 0; k < half; ++k) {
                shim_c t = w[k * step];
                shim_c u = a[i + k], v = a[i + k + half];
                double vr = v.re * t.re - v.im * t.im;
                double vi = v.re * t.im + v.im * t.re;
                a[i + k].re = u.re + vr;
                a[i + k].im = u.im + vi;
                a[i + k + half].re = u.re - vr;
                a[i + k + half].im = u.im - vi;
            }
        }
    }
}

/* Transform every line along `axis` of a row-major array with shape n[0..rank). */
static void fft_axis(shim_c *data, int rank, const ptrdiff_t *n, int axis, int sign, int nthreads) {
    ptrdiff_t L = n[axis], S = 1, O = 1;
    for (int k = axis + 1; k < rank; ++k) S *= n[k];
    for (int k = 0; k < axis; ++k) O *= n[k];
    if (L <= 1) return;
    shim_c *w = make_twiddles(L, sign);
    if (S == 1) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (ptrdiff_t o = 0; o < O; ++o) fft_line(data + o * L, L, w);
    } else {
        const ptrdiff_t B = S < 16 ? S : 16; /* lines gathered per block (S is a power of two) */
        ptrdiff_t nblk = O * (S / B);
#pragma omp parallel num_threads(nthreads)
        {
            shim_c *buf = (shim_c *)malloc((size_t)(B * L) * sizeof(shim_c));
#pragma omp for schedule(static)
            for (ptrdiff_t blk = 0; blk < nblk; ++blk) {
                ptrdiff_t o = blk / (S / B), s0 = (blk % (S / B)) * B;
                shim_c *base = data + o * L * S + s0;
                for (ptrdiff_t m = 0; m < L; ++m)
                    for (ptrdiff_t b = 0; b < B; ++b) buf[b * L + m] = base[m * S + b];
                for (ptrdiff_t b = 0; b < B; ++b) fft_line(buf + b * L, L, w);
                for (ptrdiff_t m = 0; m < L; ++m)
                    for (ptrdiff_t b = 0; b < B; ++b) base[m * S + b] = buf[b * L + m];
            }
            free(buf);
        }
    }
    free(w);
}

void qnd_shim_fft_nd(int rank, const ptrdiff_t *n, const fftw_complex *in, fftw_complex *out, int sign, int nthreads) {
    ptrdiff_t total = 1;
    for (int k = 0; k < rank; ++k) total *= n[k];
    if ((const void *)in != (const void *)out) memcpy(out, in, (size_t)total * sizeof(fftw_complex));
    for (int axis = rank - 1; axis >= 0; --axis) fft_axis((shim_c *)out, rank, n, axis, sign, nthreads < 1 ? 1 : nthreads);
}

struct qnd_shim_plan {
    int rank;
    ptrdiff_t n[8];
    fftw_complex *in, *out;
    int sign;
};

void fftw_execute(const fftw_plan p) { qnd_shim_fft_nd(p->rank, p->n, p->in, p->out, p->sign, g_nthreads); }
void fftw_destroy_plan(fftw_plan p) { free(p); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)fftw_malloc(n * sizeof(fftw_complex)); }
void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}
void fftw_free(void *p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads < 1 ? 1 : nthreads; }
void fftw_cleanup(void) {}
void fftw_cleanup_threads(void) {}

void fftw_mpi_init(void) {}
void fftw_mpi_cleanup(void) {}

ptrdiff_t fftw_mpi_local_size_1d(ptrdiff_t n0, MPI_Comm comm, int sign, unsigned flags, ptrdiff_t *local_ni,
                                 ptrdiff_t *local_i_start, ptrdiff_t *local_no, ptrdiff_t *local_o_start) {
    (void)comm; (void)sign; (void)flags;
    *local_ni = n0; *local_i_start = 0;
    *local_no = n0; *local_o_start = 0;
    return n0;
}

ptrdiff_t fftw_mpi_local_size_many(int rnk, const ptrdiff_t *n, ptrdiff_t howmany, ptrdiff_t block0, MPI_Comm comm,
                                   ptrdiff_t *local_n0, ptrdiff_t *local_0_start) {
    (void)block0; (void)comm;
    ptrdiff_t total = howmany;
    for (int k = 0; k < rnk; ++k) total *= n[k];
    *local_n0 = n[0];
    *local_0_start = 0;
    return total;
}

fftw_plan fftw_mpi_plan_dft(int rnk, const ptrdiff_t *n, fftw_complex *in, fftw_complex *out, MPI_Comm comm, int sign,
                            unsigned flags) {
    (void)comm; (void)flags;
    if (rnk < 1 || rnk > 8) return NULL;
    fftw_plan p = (fftw_plan)calloc(1, sizeof *p);
    p->rank = rnk;
    for (int k = 0; k < rnk; ++k) p->n[k] = n[k];
    p->in = in; p->out = out; p->sign = sign;
    return p;
}
