/*
 * FFTW3-MPI shim for one rank — TEST INFRASTRUCTURE ONLY.
 * With a single rank the slab decomposition is the whole grid
 * (local_n0 = N0, local_0_start = 0) and an MPI plan is a serial plan.
 */
#ifndef QND_SHIM_FFTW3_MPI_H
#define QND_SHIM_FFTW3_MPI_H

#include "fftw3.h"
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_MPI_DEFAULT_BLOCK (0)

void fftw_mpi_init(void);
void fftw_mpi_cleanup(void);
ptrdiff_t fftw_mpi_local_size_1d(ptrdiff_t n0, MPI_Comm comm, int sign, unsigned flags, ptrdiff_t *local_ni,
                                 ptrdiff_t *local_i_start, ptrdiff_t *local_no, ptrdiff_t *local_o_start);
ptrdiff_t fftw_mpi_local_size_many(int rnk, const ptrdiff_t *n, ptrdiff_t howmany, ptrdiff_t block0, MPI_Comm comm,
                                   ptrdiff_t *local_n0, ptrdiff_t *local_0_start);
fftw_plan fftw_mpi_plan_dft(int rnk, const ptrdiff_t *n, fftw_complex *in, fftw_complex *out, MPI_Comm comm, int sign,
                            unsigned flags);

#ifdef __cplusplus
}
#endif
#endif
