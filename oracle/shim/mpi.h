/*
 * Single-rank MPI shim — TEST INFRASTRUCTURE ONLY.
 *
 * Lets the reference's own C sources (every .c file in QuantumND's src/) compile and run as
 * one process without an MPI library. Only the calls those sources make are
 * provided. With one rank every collective is a copy (or a no-op) and the
 * MPI-IO reads used by Read_wavefunction_MPI (src/io_functions.c:389-420)
 * become pread(2) on a plain file descriptor.
 *
 * Nothing in the shipped CUDA library includes this header.
 */
#ifndef QND_SHIM_MPI_H
#define QND_SHIM_MPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef long long MPI_Count;
typedef struct { int fd; } *MPI_File;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_ERROR_STRING 256
#define MPI_INFO_NULL 0
#define MPI_MODE_RDONLY 2
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

/* Datatype handles encode their size in bytes (one rank: only sizes matter). */
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_LONG_LONG_INT 9          /* 8 bytes; distinct handle from MPI_DOUBLE */
#define MPI_LONG_LONG 9
#define MPI_OFFSET 10                /* 8 bytes */
#define MPI_C_DOUBLE_COMPLEX 16
#define MPI_DOUBLE_INT 17            /* struct {double; int;} padded to 16 bytes */

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MAXLOC 3

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype type, MPI_Status *st);
int MPI_File_close(MPI_File *fh);
int MPI_Error_string(int code, char *str, int *len);

#ifdef __cplusplus
}
#endif
#endif
