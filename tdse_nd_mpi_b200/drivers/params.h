/*
 * params.h — reader for QuantumND parameter files (`KEY value ...` tokens separated by white
 * space) with the reference's checks (parameters.c:11-212, 998-1135): a known key takes exactly
 * its number of values (fewer before the next known key or the end of the file, or an extra token
 * that is not a known key, is an error); an unknown key is an error. Errors print the reference's
 * messages and exit(1), as its MPI_Abort does.
 */
#ifndef QND_DRIVER_PARAMS_H
#define QND_DRIVER_PARAMS_H

#include <stdio.h>

#define QND_MAX_TOKENS 4096
#define QND_DRV_MAX_DIM 6  /* grid dimensions the drivers take (the engine's limit) */

typedef struct {
    int ntok;
    char *tok[QND_MAX_TOKENS];
} qnd_tokens;

/* Read every white-space separated token of the file (exit(1) if it cannot be opened). */
void qnd_read_tokens(const char *filename, qnd_tokens *t);
/* 1 if s is in the NULL-terminated list */
int qnd_is_key(const char *s, const char *const *keys);
/* Check that key t->tok[i] is followed by exactly n values (parameters.c:1080-1130); exit(1) otherwise. */
void qnd_expect(const qnd_tokens *t, int i, int n, const char *const *keys);
/* The value of DIMENSION (parameters.c:998-1030); exit(1) when absent. */
int qnd_find_dimension(const qnd_tokens *t);

#endif
