/* params.c — see params.h. */
#include "params.h"

#include <stdlib.h>
#include <string.h>

void qnd_read_tokens(const char *filename, qnd_tokens *t) {
    FILE *f = fopen(filename, "r");
    if (!f) {
        perror("Error opening parameter file");
        exit(1);
    }
    char buf[512];
    t->ntok = 0;
    while (fscanf(f, "%511s", buf) == 1) {
        if (t->ntok == QND_MAX_TOKENS) {
            fprintf(stderr, "ERROR: too many tokens in %s\n", filename);
            exit(1);
        }
        t->tok[t->ntok++] = strdup(buf);
    }
    fclose(f);
}

int qnd_is_key(const char *s, const char *const *keys) {
    for (int k = 0; keys[k]; ++k)
        if (strcmp(s, keys[k]) == 0) return 1;
    return 0;
}

void qnd_expect(const qnd_tokens *t, int i, int n, const char *const *keys) {
    const char *name = t->tok[i];
    for (int c = 0; c < n; ++c) {
        const int q = i + 1 + c;
        if (q >= t->ntok) {
            fprintf(stderr, "Rank 0 ERROR reading file: Parameter '%s' expected %d argument(s), but found only %d (reached EOF).\n",
                    name, n, c);
            exit(1);
        }
        if (qnd_is_key(t->tok[q], keys)) {
            fprintf(stderr, "Rank 0 ERROR reading file: Parameter '%s' expected %d argument(s), but found only %d (hit new parameter '%s').\n",
                    name, n, c, t->tok[q]);
            exit(1);
        }
    }
    const int q = i + 1 + n;
    if (q < t->ntok && !qnd_is_key(t->tok[q], keys)) {
        fprintf(stderr, "Rank 0 ERROR reading file: Parameter '%s' expected exactly %d argument(s), but found extra, unrecognized token '%s'.\n",
                name, n, t->tok[q]);
        exit(1);
    }
}

int qnd_find_dimension(const qnd_tokens *t) {
    for (int i = 0; i < t->ntok; ++i)
        if (strcmp(t->tok[i], "DIMENSION") == 0) {
            int d = 0;
            if (i + 1 >= t->ntok || sscanf(t->tok[i + 1], "%d", &d) != 1) {
                perror("The dimension is undetermined");
                exit(1);
            }
            return d;
        }
    printf("\nThe dimension is not specified\n");
    exit(1);
}
