/* Test-oracle infrastructure only.
 *
 * Replacement for BD_BOX's src/rand_move.c, linked into the oracle harness
 * in place of the original (the same link-time substitution BD_BOX itself
 * uses between its CPU and CUDA builds, src/Makefile.am:44-78).
 *
 * gauss_rand() serves consecutive float64 values from the file named by the
 * BDB_GAUSS_FILE environment variable, so that the oracle and the GPU library
 * consume the identical Gaussian stream. rand_move.c:132-168 draws them from
 * drand48_r + Marsaglia polar instead; that path is kept in the reference
 * binary (oracle/_ref/bd_box) and is not used by the harness.
 *
 * The exported names and the two MAKE_STR_IN variables mirror rand_move.h
 * (rand_move.h / rand_move.c:40-41) because input.c and restart.c bind them.
 */
#if HAVE_CONFIG_H
#include <config.h>
#endif
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rand_move.h"

MAKE_STR_IN(INT, rand_seed, 12345, "random generator seed")
MAKE_STR_IN(RAND_STATE, rand_state, 0, "inner variable")

static FILE* g_gauss = NULL;
static long long g_served = 0;

void init_rand(unsigned int seed)
{
    const char* path = getenv("BDB_GAUSS_FILE");
    (void)seed;
    if (g_gauss) return;
    if (!path) return; /* modes that draw no noise need no file */
    g_gauss = fopen(path, "rb");
    if (!g_gauss) {
        fprintf(stderr, "oracle: cannot open BDB_GAUSS_FILE=%s\n", path);
        exit(3);
    }
}

void free_rand(void)
{
    if (g_gauss) fclose(g_gauss);
    g_gauss = NULL;
}

double rand_d48(void)
{
    fprintf(stderr, "oracle: rand_d48 is not served by the Gaussian-file generator\n");
    exit(3);
    return 0.0;
}

void gauss_rand(DOUBLE* tabl, INT tabl_size)
{
    size_t got;
    if (!g_gauss) {
        fprintf(stderr, "oracle: gauss_rand called without BDB_GAUSS_FILE\n");
        exit(3);
    }
    got = fread(tabl, sizeof(DOUBLE), (size_t)tabl_size, g_gauss);
    if (got != (size_t)tabl_size) {
        fprintf(stderr, "oracle: Gaussian file exhausted after %lld values\n", g_served + (long long)got);
        exit(4);
    }
    g_served += tabl_size;
}

long long oracle_gauss_served(void) { return g_served; }

void get_state(char** state, INT* size)
{
    *state = (char*)&g_served;
    *size = (INT)sizeof(g_served);
}

void set_state(char* state, INT size)
{
    if (size != (INT)sizeof(g_served)) {
        fprintf(stderr, "oracle: random generator state size mismatch\n");
        exit(3);
    }
    memcpy(&g_served, state, sizeof(g_served));
}
