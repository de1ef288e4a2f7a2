/*
 * fd2_libm_table -- tabulates where the host C library's float acosf and
 * asinf differ from the float rounding of the double acos / asin, for every
 * float in [0, 1].
 *
 * The reference's C transport (main/kernel_cuda_c_ver1_0.cu, C branch)
 * calls acosf and asinf; their results are not the correctly rounded ones,
 * and the walk in a cylinder amplifies a 1-ulp angle difference into a
 * different photon history within a few hundred photons.  The replay mode
 * therefore applies this table on the GPU to reproduce the reference's
 * float results exactly.  Every difference on [0, 1] is one ulp; the table
 * stores, sorted, the float bit pattern of each such input with bit 31 set
 * when the library's result is one ulp below the double-rounded one.
 *
 * Output file: "FD2LIBM1", uint32 n_acos, uint32 n_asin, n_acos entries,
 * n_asin entries (little-endian).
 *
 * usage: fd2_libm_table OUTFILE
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NTHREADS 16

typedef struct {
    uint32_t lo, hi; /* inclusive bit range */
    uint32_t *acos_e, *asin_e;
    size_t n_acos, n_asin, cap_acos, cap_asin;
} job_t;

static float from_bits(uint32_t u)
{
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static uint32_t to_bits(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

static int push(uint32_t **a, size_t *n, size_t *cap, uint32_t v)
{
    if (*n == *cap) {
        size_t c = *cap ? 2 * *cap : 4096;
        uint32_t *p = (uint32_t *)realloc(*a, c * sizeof(uint32_t));
        if (!p) return -1;
        *a = p;
        *cap = c;
    }
    (*a)[(*n)++] = v;
    return 0;
}

static void *scan(void *arg)
{
    job_t *j = (job_t *)arg;
    for (uint32_t u = j->lo;; ++u) {
        const float x = from_bits(u);
        const int32_t da = (int32_t)to_bits(acosf(x)) - (int32_t)to_bits((float)acos((double)x));
        const int32_t ds = (int32_t)to_bits(asinf(x)) - (int32_t)to_bits((float)asin((double)x));
        if (da) push(&j->acos_e, &j->n_acos, &j->cap_acos, u | (da < 0 ? 0x80000000u : 0u));
        if (ds) push(&j->asin_e, &j->n_asin, &j->cap_asin, u | (ds < 0 ? 0x80000000u : 0u));
        if (da > 1 || da < -1 || ds > 1 || ds < -1) {
            fprintf(stderr, "fd2_libm_table: difference of more than one ulp at %a\n", (double)x);
            exit(2);
        }
        if (u == j->hi) break;
    }
    return NULL;
}

int main(int argc, char **argv)
{
    if (argc != 2) {
        fprintf(stderr, "usage: %s OUTFILE\n", argv[0]);
        return 2;
    }
    const uint32_t top = to_bits(1.0f);
    job_t jobs[NTHREADS];
    pthread_t th[NTHREADS];
    memset(jobs, 0, sizeof jobs);
    for (int t = 0; t < NTHREADS; ++t) {
        jobs[t].lo = (uint32_t)(((uint64_t)top + 1) * t / NTHREADS);
        jobs[t].hi = (uint32_t)(((uint64_t)top + 1) * (t + 1) / NTHREADS - 1);
        pthread_create(&th[t], NULL, scan, &jobs[t]);
    }
    uint32_t na = 0, ns = 0;
    for (int t = 0; t < NTHREADS; ++t) {
        pthread_join(th[t], NULL);
        na += (uint32_t)jobs[t].n_acos;
        ns += (uint32_t)jobs[t].n_asin;
    }
    char tmp[4096];
    snprintf(tmp, sizeof tmp, "%s.tmp", argv[1]);
    FILE *f = fopen(tmp, "wb");
    if (!f) return 1;
    int ok = fwrite("FD2LIBM1", 1, 8, f) == 8 && fwrite(&na, 4, 1, f) == 1 && fwrite(&ns, 4, 1, f) == 1;
    for (int t = 0; t < NTHREADS && ok; ++t)
        ok = fwrite(jobs[t].acos_e, 4, jobs[t].n_acos, f) == jobs[t].n_acos;
    for (int t = 0; t < NTHREADS && ok; ++t)
        ok = fwrite(jobs[t].asin_e, 4, jobs[t].n_asin, f) == jobs[t].n_asin;
    if (fclose(f) != 0 || !ok || rename(tmp, argv[1]) != 0) return 1;
    printf("fd2_libm_table: %u acosf and %u asinf corrections\n", na, ns);
    return 0;
}
