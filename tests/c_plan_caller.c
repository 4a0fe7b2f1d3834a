/* A C99 caller of the batched plan interface, as a host program would use it: synthetic inputs from
 * the library's generator, a fused plan, an autotune, one execution, and the energies printed as
 * "emp4 emp5" with 17 significant digits.  Usage: c_plan_caller nocc nvir seed */
#include <stdio.h>
#include <stdlib.h>

#include "trpdrv.h"

int main(int argc, char **argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: %s nocc nvir seed\n", argv[0]);
        return 2;
    }
    const int nocc = atoi(argv[1]), nvir = atoi(argv[2]), ncor = 0;
    const unsigned long long seed = strtoull(argv[3], NULL, 10);
    double *t[TRPDRV_T_COUNT];
    for (int w = 0; w < TRPDRV_T_COUNT; ++w) {
        const size_t n = trpdrv_tensor_elems(w, ncor, nocc, nvir);
        t[w] = (double *)malloc(sizeof(double) * n);
        if (!t[w] || trpdrv_synth_fill(w, ncor, nocc, nvir, seed, TRPDRV_DIST_UNIFORM, t[w], n) != TRPDRV_OK) {
            fprintf(stderr, "inputs: %s\n", trpdrv_last_error_message());
            return 1;
        }
    }
    trpdrv_system sys = {.ncor = ncor, .nocc = nocc, .nvir = nvir, .a = ncor + nocc + 1,
                         .eorb = t[TRPDRV_T_EORB], .t2 = t[TRPDRV_T_T2], .jvv = t[TRPDRV_T_JVV],
                         .kvv = t[TRPDRV_T_KVV], .tov = t[TRPDRV_T_TOV], .xov = t[TRPDRV_T_XOV],
                         .jov = t[TRPDRV_T_JOV], .kov = t[TRPDRV_T_KOV], .dintc = t[TRPDRV_T_DINTC],
                         .dintx = t[TRPDRV_T_DINTX], .t1v = t[TRPDRV_T_T1V]};
    trpdrv_options opt;
    trpdrv_options_default(&opt);
    trpdrv_plan *p = NULL;
    double e4 = 0.0, e5 = 0.0;
    int rc = trpdrv_plan_create(&p, &sys, 1, &opt);
    if (rc == TRPDRV_OK) rc = trpdrv_plan_upload(p, &sys, NULL);
    if (rc == TRPDRV_OK) rc = trpdrv_plan_autotune(p, NULL);
    if (rc == TRPDRV_OK) rc = trpdrv_plan_execute(p, NULL);
    if (rc == TRPDRV_OK) rc = trpdrv_plan_energies(p, &e4, &e5);
    if (p) trpdrv_plan_destroy(p);
    for (int w = 0; w < TRPDRV_T_COUNT; ++w) free(t[w]);
    if (rc != TRPDRV_OK) {
        fprintf(stderr, "%s: %s\n", trpdrv_status_string(rc), trpdrv_last_error_message());
        return 1;
    }
    printf("%.17e %.17e\n", e4, e5);
    return 0;
}
