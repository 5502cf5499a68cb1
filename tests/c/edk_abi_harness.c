/* Plain-C client of the C-ABI (what a Fortran ISO_C_BINDING caller does):
 * builds the 1 impurity + 7 bath model, applies Hmult__ to a host vector,
 * runs Lanczos pass 1 and prints E0 and the first coefficients.  Usage:
 *   edk_abi_harness <x_in.bin> <y_out.bin>    (x: dim doubles) */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "edk.h"

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    const int nc = 1, nb = 7;
    double ec[2] = {-1.0, -1.0}, u[1] = {2.0}, jj[1] = {0.0};
    double eb[2 * 49], vbc[2 * 7];
    FILE *f = fopen("model.bin", "rb");
    if (!f || fread(eb, sizeof(double), 98, f) != 98 || fread(vbc, sizeof(double), 14, f) != 14) return 3;
    fclose(f);
    edk_model m = {nc, nb, ec, eb, vbc, u, jj, 0.0, 1e-3};
    edk_ctx *ctx = NULL;
    edk_h *h = NULL;
    if (edk_ctx_create(0, NULL, &ctx) != EDK_OK) return 4;
    if (edk_h_create(ctx, &m, 4, 4, &h) != EDK_OK) { fprintf(stderr, "%s\n", edk_ctx_last_error(ctx)); return 5; }
    int64_t dim, du, dd;
    edk_h_dims(h, &dim, &du, &dd);
    double *x = malloc(sizeof(double) * dim), *y = malloc(sizeof(double) * dim);
    f = fopen(argv[1], "rb");
    if (!f || fread(x, sizeof(double), dim, f) != (size_t)dim) return 6;
    fclose(f);
    if (edk_hmult_host(h, EDK_F64, dim, x, y) != EDK_OK) return 7;
    f = fopen(argv[2], "wb");
    fwrite(y, sizeof(double), dim, f);
    fclose(f);
    double diag[1002], sub[1002], vecp[1002];
    edk_lanczos_opts o;
    memset(&o, 0, sizeof o);
    o.nitermax = 1000; o.neigen = 1; o.tolerance = 1e-12; o.demax = 1e300;
    o.cutoff_min_lanczos_vec = 1e-25; o.dtype = EDK_F64; o.check_every = 4;
    edk_lanczos_result r;
    memset(&r, 0, sizeof r);
    r.diag = diag; r.subdiag = sub; r.vecp = vecp;
    if (edk_lanczos_e0(h, &o, &r) != EDK_OK) return 8;
    /* invalid input is an error code, not a crash */
    edk_h *bad = NULL;
    int rc = edk_h_create(ctx, &m, 99, 4, &bad);
    printf("dim %lld E0 %.15f niter %d alpha1 %.15f invalid_rc %d\n", (long long)dim, r.E[0], r.niter, diag[0], rc);
    edk_h_destroy(h);
    edk_ctx_destroy(ctx);
    free(x); free(y);
    return rc == EDK_ERR_INVALID ? 0 : 9;
}
