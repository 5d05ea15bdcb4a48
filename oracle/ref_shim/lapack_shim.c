/*
 * lapack_shim.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The three LAPACK routines the reference calls through raw Fortran-ABI
 * declarations (Old-BVE-code/helpers.h:15-19: dgesv_, dgetrf_, dgetrs_),
 * written from the textbook algorithm because neither Accelerate nor a
 * system LAPACK exists here.  dgetrf_ is the unblocked right-looking LU
 * with partial pivoting in dgetf2 order (first maximal |a(i,k)| pivot, full
 * row swap, column scaled by the reciprocal of the pivot, rank-1 update);
 * dgetrs_ applies the row swaps, then unit-lower forward and upper backward
 * substitution.  This is the arithmetic the oracle pins (fss_oracle.c
 * lu_solve3) and the GPU tree build reproduces.
 */
#include <math.h>

int dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info) {
    int M = *m, N = *n, L = *lda, K = (M < N) ? M : N;
    *info = 0;
    for (int k = 0; k < K; k++) {
        int p = k;
        double mx = fabs(a[k + k * L]);
        for (int i = k + 1; i < M; i++)
            if (fabs(a[i + k * L]) > mx) { mx = fabs(a[i + k * L]); p = i; }
        ipiv[k] = p + 1;
        if (a[p + k * L] == 0.0) { if (*info == 0) *info = k + 1; continue; }
        if (p != k)
            for (int j = 0; j < N; j++) { double t = a[k + j * L]; a[k + j * L] = a[p + j * L]; a[p + j * L] = t; }
        double r = 1.0 / a[k + k * L];
        for (int i = k + 1; i < M; i++) a[i + k * L] *= r;
        for (int j = k + 1; j < N; j++)
            for (int i = k + 1; i < M; i++) a[i + j * L] -= a[i + k * L] * a[k + j * L];
    }
    return 0;
}

int dgetrs_(char *trans, int *n, int *nrhs, double *a, int *lda, int *ipiv, double *b, int *ldb, int *info) {
    (void)trans; /* the reference only passes 'N' */
    int N = *n, L = *lda, B = *ldb;
    *info = 0;
    for (int c = 0; c < *nrhs; c++) {
        double *x = b + c * B;
        for (int k = 0; k < N; k++) { int p = ipiv[k] - 1; if (p != k) { double t = x[k]; x[k] = x[p]; x[p] = t; } }
        for (int k = 0; k < N; k++) for (int i = k + 1; i < N; i++) x[i] -= a[i + k * L] * x[k];
        for (int k = N - 1; k >= 0; k--) { x[k] /= a[k + k * L]; for (int i = 0; i < k; i++) x[i] -= a[i + k * L] * x[k]; }
    }
    return 0;
}

int dgesv_(int *n, int *nrhs, double *a, int *lda, int *ipiv, double *b, int *ldb, int *info) {
    dgetrf_(n, n, a, lda, ipiv, info);
    if (*info != 0) return 0;
    char t = 'N';
    return dgetrs_(&t, n, nrhs, a, lda, ipiv, b, ldb, info);
}
