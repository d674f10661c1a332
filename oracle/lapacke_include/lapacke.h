/*
 * The one LAPACKE call of the reference's eigenvalue analysis
 * (pgabor/sdddst src/spectral_decompositor.cpp:188), declared for compiling
 * that file in place against oracle/lapacke_shim.c.  Test infrastructure only.
 */
#ifndef SDDDST_ORACLE_LAPACKE_SHIM_H
#define SDDDST_ORACLE_LAPACKE_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

typedef int lapack_int;

lapack_int LAPACKE_dsyevd(int matrix_layout, char jobz, char uplo, lapack_int n, double *a, lapack_int lda,
                          double *w);

/* the matrix most recently passed to LAPACKE_dsyevd (n x n, as passed) */
long lapacke_shim_last_input(double *out, long cap);

#ifdef __cplusplus
}
#endif

#endif
