/*
 * LAPACKE_dsyevd for the reference's eigenvalue analysis compiled in place
 * (test infrastructure only; LAPACKE is not installed here).
 *
 * The reference calls LAPACKE_dsyevd(LAPACK_COL_MAJOR, 'v', 'U', n, H, n, w)
 * on its symmetric Hessian (src/spectral_decompositor.cpp:188).  This shim
 * keeps a copy of the matrix it is given (lapacke_shim_last_input) and
 * returns the eigenpairs from the cyclic Jacobi method with a threshold
 * sweep (Golub and Van Loan, Matrix Computations, 4th ed., 8.5.2-8.5.3):
 * eigenvalues ascending in w, unit eigenvectors in the columns of the
 * column-major array a, as dsyevd returns them.  O(n^3) per sweep; meant
 * for the small matrices of the parity tests.
 */
#include "lapacke.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static double *g_last = NULL;
static long g_last_n = 0;

long lapacke_shim_last_input(double *out, long cap)
{
    long m = g_last_n * g_last_n;
    if (out && cap >= m) memcpy(out, g_last, sizeof(double) * (size_t)m);
    return g_last_n;
}

lapack_int LAPACKE_dsyevd(int layout, char jobz, char uplo, lapack_int n, double *a, lapack_int lda, double *w)
{
    (void)uplo;
    if (n < 0 || lda < n || (layout != LAPACK_COL_MAJOR && layout != LAPACK_ROW_MAJOR)) return -1;
    free(g_last);
    g_last = (double *)malloc(sizeof(double) * (size_t)n * (size_t)n + 8);
    g_last_n = n;
    for (int j = 0; j < n; ++j) memcpy(g_last + (size_t)j * n, a + (size_t)j * lda, sizeof(double) * (size_t)n);
    /* full symmetric working copy from the upper triangle (column-major view) */
    double *A = (double *)malloc(sizeof(double) * (size_t)n * (size_t)n + 8);
    double *V = (double *)calloc((size_t)n * (size_t)n + 1, sizeof(double));
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) {
            double v = layout == LAPACK_COL_MAJOR ? a[(size_t)j * lda + i] : a[(size_t)i * lda + j];
            A[(size_t)j * n + i] = v;
            A[(size_t)i * n + j] = v;
        }
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    double fro = 0.0;
    for (size_t k = 0; k < (size_t)n * n; ++k) fro += A[k] * A[k];
    fro = sqrt(fro);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < j; ++i) off += 2.0 * A[(size_t)j * n + i] * A[(size_t)j * n + i];
        if (sqrt(off) <= 1e-17 * fro) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A[(size_t)q * n + p];
                if (apq == 0.0) continue;
                double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                /* symmetric Schur decomposition of the 2x2 block */
                double tau = (aqq - app) / (2.0 * apq);
                double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) { /* A <- A J (columns p, q) */
                    double akp = A[(size_t)p * n + k], akq = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * akp - s * akq;
                    A[(size_t)q * n + k] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) { /* A <- J^T A (rows p, q) */
                    double apk = A[(size_t)k * n + p], aqk = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * apk - s * aqk;
                    A[(size_t)k * n + q] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) { /* V <- V J */
                    double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
                    V[(size_t)p * n + k] = c * vkp - s * vkq;
                    V[(size_t)q * n + k] = s * vkp + c * vkq;
                }
            }
    }
    /* ascending order (selection sort of the diagonal) */
    int *ord = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) ord[i] = i;
    for (int i = 0; i < n; ++i) {
        int b = i;
        for (int k = i + 1; k < n; ++k)
            if (A[(size_t)ord[k] * n + ord[k]] < A[(size_t)ord[b] * n + ord[b]]) b = k;
        int t = ord[i];
        ord[i] = ord[b];
        ord[b] = t;
    }
    for (int i = 0; i < n; ++i) w[i] = A[(size_t)ord[i] * n + ord[i]];
    if (jobz == 'v' || jobz == 'V')
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k) {
                double v = V[(size_t)ord[i] * n + k];
                if (layout == LAPACK_COL_MAJOR) a[(size_t)i * lda + k] = v;
                else a[(size_t)k * lda + i] = v;
            }
    free(ord);
    free(A);
    free(V);
    return 0;
}
