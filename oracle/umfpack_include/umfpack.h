/*
 * Project-written prototype header that stands in for SuiteSparse UMFPACK's
 * <umfpack.h> when the reference hot path is compiled in place for the oracle.
 * It declares only the five double/int entry points the reference calls
 * (src/simulation.cpp:83,388-395 of pgabor/sdddst) and the UMFPACK_A system
 * selector.  The implementation is oracle/umfpack_shim.c (a banded LU with
 * partial pivoting and iterative refinement), not UMFPACK.
 *
 * Test infrastructure only: nothing in the product library includes this.
 */
#ifndef SDDDST_ORACLE_UMFPACK_SHIM_H
#define SDDDST_ORACLE_UMFPACK_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

#define UMFPACK_A 0
#define UMFPACK_OK 0
#define UMFPACK_WARNING_singular_matrix 1
#define UMFPACK_ERROR_out_of_memory (-1)
#define UMFPACK_ERROR_invalid_system (-13)

int umfpack_di_symbolic(int n_row, int n_col, const int Ap[], const int Ai[],
                        const double Ax[], void **Symbolic,
                        const double Control[], double Info[]);
int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[],
                       void *Symbolic, void **Numeric,
                       const double Control[], double Info[]);
int umfpack_di_solve(int sys, const int Ap[], const int Ai[], const double Ax[],
                     double X[], const double B[], void *Numeric,
                     const double Control[], double Info[]);
void umfpack_di_free_symbolic(void **Symbolic);
void umfpack_di_free_numeric(void **Numeric);

#ifdef __cplusplus
}
#endif

#endif
