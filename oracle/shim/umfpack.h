/*
 * Declaration-only stand-in for SuiteSparse UMFPACK's public header, written for
 * this project so that the reference sources compile here without SuiteSparse.
 *
 * Only the names the reference uses are declared (src/la/bcgstab_solver.c:5-7,
 * 371-420).  The constants carry the values of UMFPACK's documented public API
 * (SuiteSparse 7.x user guide): control/info array sizes, the ordering selector
 * slot and its choices, and the "solve with the transposed matrix" system code.
 *
 * The implementation behind these names is oracle/shim/ref_shim.c: an exact
 * banded LU with partial pivoting.  It is NOT UMFPACK; it reproduces what the
 * reference asks of UMFPACK (an exact factor-and-solve of A x = b) so that the
 * reference's BiCGStab converges the same way it does with the real library.
 *
 * Test infrastructure only: nothing in the product links this header.
 */
#ifndef ORACLE_SHIM_UMFPACK_H
#define ORACLE_SHIM_UMFPACK_H

#define UMFPACK_CONTROL 20
#define UMFPACK_INFO 90

#define UMFPACK_ORDERING 10
#define UMFPACK_ORDERING_CHOLMOD 0
#define UMFPACK_ORDERING_AMD 1
#define UMFPACK_ORDERING_GIVEN 2
#define UMFPACK_ORDERING_METIS 3
#define UMFPACK_ORDERING_BEST 4
#define UMFPACK_ORDERING_NONE 5

/* system codes for umfpack_di_solve */
#define UMFPACK_A 0
#define UMFPACK_At 1
#define UMFPACK_Aat 2

#define UMFPACK_OK 0
#define UMFPACK_ERROR_out_of_memory (-1)
#define UMFPACK_ERROR_invalid_matrix (-8)
#define UMFPACK_WARNING_singular_matrix 1

void umfpack_di_defaults(double Control[UMFPACK_CONTROL]);
int umfpack_di_symbolic(int n_row, int n_col, const int Ap[], const int Ai[],
                        const double Ax[], void **Symbolic,
                        const double Control[UMFPACK_CONTROL],
                        double Info[UMFPACK_INFO]);
int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[],
                       void *Symbolic, void **Numeric,
                       const double Control[UMFPACK_CONTROL],
                       double Info[UMFPACK_INFO]);
int umfpack_di_solve(int sys, const int Ap[], const int Ai[], const double Ax[],
                     double X[], const double B[], void *Numeric,
                     const double Control[UMFPACK_CONTROL],
                     double Info[UMFPACK_INFO]);
void umfpack_di_free_symbolic(void **Symbolic);
void umfpack_di_free_numeric(void **Numeric);

#endif
