/*
 * Link shim that lets the reference's own C sources (compiled unmodified from the
 * reference tree) link and run here, where SuiteSparse, SCOTCH and HDF5 are not
 * installed.  Test infrastructure only: it is linked into oracle/_ref/ and never
 * into the product library.
 *
 *  - umfpack_di_*: the reference factors its whole scaled matrix every Newton
 *    iteration and uses the factors as the BiCGStab preconditioner
 *    (src/la/bcgstab_solver.c:371-420, called at src/newton/fe_newton.c:513).
 *    UMFPACK receives the CSR arrays as if they were CSC and solves with
 *    UMFPACK_Aat, i.e. it solves A x = b for the CSR matrix A.  This shim does
 *    the same solve with a banded LU with partial pivoting (the classic
 *    band-storage Gaussian elimination: row interchanges inside the band, fill
 *    confined to kl extra super-diagonals).  It is exact up to rounding, like
 *    UMFPACK, but its rounding differs, so BiCGStab iterates agree with a real
 *    UMFPACK build only to the solver tolerance.
 *  - sflags.c does not compile without _HDF5 (a field declared under that
 *    macro is assigned unconditionally); oracle/ref_harness.c supplies the
 *    zeroed flag block its only caller needs (smodel_super_alloc_init.c:31).
 *  - hdf5_init / hdf5_write_grid / xmf_init are not referenced once
 *    smodel_design_xmf.c is left out of the build.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "umfpack.h"

typedef struct {
    int n, kl, ku, ldab;   /* band storage: ldab = 2*kl + ku + 1 rows */
    double *ab;            /* column-major band: A(i,j) at ab[(kl+ku+i-j) + j*ldab] */
    int *ipiv;
} shim_lu;

typedef struct { int n, kl, ku; } shim_sym;

void umfpack_di_defaults(double Control[UMFPACK_CONTROL]) {
    for (int i = 0; i < UMFPACK_CONTROL; i++) Control[i] = 0.0;
}

/* The matrix UMFPACK would see is C (CSC from Ap/Ai); we factor A = C^T, whose
 * row j holds the entries Ai[Ap[j]..Ap[j+1]) with values Ax. */
int umfpack_di_symbolic(int n_row, int n_col, const int Ap[], const int Ai[],
                        const double Ax[], void **Symbolic,
                        const double Control[UMFPACK_CONTROL],
                        double Info[UMFPACK_INFO]) {
    (void)Ax; (void)Control; (void)Info;
    if (n_row != n_col) return UMFPACK_ERROR_invalid_matrix;
    shim_sym *s = (shim_sym *)calloc(1, sizeof(shim_sym));
    s->n = n_row;
    for (int j = 0; j < n_row; j++) {
        for (int k = Ap[j]; k < Ap[j + 1]; k++) {
            int c = Ai[k];
            if (c - j > s->ku) s->ku = c - j;   /* row j, column c of A */
            if (j - c > s->kl) s->kl = j - c;
        }
    }
    *Symbolic = s;
    return UMFPACK_OK;
}

int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[],
                       void *Symbolic, void **Numeric,
                       const double Control[UMFPACK_CONTROL],
                       double Info[UMFPACK_INFO]) {
    (void)Control; (void)Info;
    shim_sym *s = (shim_sym *)Symbolic;
    int n = s->n, kl = s->kl, ku = s->ku;
    shim_lu *f = (shim_lu *)calloc(1, sizeof(shim_lu));
    f->n = n; f->kl = kl; f->ku = ku; f->ldab = 2 * kl + ku + 1;
    f->ab = (double *)calloc((size_t)f->ldab * (size_t)n, sizeof(double));
    f->ipiv = (int *)malloc(sizeof(int) * (size_t)n);
    if (!f->ab || !f->ipiv) return UMFPACK_ERROR_out_of_memory;
#define AB(i, j) f->ab[(size_t)(kl + ku + (i) - (j)) + (size_t)(j) * (size_t)f->ldab]
    for (int i = 0; i < n; i++)
        for (int k = Ap[i]; k < Ap[i + 1]; k++) AB(i, Ai[k]) += Ax[k];
    int status = UMFPACK_OK;
    int kuf = kl + ku; /* upper bandwidth of U after row interchanges */
    for (int j = 0; j < n; j++) {
        int imax = j, iend = (j + kl < n - 1) ? j + kl : n - 1;
        double amax = fabs(AB(j, j));
        for (int i = j + 1; i <= iend; i++)
            if (fabs(AB(i, j)) > amax) { amax = fabs(AB(i, j)); imax = i; }
        f->ipiv[j] = imax;
        int cend = (j + kuf < n - 1) ? j + kuf : n - 1;
        if (amax == 0.0) { status = UMFPACK_WARNING_singular_matrix; continue; }
        if (imax != j)
            for (int c = j; c <= cend; c++) { double t = AB(j, c); AB(j, c) = AB(imax, c); AB(imax, c) = t; }
        double piv = AB(j, j);
        for (int i = j + 1; i <= iend; i++) {
            double l = AB(i, j) / piv;
            AB(i, j) = l;
            if (l != 0.0)
                for (int c = j + 1; c <= cend; c++) AB(i, c) -= l * AB(j, c);
        }
    }
#undef AB
    *Numeric = f;
    return status;
}

int umfpack_di_solve(int sys, const int Ap[], const int Ai[], const double Ax[],
                     double X[], const double B[], void *Numeric,
                     const double Control[UMFPACK_CONTROL],
                     double Info[UMFPACK_INFO]) {
    (void)Ap; (void)Ai; (void)Ax; (void)Control; (void)Info;
    if (sys != UMFPACK_Aat) {
        fprintf(stderr, "umfpack shim: only UMFPACK_Aat is provided\n");
        return UMFPACK_ERROR_invalid_matrix;
    }
    shim_lu *f = (shim_lu *)Numeric;
    int n = f->n, kl = f->kl, ku = f->ku, kuf = kl + ku;
#define AB(i, j) f->ab[(size_t)(kl + ku + (i) - (j)) + (size_t)(j) * (size_t)f->ldab]
    double *y = (double *)malloc(sizeof(double) * (size_t)n);
    memcpy(y, B, sizeof(double) * (size_t)n);
    for (int j = 0; j < n; j++) {            /* L y = P b */
        int p = f->ipiv[j];
        if (p != j) { double t = y[j]; y[j] = y[p]; y[p] = t; }
        int iend = (j + kl < n - 1) ? j + kl : n - 1;
        for (int i = j + 1; i <= iend; i++) y[i] -= AB(i, j) * y[j];
    }
    for (int j = n - 1; j >= 0; j--) {       /* U x = y */
        int cend = (j + kuf < n - 1) ? j + kuf : n - 1;
        double s = y[j];
        for (int c = j + 1; c <= cend; c++) s -= AB(j, c) * X[c];
        X[j] = s / AB(j, j);
    }
#undef AB
    free(y);
    return UMFPACK_OK;
}

void umfpack_di_free_symbolic(void **Symbolic) {
    if (Symbolic && *Symbolic) { free(*Symbolic); *Symbolic = NULL; }
}

void umfpack_di_free_numeric(void **Numeric) {
    if (Numeric && *Numeric) {
        shim_lu *f = (shim_lu *)*Numeric;
        free(f->ab); free(f->ipiv); free(f);
        *Numeric = NULL;
    }
}
