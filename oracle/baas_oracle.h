/*
 * baas_oracle.h -- TEST INFRASTRUCTURE ONLY: plain-C restatement of the reference's serial
 * numeric routines on the hot path, used to check the CUDA library (never linked into it).
 * CSR arrays are 0-based with strictly ascending columns in each row.
 */
#ifndef BAAS_ORACLE_H
#define BAAS_ORACLE_H

/* x = L^-1 b, L lower with the diagonal last in each row (merge/SpTRSV.cpp:24-39). */
void orc_lower_solve(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x);

/* x = U^-1 b, U upper with the diagonal first; off-diagonal sum taken from the last entry
 * down (the p2p backward sweep's order, merge/SpTRSV.cpp:642-652). */
void orc_upper_solve_desc(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x);

/* Same, off-diagonal sum ascending (upper_csr_trsv_serial, merge/SpTRSV.cpp:580-599). */
void orc_upper_solve_asc(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x);

/* Up-looking IC0 in place on lu (pre-filled with A's values), merge/IC.cpp:32-89.
 * Returns the number of pivots left unchanged because A_ii - dv <= 0. */
int orc_ic0(int n, const int *rowptr, const int *colidx, const int *diagptr, double *lu);

/* Up-looking ILU0 in place on lu, merge/ILU.cpp:350-386. Returns the number of zero pivots. */
int orc_ilu0(int n, const int *rowptr, const int *colidx, const int *diagptr, double *lu);

/* y = alpha * A x + beta * y, blas/spmv.cpp:29-45. */
void orc_spmv(int n, const int *rowptr, const int *colidx, const double *val, const double *x, double *y, double alpha,
              double beta);

/* Sequential dot product (blas/blasone.cpp:7-16 with one thread). */
double orc_dot(const double *x, const double *y, int n);

/* IC0-preconditioned CG (the pcg_opt loop, test/iccg_level_merge.cpp:458-503, with its
 * IC0_preconditioner split :809-906), serial routines, stopping once ||r||/||r0|| < tol.
 * x holds the initial guess. Returns the iteration count; *relres gets the final ratio. */
int orc_pcg(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x, int maxiter,
            double tol, double *relres, double *unused);

#endif
