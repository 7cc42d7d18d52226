/*
 * baas_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle). A plain-C restatement of the
 * reference's serial numeric routines for the sparse hot path; the CUDA library is checked
 * against it and against the reference compiled from its sources (oracle/_ref). Built with
 * -ffp-contract=off so every a*b+c is a rounded multiply then a rounded add, as in the
 * reference's ISO C++ build.
 *
 * Parity pin: tests/test_oracle.py compares every function here with the reference's own
 * routine (oracle/_ref/libbaas_ref.so) bit for bit, and with the committed golden vectors in
 * tests/golden/ that the reference produced (tests/golden/make_golden.py).
 */
#include "baas_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* merge/SpTRSV.cpp:24-39 */
void orc_lower_solve(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x) {
    for (int i = 0; i < n; i++) {
        double sum = 0.0;
        for (int j = rowptr[i]; j < rowptr[i + 1] - 1; j++) sum += val[j] * x[colidx[j]];
        x[i] = (b[i] - sum) / val[rowptr[i + 1] - 1];
    }
}

/* merge/SpTRSV.cpp:642-652 (rows in any topological order give the same values; serial) */
void orc_upper_solve_desc(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x) {
    for (int i = n - 1; i >= 0; i--) {
        double sum = 0.0;
        for (int j = rowptr[i + 1] - 1; j > rowptr[i]; j--) sum += x[colidx[j]] * val[j];
        x[i] = (b[i] - sum) / val[rowptr[i]];
    }
}

/* merge/SpTRSV.cpp:580-599 */
void orc_upper_solve_asc(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x) {
    for (int i = n - 1; i >= 0; i--) {
        double sum = 0.0;
        for (int j = rowptr[i] + 1; j < rowptr[i + 1]; j++) sum += val[j] * x[colidx[j]];
        x[i] = (b[i] - sum) / val[rowptr[i]];
    }
}

/* merge/IC.cpp:6-29 */
static double sparse_dot(int l1, int u1, int l2, int u2, const int *idx, const double *data) {
    double r = 0.0;
    while (l1 < u1 && l2 < u2) {
        if (idx[l1] == idx[l2])
            r += data[l1++] * data[l2++];
        else if (idx[l1] < idx[l2])
            l1++;
        else
            l2++;
    }
    return r;
}

/* merge/IC.cpp:32-89 (the p2p routine :296-393 computes the same row updates; its A_ij is
 * lu[k], identical because lu starts as A's values) */
int orc_ic0(int n, const int *rowptr, const int *colidx, const int *diagptr, double *lu) {
    int bad = 0;
    for (int i = 0; i < n; i++) {
        for (int k = rowptr[i]; k < diagptr[i]; k++) {
            const int j = colidx[k];
            const double dp = sparse_dot(rowptr[i], diagptr[i], rowptr[j], diagptr[j], colidx, lu);
            lu[k] = (lu[k] - dp) / lu[diagptr[j]];
        }
        const double dv = sparse_dot(rowptr[i], diagptr[i], rowptr[i], diagptr[i], colidx, lu);
        const double aii = lu[diagptr[i]];
        if (aii - dv > 0)
            lu[diagptr[i]] = sqrt(aii - dv);
        else
            bad++;
    }
    return bad;
}

/* merge/ILU.cpp:350-386 */
int orc_ilu0(int n, const int *rowptr, const int *colidx, const int *diagptr, double *lu) {
    int bad = 0;
    for (int i = 0; i < n; i++) {
        for (int j = rowptr[i]; j < diagptr[i]; j++) {
            const int c = colidx[j];
            const double pivot = lu[diagptr[c]];
            if (pivot == 0.0) bad++;
            const double tmp = lu[j] /= pivot;
            int k1 = j + 1, k2 = diagptr[c] + 1;
            while (k1 < rowptr[i + 1] && k2 < rowptr[c + 1]) {
                if (colidx[k1] < colidx[k2])
                    k1++;
                else if (colidx[k1] > colidx[k2])
                    k2++;
                else {
                    lu[k1] -= tmp * lu[k2];
                    k1++;
                    k2++;
                }
            }
        }
    }
    return bad;
}

/* blas/spmv.cpp:29-45 */
void orc_spmv(int n, const int *rowptr, const int *colidx, const double *val, const double *x, double *y, double alpha,
              double beta) {
    for (int i = 0; i < n; i++) {
        double sum = 0.0;
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) sum += val[j] * x[colidx[j]];
        y[i] = alpha * sum + beta * y[i];
    }
}

double orc_dot(const double *x, const double *y, int n) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}

int orc_pcg(int n, const int *rowptr, const int *colidx, const double *val, const double *b, double *x, int maxiter,
            double tol, double *relres, double *unused) {
    (void)unused;
    const int nnz = rowptr[n];
    int *diag = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) {
        int e = rowptr[i];
        while (e < rowptr[i + 1] && colidx[e] < i) e++;
        diag[i] = e;
    }
    /* IC0_preconditioner: L = lower part (diagonal last), U = L^T (diagonal first) */
    const int nnzL = (nnz + n) / 2;
    int *Lrp = (int *)calloc((size_t)n + 1, sizeof(int)), *Urp = (int *)calloc((size_t)n + 1, sizeof(int));
    int *Lci = (int *)malloc(sizeof(int) * (size_t)nnzL), *Uci = (int *)malloc(sizeof(int) * (size_t)nnzL);
    double *Lv = (double *)malloc(sizeof(double) * (size_t)nnzL), *Uv = (double *)malloc(sizeof(double) * (size_t)nnzL);
    double *lu = (double *)malloc(sizeof(double) * (size_t)nnz);
    memcpy(lu, val, sizeof(double) * (size_t)nnz);
    for (int i = 0; i < n; i++) {
        Lrp[i + 1] = Lrp[i] + diag[i] - rowptr[i] + 1;
        Urp[i + 1] = Urp[i] + rowptr[i + 1] - diag[i];
    }
    for (int i = 0; i < n; i++) {
        memcpy(Lci + Lrp[i], colidx + rowptr[i], sizeof(int) * (size_t)(diag[i] - rowptr[i] + 1));
        memcpy(Uci + Urp[i], colidx + diag[i], sizeof(int) * (size_t)(rowptr[i + 1] - diag[i]));
    }
    orc_ic0(n, rowptr, colidx, diag, lu);
    int *ucur = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    memcpy(ucur, Urp, sizeof(int) * (size_t)(n + 1));
    for (int i = 0; i < n; i++)
        for (int j = rowptr[i]; j <= diag[i]; j++) {
            Lv[Lrp[i] + j - rowptr[i]] = lu[j];
            Uv[ucur[colidx[j]]++] = lu[j];
        }

    double *r = (double *)malloc(sizeof(double) * (size_t)n), *z = (double *)malloc(sizeof(double) * (size_t)n);
    double *y = (double *)malloc(sizeof(double) * (size_t)n), *p = (double *)malloc(sizeof(double) * (size_t)n);
    double *Ap = (double *)calloc((size_t)n, sizeof(double));
    memcpy(r, b, sizeof(double) * (size_t)n);
    orc_spmv(n, rowptr, colidx, val, x, r, -1.0, 1.0);
    const double norm0 = sqrt(orc_dot(r, r, n));
    double rel = 1.0;
    orc_lower_solve(n, Lrp, Lci, Lv, r, y);
    orc_upper_solve_desc(n, Urp, Uci, Uv, y, z);
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = orc_dot(r, z, n);
    int k = 1, iters = 0;
    while (k <= maxiter) {
        const double old_rz = rz;
        orc_spmv(n, rowptr, colidx, val, p, Ap, 1.0, 0.0);
        const double alpha = old_rz / orc_dot(p, Ap, n);
        for (int i = 0; i < n; i++) x[i] = x[i] + alpha * p[i];
        for (int i = 0; i < n; i++) r[i] = r[i] + (-alpha) * Ap[i];
        rel = sqrt(orc_dot(r, r, n)) / norm0;
        iters = k;
        if (rel < tol) break;
        orc_lower_solve(n, Lrp, Lci, Lv, r, y);
        orc_upper_solve_desc(n, Urp, Uci, Uv, y, z);
        rz = orc_dot(r, z, n);
        const double beta = rz / old_rz;
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        ++k;
    }
    if (relres) *relres = rel;
    free(diag);
    free(Lrp);
    free(Urp);
    free(Lci);
    free(Uci);
    free(Lv);
    free(Uv);
    free(lu);
    free(ucur);
    free(r);
    free(z);
    free(y);
    free(p);
    free(Ap);
    return iters;
}
