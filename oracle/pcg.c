/* Jacobi-preconditioned conjugate gradient on a CSR matrix, FP64 -- TEST
 * INFRASTRUCTURE (oracle).  Restates cpu_conjugate_gradient
 * (src/linear_system_solver_library/linear_system_solver.c:47-183): the same
 * recurrences, the same iteration count convention (its starts at 1 and the
 * loop runs while its < max_its) and the same stopping test on the absolute
 * r.r <= tol.  The diagonal is the first entry of every row, as elements[0]
 * is in the reference.
 */
#include <stdlib.h>

#include "oracle.h"

static double row_dot(const orc_csr *A, int32_t i, const double *v) {
    double s = 0.0;
    for (int32_t e = A->row_ptr[i]; e < A->row_ptr[i + 1]; ++e) s += A->val[e] * v[A->col[e]];
    return s;
}

static double inv_diag(const orc_csr *A, int32_t i) {
    double d = A->val[A->row_ptr[i]];
    if (d == 0.0) d = 1.0;
    return 1.0 / d;
}

void orc_pcg(const orc_csr *A, const double *b, double *x, double tol, int max_its, int use_preconditioner,
             uint32_t *its_out, double *error_out) {
    const int32_t n = A->n;
    double *r = malloc(sizeof(double) * (size_t)n), *z = malloc(sizeof(double) * (size_t)n);
    double *p = malloc(sizeof(double) * (size_t)n), *ap = malloc(sizeof(double) * (size_t)n);
    uint32_t its = 1;
    double rTr = 0.0, rTz = 0.0, error;

#pragma omp parallel for reduction(+ : rTr, rTz)
    for (int32_t i = 0; i < n; ++i) {
        r[i] = b[i] - row_dot(A, i, x);
        if (use_preconditioner) {
            z[i] = inv_diag(A, i) * r[i];
            rTz += r[i] * z[i];
            p[i] = z[i];
        } else {
            p[i] = r[i];
        }
        rTr += r[i] * r[i];
    }
    error = rTr;

    if (error >= tol) {
        while (its < (uint32_t)max_its) {
            double pTAp = 0.0;
#pragma omp parallel for reduction(+ : pTAp)
            for (int32_t i = 0; i < n; ++i) {
                ap[i] = row_dot(A, i, p);
                pTAp += p[i] * ap[i];
            }
            const double alpha = (use_preconditioner ? rTz : rTr) / pTAp;
            double r1Tr1 = 0.0, r1Tz1 = 0.0;
#pragma omp parallel for reduction(+ : r1Tr1, r1Tz1)
            for (int32_t i = 0; i < n; ++i) {
                x[i] += alpha * p[i];
                r[i] -= alpha * ap[i];
                if (use_preconditioner) {
                    z[i] = inv_diag(A, i) * r[i];
                    r1Tz1 += z[i] * r[i];
                }
                r1Tr1 += r[i] * r[i];
            }
            const double beta = use_preconditioner ? r1Tz1 / rTz : r1Tr1 / rTr;
            error = r1Tr1;
            its++;
            if (error <= tol) break;
#pragma omp parallel for
            for (int32_t i = 0; i < n; ++i) p[i] = (use_preconditioner ? z[i] : r[i]) + beta * p[i];
            rTz = r1Tz1;
            rTr = r1Tr1;
        }
    }
    free(r); free(z); free(p); free(ap);
    *its_out = its;
    *error_out = error;
}
