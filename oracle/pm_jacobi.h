/*
 * pm_jacobi.h -- cyclic Jacobi eigen-decomposition of a small real symmetric
 * matrix (TEST INFRASTRUCTURE for the oracle; the GPU path has its own).
 *
 * Written from the textbook method (cyclic-by-row sweeps, Rutishauser's stable
 * rotation update).  Input: a[n*n] full symmetric (overwritten); output: w[n]
 * unordered eigenvalues, v[n*n] row-major with eigenvector j in column j.  It
 * stands in for GSL's gsl_eigen_symmv, which the reference's mil_svd
 * (milosUtils.c:237-271) calls; the pseudo-inverse that mil_svd forms from it
 * does not depend on eigenvalue order or eigenvector signs.
 */
#ifndef PM_JACOBI_H
#define PM_JACOBI_H
#include <math.h>
#include <stddef.h>

static void pm_jacobi_eigen(double *a, size_t n, double *w, double *v) {
  size_t i, j, p, q, k;
  int sweep;
  for (i = 0; i < n; i++)
    for (j = 0; j < n; j++) v[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, diag = 0.0;
    for (p = 0; p < n; p++) {
      diag += a[p * n + p] * a[p * n + p];
      for (q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
    }
    if (off == 0.0 || off <= 1e-36 * diag) break;
    for (p = 0; p + 1 < n; p++) {
      for (q = p + 1; q < n; q++) {
        double apq = a[p * n + q], app, aqq, theta, t, c, s, tau;
        if (apq == 0.0) continue;
        app = a[p * n + p];
        aqq = a[q * n + q];
        theta = (aqq - app) / (2.0 * apq);
        t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        if (!isfinite(t)) t = 0.0; /* theta overflowed: apq is negligible */
        c = 1.0 / sqrt(t * t + 1.0);
        s = t * c;
        tau = s / (1.0 + c);
        a[p * n + p] = app - t * apq;
        a[q * n + q] = aqq + t * apq;
        a[p * n + q] = 0.0;
        a[q * n + p] = 0.0;
        for (k = 0; k < n; k++) {
          double vkp, vkq;
          if (k != p && k != q) {
            double akp = a[k * n + p], akq = a[k * n + q];
            a[k * n + p] = akp - s * (akq + tau * akp);
            a[k * n + q] = akq + s * (akp - tau * akq);
            a[p * n + k] = a[k * n + p];
            a[q * n + k] = a[k * n + q];
          }
          vkp = v[k * n + p];
          vkq = v[k * n + q];
          v[k * n + p] = vkp - s * (vkq + tau * vkp);
          v[k * n + q] = vkq + s * (vkp - tau * vkq);
        }
      }
    }
  }
  for (i = 0; i < n; i++) w[i] = a[i * n + i];
}
#endif
