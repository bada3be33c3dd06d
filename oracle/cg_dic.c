/* CPU oracle: restatement of the reference's Fortran MEX PCG solver.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU stand-in); the
 * product never links or calls this file.
 *
 * Follows solvers/pressure/cg.F of bsanderse/INS2D:
 *   cg           cg.F:158-280  (x0 = x_in, relative test ||r||^2/||y||^2 <= tol^2
 *                               after the x,r update; iter = the iteration
 *                               that met it; error after maxit iterations)
 *   matvec_prod  cg.F:285-312  (symmetric product from the main + lower
 *                               diagonals in spdiags storage)
 *   precond      cg.F:317-390  (forward/backward DIC sweeps)
 *   make_cholinc cg.F:394-429  (diagonal incomplete Cholesky pivots)
 * Storage: A is N x nd, column-major (Fortran), column 0 the main diagonal
 * and column k the lower diagonal at distance dia[k] (so A(i,k) multiplies
 * x(i+dia[k]) in row i and x(i) in row i+dia[k]).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define AIK(A, N, i, k) ((A)[(size_t)(k) * (size_t)(N) + (size_t)(i)])

static void matvec_prod(long N, const double *A, const long *dia, long nd,
                        const double *x, double *y) {
  for (long i = 0; i < N; ++i) y[i] = AIK(A, N, i, 0) * x[i];
  for (long j = 1; j < nd; ++j) {
    long dj = dia[j];
    for (long i = 0; i < N - dj; ++i) {
      y[i] += AIK(A, N, i, j) * x[i + dj];
      y[i + dj] += AIK(A, N, i, j) * x[i];
    }
  }
}

/* dia2 has nd+1 entries, dia2[nd] = N (1-based ranges of cg.F:350,371). */
static void precond(long N, const double *A, const long *dia2, long nd,
                    const double *D, const double *y, double *x, double *q) {
  q[0] = y[0] / D[0];
  for (long j = 1; j < nd; ++j) {
    for (long i1 = dia2[j] + 1; i1 <= dia2[j + 1]; ++i1) {
      long i = i1 - 1;
      double s = 0.0;
      for (long k = 1; k <= j; ++k) s -= AIK(A, N, i - dia2[k], k) * q[i - dia2[k]];
      q[i] = (y[i] + s) / D[i];
    }
  }
  x[N - 1] = q[N - 1];
  for (long j = 1; j < nd; ++j) {
    for (long i1 = N - dia2[j]; i1 >= N - dia2[j + 1] + 1; --i1) {
      long i = i1 - 1;
      double s = 0.0;
      for (long k = 1; k <= j; ++k) s -= AIK(A, N, i, k) * x[i + dia2[k]];
      x[i] = q[i] + s / D[i];
    }
  }
}

static void make_cholinc(long N, const double *A, const long *dia2, long nd, double *D) {
  D[0] = AIK(A, N, 0, 0);
  for (long j = 1; j < nd; ++j) {
    for (long i1 = dia2[j] + 1; i1 <= dia2[j + 1]; ++i1) {
      long i = i1 - 1;
      double s = 0.0;
      for (long k = 1; k <= j; ++k) {
        double a = AIK(A, N, i - dia2[k], k);
        s -= (a * a) / D[i - dia2[k]];
      }
      D[i] = AIK(A, N, i, 0) + s;
    }
  }
}

/* Returns 0 on convergence, 1 when maxit iterations did not converge
 * (cg.F:262 mexErrMsgTxt), 2 on allocation failure. */
int oracle_cg_dic(long N, const double *A, const long *dia, long nd, const double *y,
                  double tol, const double *x_in, long maxit, double *x, long *iter,
                  double *norm1, double *norm2) {
  double tol2 = tol * tol;
  if (nd == 1 && dia[0] == 0) {
    for (long i = 0; i < N; ++i) x[i] = y[i] / AIK(A, N, i, 0);
    *iter = 1;
    *norm1 = 0.0;
    *norm2 = 0.0;
    return 0;
  }
  long *dia2 = (long *)malloc(sizeof(long) * (size_t)(nd + 1));
  double *D = (double *)malloc(sizeof(double) * (size_t)N);
  double *r = (double *)malloc(sizeof(double) * (size_t)N);
  double *p = (double *)malloc(sizeof(double) * (size_t)N);
  double *z = (double *)malloc(sizeof(double) * (size_t)N);
  double *q = (double *)malloc(sizeof(double) * (size_t)N);
  double *tv = (double *)malloc(sizeof(double) * (size_t)N);
  int status = 0;
  if (!dia2 || !D || !r || !p || !z || !q || !tv) {
    status = 2;
    goto done;
  }
  memcpy(dia2, dia, sizeof(long) * (size_t)nd);
  dia2[nd] = N;
  memcpy(x, x_in, sizeof(double) * (size_t)N);
  make_cholinc(N, A, dia2, nd, D);
  matvec_prod(N, A, dia, nd, x, tv);
  for (long i = 0; i < N; ++i) r[i] = y[i] - tv[i];
  precond(N, A, dia2, nd, D, r, z, q);
  memcpy(p, z, sizeof(double) * (size_t)N);
  double nr0 = 0.0;
  for (long i = 0; i < N; ++i) nr0 += y[i] * y[i];
  double nr = nr0;
  if (nr0 <= tol2) {
    *iter = 0;
    *norm1 = 0.0;
    *norm2 = 0.0;
    goto done;
  }
  double rz = 0.0;
  for (long i = 0; i < N; ++i) rz += r[i] * z[i];
  double maxx = 0, minx = 0, maxres = 0;
  long it;
  for (it = 1; it <= maxit; ++it) {
    matvec_prod(N, A, dia, nd, p, tv);
    double temp = 0.0;
    for (long i = 0; i < N; ++i) temp += p[i] * tv[i];
    double alpha = rz / temp;
    for (long i = 0; i < N; ++i) x[i] += alpha * p[i];
    for (long i = 0; i < N; ++i) r[i] -= alpha * tv[i];
    nr = 0.0;
    for (long i = 0; i < N; ++i) nr += r[i] * r[i];
    nr = nr / nr0;
    maxx = x[0];
    minx = x[0];
    maxres = fabs(r[0]);
    for (long i = 1; i < N; ++i) {
      if (x[i] > maxx) maxx = x[i];
      if (x[i] < minx) minx = x[i];
      if (fabs(r[i]) > maxres) maxres = fabs(r[i]);
    }
    if (nr <= tol2) break;
    precond(N, A, dia2, nd, D, r, z, q);
    double rz_old = rz;
    rz = 0.0;
    for (long i = 0; i < N; ++i) rz += r[i] * z[i];
    for (long i = 0; i < N; ++i) p[i] = z[i] + p[i] * (rz / rz_old);
  }
  if (it > maxit) {
    status = 1;
    *iter = maxit;
    *norm1 = sqrt(nr);
    goto done;
  }
  *iter = it;
  *norm1 = sqrt(nr);
  *norm2 = maxres / (maxx - minx);
done:
  free(dia2);
  free(D);
  free(r);
  free(p);
  free(z);
  free(q);
  free(tv);
  return status;
}
