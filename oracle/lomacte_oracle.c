/*
 * lomacte_oracle.c -- CPU FP64 oracle for the lomacte RK3 substep.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  The
 * product library never links or calls this file.  See lomacte_oracle.h for
 * the list of reference files restated here.  Every routine cites the
 * reference routine (file:line, paths inside Beovulfo/LoMa_phD) it follows.
 *
 * Parity pinning: the FFT conventions are pinned by the reference's own
 * golden vectors (branches/reactml/benchmark_fft/ cfttest_double.txt, rffttest_double.txt); the compact
 * derivatives by the analytic-derivative harness pattern of
 * trunk/mixing/test/test.f:182-200 and benchmark_fft/main.f:46-74; the full
 * substep is pinned by restatement only (the Fortran cannot be built here).
 */
#include "lomacte_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------ */
/* RK3 coefficients: modulos.f:193-209 (module rkcoef).                */
/* ------------------------------------------------------------------ */
static void rk_coefs(double gama[3], double xi[3], double alpha[3],
                     double beta[3]) {
  const double p0 = 5.0 / 66.0, p1 = -1.0;
  xi[0] = 0.0;
  xi[1] = -17.0 / 60.0;
  xi[2] = -5.0 / 12.0;
  gama[0] = 8.0 / 15.0;
  gama[1] = 5.0 / 12.0;
  gama[2] = 3.0 / 4.0;
  double b3 = (p1 * (gama[0] * gama[2] + gama[1] * gama[2] + xi[1] * gama[2] +
                     gama[0] * xi[2]) -
               gama[0] * gama[1] * gama[2] - gama[0] * gama[1] * xi[2]) /
              (p1 - gama[0] * gama[1]);
  beta[0] = gama[0] - p0;
  beta[1] = p1;
  beta[2] = b3;
  alpha[0] = p0;
  alpha[1] = gama[1] + xi[1] - p1;
  alpha[2] = gama[2] + xi[2] - beta[2];
}

/* ------------------------------------------------------------------ */
/* FFT written from the DFT definition (mixed-radix, recursive DIT).   */
/* Conventions follow cftsingle.f:2-68 and rftsingle.f:25-95: the      */
/* direct transform (iopt<0) is exp(-i..) scaled by 1/n, the inverse   */
/* is exp(+i..) unscaled.                                              */
/* ------------------------------------------------------------------ */
typedef struct {
  int n, nf, fac[40];
  cplx *w; /* w[t] = exp(-2 pi i t / n) */
} fftplan;

static void plan_init(fftplan *p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
  for (int f = 3; m > 1;) {
    if (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
    else f += 2;
  }
  p->w = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  for (int t = 0; t < n; t++) {
    double a = 2.0 * M_PI * (double)t / (double)n;
    p->w[t] = cos(a) - I * sin(a);
  }
}
static void plan_free(fftplan *p) { free(p->w); }

/* out[k] = sum_j in[j*is] W^{jk}, W = exp(sign*2 pi i/n); n divides P->n */
static void dft_rec(const fftplan *P, int n, int fi, const cplx *in, int is,
                    cplx *out, int sign) {
  if (n == 1) { out[0] = in[0]; return; }
  int p = P->fac[fi], m = n / p, N = P->n, step = N / n;
  for (int r = 0; r < p; r++) dft_rec(P, m, fi + 1, in + (size_t)r * is, is * p, out + (size_t)r * m, sign);
  cplx t[64];
  for (int k = 0; k < m; k++) {
    for (int r = 0; r < p; r++) {
      cplx w = P->w[((size_t)r * k * step) % N];
      if (sign > 0) w = conj(w);
      t[r] = out[(size_t)r * m + k] * w;
    }
    for (int q = 0; q < p; q++) {
      cplx s = 0;
      for (int r = 0; r < p; r++) {
        cplx w = P->w[((size_t)((r * q) % p) * (N / p)) % N];
        if (sign > 0) w = conj(w);
        s += t[r] * w;
      }
      out[(size_t)q * m + k] = s;
    }
  }
}

/* unnormalised c2c of length P->n: out = sum in exp(sign 2 pi i jk/n) */
static void cfft(const fftplan *P, const cplx *in, cplx *out, int sign) {
  dft_rec(P, P->n, 0, in, 1, out, sign);
}

/* ------------------------------------------------------------------ */
/* Band storage helpers.  A(i,j) of the reference (band i, row j,      */
/* 1-based) is a[(j-1)*nb + (i-1)] here.                               */
/* ------------------------------------------------------------------ */
#define B7(a, i, j) a[((j)-1) * 7 + ((i)-1)]
#define B5(a, i, j) a[((j)-1) * 5 + ((i)-1)]

/* gaussj: Gauss-Jordan elimination with full pivoting, the published
 * algorithm used at cfdiff.f:1144-1223.  a is column-major a(np,np). */
static void gaussj(double *a, int n, int np, double *b, int m, int mp) {
  int indxc[64], indxr[64], ipiv[64];
  int irow = 0, icol = 0;
#define A(i, j) a[((j)-1) * np + ((i)-1)]
#define BB(i, j) b[((j)-1) * np + ((i)-1)]
  (void)mp;
  for (int j = 1; j <= n; j++) ipiv[j] = 0;
  for (int i = 1; i <= n; i++) {
    double big = 0.0;
    for (int j = 1; j <= n; j++)
      if (ipiv[j] != 1)
        for (int k = 1; k <= n; k++)
          if (ipiv[k] == 0 && fabs(A(j, k)) >= big) {
            big = fabs(A(j, k));
            irow = j;
            icol = k;
          }
    ipiv[icol] += 1;
    if (irow != icol) {
      for (int l = 1; l <= n; l++) { double d = A(irow, l); A(irow, l) = A(icol, l); A(icol, l) = d; }
      for (int l = 1; l <= m; l++) { double d = BB(irow, l); BB(irow, l) = BB(icol, l); BB(icol, l) = d; }
    }
    indxr[i] = irow;
    indxc[i] = icol;
    double pivinv = 1.0 / A(icol, icol);
    A(icol, icol) = 1.0;
    for (int l = 1; l <= n; l++) A(icol, l) *= pivinv;
    for (int l = 1; l <= m; l++) BB(icol, l) *= pivinv;
    for (int ll = 1; ll <= n; ll++)
      if (ll != icol) {
        double dum = A(ll, icol);
        A(ll, icol) = 0.0;
        for (int l = 1; l <= n; l++) A(ll, l) -= A(icol, l) * dum;
        for (int l = 1; l <= m; l++) BB(ll, l) -= BB(icol, l) * dum;
      }
  }
  for (int l = n; l >= 1; l--)
    if (indxr[l] != indxc[l])
      for (int k = 1; k <= n; k++) {
        double d = A(k, indxr[l]);
        A(k, indxr[l]) = A(k, indxc[l]);
        A(k, indxc[l]) = d;
      }
#undef A
#undef BB
}

/* pred1m6o: cfdiff.f:24-182.  Columns of d(ny,7) for the LHS
 * (den,ben,aln,one,alp,bep,dep) and RHS (a3n..a3p) of the first
 * derivative on uniform eta in [-1,1]. */
static void pred1m6o(int ny, double *l /*ny x 7*/, double *r /*ny x 7*/) {
#define L(j, c) l[((c)-1) * ny + ((j)-1)]
#define R(j, c) r[((c)-1) * ny + ((j)-1)]
  double h = 2.0 / (double)(ny - 1);
  double aaa = 0.56926818603810, bbb = 0.31997939759919, ccc = 0.03751544855390;
  double alpha = -3.0 / 4.0 + (33.0 / 20.0) * ccc + (239.0 / 180.0) * aaa + (82.0 / 45.0) * bbb;
  double beta = 3.0 / 10.0 + (24.0 / 25.0) * ccc - (88.0 / 225.0) * aaa + (34.0 / 225.0) * bbb;
  double delta = -1.0 / 20.0 + (39.0 / 100.0) * ccc + (19.0 / 300.0) * aaa + (2.0 / 75.0) * bbb;
  for (int j = 1; j <= ny; j++) L(j, 4) = 1.0;
  for (int j = 4; j <= ny - 3; j++) {
    L(j, 1) = delta; L(j, 2) = beta; L(j, 3) = alpha;
    L(j, 5) = alpha; L(j, 6) = beta; L(j, 7) = delta;
    R(j, 1) = -ccc / h; R(j, 2) = -bbb / h; R(j, 3) = -aaa / h; R(j, 4) = 0.0;
    R(j, 5) = aaa / h; R(j, 6) = bbb / h; R(j, 7) = ccc / h;
  }
  /* j=1 (cfdiff.f:83-98) */
  L(1, 1) = 0; L(1, 2) = 0; L(1, 3) = 0; L(1, 5) = 1; L(1, 6) = 0; L(1, 7) = 0;
  R(1, 1) = 0; R(1, 2) = 0; R(1, 3) = 0; R(1, 4) = -2.0 / h; R(1, 5) = 2.0 / h; R(1, 6) = 0; R(1, 7) = 0;
  /* j=2 (cfdiff.f:100-115) */
  L(2, 1) = 0; L(2, 2) = 0; L(2, 3) = 0.25; L(2, 5) = 0.25; L(2, 6) = 0; L(2, 7) = 0;
  R(2, 1) = 0; R(2, 2) = 0; R(2, 3) = -3.0 / 4.0 / h; R(2, 4) = 0; R(2, 5) = 3.0 / 4.0 / h; R(2, 6) = 0; R(2, 7) = 0;
  /* j=3 (cfdiff.f:118-132) */
  L(3, 1) = 0; L(3, 2) = 1.0 / 36.0; L(3, 3) = 4.0 / 9.0; L(3, 5) = 4.0 / 9.0; L(3, 6) = 1.0 / 36.0; L(3, 7) = 0;
  R(3, 1) = 0; R(3, 2) = -25.0 / 216.0 / h; R(3, 3) = -20.0 / 27.0 / h; R(3, 4) = 0;
  R(3, 5) = 20.0 / 27.0 / h; R(3, 6) = 25.0 / 216.0 / h; R(3, 7) = 0;
  /* mirrored ends (cfdiff.f:136-179) */
  for (int e = 1; e <= 3; e++) {
    int j = ny + 1 - e;
    L(j, 1) = L(e, 7); L(j, 2) = L(e, 6); L(j, 3) = L(e, 5);
    L(j, 5) = L(e, 3); L(j, 6) = L(e, 2); L(j, 7) = L(e, 1);
    R(j, 1) = -R(e, 7); R(j, 2) = -R(e, 6); R(j, 3) = -R(e, 5); R(j, 4) = -R(e, 4);
    R(j, 5) = -R(e, 3); R(j, 6) = -R(e, 2); R(j, 7) = -R(e, 1);
  }
#undef L
#undef R
}

/* prederiv2: cfdiff.f:196-501.  Second derivative on the actual y, from
 * Taylor-matching systems solved with gaussj. */
static void prederiv2(int ny, double *l /*ny x 5*/, double *r /*ny x 5*/,
                      const double *x /*1-based via X()*/) {
#define L(j, c) l[((c)-1) * ny + ((j)-1)]
#define R(j, c) r[((c)-1) * ny + ((j)-1)]
#define X(j) x[(j)-1]
  double c[81], b[9];
#define C(i, j) c[((j)-1) * 9 + ((i)-1)]
  for (int j = 1; j <= ny; j++) L(j, 3) = 1.0;
  for (int j = 3; j <= ny - 2; j++) {
    double d[4] = {X(j - 2) - X(j), X(j - 1) - X(j), X(j + 1) - X(j), X(j + 2) - X(j)};
    C(1, 1) = 0; C(1, 2) = 0; C(1, 3) = 0; C(1, 4) = 0; C(1, 5) = 1; C(1, 6) = 1; C(1, 7) = 1; C(1, 8) = 1; C(1, 9) = 1; b[0] = 0;
    C(2, 1) = 0; C(2, 2) = 0; C(2, 3) = 0; C(2, 4) = 0; C(2, 5) = d[0]; C(2, 6) = d[1]; C(2, 7) = 0; C(2, 8) = d[2]; C(2, 9) = d[3]; b[1] = 0;
    C(3, 1) = 2; C(3, 2) = 2; C(3, 3) = 2; C(3, 4) = 2;
    C(3, 5) = -d[0] * d[0]; C(3, 6) = -d[1] * d[1]; C(3, 7) = 0; C(3, 8) = -d[2] * d[2]; C(3, 9) = -d[3] * d[3]; b[2] = -2;
    for (int n = 3; n <= 8; n++) {
      double nn = (double)(n * (n - 1));
      C(n + 1, 1) = nn * pow(d[0], n - 2); C(n + 1, 2) = nn * pow(d[1], n - 2);
      C(n + 1, 3) = nn * pow(d[2], n - 2); C(n + 1, 4) = nn * pow(d[3], n - 2);
      C(n + 1, 5) = -pow(d[0], n); C(n + 1, 6) = -pow(d[1], n); C(n + 1, 7) = 0;
      C(n + 1, 8) = -pow(d[2], n); C(n + 1, 9) = -pow(d[3], n); b[n] = 0;
    }
    gaussj(c, 9, 9, b, 1, 1);
    L(j, 1) = b[0]; L(j, 2) = b[1]; L(j, 4) = b[2]; L(j, 5) = b[3];
    R(j, 1) = b[4]; R(j, 2) = b[5]; R(j, 3) = b[6]; R(j, 4) = b[7]; R(j, 5) = b[8];
  }
  { /* j=1 (cfdiff.f:283-335) */
    int j = 1;
    double d1 = X(j + 1) - X(j), d2 = X(j + 2) - X(j);
    C(1, 1) = 0; C(1, 2) = 0; C(1, 3) = 1; C(1, 4) = 1; C(1, 5) = 1; b[0] = 0;
    C(2, 1) = 0; C(2, 2) = 0; C(2, 3) = 0; C(2, 4) = d1; C(2, 5) = d2; b[1] = 0;
    C(3, 1) = 2; C(3, 2) = 2; C(3, 3) = 0; C(3, 4) = -d1 * d1; C(3, 5) = -d2 * d2; b[2] = -2;
    for (int n = 3; n <= 4; n++) {
      double nn = (double)(n * (n - 1));
      C(n + 1, 1) = nn * pow(d1, n - 2); C(n + 1, 2) = nn * pow(d2, n - 2); C(n + 1, 3) = 0;
      C(n + 1, 4) = -pow(d1, n); C(n + 1, 5) = -pow(d2, n); b[n] = 0;
    }
    gaussj(c, 5, 9, b, 1, 1);
    L(j, 1) = 0; L(j, 2) = 0; L(j, 4) = b[0]; L(j, 5) = b[1];
    R(j, 1) = 0; R(j, 2) = 0; R(j, 3) = b[2]; R(j, 4) = b[3]; R(j, 5) = b[4];
  }
  { /* j=2 (cfdiff.f:338-387) */
    int j = 2;
    double dm1 = X(j - 1) - X(j), d1 = X(j + 1) - X(j), d2 = X(j + 2) - X(j);
    C(1, 1) = 0; C(1, 2) = 0; C(1, 3) = 0; C(1, 4) = 1; C(1, 5) = 1; C(1, 6) = 1; C(1, 7) = 1; b[0] = 0;
    C(2, 1) = 0; C(2, 2) = 0; C(2, 3) = 0; C(2, 4) = dm1; C(2, 5) = 0; C(2, 6) = d1; C(2, 7) = d2; b[1] = 0;
    C(3, 1) = 2; C(3, 2) = 2; C(3, 3) = 2; C(3, 4) = -dm1 * dm1; C(3, 5) = 0; C(3, 6) = -d1 * d1; C(3, 7) = -d2 * d2; b[2] = -2;
    for (int n = 3; n <= 6; n++) {
      double nn = (double)(n * (n - 1));
      C(n + 1, 1) = nn * pow(dm1, n - 2); C(n + 1, 2) = nn * pow(d1, n - 2); C(n + 1, 3) = nn * pow(d2, n - 2);
      C(n + 1, 4) = -pow(dm1, n); C(n + 1, 5) = 0; C(n + 1, 6) = -pow(d1, n); C(n + 1, 7) = -pow(d2, n); b[n] = 0;
    }
    gaussj(c, 7, 9, b, 1, 1);
    L(j, 1) = 0; L(j, 2) = b[0]; L(j, 4) = b[1]; L(j, 5) = b[2];
    R(j, 1) = 0; R(j, 2) = b[3]; R(j, 3) = b[4]; R(j, 4) = b[5]; R(j, 5) = b[6];
  }
  { /* j=ny-1 (cfdiff.f:391-441) */
    int j = ny - 1;
    double dm2 = X(j - 2) - X(j), dm1 = X(j - 1) - X(j), d1 = X(j + 1) - X(j);
    C(1, 1) = 0; C(1, 2) = 0; C(1, 3) = 0; C(1, 4) = 1; C(1, 5) = 1; C(1, 6) = 1; C(1, 7) = 1; b[0] = 0;
    C(2, 1) = 0; C(2, 2) = 0; C(2, 3) = 0; C(2, 4) = dm2; C(2, 5) = dm1; C(2, 6) = 0; C(2, 7) = d1; b[1] = 0;
    C(3, 1) = 2; C(3, 2) = 2; C(3, 3) = 2; C(3, 4) = -dm2 * dm2; C(3, 5) = -dm1 * dm1; C(3, 6) = 0; C(3, 7) = -d1 * d1; b[2] = -2;
    for (int n = 3; n <= 6; n++) {
      double nn = (double)(n * (n - 1));
      C(n + 1, 1) = nn * pow(dm2, n - 2); C(n + 1, 2) = nn * pow(dm1, n - 2); C(n + 1, 3) = nn * pow(d1, n - 2);
      C(n + 1, 4) = -pow(dm2, n); C(n + 1, 5) = -pow(dm1, n); C(n + 1, 6) = 0; C(n + 1, 7) = -pow(d1, n); b[n] = 0;
    }
    gaussj(c, 7, 9, b, 1, 1);
    L(j, 1) = b[0]; L(j, 2) = b[1]; L(j, 4) = b[2]; L(j, 5) = 0;
    R(j, 1) = b[3]; R(j, 2) = b[4]; R(j, 3) = b[5]; R(j, 4) = b[6]; R(j, 5) = 0;
  }
  { /* j=ny (cfdiff.f:445-498) */
    int j = ny;
    double dm1 = X(j - 1) - X(j), dm2 = X(j - 2) - X(j);
    C(1, 1) = 0; C(1, 2) = 0; C(1, 3) = 1; C(1, 4) = 1; C(1, 5) = 1; b[0] = 0;
    C(2, 1) = 0; C(2, 2) = 0; C(2, 3) = 0; C(2, 4) = dm1; C(2, 5) = dm2; b[1] = 0;
    C(3, 1) = 2; C(3, 2) = 2; C(3, 3) = 0; C(3, 4) = -dm1 * dm1; C(3, 5) = -dm2 * dm2; b[2] = -2;
    for (int n = 3; n <= 4; n++) {
      double nn = (double)(n * (n - 1));
      C(n + 1, 1) = nn * pow(dm1, n - 2); C(n + 1, 2) = nn * pow(dm2, n - 2); C(n + 1, 3) = 0;
      C(n + 1, 4) = -pow(dm1, n); C(n + 1, 5) = -pow(dm2, n); b[n] = 0;
    }
    gaussj(c, 5, 9, b, 1, 1);
    L(j, 1) = b[1]; L(j, 2) = b[0]; L(j, 4) = 0; L(j, 5) = 0;
    R(j, 1) = b[4]; R(j, 2) = b[3]; R(j, 3) = b[2]; R(j, 4) = 0; R(j, 5) = 0;
  }
#undef C
#undef X
#undef L
#undef R
}

/* bandec / banbks (5-band, cfdiff.f:954-1022) */
static void bandec(double *a, int n) {
  for (int j = 1; j <= 3; j++) B5(a, j, 1) = B5(a, j + 2, 1);
  for (int j = 1; j <= 4; j++) B5(a, j, 2) = B5(a, j + 1, 2);
  for (int k = 1; k <= n - 2; k++) {
    B5(a, 1, k) = 1.0 / B5(a, 1, k);
    B5(a, 4, k) = B5(a, 1, k + 1) * B5(a, 1, k);
    B5(a, 1, k + 1) = B5(a, 2, k + 1) - B5(a, 4, k) * B5(a, 2, k);
    B5(a, 2, k + 1) = B5(a, 3, k + 1) - B5(a, 4, k) * B5(a, 3, k);
    B5(a, 3, k + 1) = B5(a, 4, k + 1);
    B5(a, 5, k) = B5(a, 1, k + 2) * B5(a, 1, k);
    B5(a, 1, k + 2) = B5(a, 2, k + 2) - B5(a, 5, k) * B5(a, 2, k);
    B5(a, 2, k + 2) = B5(a, 3, k + 2) - B5(a, 5, k) * B5(a, 3, k);
    B5(a, 3, k + 2) = B5(a, 4, k + 2);
    B5(a, 4, k + 2) = B5(a, 5, k + 2);
  }
  B5(a, 1, n - 1) = 1.0 / B5(a, 1, n - 1);
  B5(a, 4, n - 1) = B5(a, 1, n) * B5(a, 1, n - 1);
  B5(a, 1, n) = B5(a, 2, n) - B5(a, 4, n - 1) * B5(a, 2, n - 1);
  B5(a, 2, n) = B5(a, 3, n) - B5(a, 4, n - 1) * B5(a, 3, n - 1);
  B5(a, 3, n) = B5(a, 4, n);
  B5(a, 1, n) = 1.0 / B5(a, 1, n);
}

/* works on a real vector b(1..n) stored 0-based */
static void banbks(const double *a, int n, double *b) {
#define V(k) b[(k)-1]
  for (int k = 1; k <= n - 2; k++) {
    V(k + 1) -= B5(a, 4, k) * V(k);
    V(k + 2) -= B5(a, 5, k) * V(k);
  }
  V(n) -= B5(a, 4, n - 1) * V(n - 1);
  V(n) = V(n) * B5(a, 1, n);
  V(n - 1) = (V(n - 1) - B5(a, 2, n - 1) * V(n)) * B5(a, 1, n - 1);
  for (int i = n - 2; i >= 1; i--) V(i) = (V(i) - B5(a, 2, i) * V(i + 1) - B5(a, 3, i) * V(i + 2)) * B5(a, 1, i);
#undef V
}

/* banbks7 / bandec7 (cfdiff.f:1025-1137) */
static void banbks7(const double *a, int n, double *b) {
#define V(k) b[(k)-1]
  for (int k = 1; k <= n - 3; k++) {
    V(k + 1) -= B7(a, 5, k) * V(k);
    V(k + 2) -= B7(a, 6, k) * V(k);
    V(k + 3) -= B7(a, 7, k) * V(k);
  }
  V(n - 1) -= B7(a, 5, n - 2) * V(n - 2);
  V(n) -= B7(a, 6, n - 2) * V(n - 2);
  V(n) -= B7(a, 5, n - 1) * V(n - 1);
  V(n) = V(n) * B7(a, 1, n);
  V(n - 1) = (V(n - 1) - B7(a, 2, n - 1) * V(n)) * B7(a, 1, n - 1);
  V(n - 2) = (V(n - 2) - B7(a, 2, n - 2) * V(n - 1) - B7(a, 3, n - 2) * V(n)) * B7(a, 1, n - 2);
  for (int i = n - 3; i >= 1; i--)
    V(i) = (V(i) - B7(a, 2, i) * V(i + 1) - B7(a, 3, i) * V(i + 2) - B7(a, 4, i) * V(i + 3)) * B7(a, 1, i);
#undef V
}

static void bandec7(double *a, int n) {
  for (int j = 1; j <= 4; j++) B7(a, j, 1) = B7(a, j + 3, 1);
  for (int j = 1; j <= 5; j++) B7(a, j, 2) = B7(a, j + 2, 2);
  for (int j = 1; j <= 6; j++) B7(a, j, 3) = B7(a, j + 1, 3);
  for (int k = 1; k <= n - 3; k++) {
    B7(a, 1, k) = 1.0 / B7(a, 1, k);
    B7(a, 5, k) = B7(a, 1, k + 1) * B7(a, 1, k);
    B7(a, 1, k + 1) = B7(a, 2, k + 1) - B7(a, 5, k) * B7(a, 2, k);
    B7(a, 2, k + 1) = B7(a, 3, k + 1) - B7(a, 5, k) * B7(a, 3, k);
    B7(a, 3, k + 1) = B7(a, 4, k + 1) - B7(a, 5, k) * B7(a, 4, k);
    B7(a, 4, k + 1) = B7(a, 5, k + 1);
    B7(a, 6, k) = B7(a, 1, k + 2) * B7(a, 1, k);
    B7(a, 1, k + 2) = B7(a, 2, k + 2) - B7(a, 6, k) * B7(a, 2, k);
    B7(a, 2, k + 2) = B7(a, 3, k + 2) - B7(a, 6, k) * B7(a, 3, k);
    B7(a, 3, k + 2) = B7(a, 4, k + 2) - B7(a, 6, k) * B7(a, 4, k);
    B7(a, 4, k + 2) = B7(a, 5, k + 2);
    B7(a, 5, k + 2) = B7(a, 6, k + 2);
    B7(a, 7, k) = B7(a, 1, k + 3) * B7(a, 1, k);
    B7(a, 1, k + 3) = B7(a, 2, k + 3) - B7(a, 7, k) * B7(a, 2, k);
    B7(a, 2, k + 3) = B7(a, 3, k + 3) - B7(a, 7, k) * B7(a, 3, k);
    B7(a, 3, k + 3) = B7(a, 4, k + 3) - B7(a, 7, k) * B7(a, 4, k);
    B7(a, 4, k + 3) = B7(a, 5, k + 3);
    B7(a, 5, k + 3) = B7(a, 6, k + 3);
    B7(a, 6, k + 3) = B7(a, 7, k + 3);
  }
  B7(a, 1, n - 2) = 1.0 / B7(a, 1, n - 2);
  B7(a, 5, n - 2) = B7(a, 1, n - 1) * B7(a, 1, n - 2);
  B7(a, 1, n - 1) = B7(a, 2, n - 1) - B7(a, 5, n - 2) * B7(a, 2, n - 2);
  B7(a, 2, n - 1) = B7(a, 3, n - 1) - B7(a, 5, n - 2) * B7(a, 3, n - 2);
  B7(a, 3, n - 1) = B7(a, 4, n - 1) - B7(a, 5, n - 2) * B7(a, 4, n - 2);
  B7(a, 4, n - 1) = B7(a, 5, n - 1);
  B7(a, 6, n - 2) = B7(a, 1, n) * B7(a, 1, n - 2);
  B7(a, 1, n) = B7(a, 2, n) - B7(a, 6, n - 2) * B7(a, 2, n - 2);
  B7(a, 2, n) = B7(a, 3, n) - B7(a, 6, n - 2) * B7(a, 3, n - 2);
  B7(a, 3, n) = B7(a, 4, n) - B7(a, 6, n - 2) * B7(a, 4, n - 2);
  B7(a, 4, n) = B7(a, 5, n);
  B7(a, 5, n) = B7(a, 6, n);
  B7(a, 1, n - 1) = 1.0 / B7(a, 1, n - 1);
  B7(a, 5, n - 1) = B7(a, 1, n) * B7(a, 1, n - 1);
  B7(a, 1, n) = B7(a, 2, n) - B7(a, 5, n - 1) * B7(a, 2, n - 1);
  B7(a, 2, n) = B7(a, 3, n) - B7(a, 5, n - 1) * B7(a, 3, n - 1);
  B7(a, 3, n) = B7(a, 4, n) - B7(a, 5, n - 1) * B7(a, 4, n - 1);
  B7(a, 4, n) = B7(a, 5, n);
  B7(a, 1, n) = 1.0 / B7(a, 1, n);
}

/* Band matrix-vector products with the reference's truncated edge rows:
 * the 7-band one of deryr2 / calcrhsd1 (cfdiff.f:533-584, laps.f:97-127)
 * and the 5-band one of deryyr2 (cfdiff.f:750-781).  Edge rows only use
 * the in-range columns, exactly as the reference spells them out. */
static void matvec7(const double *m, int n, const double *u, double *out) {
  for (int j = 1; j <= n; j++) {
    double s = 0.0;
    int lo = j - 3 < 1 ? 1 : j - 3, hi = j + 3 > n ? n : j + 3;
    for (int c = lo; c <= hi; c++) s += B7(m, c - j + 4, j) * u[c - 1];
    out[j - 1] = s;
  }
}
static void matvec5(const double *m, int n, const double *u, double *out) {
  for (int j = 1; j <= n; j++) {
    double s = 0.0;
    int lo = j - 2 < 1 ? 1 : j - 2, hi = j + 2 > n ? n : j + 2;
    for (int c = lo; c <= hi; c++) s += B5(m, c - j + 3, j) * u[c - 1];
    out[j - 1] = s;
  }
}

/* ------------------------------------------------------------------ */
/* Oracle object                                                       */
/* ------------------------------------------------------------------ */
struct lmo {
  int mgalx, mgalz, my, mx, nkx, mz, nz1, nz2, nmode;
  double Re, alp, bet, peclet, cfl, ire;
  int ncfl, dtmode, nthreads;
  double *y, *hy, *trp, *fmap;
  double *prem1, *dt11, *dt12, *prem3, *dt21, *dt22; /* band [row][band] */
  double *kxv, *kzv; /* wavenumbers: kx(i)=alp*i, kz(k) signed */
  double gama[3], xi[3], alpha[3], beta[3];
  /* state, reference layout [kx][kz][y] */
  cplx *vor, *phi, *psi, *scal;
  cplx *ten12p, *ten13p; /* RHS(Omega_y), RHS(phi) of the previous substep */
  double *rhst;          /* physical RHS(T) of the previous substep [line][x] */
  double *u00wk, *v00wk, *w00wk, *rf0u, *rf0w, *rf0v;
  double Deltat, time, dtr, rhobot, rhotop;
  int icfl, istep_total;
  int variant;  /* 0: trunk/lomacte3 (2017), 1: trunk/lomacte (2014) */
  cplx *rts;    /* 2014 variant: spectral RHS(T) of the previous substep */
  double diag[LMO_NDIAG];
  fftplan px, pz;
  /* work buffers: spectral [kx][kz][y] (size nmode*my) */
  cplx *w_mx, *w_my, *w_mz, *w_nx, *w_ny, *w_nz, *w_t12, *w_t13, *w_t23, *w_drho, *w_chwk, *w_chwk2;
  /* line buffers [line][kx] complex, line = z + mgalz*y: 8 inputs and 11
   * outputs of the transforms, 12 and 12 with the passive scalar */
  cplx *ln[18];
  /* passive scalar Z (the extension restated in lomacte_oracle.h): state,
   * spectral work (lap Z, dZ/dx, dZ/dy, dZ/dz, Delta Z), physical RHS(Z) of
   * the previous substep, wall values of its 00 mode, Re*Sc */
  int scalar;
  double pez, zbot, ztop;
  cplx *zsc, *w_zlap, *w_zx, *w_zy, *w_zz, *w_dz;
  double *rhsz;
  /* variable viscosity mu = k = rho D = T^vsig (the extension restated in
   * lomacte_oracle.h): on/off, the exponent, and the six spectral inputs
   * d(rho u)/dx, d(rho v)/dy, d(rho w)/dz, and the symmetric sums
   * d(rho u)/dy + d(rho v)/dx, d(rho u)/dz + d(rho w)/dx,
   * d(rho v)/dz + d(rho w)/dy */
  int vs;
  double vsig;
  cplx *w_g[6];
  /* statistics (cross.f:578-585, 794-812, 1583-1607; escru.f:276-580):
   * st[LMO_NSTAT][my] raw accumulators in the order of the .sta record,
   * sp[nkx][12][nsp][nz1+1] spectra, uner[9] energies of the last
   * accumulating step, jsp the 0-based rows of the spectra planes */
  int istati, nsp, nacum, nacumsp;
  int *jsp;
  double sigma;
  double *st, *sp, uner[9];
  /* timing samples (lmo_set_sample): with smp > 1 the parallel loops of a
   * substep visit only the units (modes, kx planes of a field, physical
   * lines) whose index is smph modulo smp, i.e. 1/smp of the work */
  int smp, smph;
};

static inline int skip_unit(const lmo *o, long u) { return o->smp > 1 && (int)(u % o->smp) != o->smph; }

#define SIDX(o, i, k, j) (((size_t)(i) * (o)->mz + (k)) * (o)->my + (j))

static void *xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

lmo *lmo_create(int mgalx, int mgalz, int my, const double *y, double Re,
                double alp, double bet, double peclet, double cfl, int ncfl,
                int dtmode, double dt0, int nthreads) {
  if (mgalx < 6 || mgalz < 3 || my < 9) return NULL;
  lmo *o = (lmo *)xcalloc(1, sizeof(lmo));
  o->mgalx = mgalx; o->mgalz = mgalz; o->my = my;
  o->mx = 2 * (mgalx / 3); o->nkx = o->mx / 2;
  o->mz = 2 * (mgalz / 3) - 1; o->nz1 = (o->mz - 1) / 2; o->nz2 = mgalz - o->nz1;
  o->nmode = o->nkx * o->mz;
  o->Re = Re; o->alp = alp; o->bet = bet; o->peclet = peclet; o->cfl = cfl;
  o->ire = 1.0 / Re; o->ncfl = ncfl < 1 ? 1 : ncfl; o->dtmode = dtmode;
  o->nthreads = nthreads;
  rk_coefs(o->gama, o->xi, o->alpha, o->beta);
  o->y = (double *)xcalloc(my, 8); memcpy(o->y, y, sizeof(double) * my);
  o->hy = (double *)xcalloc(my, 8); o->trp = (double *)xcalloc(my, 8); o->fmap = (double *)xcalloc(my, 8);
  /* main.f:689-696 */
  for (int j = 2; j <= my - 1; j++) {
    o->trp[j - 1] = 0.25 * (y[j] - y[j - 2]);
    o->hy[j - 1] = (y[j] - y[j - 2]) / 2.0;
  }
  o->trp[0] = 0.25 * (y[1] - y[0]);
  o->trp[my - 1] = 0.25 * (y[my - 1] - y[my - 2]);
  o->hy[0] = (y[1] - y[0]) / 2.0;
  o->hy[my - 1] = (y[my - 1] - y[my - 2]) / 2.0;
  /* derivadas: cfdiff.f:869-941 */
  double *d11 = xcalloc((size_t)my * 7, 8), *d12 = xcalloc((size_t)my * 7, 8);
  double *d21 = xcalloc((size_t)my * 5, 8), *d22 = xcalloc((size_t)my * 5, 8);
  pred1m6o(my, d11, d12);
  prederiv2(my, d21, d22, y);
  o->prem1 = xcalloc((size_t)my * 7, 8); o->dt11 = xcalloc((size_t)my * 7, 8); o->dt12 = xcalloc((size_t)my * 7, 8);
  o->prem3 = xcalloc((size_t)my * 5, 8); o->dt21 = xcalloc((size_t)my * 5, 8); o->dt22 = xcalloc((size_t)my * 5, 8);
  for (int j = 1; j <= my; j++)
    for (int i = 1; i <= 7; i++) {
      B7(o->prem1, i, j) = d11[(i - 1) * my + j - 1];
      B7(o->dt11, i, j) = d11[(i - 1) * my + j - 1];
      B7(o->dt12, i, j) = d12[(i - 1) * my + j - 1];
    }
  for (int j = 1; j <= my; j++)
    for (int i = 1; i <= 5; i++) {
      B5(o->prem3, i, j) = d21[(i - 1) * my + j - 1];
      B5(o->dt21, i, j) = d21[(i - 1) * my + j - 1];
      B5(o->dt22, i, j) = d22[(i - 1) * my + j - 1];
    }
  free(d11); free(d12); free(d21); free(d22);
  bandec7(o->prem1, my);
  bandec(o->prem3, my);
  matvec7(o->dt12, my, o->y, o->fmap);
  banbks7(o->prem1, my, o->fmap);
  for (int j = 0; j < my; j++) o->fmap[j] = 1.0 / o->fmap[j];
  /* wavenumbers: main.f:769-800 */
  o->kxv = xcalloc(o->nkx, 8); o->kzv = xcalloc(o->mz, 8);
  for (int i = 0; i < o->nkx; i++) o->kxv[i] = alp * i;
  for (int k = 0; k <= o->nz1; k++) o->kzv[k] = bet * k;
  for (int k = o->nz1 + 1; k < o->mz; k++) o->kzv[k] = -bet * (o->mz - k);
  size_t ns = (size_t)o->nmode * my;
  cplx **bufs[] = {&o->vor, &o->phi, &o->psi, &o->scal, &o->ten12p, &o->ten13p,
                   &o->w_mx, &o->w_my, &o->w_mz, &o->w_nx, &o->w_ny, &o->w_nz,
                   &o->w_t12, &o->w_t13, &o->w_t23, &o->w_drho, &o->w_chwk, &o->w_chwk2, &o->rts};
  for (size_t b = 0; b < sizeof(bufs) / sizeof(bufs[0]); b++) *bufs[b] = xcalloc(ns, sizeof(cplx));
  size_t nl = (size_t)mgalz * my;
  for (int f = 0; f < 12; f++) o->ln[f] = xcalloc(nl * o->nkx, sizeof(cplx));
  o->rhst = xcalloc(nl * mgalx, 8);
  o->u00wk = xcalloc(my, 8); o->v00wk = xcalloc(my, 8); o->w00wk = xcalloc(my, 8);
  o->rf0u = xcalloc(my, 8); o->rf0w = xcalloc(my, 8); o->rf0v = xcalloc(my, 8);
  plan_init(&o->px, mgalx);
  plan_init(&o->pz, mgalz);
  o->Deltat = dt0; o->icfl = 1; o->dtr = dt0;
  return o;
}

void lmo_destroy(lmo *o) {
  if (!o) return;
  void *p[] = {o->y, o->hy, o->trp, o->fmap, o->prem1, o->dt11, o->dt12, o->prem3, o->dt21, o->dt22,
               o->kxv, o->kzv, o->vor, o->phi, o->psi, o->scal, o->ten12p, o->ten13p, o->rhst,
               o->u00wk, o->v00wk, o->w00wk, o->rf0u, o->rf0w, o->rf0v, o->w_mx, o->w_my, o->w_mz,
               o->w_nx, o->w_ny, o->w_nz, o->w_t12, o->w_t13, o->w_t23, o->w_drho, o->w_chwk, o->w_chwk2,
               o->rts};
  for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) free(p[i]);
  for (int f = 0; f < 18; f++) free(o->ln[f]);
  for (int f = 0; f < 6; f++) free(o->w_g[f]);
  free(o->jsp); free(o->st); free(o->sp);
  free(o->zsc); free(o->w_zlap); free(o->w_zx); free(o->w_zy); free(o->w_zz); free(o->w_dz); free(o->rhsz);
  plan_free(&o->px); plan_free(&o->pz);
  free(o);
}

/* State I/O.  The RK3 memory (previous RHS) is reset, as in a fresh run:
 * main.f zeroes the whole work pool before cross1 (main.f:171-174). */
int lmo_set_state(lmo *o, const double *vor, const double *phi, const double *psi,
                  const double *scal, const double *u00, const double *v00,
                  const double *w00, double time) {
  size_t ns = (size_t)o->nmode * o->my;
  memcpy(o->vor, vor, ns * sizeof(cplx)); memcpy(o->phi, phi, ns * sizeof(cplx));
  memcpy(o->psi, psi, ns * sizeof(cplx)); memcpy(o->scal, scal, ns * sizeof(cplx));
  memset(o->ten12p, 0, ns * sizeof(cplx)); memset(o->ten13p, 0, ns * sizeof(cplx));
  memset(o->rts, 0, ns * sizeof(cplx));
  memset(o->rhst, 0, (size_t)o->mgalz * o->my * o->mgalx * 8);
  if (o->rhsz) memset(o->rhsz, 0, (size_t)o->mgalz * o->my * o->mgalx * 8);
  /* cross.f:276-280 (first step copies the 00 modes to the work vectors) */
  memcpy(o->u00wk, u00, o->my * 8); memcpy(o->v00wk, v00, o->my * 8); memcpy(o->w00wk, w00, o->my * 8);
  memset(o->rf0u, 0, o->my * 8); memset(o->rf0w, 0, o->my * 8); memset(o->rf0v, 0, o->my * 8);
  o->time = time;
  /* cross.f:211-213 */
  o->rhobot = 1.0 / creal(o->scal[SIDX(o, 0, 0, 0)]);
  o->rhotop = 1.0 / creal(o->scal[SIDX(o, 0, 0, o->my - 1)]);
  o->icfl = 1; o->istep_total = 0;
  return 0;
}

int lmo_get_state(const lmo *o, double *vor, double *phi, double *psi, double *scal,
                  double *u00, double *v00, double *w00, double *time) {
  size_t ns = (size_t)o->nmode * o->my;
  if (vor) memcpy(vor, o->vor, ns * sizeof(cplx));
  if (phi) memcpy(phi, o->phi, ns * sizeof(cplx));
  if (psi) memcpy(psi, o->psi, ns * sizeof(cplx));
  if (scal) memcpy(scal, o->scal, ns * sizeof(cplx));
  if (u00) memcpy(u00, o->u00wk, o->my * 8);
  if (v00) memcpy(v00, o->v00wk, o->my * 8);
  if (w00) memcpy(w00, o->w00wk, o->my * 8);
  if (time) *time = o->time;
  return 0;
}

/* ------------------------------------------------------------------ */
/* y-operators on complex pencils (componentwise, real operators).     */
/* ------------------------------------------------------------------ */
/* deryr2: cfdiff.f:518-601 */
static void deryr2_c(const lmo *o, const cplx *u, cplx *du, double *w1, double *w2, double *t1, double *t2) {
  int my = o->my;
  for (int j = 0; j < my; j++) { t1[j] = creal(u[j]); t2[j] = cimag(u[j]); }
  matvec7(o->dt12, my, t1, w1); matvec7(o->dt12, my, t2, w2);
  banbks7(o->prem1, my, w1); banbks7(o->prem1, my, w2);
  for (int j = 0; j < my; j++) du[j] = w1[j] * o->fmap[j] + I * (w2[j] * o->fmap[j]);
}
/* deryyr2: cfdiff.f:735-797 */
static void deryyr2_c(const lmo *o, const cplx *u, cplx *du, double *w1, double *w2, double *t1, double *t2) {
  int my = o->my;
  for (int j = 0; j < my; j++) { t1[j] = creal(u[j]); t2[j] = cimag(u[j]); }
  matvec5(o->dt22, my, t1, w1); matvec5(o->dt22, my, t2, w2);
  banbks(o->prem3, my, w1); banbks(o->prem3, my, w2);
  for (int j = 0; j < my; j++) du[j] = w1[j] + I * w2[j];
}

/* deryr / deryyr on one real FP64 vector: cfdiff.f:615-710 */
void lmo_deryr(const lmo *o, const double *u, double *du) {
  double *f = malloc(sizeof(double) * o->my);
  matvec7(o->dt12, o->my, u, f);
  banbks7(o->prem1, o->my, f);
  for (int j = 0; j < o->my; j++) du[j] = f[j] * o->fmap[j];
  free(f);
}
void lmo_deryyr(const lmo *o, const double *u, double *du) {
  double *f = malloc(sizeof(double) * o->my);
  matvec5(o->dt22, o->my, u, f);
  banbks(o->prem3, o->my, f);
  memcpy(du, f, sizeof(double) * o->my);
  free(f);
}

/* inty8: laps.f:484-575.  Integrates du once with the compact scheme,
 * u(1) = 0. */
void lmo_inty8(const lmo *o, const double *du, double *u) {
  int my = o->my;
  double *wk2 = malloc(sizeof(double) * 7 * my), *f = malloc(sizeof(double) * my), *v = malloc(sizeof(double) * my);
  memcpy(wk2, o->dt12, sizeof(double) * 7 * my);
  bandec7(wk2, my);
  /* dt12 annihilates constants, so the last pivot of its LU is zero in
   * exact arithmetic and round-off as computed by laps.f:523.  Only
   * u - u(1) is used (laps.f:567-571) and it does not depend on the last
   * unknown: set the reciprocal last pivot to 0 (last unknown = 0). */
  B7(wk2, 1, my) = 0.0;
  for (int j = 0; j < my; j++) f[j] = du[j] / o->fmap[j];
  matvec7(o->dt11, my, f, v);
  banbks7(wk2, my, v);
  for (int j = 0; j < my; j++) u[j] = v[j] - v[0];
  free(wk2); free(f); free(v);
}

/* calcrhslap: laps.f:17-47 (rows 1 and my zeroed) */
static void calcrhslap(const lmo *o, const double *f, double *r) {
  int my = o->my;
  matvec5(o->dt21, my, f, r);
  r[0] = 0.0;
  r[my - 1] = 0.0;
}

/* Poisson operator wk1 = dt22 - rK*dt21 with identity rows 1 and my,
 * factorised with bandec: laps.f:349-366 / laps.f:648-665. */
static void poisson_factor(const lmo *o, double rk, double *wk1) {
  int my = o->my;
  for (int j = 2; j <= my - 1; j++)
    for (int i = 1; i <= 5; i++) B5(wk1, i, j) = B5(o->dt22, i, j) - rk * B5(o->dt21, i, j);
  for (int i = 1; i <= 5; i++) { B5(wk1, i, 1) = 0.0; B5(wk1, i, my) = 0.0; }
  B5(wk1, 3, 1) = 1.0;
  B5(wk1, 3, my) = 1.0;
  bandec(wk1, my);
}

/* Lapvdvhom: laps.f:319-477.  Solves v'' - rK v = phi with v=0 at both
 * walls and returns v and dv/dy (rK=0 -> zeros). */
static void lapvdvhom_c(const lmo *o, const cplx *phi, cplx *v, cplx *dvdy, double rk, double *scratch) {
  int my = o->my;
  if (rk == 0.0) {
    for (int j = 0; j < my; j++) { v[j] = 0; dvdy[j] = 0; }
    return;
  }
  double *wk1 = scratch, *d1 = scratch + 5 * my, *d2 = d1 + my, *f1 = d2 + my, *f2 = f1 + my, *fw = f2 + my;
  poisson_factor(o, rk, wk1);
  for (int j = 0; j < my; j++) { d1[j] = creal(phi[j]); d2[j] = cimag(phi[j]); }
  matvec5(o->dt21, my, d1, f1); matvec5(o->dt21, my, d2, f2);
  f1[0] = 0; f2[0] = 0; f1[my - 1] = 0; f2[my - 1] = 0;
  banbks(wk1, my, f1);
  banbks(wk1, my, f2);
  for (int j = 0; j < my; j++) v[j] = f1[j] + I * f2[j];
  matvec7(o->dt12, my, f1, fw); banbks7(o->prem1, my, fw);
  for (int j = 0; j < my; j++) d1[j] = fw[j] * o->fmap[j];
  matvec7(o->dt12, my, f2, fw); banbks7(o->prem1, my, fw);
  for (int j = 0; j < my; j++) dvdy[j] = d1[j] + I * (fw[j] * o->fmap[j]);
}

/* solvepsi: laps.f:580-730.  Solves psi'' - rK psi = phi with
 * dpsi/dy = 0 at both walls (influence-matrix method with two
 * homogeneous solutions and a 2x2 gaussj), returns psi and dpsi/dy. */
static void solvepsi_c(const lmo *o, const cplx *phi, cplx *v, cplx *dvdy, double rk, double *scratch) {
  int my = o->my;
  if (rk == 0.0) {
    for (int j = 0; j < my; j++) { v[j] = 0; dvdy[j] = 0; }
    return;
  }
  const double Cvtop = 0.0, Cdyvtop = 1.0, BC_top = 0.0, Cvbot = 0.0, Cdyvbot = 1.0, BC_bot = 0.0;
  double *wk1 = scratch, *v1 = wk1 + 5 * my, *v2 = v1 + my, *vpr = v2 + my, *vpi = vpr + my;
  double *dvpr = vpi + my, *dvpi = dvpr + my, *dv1 = dvpi + my, *dv2 = dv1 + my;
  poisson_factor(o, rk, wk1);
  for (int j = 0; j < my; j++) { v1[j] = creal(phi[j]); v2[j] = cimag(phi[j]); }
  calcrhslap(o, v1, vpr);
  calcrhslap(o, v2, vpi);
  v1[0] = 1.0; v2[0] = 0.0;
  for (int j = 1; j < my - 1; j++) { v1[j] = 0.0; v2[j] = 0.0; }
  v1[my - 1] = 0.0; v2[my - 1] = 1.0;
  banbks(wk1, my, vpr); banbks(wk1, my, vpi); banbks(wk1, my, v1); banbks(wk1, my, v2);
  matvec7(o->dt12, my, vpr, dvpr); matvec7(o->dt12, my, vpi, dvpi);
  matvec7(o->dt12, my, v1, dv1); matvec7(o->dt12, my, v2, dv2);
  banbks7(o->prem1, my, dvpr); banbks7(o->prem1, my, dvpi);
  banbks7(o->prem1, my, dv1); banbks7(o->prem1, my, dv2);
  double AA[4], coef[4];
  const double *fm = o->fmap;
  AA[0] = Cvbot + Cdyvbot * dv1[0] * fm[0];          /* AA(1,1) */
  AA[2] = Cdyvbot * dv2[0] * fm[0];                  /* AA(1,2) */
  AA[1] = Cdyvtop * dv1[my - 1] * fm[my - 1];        /* AA(2,1) */
  AA[3] = Cvtop + Cdyvtop * dv2[my - 1] * fm[my - 1]; /* AA(2,2) */
  coef[0] = BC_bot - Cdyvbot * dvpr[0] * fm[0];
  coef[1] = BC_top - Cdyvtop * dvpr[my - 1] * fm[my - 1];
  coef[2] = BC_bot - Cdyvbot * dvpi[0] * fm[0];
  coef[3] = BC_top - Cdyvtop * dvpi[my - 1] * fm[my - 1];
  gaussj(AA, 2, 2, coef, 2, 2);
  for (int j = 0; j < my; j++) {
    v[j] = (vpr[j] + coef[0] * v1[j] + coef[1] * v2[j]) + I * (vpi[j] + coef[2] * v1[j] + coef[3] * v2[j]);
    dvdy[j] = fm[j] * (dvpr[j] + coef[0] * dv1[j] + coef[1] * dv2[j]) +
              I * (fm[j] * (dvpi[j] + coef[2] * dv1[j] + coef[3] * dv2[j]));
  }
}

void lmo_lapvdvhom(const lmo *o, const double *phi, double *v, double *dvdy, double rk) {
  double *s = malloc(sizeof(double) * 16 * o->my);
  lapvdvhom_c(o, (const cplx *)phi, (cplx *)v, (cplx *)dvdy, rk, s);
  free(s);
}
void lmo_solvepsi(const lmo *o, const double *phi, double *v, double *dvdy, double rk) {
  double *s = malloc(sizeof(double) * 16 * o->my);
  solvepsi_c(o, (const cplx *)phi, (cplx *)v, (cplx *)dvdy, rk, s);
  free(s);
}

/* ------------------------------------------------------------------ */
/* Transforms (fou3D.f)                                                 */
/* ------------------------------------------------------------------ */
/* spectral kz index -> padded physical-FFT index (localyz2zy,
 * fou3D.f:103-145): k<=nz1 stays, k>nz1 moves to k+(mgalz-mz). */
static inline int kz_pad(const lmo *o, int k) { return k <= o->nz1 ? k : k + (o->mgalz - o->mz); }

/* foup2 inverse half for one kx plane: localyz2zy + fourz(+1)
 * (fou3D.f:80-145), writing the x-lines buffer [line][kx]. */
static void zinv_plane(const lmo *o, int i, const cplx *spec, cplx *lines, cplx *buf, cplx *out) {
  int my = o->my, mgalz = o->mgalz, nkx = o->nkx;
  for (int j = 0; j < my; j++) {
    for (int z = 0; z < mgalz; z++) buf[z] = 0;
    for (int k = 0; k < o->mz; k++) buf[kz_pad(o, k)] = spec[SIDX(o, i, k, j)];
    cfft(&o->pz, buf, out, +1);
    for (int z = 0; z < mgalz; z++) lines[((size_t)j * mgalz + z) * nkx + i] = out[z];
  }
}
/* foup2 forward half: fourz(-1) + truncation + localzy2yz (fou3D.f:149-189) */
static void zfwd_plane(const lmo *o, int i, const cplx *lines, cplx *spec, cplx *buf, cplx *out) {
  int my = o->my, mgalz = o->mgalz, nkx = o->nkx;
  double dn = 1.0 / (double)mgalz;
  for (int j = 0; j < my; j++) {
    for (int z = 0; z < mgalz; z++) buf[z] = lines[((size_t)j * mgalz + z) * nkx + i];
    cfft(&o->pz, buf, out, -1);
    for (int k = 0; k < o->mz; k++) spec[SIDX(o, i, k, j)] = out[kz_pad(o, k)] * dn;
  }
}

/* fourx inverse (fou3D.f:29-60 + rftsingle.f:25-95) of two lines at once:
 * kx modes 0..nkx-1 (Im of mode 0 dropped, higher modes zero) -> two real
 * lines, via one complex transform of A + iB. */
static void xinv2(const lmo *o, const cplx *A, const cplx *B, double *a, double *b, cplx *buf, cplx *out) {
  int n = o->mgalx, nk = o->nkx;
  for (int k = 0; k < n; k++) buf[k] = 0;
  buf[0] = creal(A[0]) + I * creal(B[0]);
  for (int k = 1; k < nk; k++) {
    buf[k] = A[k] + I * B[k];
    buf[n - k] = conj(A[k]) + I * conj(B[k]);
  }
  cfft(&o->px, buf, out, +1);
  for (int x = 0; x < n; x++) { a[x] = creal(out[x]); b[x] = cimag(out[x]); }
}
/* fourx direct of two real lines, scaled by 1/n, truncated to kx<nkx and
 * Im(mode 0) = 0 (rftsingle.f:62-72, fou3D.f:43-46, cross.f:1723-1760). */
static void xfwd2(const lmo *o, const double *a, const double *b, cplx *A, cplx *B, cplx *buf, cplx *out) {
  int n = o->mgalx, nk = o->nkx;
  double dn = 1.0 / (double)n;
  for (int x = 0; x < n; x++) buf[x] = a[x] + I * (b ? b[x] : 0.0);
  cfft(&o->px, buf, out, -1);
  A[0] = creal(out[0]) * dn;
  if (B) B[0] = cimag(out[0]) * dn;
  for (int k = 1; k < nk; k++) {
    cplx c1 = out[k], c2 = conj(out[n - k]);
    A[k] = 0.5 * (c1 + c2) * dn;
    if (B) B[k] = -0.5 * I * (c1 - c2) * dn;
  }
}

/* Public single-vector FFT entry points for the golden-vector tests. */
void lmo_cft(int n, double *c, int iopt) {
  fftplan p; plan_init(&p, n);
  cplx *in = malloc(sizeof(cplx) * n), *out = malloc(sizeof(cplx) * n);
  memcpy(in, c, sizeof(cplx) * n);
  cfft(&p, in, out, iopt < 0 ? -1 : +1);
  double s = iopt < 0 ? 1.0 / n : 1.0;
  for (int k = 0; k < n; k++) { c[2 * k] = creal(out[k]) * s; c[2 * k + 1] = cimag(out[k]) * s; }
  free(in); free(out); plan_free(&p);
}
void lmo_rft(int n, double *c, int iopt) {
  fftplan p; plan_init(&p, n);
  cplx *in = malloc(sizeof(cplx) * n), *out = malloc(sizeof(cplx) * n);
  if (iopt < 0) {
    for (int x = 0; x < n; x++) in[x] = c[x];
    cfft(&p, in, out, -1);
    for (int k = 0; k <= n / 2; k++) { c[2 * k] = creal(out[k]) / n; c[2 * k + 1] = cimag(out[k]) / n; }
    c[1] = 0.0;
    c[n + 1] = 0.0;
  } else {
    for (int k = 0; k < n; k++) in[k] = 0;
    in[0] = c[0];
    for (int k = 1; k < n / 2; k++) { in[k] = c[2 * k] + I * c[2 * k + 1]; in[n - k] = conj(in[k]); }
    in[n / 2] = c[n];
    cfft(&p, in, out, +1);
    for (int x = 0; x < n; x++) c[x] = creal(out[x]);
  }
  free(in); free(out); plan_free(&p);
}

/* ------------------------------------------------------------------ */
/* phys2: cross.f:1440-1828.  Per (z,y) line: 8 inverse x-transforms,  */
/* FP64 products, T update, d(rho)/dt source, CFL maxima, 11 direct    */
/* x-transforms with dealiasing.                                       */
/* lines in : 0 rhou 1 rhov 2 rhow 3 lapT 4 dTdx 5 dTdy 6 dTdz 7 T       */
/* lines out: 0 u 1 v 2 w 3 rhouu 4 rhovv 5 rhoww 6 rhouv 7 rhouw       */
/*            8 rhovw 9 drho 10 DT                                     */
/* ------------------------------------------------------------------ */
static void phys2(lmo *o, int rk, double dtxi, double dtgamma, double dtbeta, int do_cfl, int do_mass,
                  double *cflout /*4*/, double *rhom /*my*/) {
  int mgalx = o->mgalx, mgalz = o->mgalz, my = o->my, nkx = o->nkx;
  size_t nlines = (size_t)mgalz * my;
  /* statistics of the physical fields (cross.f:1583-1607), per line, added
   * into the profiles in line order after the parallel loop */
  const int do_st = o->istati && rk == 0 && o->st;
  double *lst = do_st ? xcalloc(nlines * 9, 8) : NULL;
  double cflx = 0, cfly = 0, cflz = 0, cflT = 0;
  double hxalp = o->alp * (mgalx - 1) / M_PI, hzbet = o->bet * (mgalz - 1) / M_PI;
  double ab = o->alpha[rk] / o->beta[rk];
#pragma omp parallel num_threads(o->nthreads)
  {
    double *ph = malloc(sizeof(double) * mgalx * 18), *out = malloc(sizeof(double) * mgalx * 12);
    cplx *buf = malloc(sizeof(cplx) * mgalx), *fo = malloc(sizeof(cplx) * mgalx);
    cplx *spec = malloc(sizeof(cplx) * nkx * 12);
#pragma omp for schedule(static)
    for (long L = 0; L < (long)nlines; L++) {
      if (skip_unit(o, L)) continue;
      int jj = (int)(L / mgalz); /* y index (cross.f:1583) */
      const int vb = o->scalar ? 12 : 8, nin = vb + (o->vs ? 6 : 0), nout = o->scalar ? 12 : 11;
      cplx *sp[18];
      for (int f = 0; f < nin; f++) sp[f] = o->ln[f] + (size_t)L * nkx;
      double *p[18];
      for (int f = 0; f < nin; f++) p[f] = ph + (size_t)f * mgalx;
      for (int f = 0; f < nin; f += 2) xinv2(o, sp[f], sp[f + 1], p[f], p[f + 1], buf, fo);
      double *ru = p[0], *rv = p[1], *rw = p[2], *lapT = p[3], *tx = p[4], *ty = p[5], *tz = p[6], *T = p[7];
      double *rh = o->rhst + (size_t)L * mgalx;
      double *q[12];
      for (int f = 0; f < nout; f++) q[f] = out + (size_t)f * mgalx;
      double lmx = 0, lmy = 0, lmz = 0, Tmax = 0, rsum = 0;
      for (int x = 0; x < mgalx; x++) {
        double u = ru[x] * T[x], v = rv[x] * T[x], w = rw[x] * T[x]; /* cross.f:1613-1622 */
        double tnext = T[x] + dtxi * rh[x];                            /* cross.f:1625-1629 */
        double d8 = dtxi * rh[x];
        double rhs = -u * tx[x] - v * ty[x] - w * tz[x] + T[x] * lapT[x] / o->peclet; /* cross.f:1631-1637 */
        double tsg = 1.0; /* mu = k = rho D = T^sigma */
        if (o->vs) { /* branches/loma/src/cross.f:1591-1596 */
          tsg = pow(T[x], o->vsig);
          const double g2 = tx[x] * tx[x] + ty[x] * ty[x] + tz[x] * tz[x];
          rhs = -u * tx[x] - v * ty[x] - w * tz[x] + tsg * (T[x] * lapT[x] + o->vsig * g2) / o->peclet;
        }
        rh[x] = rhs;
        tnext = tnext + dtgamma * rhs; /* cross.f:1640-1643 */
        d8 = d8 + dtgamma * rhs;
        q[10][x] = d8;                     /* DT (cross.f:1645-1647) */
        if (o->scalar) { /* the passive scalar, advanced as T is */
          const double *zl = p[8], *zx = p[9], *zy = p[10], *zz = p[11];
          double *rz = o->rhsz + (size_t)L * mgalx;
          double dz = dtxi * rz[x];
          double rzs = -u * zx[x] - v * zy[x] - w * zz[x] + T[x] * zl[x] / o->pez;
          if (o->vs) /* rho D = T^sigma */
            rzs = -u * zx[x] - v * zy[x] - w * zz[x] +
                  tsg * (T[x] * zl[x] + o->vsig * (tx[x] * zx[x] + ty[x] * zy[x] + tz[x] * zz[x])) / o->pez;
          rz[x] = rzs;
          q[11][x] = dz + dtgamma * rzs;
        }
        q[0][x] = u; q[1][x] = v; q[2][x] = w;
        q[3][x] = ru[x] * u; q[4][x] = rv[x] * v; q[5][x] = rw[x] * w; /* cross.f:1655-1659 */
        q[6][x] = ru[x] * v; q[7][x] = ru[x] * w; q[8][x] = rv[x] * w; /* cross.f:1662-1666 */
        if (o->vs) { /* minus the variable part of the stress, 2 (T^sigma - 1) S_ij / Re */
          const double *g0 = p[vb], *g1 = p[vb + 1], *g2 = p[vb + 2], *g3 = p[vb + 3], *g4 = p[vb + 4],
                       *g5 = p[vb + 5];
          const double c = o->ire * (tsg - 1.0), Tx = T[x];
          q[3][x] -= 2.0 * c * (Tx * g0[x] + ru[x] * tx[x]);
          q[4][x] -= 2.0 * c * (Tx * g1[x] + rv[x] * ty[x]);
          q[5][x] -= 2.0 * c * (Tx * g2[x] + rw[x] * tz[x]);
          q[6][x] -= c * (Tx * g3[x] + ru[x] * ty[x] + rv[x] * tx[x]);
          q[7][x] -= c * (Tx * g4[x] + ru[x] * tz[x] + rw[x] * tx[x]);
          q[8][x] -= c * (Tx * g5[x] + rv[x] * tz[x] + rw[x] * ty[x]);
        }
        q[9][x] = (d8 / (T[x] * tnext)) / dtbeta - ab * rhs / (T[x] * T[x]); /* cross.f:1669-1673 */
        if (do_cfl) {
          lmx = fmax(lmx, fabs(u)); lmy = fmax(lmy, fabs(v)); lmz = fmax(lmz, fabs(w)); Tmax = fmax(Tmax, T[x]);
        }
        if (do_mass) rsum += 1.0 / T[x];
      }
      if (do_st) { /* cross.f:1587-1607 */
        double *a = lst + (size_t)L * 9;
        for (int x = 0; x < mgalx; x++) {
          double uu = ru[x] * T[x];
          a[0] += uu * ru[x]; a[1] += uu * rv[x]; a[2] += uu * rw[x];
        }
        for (int x = 0; x < mgalx; x++) {
          double vv = rv[x] * T[x];
          a[3] += vv * rv[x]; a[4] += vv * rw[x];
        }
        for (int x = 0; x < mgalx; x++) {
          double ww = rw[x] * T[x];
          a[5] += ww * rw[x];
        }
        for (int x = 0; x < mgalx; x++) {
          a[6] += 1.0 / T[x];
          a[7] += pow(T[x], o->sigma);
          a[8] += pow(T[x], o->sigma + 1.0);
        }
      }
      if (do_cfl) { /* cross.f:1690-1708 */
        double DD = (o->scalar ? fmax(1.0 / o->peclet, 1.0 / o->pez) : 1.0 / o->peclet) *
                    (o->vs ? pow(Tmax, 1.0 + o->vsig) : Tmax);
        double c0 = lmy / o->hy[jj];
        double cT = 2 * DD * ((hxalp / 2) * (hxalp / 2) + (hzbet / 2) * (hzbet / 2) + (1 / o->hy[jj]) * (1 / o->hy[jj]));
#pragma omp critical
        {
          cflx = fmax(cflx, lmx); cflz = fmax(cflz, lmz); cfly = fmax(cfly, c0); cflT = fmax(cflT, cT);
        }
      }
      if (do_mass) {
#pragma omp atomic
        rhom[jj] += rsum;
      }
      cplx *so[12];
      for (int f = 0; f < nout; f++) so[f] = spec + (size_t)f * nkx;
      for (int f = 0; f < 10; f += 2) xfwd2(o, q[f], q[f + 1], so[f], so[f + 1], buf, fo);
      if (o->scalar) xfwd2(o, q[10], q[11], so[10], so[11], buf, fo);  /* (DT, DZ) */
      else xfwd2(o, q[10], NULL, so[10], NULL, buf, fo);
      for (int f = 0; f < nout; f++) memcpy(o->ln[f] + (size_t)L * nkx, so[f], sizeof(cplx) * nkx);
    }
    free(ph); free(out); free(buf); free(fo); free(spec);
  }
  cflout[0] = cflx; cflout[1] = cfly; cflout[2] = cflz; cflout[3] = cflT;
  if (do_st) {
    static const int dst[9] = {LMO_S_RUU, LMO_S_RUV, LMO_S_RUW, LMO_S_RVV, LMO_S_RVW,
                               LMO_S_RWW, LMO_S_RHOM, LMO_S_MUM, LMO_S_NUM};
    for (size_t L = 0; L < nlines; L++) {
      int jj = (int)(L / mgalz);
      for (int q = 0; q < 9; q++) o->st[(size_t)dst[q] * my + jj] += lst[L * 9 + q];
    }
    free(lst);
  }
}

/* foup2: cross.f:1282-1430 */
static void foup2(lmo *o, int rk, double dtxi, double dtgamma, double dtbeta, int do_cfl, int do_diag,
                  cplx *in8[18], cplx *out11[12]) {
  const int nin = (o->scalar ? 12 : 8) + (o->vs ? 6 : 0), nout = o->scalar ? 12 : 11;
  int nkx = o->nkx, mgalz = o->mgalz;
#pragma omp parallel num_threads(o->nthreads)
  {
    cplx *buf = malloc(sizeof(cplx) * mgalz), *out = malloc(sizeof(cplx) * mgalz);
#pragma omp for collapse(2) schedule(static)
    for (int f = 0; f < nin; f++)
      for (int i = 0; i < nkx; i++)
        if (!skip_unit(o, (long)f * nkx + i)) zinv_plane(o, i, in8[f], o->ln[f], buf, out);
    free(buf); free(out);
  }
  double cfl[4];
  double *rhom = xcalloc(o->my, 8);
  phys2(o, rk, dtxi, dtgamma, dtbeta, do_cfl, do_diag, cfl, rhom);
#pragma omp parallel num_threads(o->nthreads)
  {
    cplx *buf = malloc(sizeof(cplx) * mgalz), *out = malloc(sizeof(cplx) * mgalz);
#pragma omp for collapse(2) schedule(static)
    for (int f = 0; f < nout; f++)
      for (int i = 0; i < nkx; i++)
        if (!skip_unit(o, (long)f * nkx + i)) zfwd_plane(o, i, o->ln[f], out11[f], buf, out);
    free(buf); free(out);
  }
  if (do_diag) {
    /* momentum thickness: cross.f:1416-1429 (u00 = out11[0] mode 00) */
    const cplx *u = out11[0];
    int my = o->my;
    double dm = 0.0;
    for (int j = 1; j <= my - 2; j++) {
      double a = creal(u[j + 1]), b = creal(u[j - 1]);
      dm += o->trp[j] * (a * a + b * b);
    }
    {
      double a = creal(u[1]), b = creal(u[0]), c = creal(u[my - 1]), d = creal(u[my - 2]);
      dm += o->trp[0] * (a * a + b * b) + o->trp[my - 1] * (c * c + d * d);
    }
    double du = creal(u[my - 1]) - creal(u[0]);
    o->diag[2] = 0.25 * (o->y[my - 1] - o->y[0]) - dm / (du * du);
    /* masst: escru.f:372-376 with one accumulation (plane mean of 1/T) */
    double fac = 1.0 / ((double)o->mgalx * o->mgalz), mt = 0.0;
    for (int j = 0; j < my; j++) mt += fac * rhom[j] * o->hy[j];
    o->diag[6] = mt;
  }
  free(rhom);
  if (do_cfl) { /* cross.f:1778-1826, single compute rank */
    double hxalp = o->alp * (o->mgalx - 1) / M_PI, hzbet = o->bet * (o->mgalz - 1) / M_PI;
    double cflx = cfl[0] * hxalp * 0.5, cflz = cfl[2] * hzbet * 0.5;
    double reig = cflx + cfl[1] + cflz + cfl[3];
    o->dtr = (double)(float)(o->cfl / reig); /* dtr is real*4 */
  }
}

/* ------------------------------------------------------------------ */
/* Statistics: addstats1 (cross.f:1981-2064), addstats2                */
/* (cross.f:2070-2290).  Weights: kx plane 0 once, the others twice    */
/* (the conjugate half of the x spectrum).                             */
/* ------------------------------------------------------------------ */
static inline double cabs2(cplx c) { return creal(c) * creal(c) + cimag(c) * cimag(c); }
static inline size_t spidx(const lmo *o, int i, int var, int iy, int k) {
  return (((size_t)i * 12 + var) * o->nsp + iy) * (o->nz1 + 1) + k;
}
/* |kz| index of kz index kk (icx, main.f:769-782) */
static inline int icx(const lmo *o, int kk) { return kk <= o->nz1 ? kk : o->mz - kk; }

static void addstats1(lmo *o, const cplx *ru, const cplx *rv, const cplx *rw, const cplx *T) {
  int my = o->my, mz = o->mz;
  double *Tp = o->st + (size_t)LMO_S_TP * my;
  for (int i = 0; i < o->nkx; i++) {
    double f = i == 0 ? 1.0 : 2.0;
    for (int iy = 0; iy < o->nsp; iy++) { /* cross.f:2005-2031 */
      int j = o->jsp[iy];
      for (int kk = 0; kk < mz; kk++) {
        int k = icx(o, kk);
        size_t b = SIDX(o, i, kk, j);
        o->sp[spidx(o, i, 8, iy, k)] += f * cabs2(ru[b]);
        o->sp[spidx(o, i, 9, iy, k)] += f * cabs2(rv[b]);
        o->sp[spidx(o, i, 10, iy, k)] += f * cabs2(rw[b]);
        o->sp[spidx(o, i, 11, iy, k)] += f * cabs2(T[b]);
      }
    }
    for (int kk = 0; kk < mz; kk++) /* cross.f:2034-2046 */
      for (int j = 0; j < my; j++) Tp[j] += f * cabs2(T[SIDX(o, i, kk, j)]);
  }
  for (int j = 0; j < my; j++) { /* cross.f:2050-2058 */
    o->st[(size_t)LMO_S_RUM * my + j] += creal(ru[j]);
    o->st[(size_t)LMO_S_RVM * my + j] += creal(rv[j]);
    o->st[(size_t)LMO_S_RWM * my + j] += creal(rw[j]);
    o->st[(size_t)LMO_S_TM * my + j] += creal(T[j]);
  }
}

static void addstats2(lmo *o, const cplx *u1, const cplx *u2, const cplx *u3) {
  int my = o->my, mz = o->mz, nkx = o->nkx;
  size_t ns = (size_t)o->nmode * my;
  /* du/dy, dv/dy, dw/dy (cross.f:749-750 and 2152) */
  cplx *du = xcalloc(ns, sizeof(cplx)), *dv = xcalloc(ns, sizeof(cplx)), *dw = xcalloc(ns, sizeof(cplx));
#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 4 * my);
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      size_t b = (size_t)m * my;
      deryr2_c(o, u1 + b, du + b, s, s + my, s + 2 * my, s + 3 * my);
      deryr2_c(o, u2 + b, dv + b, s, s + my, s + 2 * my, s + 3 * my);
      deryr2_c(o, u3 + b, dw + b, s, s + my, s + 2 * my, s + 3 * my);
    }
    free(s);
  }
  double *P[11];
  for (int q = 0; q < 11; q++) P[q] = o->st + (size_t)(LMO_S_UP + q) * my;
  double *thep = o->st + (size_t)LMO_S_THEP * my, *theup = o->st + (size_t)LMO_S_THEUP * my;
  for (int q = 0; q < 9; q++) o->uner[q] = 0.0; /* cross.f:801-803 */
  for (int i = 0; i < nkx; i++) {
    double f = i == 0 ? 1.0 : 2.0, a = o->kxv[i];
    for (int kk = 0; kk < mz; kk++) {
      double bz = o->kzv[kk];
      for (int j = 0; j < my; j++) {
        size_t b = SIDX(o, i, kk, j);
        cplx u = u1[b], v = u2[b], w = u3[b];
        cplx o1 = dw[b] - I * bz * v, o2 = I * bz * u - I * a * w, o3 = I * a * v - du[b]; /* cross.f:755-766 */
        double e[9];
        e[0] = f * cabs2(u); e[1] = f * cabs2(v); e[2] = f * cabs2(w);       /* cross.f:2153-2182 */
        e[3] = f * creal(u * conj(v)); e[4] = f * creal(u * conj(w));
        e[5] = f * creal(w * conj(v));
        e[6] = f * cabs2(o1); e[7] = f * cabs2(o2); e[8] = f * cabs2(o3);
        for (int q = 0; q < 9; q++) P[q][j] += e[q];
        cplx cc = I * a * u + dv[b] + I * bz * w; /* cross.f:2184-2188 */
        thep[j] += f * cabs2(cc);
        theup[j] += f * creal(cc * conj(v));
        double aa = (a * a + bz * bz) * (cabs2(u) + cabs2(v) + cabs2(w)) + cabs2(dv[b]); /* cross.f:2190-2203 */
        cplx c1 = o1 + I * bz * v, c3 = o3 - I * a * v;
        aa += cabs2(c1) + cabs2(c3);
        P[10][j] += f * aa;
        for (int q = 0; q < 9; q++) o->uner[q] += e[q] * o->hy[j]; /* cross.f:2207-2210 */
      }
    }
    for (int iy = 0; iy < o->nsp; iy++) { /* cross.f:2100-2147 */
      int j = o->jsp[iy];
      for (int kk = 0; kk < mz; kk++) {
        int k = icx(o, kk);
        double bz = o->kzv[kk];
        size_t b = SIDX(o, i, kk, j);
        cplx u = u1[b], v = u2[b], w = u3[b];
        cplx o1 = dw[b] - I * bz * v, o2 = I * bz * u - I * a * w, o3 = I * a * v - du[b];
        cplx uv = u * conj(v);
        double c[8] = {cabs2(u), cabs2(v), cabs2(w), creal(uv), cimag(uv), cabs2(o1), cabs2(o2), cabs2(o3)};
        for (int q = 0; q < 8; q++) o->sp[spidx(o, i, q, iy, k)] += f * c[q];
      }
    }
  }
  for (int j = 0; j < my; j++) { /* cross.f:2279-2289, kx = kz = 0 */
    cplx o1 = dw[j], o3 = -du[j];
    o->st[(size_t)LMO_S_UM * my + j] += creal(u1[j]);
    o->st[(size_t)LMO_S_VM * my + j] += creal(u2[j]);
    o->st[(size_t)LMO_S_WM * my + j] += creal(u3[j]);
    o->st[(size_t)LMO_S_W1M * my + j] += creal(o1);
    o->st[(size_t)LMO_S_W2M * my + j] += 0.0;
    o->st[(size_t)LMO_S_W3M * my + j] += creal(o3);
    o->st[(size_t)LMO_S_THEM * my + j] += creal(dv[j]);
  }
  free(du); free(dv); free(dw);
}

/* ------------------------------------------------------------------ */
/* Variable viscosity (extension): the spectral inputs of the strain   */
/* rates.  In physical space d(u_i)/dx_j = T d(rho u_i)/dx_j +         */
/* rho u_i dT/dx_j, so S_ij needs d(rho u_i)/dx_j only in the sums     */
/* d(rho u_i)/dx_j + d(rho u_j)/dx_i: g[0..2] the diagonal ones        */
/* (halved), g[3..5] the pairs 12, 13, 23.  y derivatives by deryr2    */
/* (cfdiff.f:518-601), as every first y derivative of the substep.     */
/* ------------------------------------------------------------------ */
static void strain_inputs(lmo *o, const cplx *ru, const cplx *rv, const cplx *rw) {
  int my = o->my, mz = o->mz;
#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 4 * my);
    cplx *dy = malloc(sizeof(cplx) * 3 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      if (skip_unit(o, m)) continue;
      double kx = o->kxv[m / mz], kz = o->kzv[m % mz];
      size_t b = (size_t)m * my;
      deryr2_c(o, ru + b, dy, w1, w2, tt1, tt2);
      deryr2_c(o, rv + b, dy + my, w1, w2, tt1, tt2);
      deryr2_c(o, rw + b, dy + 2 * my, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        o->w_g[0][b + j] = I * kx * ru[b + j];
        o->w_g[1][b + j] = dy[my + j];
        o->w_g[2][b + j] = I * kz * rw[b + j];
        o->w_g[3][b + j] = dy[j] + I * kx * rv[b + j];
        o->w_g[4][b + j] = I * kz * ru[b + j] + I * kx * rw[b + j];
        o->w_g[5][b + j] = I * kz * rv[b + j] + dy[2 * my + j];
      }
    }
    free(s); free(dy);
  }
}

/* ------------------------------------------------------------------ */
/* One RK3 substep: cross.f:307-1141                                   */
/* ------------------------------------------------------------------ */
static void substep(lmo *o, int r /*0..2*/, int ihist) {
  int my = o->my, nkx = o->nkx, mz = o->mz;
  double dtxi = o->Deltat * o->xi[r], dtgamma = o->Deltat * o->gama[r], dtbeta = o->Deltat * o->beta[r];
  double ire = o->ire;
  /* BCs: cross.f:315-349 */
  for (int m = 0; m < o->nmode; m++) {
    cplx *vv = o->vor + (size_t)m * my, *pp = o->phi + (size_t)m * my, *ss = o->scal + (size_t)m * my;
    vv[0] = vv[1];
    vv[my - 1] = vv[my - 2];
    pp[0] = 0; pp[my - 1] = 0;
    ss[0] = 0; ss[my - 1] = 0;
  }
  o->scal[0] = 1.0 / o->rhobot;
  o->scal[my - 1] = 1.0 / o->rhotop;
  if (o->scalar) { /* Z: zero at the walls, its mean held at the wall values */
    for (int m = 0; m < o->nmode; m++) {
      cplx *zz = o->zsc + (size_t)m * my;
      zz[0] = 0; zz[my - 1] = 0;
    }
    o->zsc[0] = o->zbot;
    o->zsc[my - 1] = o->ztop;
  }

  cplx *mxw = o->w_mx, *myw = o->w_my, *mzw = o->w_mz, *nxw = o->w_nx, *nyw = o->w_ny, *nzw = o->w_nz;
  cplx *t12 = o->w_t12, *t13 = o->w_t13, *t23 = o->w_t23, *drho = o->w_drho, *chwk = o->w_chwk, *chwk2 = o->w_chwk2;

#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 20 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my, *sc = s + 4 * my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      if (skip_unit(o, m)) continue;
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k], rK = kx * kx + kz * kz;
      size_t b = (size_t)m * my;
      /* save vor and psi: cross.f:353-360 */
      for (int j = 0; j < my; j++) { nxw[b + j] = o->vor[b + j]; nyw[b + j] = o->psi[b + j]; }
      /* (1) Lapvdvhom: cross.f:365-372 */
      lapvdvhom_c(o, o->phi + b, myw + b, nzw + b, rK, sc);
      /* (2) mx, mz: cross.f:395-407 ; tempa=i kx/k2, tempb=i kz/k2 (cross.f:133-154) */
      cplx ta = 0, tb = 0;
      if (rK != 0.0) { ta = I * kx / rK; tb = I * kz / rK; }
      for (int j = 0; j < my; j++) {
        mxw[b + j] = nzw[b + j] * ta - nxw[b + j] * tb;
        mzw[b + j] = nzw[b + j] * tb + nxw[b + j] * ta;
      }
      /* drho = scal: cross.f:410-416 ; xi-update: cross.f:420-430 */
      for (int j = 0; j < my; j++) {
        drho[b + j] = o->scal[b + j];
        o->vor[b + j] = o->vor[b + j] + o->ten12p[b + j] * dtxi;
        o->phi[b + j] = o->phi[b + j] + o->ten13p[b + j] * dtxi;
      }
      /* d(psi)/dy: cross.f:434-437 */
      deryr2_c(o, nyw + b, t23 + b, w1, w2, tt1, tt2);
      /* rho u_i: cross.f:463-482 */
      for (int j = 0; j < my; j++) {
        mxw[b + j] = mxw[b + j] + I * kx * nyw[b + j];
        mzw[b + j] = mzw[b + j] + I * kz * nyw[b + j];
        myw[b + j] = myw[b + j] + t23[b + j];
      }
      /* T derivatives: cross.f:521-554 */
      deryr2_c(o, drho + b, t13 + b, w1, w2, tt1, tt2);
      deryyr2_c(o, drho + b, nyw + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        nyw[b + j] = nyw[b + j] - rK * drho[b + j];
        t23[b + j] = I * kz * drho[b + j];
        t12[b + j] = I * kx * drho[b + j];
      }
      if (o->scalar) { /* the same derivatives of Z */
        const cplx *z = o->zsc + b;
        deryr2_c(o, z, o->w_zy + b, w1, w2, tt1, tt2);
        deryyr2_c(o, z, o->w_zlap + b, w1, w2, tt1, tt2);
        for (int j = 0; j < my; j++) {
          o->w_zlap[b + j] = o->w_zlap[b + j] - rK * z[j];
          o->w_zx[b + j] = I * kx * z[j];
          o->w_zz[b + j] = I * kz * z[j];
        }
      }
    }
    free(s);
  }
  /* 00 modes into rho u_i, then xi-update of u00/w00: cross.f:486-499 */
  for (int j = 0; j < my; j++) {
    mxw[j] = o->u00wk[j];
    myw[j] = o->v00wk[j];
    mzw[j] = o->w00wk[j];
  }
  for (int j = 1; j < my - 1; j++) {
    o->u00wk[j] += dtxi * o->rf0u[j];
    o->w00wk[j] += dtxi * o->rf0w[j];
  }
  if (o->vs) strain_inputs(o, mxw, myw, mzw);
  const int do_st = o->istati && r == 0 && o->st;
  if (do_st) addstats1(o, mxw, myw, mzw, drho); /* cross.f:578-585 */
  /* (5) foup2 */
  int do_cfl = (r == 0 && o->icfl == 1 && o->dtmode == 0);
  cplx *in8[18] = {mxw, myw, mzw, nyw, t12, t13, t23, drho, o->w_zlap, o->w_zx, o->w_zy, o->w_zz};
  if (o->vs) {
    const int vb = o->scalar ? 12 : 8;
    for (int f = 0; f < 6; f++) in8[vb + f] = o->w_g[f];
  }
  cplx *out11[12] = {mxw, myw, mzw, nxw, nyw, nzw, t12, t13, t23, drho, chwk2, o->w_dz};
  foup2(o, r, dtxi, dtgamma, dtbeta, do_cfl, ihist && r == 0, in8, out11);
  if (do_st) { /* cross.f:796-812 (u, v, w are not changed in between) */
    o->nacum++;
    o->nacumsp++;
    addstats2(o, mxw, myw, mzw);
  }

#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 20 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      if (skip_unit(o, m)) continue;
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k];
      size_t b = (size_t)m * my;
      /* (6a) T update: cross.f:619-627 */
      for (int j = 0; j < my; j++) o->scal[b + j] = o->scal[b + j] + chwk2[b + j];
      if (o->scalar)
        for (int j = 0; j < my; j++) o->zsc[b + j] = o->zsc[b + j] + o->w_dz[b + j];
      /* (6b) Nx, Ny, Nz: cross.f:652-682 */
      deryr2_c(o, nyw + b, nyw + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) nyw[b + j] = -I * kx * t12[b + j] - nyw[b + j] - I * kz * t23[b + j];
    }
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      if (skip_unit(o, m)) continue;
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k];
      size_t b = (size_t)m * my;
      deryr2_c(o, t12 + b, t12 + b, w1, w2, tt1, tt2);
      deryr2_c(o, t23 + b, t23 + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        nxw[b + j] = -I * kx * nxw[b + j] - t12[b + j] - I * kz * t13[b + j];
        nzw[b + j] = -I * kx * t13[b + j] - t23[b + j] - I * kz * nzw[b + j];
      }
    }
    free(s);
  }
  /* 00 modes: cross.f:686-722 */
  {
    double *dudy = xcalloc(my, 8);
    for (int j = 0; j < my; j++) { o->rf0u[j] = creal(mxw[j]); o->rf0w[j] = creal(mzw[j]); }
    if (r == 2 && ihist) {
      lmo_deryr(o, o->rf0u, dudy);
      double dw = 0.0;
      for (int j = 0; j < my; j++) dw = fmax(fabs(dudy[j]), dw);
      o->diag[3] = 1.0 / dw;
      o->diag[4] = o->diag[3] * o->Re;
    }
    lmo_deryyr(o, o->rf0u, o->rf0u);
    lmo_deryyr(o, o->rf0w, o->rf0w);
    for (int j = 0; j < my; j++) {
      o->rf0u[j] = -creal(t12[j]) + ire * o->rf0u[j];
      o->rf0w[j] = -creal(t23[j]) + ire * o->rf0w[j];
    }
    if (r == 2 && ihist) {
      double hu = 0, hw = 0;
      for (int j = 0; j < my; j++) { hu += o->rf0u[j] * o->hy[j]; hw += o->rf0w[j] * o->hy[j]; }
      o->diag[10] = 0.25 * hu;
      o->diag[11] = 0.25 * hw;
    }
    free(dudy);
  }
#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 24 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my, *sc = s + 4 * my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      if (skip_unit(o, m)) continue;
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k], rK = kx * kx + kz * kz;
      size_t b = (size_t)m * my;
      /* vorticities: cross.f:748-767 */
      deryr2_c(o, mxw + b, t12 + b, w1, w2, tt1, tt2);
      deryr2_c(o, mzw + b, t23 + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        t23[b + j] = t23[b + j] - I * kz * myw[b + j];
        t13[b + j] = I * kz * mxw[b + j] - I * kx * mzw[b + j];
        t12[b + j] = I * kx * myw[b + j] - t12[b + j];
      }
      /* Laplacians: cross.f:821-857 */
      deryyr2_c(o, t13 + b, chwk + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) t13[b + j] = chwk[b + j] - rK * t13[b + j];
      for (int j = 0; j < my; j++) t23[b + j] = I * kz * t23[b + j] - I * kx * t12[b + j];
      deryyr2_c(o, t23 + b, chwk + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) t23[b + j] = chwk[b + j] - rK * t23[b + j];
      /* RHS(Omega_y), RHS(phi): cross.f:885-921 */
      for (int j = 0; j < my; j++) t12[b + j] = I * kz * nxw[b + j] - I * kx * nzw[b + j] + ire * t13[b + j];
      for (int j = 0; j < my; j++) nxw[b + j] = I * kx * nxw[b + j] + I * kz * nzw[b + j];
      deryr2_c(o, nxw + b, nxw + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) t13[b + j] = -rK * nyw[b + j] - nxw[b + j] - ire * t23[b + j];
      /* RK3 update: cross.f:966-981 */
      for (int j = 0; j < my; j++) {
        o->vor[b + j] = o->vor[b + j] + dtgamma * t12[b + j];
        o->phi[b + j] = o->phi[b + j] + dtgamma * t13[b + j];
        o->ten12p[b + j] = t12[b + j];
        o->ten13p[b + j] = t13[b + j];
      }
      /* psi(n+1): cross.f:1092-1104 */
      solvepsi_c(o, drho + b, o->psi + b, chwk + b, rK, sc);
    }
    free(s);
  }
  /* 00 modes: cross.f:1006-1074 */
  {
    for (int j = 1; j < my - 1; j++) {
      o->u00wk[j] += dtgamma * o->rf0u[j];
      o->w00wk[j] += dtgamma * o->rf0w[j];
    }
    double mu = 0, mv = 0, mw = 0;
    for (int j = 0; j < my; j++) {
      mu += o->u00wk[j] * o->hy[j];
      mv += o->v00wk[j] * o->hy[j];
      mw += o->w00wk[j] * o->hy[j];
    }
    o->diag[7] = mu; o->diag[8] = mv; o->diag[9] = mw;
    double *d00 = xcalloc(my, 8);
    for (int j = 0; j < my; j++) d00[j] = creal(drho[j]);
    lmo_inty8(o, d00, o->rf0v);
    double trapz = -o->rf0v[my - 1];
    o->diag[5] = trapz;
    for (int j = 0; j < my; j++) o->v00wk[j] = o->rf0v[j] + trapz / (1.0 + sqrt(o->rhotop / o->rhobot));
    free(d00);
  }
  (void)nkx;
}

/* ------------------------------------------------------------------ */
/* The 2014 variant, trunk/lomacte/src/cross.f (below "lomacte/"):     */
/* spectral T with its own RK3 RHS, d(rho) from a transform round trip */
/* of T and Delta T, psi by the Dirichlet Poisson solver and rho v00   */
/* by a cumulative trapezoid.                                          */
/* ------------------------------------------------------------------ */

/* phys2 of lomacte/cross.f:1268-1578 on all lines: u_i, RHS(T) with
 * Pe = Re (lomacte/cross.f:1301), the six products; CFL maxima. */
static void phys2_14(lmo *o, int do_cfl, int do_mass, double *cflout /*3*/, double *rhom) {
  int mgalx = o->mgalx, mgalz = o->mgalz, my = o->my, nkx = o->nkx;
  size_t nlines = (size_t)mgalz * my;
  double cflx = 0, cfly = 0, cflz = 0;
  const double pe = o->Re;
#pragma omp parallel num_threads(o->nthreads)
  {
    double *ph = malloc(sizeof(double) * mgalx * 8), *out = malloc(sizeof(double) * mgalx * 10);
    cplx *buf = malloc(sizeof(cplx) * mgalx), *fo = malloc(sizeof(cplx) * mgalx);
    cplx *spec = malloc(sizeof(cplx) * nkx * 10);
#pragma omp for schedule(static)
    for (long L = 0; L < (long)nlines; L++) {
      int jj = (int)(L / mgalz);
      cplx *sp[8];
      double *p[8];
      for (int f = 0; f < 8; f++) { sp[f] = o->ln[f] + (size_t)L * nkx; p[f] = ph + (size_t)f * mgalx; }
      for (int f = 0; f < 8; f += 2) xinv2(o, sp[f], sp[f + 1], p[f], p[f + 1], buf, fo);
      double *ru = p[0], *rv = p[1], *rw = p[2], *lapT = p[3], *tx = p[4], *ty = p[5], *tz = p[6], *T = p[7];
      double *q[10];
      for (int f = 0; f < 10; f++) q[f] = out + (size_t)f * mgalx;
      double lmx = 0, lmy = 0, lmz = 0, rsum = 0;
      for (int x = 0; x < mgalx; x++) {
        double u = ru[x] * T[x], v = rv[x] * T[x], w = rw[x] * T[x]; /* lomacte/cross.f:1440-1449 */
        q[9][x] = -u * tx[x] - v * ty[x] - w * tz[x] + (1 / pe) * T[x] * lapT[x]; /* :1452-1456 */
        q[0][x] = u; q[1][x] = v; q[2][x] = w;
        q[3][x] = ru[x] * u; q[4][x] = rv[x] * v; q[5][x] = rw[x] * w; /* :1465-1469 */
        q[6][x] = ru[x] * v; q[7][x] = ru[x] * w; q[8][x] = rv[x] * w; /* :1472-1476 */
        if (do_cfl) { lmx = fmax(lmx, fabs(u)); lmy = fmax(lmy, fabs(v)); lmz = fmax(lmz, fabs(w)); }
        if (do_mass) rsum += 1.0 / T[x];
      }
      if (do_cfl) { /* :1492-1503 */
#pragma omp critical
        { cflx = fmax(cflx, lmx); cflz = fmax(cflz, lmz); cfly = fmax(cfly, lmy / o->hy[jj]); }
      }
      if (do_mass) {
#pragma omp atomic
        rhom[jj] += rsum;
      }
      cplx *so[10];
      for (int f = 0; f < 10; f++) so[f] = spec + (size_t)f * nkx;
      for (int f = 0; f < 10; f += 2) xfwd2(o, q[f], q[f + 1], so[f], so[f + 1], buf, fo);
      for (int f = 0; f < 10; f++) memcpy(o->ln[f] + (size_t)L * nkx, so[f], sizeof(cplx) * nkx);
    }
    free(ph); free(out); free(buf); free(fo); free(spec);
  }
  cflout[0] = cflx; cflout[1] = cfly; cflout[2] = cflz;
}

/* foup2 of lomacte/cross.f:1109-1258 and the Deltat of phys2
 * (lomacte/cross.f:1547-1574): applied at once, in the first substep. */
static void foup2_14(lmo *o, int do_cfl, int do_diag, cplx *in8[8], cplx *out10[10]) {
  int nkx = o->nkx, mgalz = o->mgalz, my = o->my;
#pragma omp parallel num_threads(o->nthreads)
  {
    cplx *buf = malloc(sizeof(cplx) * mgalz), *out = malloc(sizeof(cplx) * mgalz);
#pragma omp for collapse(2) schedule(static)
    for (int f = 0; f < 8; f++)
      for (int i = 0; i < nkx; i++) zinv_plane(o, i, in8[f], o->ln[f], buf, out);
    free(buf); free(out);
  }
  double cfl[3];
  double *rhom = xcalloc(my, 8);
  phys2_14(o, do_cfl, do_diag, cfl, rhom);
#pragma omp parallel num_threads(o->nthreads)
  {
    cplx *buf = malloc(sizeof(cplx) * mgalz), *out = malloc(sizeof(cplx) * mgalz);
#pragma omp for collapse(2) schedule(static)
    for (int f = 0; f < 10; f++)
      for (int i = 0; i < nkx; i++) zfwd_plane(o, i, o->ln[f], out10[f], buf, out);
    free(buf); free(out);
  }
  if (do_diag) { /* dm: lomacte/cross.f:1240-1256; masst as in the 2017 path */
    const cplx *u = out10[0];
    double dm = 0.0;
    for (int j = 1; j <= my - 2; j++) {
      double a = creal(u[j + 1]), b = creal(u[j - 1]);
      dm += o->trp[j] * (a * a + b * b);
    }
    {
      double a = creal(u[1]), b = creal(u[0]), c = creal(u[my - 1]), d = creal(u[my - 2]);
      dm += o->trp[0] * (a * a + b * b) + o->trp[my - 1] * (c * c + d * d);
    }
    double du = creal(u[my - 1]) - creal(u[0]);
    o->diag[2] = 0.25 * (o->y[my - 1] - o->y[0]) - dm / (du * du);
    double fac = 1.0 / ((double)o->mgalx * o->mgalz), mt = 0.0;
    for (int j = 0; j < my; j++) mt += fac * rhom[j] * o->hy[j];
    o->diag[6] = mt;
  }
  free(rhom);
  if (do_cfl) {
    double hxalp = o->alp * (o->mgalx - 1) / M_PI, hzbet = o->bet * (o->mgalz - 1) / M_PI;
    double hmin = o->hy[0];
    for (int j = 1; j < my; j++) hmin = fmin(hmin, o->hy[j]);
    double hyy = 1.0 / hmin;
    hyy = 2.0 / o->Re * pow(fmax(hyy, fmax(hxalp / 2, hzbet / 2)), 2); /* viscous limit */
    double c0 = fmax(cfl[0] * hxalp, fmax(cfl[1], cfl[2] * hzbet));
    double reig = fmax(c0, hyy);
    o->Deltat = (double)(float)(o->cfl / reig); /* Deltat is real*4 */
  }
}

/* tauij2 / tensor2 of lomacte/cross.f:1738-1908: d(rho) = 1/(T + Delta T)
 * - 1/T = -Delta T / (T (T + Delta T)) in physical space. */
static void tauij2_14(lmo *o, cplx *T, cplx *dT) {
  int nkx = o->nkx, mgalz = o->mgalz, mgalx = o->mgalx, my = o->my;
  cplx *in2[2] = {T, dT};
#pragma omp parallel num_threads(o->nthreads)
  {
    cplx *buf = malloc(sizeof(cplx) * mgalz), *out = malloc(sizeof(cplx) * mgalz);
#pragma omp for collapse(2) schedule(static)
    for (int f = 0; f < 2; f++)
      for (int i = 0; i < nkx; i++) zinv_plane(o, i, in2[f], o->ln[f], buf, out);
    free(buf); free(out);
  }
  size_t nlines = (size_t)mgalz * my;
#pragma omp parallel num_threads(o->nthreads)
  {
    double *a = malloc(sizeof(double) * mgalx * 2), *b = a + mgalx;
    cplx *buf = malloc(sizeof(cplx) * mgalx), *fo = malloc(sizeof(cplx) * mgalx);
#pragma omp for schedule(static)
    for (long L = 0; L < (long)nlines; L++) {
      cplx *s0 = o->ln[0] + (size_t)L * nkx, *s1 = o->ln[1] + (size_t)L * nkx;
      xinv2(o, s0, s1, a, b, buf, fo);
      for (int x = 0; x < mgalx; x++) a[x] = -b[x] / (a[x] * (a[x] + b[x])); /* :1881 */
      xfwd2(o, a, NULL, s0, NULL, buf, fo);
    }
    free(a); free(buf); free(fo);
  }
#pragma omp parallel num_threads(o->nthreads)
  {
    cplx *buf = malloc(sizeof(cplx) * mgalz), *out = malloc(sizeof(cplx) * mgalz);
#pragma omp for schedule(static)
    for (int i = 0; i < nkx; i++) zfwd_plane(o, i, o->ln[0], T, buf, out);
    free(buf); free(out);
  }
}

/* One RK3 substep of the 2014 variant: lomacte/cross.f:286-989. */
static void substep14(lmo *o, int r, int ihist) {
  int my = o->my, mz = o->mz;
  double dtxi = o->Deltat * o->xi[r];
  double ire = o->ire;
  cplx *mxw = o->w_mx, *myw = o->w_my, *mzw = o->w_mz, *nxw = o->w_nx, *nyw = o->w_ny, *nzw = o->w_nz;
  cplx *t12 = o->w_t12, *t13 = o->w_t13, *t23 = o->w_t23, *drho = o->w_drho, *chwk = o->w_chwk, *chwk2 = o->w_chwk2;
#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 20 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my, *sc = s + 4 * my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k], rK = kx * kx + kz * kz;
      size_t b = (size_t)m * my;
      /* work copies and BCs: lomacte/cross.f:293-320 */
      for (int j = 0; j < my; j++) { nxw[b + j] = o->vor[b + j]; nyw[b + j] = o->psi[b + j]; }
      nxw[b + 1] = nxw[b + 2];
      nxw[b + 0] = nxw[b + 2];
      nxw[b + my - 2] = nxw[b + my - 3];
      nxw[b + my - 1] = nxw[b + my - 2];
      o->phi[b] = 0;
      o->phi[b + my - 1] = 0;
      /* (1) Lapvdvhom: :322-329 */
      lapvdvhom_c(o, o->phi + b, myw + b, nzw + b, rK, sc);
      /* (2) mx, mz: :353-366 */
      cplx ta = 0, tb = 0;
      if (rK != 0.0) { ta = I * kx / rK; tb = I * kz / rK; }
      for (int j = 0; j < my; j++) {
        mxw[b + j] = nzw[b + j] * ta - nxw[b + j] * tb;
        mzw[b + j] = nzw[b + j] * tb + nxw[b + j] * ta;
      }
      /* T saved, xi-updates (T too, from its spectral RHS): :368-396 */
      for (int j = 0; j < my; j++) {
        drho[b + j] = o->scal[b + j];
        o->vor[b + j] = o->vor[b + j] + o->ten12p[b + j] * dtxi;
        o->phi[b + j] = o->phi[b + j] + o->ten13p[b + j] * dtxi;
        o->scal[b + j] = o->scal[b + j] + o->rts[b + j] * dtxi;
        chwk2[b + j] = o->rts[b + j] * dtxi;
      }
      /* d(psi)/dy and rho u_i: :400-444 */
      deryr2_c(o, nyw + b, t23 + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        mxw[b + j] = mxw[b + j] + I * kx * nyw[b + j];
        mzw[b + j] = mzw[b + j] + I * kz * nyw[b + j];
        myw[b + j] = myw[b + j] + t23[b + j];
      }
      /* (4) derivatives of the saved T: :486-519 */
      deryr2_c(o, drho + b, t13 + b, w1, w2, tt1, tt2);
      deryyr2_c(o, drho + b, nyw + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        nyw[b + j] = nyw[b + j] - rK * drho[b + j];
        t23[b + j] = I * kz * drho[b + j];
        t12[b + j] = I * kx * drho[b + j];
      }
    }
    free(s);
  }
  /* 00 modes: :447-461 */
  for (int j = 0; j < my; j++) { mxw[j] = o->u00wk[j]; myw[j] = o->v00wk[j]; mzw[j] = o->w00wk[j]; }
  for (int j = 1; j < my - 1; j++) {
    o->u00wk[j] += dtxi * o->rf0u[j];
    o->w00wk[j] += dtxi * o->rf0w[j];
  }
  /* (5) foup2, new Deltat in the first substep of a CFL step: :544-556 */
  int do_cfl = (r == 0 && o->icfl == 1 && o->dtmode == 0);
  cplx *rtn = chwk; /* RHS(T) of this substep */
  cplx *in8[8] = {mxw, myw, mzw, nyw, t12, t13, t23, drho};
  cplx *out10[10] = {mxw, myw, mzw, nxw, nyw, nzw, t12, t13, t23, rtn};
  foup2_14(o, do_cfl, ihist && r == 0, in8, out10);
  if (r == 0) o->diag[1] = o->Deltat;
  double dtgamma = o->Deltat * o->gama[r];
  dtxi = o->Deltat * o->xi[r];
#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 20 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k];
      size_t b = (size_t)m * my;
      /* (6a) T: :563-570 */
      for (int j = 0; j < my; j++) {
        o->scal[b + j] = o->scal[b + j] + dtgamma * rtn[b + j];
        chwk2[b + j] = chwk2[b + j] + dtgamma * rtn[b + j];
        o->rts[b + j] = rtn[b + j];
      }
      /* (6b) N_x, N_y, N_z: :594-625 */
      deryr2_c(o, nyw + b, nyw + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) nyw[b + j] = -I * kx * t12[b + j] - nyw[b + j] - I * kz * t23[b + j];
      deryr2_c(o, t12 + b, t12 + b, w1, w2, tt1, tt2);
      deryr2_c(o, t23 + b, t23 + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        nxw[b + j] = -I * kx * nxw[b + j] - t12[b + j] - I * kz * t13[b + j];
        nzw[b + j] = -I * kx * t13[b + j] - t23[b + j] - I * kz * nzw[b + j];
      }
    }
    free(s);
  }
  /* 00 modes: :628-653 (dw and the hy-weighted H00 as in the 2017 path) */
  {
    double *dudy = xcalloc(my, 8);
    for (int j = 0; j < my; j++) { o->rf0u[j] = creal(mxw[j]); o->rf0w[j] = creal(mzw[j]); }
    if (r == 2 && ihist) {
      lmo_deryr(o, o->rf0u, dudy);
      double dw = 0.0;
      for (int j = 0; j < my; j++) dw = fmax(fabs(dudy[j]), dw);
      o->diag[3] = 1.0 / dw;
      o->diag[4] = o->diag[3] * o->Re;
    }
    lmo_deryyr(o, o->rf0u, o->rf0u);
    lmo_deryyr(o, o->rf0w, o->rf0w);
    for (int j = 0; j < my; j++) {
      o->rf0u[j] = creal(nxw[j]) + ire * o->rf0u[j];
      o->rf0w[j] = creal(nzw[j]) + ire * o->rf0w[j];
    }
    if (r == 2 && ihist) {
      double hu = 0, hw = 0;
      for (int j = 0; j < my; j++) { hu += o->rf0u[j] * o->hy[j]; hw += o->rf0w[j] * o->hy[j]; }
      o->diag[10] = 0.25 * hu;
      o->diag[11] = 0.25 * hw;
    }
    free(dudy);
  }
  /* d(rho) from T and Delta T: :877 */
  tauij2_14(o, drho, chwk2);
  const double den = dtgamma + dtxi;
#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 24 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my, *sc = s + 4 * my;
    cplx *c1 = malloc(sizeof(cplx) * 2 * my), *c2 = c1 + my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k], rK = kx * kx + kz * kz;
      size_t b = (size_t)m * my;
      /* vorticities, Laplacians, RHS(Omega_y), RHS(phi): :656-872 */
      deryr2_c(o, mxw + b, t12 + b, w1, w2, tt1, tt2);
      deryr2_c(o, mzw + b, t23 + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        t23[b + j] = t23[b + j] - I * kz * myw[b + j];
        t13[b + j] = I * kz * mxw[b + j] - I * kx * mzw[b + j];
        t12[b + j] = I * kx * myw[b + j] - t12[b + j];
      }
      deryyr2_c(o, t13 + b, c1, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) t13[b + j] = c1[j] - rK * t13[b + j];
      for (int j = 0; j < my; j++) t23[b + j] = I * kz * t23[b + j] - I * kx * t12[b + j];
      deryyr2_c(o, t23 + b, c1, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) t23[b + j] = c1[j] - rK * t23[b + j];
      for (int j = 0; j < my; j++) t12[b + j] = I * kz * nxw[b + j] - I * kx * nzw[b + j] + ire * t13[b + j];
      for (int j = 0; j < my; j++) nxw[b + j] = I * kx * nxw[b + j] + I * kz * nzw[b + j];
      deryr2_c(o, nxw + b, nxw + b, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) t13[b + j] = -rK * nyw[b + j] - nxw[b + j] - ire * t23[b + j];
      /* (10) RK3 update: :912-928 */
      for (int j = 0; j < my; j++) {
        o->vor[b + j] = o->vor[b + j] + dtgamma * t12[b + j];
        o->phi[b + j] = o->phi[b + j] + dtgamma * t13[b + j];
        o->ten12p[b + j] = t12[b + j];
        o->ten13p[b + j] = t13[b + j];
      }
      /* psi(n+1) = Lapvdvhom(-d(rho)/(dt (gamma + xi))): :974-983 */
      for (int j = 0; j < my; j++) c2[j] = -drho[b + j] / den;
      lapvdvhom_c(o, c2, o->psi + b, c1, rK, sc);
    }
    free(s);
    free(c1);
  }
  /* 00 modes: :950-1002 */
  {
    for (int j = 1; j < my - 1; j++) {
      o->u00wk[j] += dtgamma * o->rf0u[j];
      o->w00wk[j] += dtgamma * o->rf0w[j];
    }
    double mu = 0, mv = 0, mw = 0;
    for (int j = 0; j < my; j++) {
      mu += o->u00wk[j] * o->hy[j];
      mv += o->v00wk[j] * o->hy[j];
      mw += o->w00wk[j] * o->hy[j];
    }
    o->diag[7] = mu; o->diag[8] = mv; o->diag[9] = mw;
    /* cumulative trapezoid of d(rho)00 / (dt (gamma + xi)) */
    o->rf0v[0] = 0.0;
    for (int j = 0; j < my - 1; j++)
      o->rf0v[j + 1] = o->rf0v[j] + 0.5 * (o->y[j + 1] - o->y[j]) * (creal(drho[j + 1]) / den + creal(drho[j]) / den);
    double trapz = o->rf0v[my - 1];
    o->diag[5] = trapz;
    for (int j = 0; j < my; j++) {
      o->rf0v[j] = o->rf0v[j] - o->rhobot * trapz / (o->rhotop + o->rhobot);
      o->v00wk[j] = -o->rf0v[j];
    }
  }
}

/* Time loop body: cross.f:225-1226 (images, .sta/.spe and .cf output are the
 * caller's business); the 2014 variant follows lomacte/cross.f:212-1040,
 * whose Deltat changes inside the first substep of a CFL step. */
int lmo_step(lmo *o, int nsteps) {
  for (int s = 0; s < nsteps; s++) {
    int istep = ++o->istep_total;
    if (o->dtmode == 0 && (istep - 1) % o->ncfl == 0) o->icfl = 1;
    int ihist = 1; /* diagnostics every step */
    o->diag[0] = o->time;
    o->diag[1] = o->Deltat;
    if (o->variant == 1) {
      for (int r = 0; r < 3; r++) substep14(o, r, ihist);
      o->time += o->Deltat;
      o->icfl = 0;
      o->diag[12] = o->Deltat;
      continue;
    }
    for (int r = 0; r < 3; r++) substep(o, r, ihist);
    o->time += o->Deltat;
    if (o->dtmode == 0 && o->icfl == 1) {
      o->icfl = 0;
      o->Deltat = o->dtr;
    }
    o->diag[12] = o->Deltat;
  }
  return 0;
}

/* Physical fields of the current state on chosen y planes: the quantities
 * of tofis_loma's escrphys (trunk/tofis_loma/src/escru.f:11-314, with the
 * y work of uvw.f:7-94), formed from the solver's own rho u_i (Lapvdvhom
 * with the wall conditions of Omega_y and phi, cross.f:315-335, 365-499;
 * T and Z as stored, as tofis_loma reads them):
 * u = T rho u, v, w, T, and the vorticity omega = curl(T rho u) = T C +
 * grad T x rho u with C = curl(rho u) (C_y is Omega_y), then Z with the
 * scalar.  out[p][q][z][x] (x fastest), q = 0..6 (7 with the scalar);
 * jplanes 1-based.  The state is not changed. */
int lmo_physical(const lmo *o, int nplanes, const int *jplanes, double *out) {
  if (!o || nplanes < 0 || (nplanes && (!jplanes || !out)) || o->variant) return -1;
  for (int p = 0; p < nplanes; p++)
    if (jplanes[p] < 1 || jplanes[p] > o->my) return -1;
  const int my = o->my, mz = o->mz, mgalx = o->mgalx, mgalz = o->mgalz, nkx = o->nkx;
  const int nf = o->scalar ? 11 : 10, nq = o->scalar ? 8 : 7;
  const size_t ns = (size_t)o->nmode * my, nl = (size_t)mgalz * my * nkx;
  cplx *f[11], *ln[11];
  for (int q = 0; q < nf; q++) { f[q] = xcalloc(ns, sizeof(cplx)); ln[q] = xcalloc(nl, sizeof(cplx)); }
  /* f: 0 rho u, 1 rho v, 2 rho w, 3 T, 4 dT/dx, 5 dT/dy, 6 dT/dz, 7 C_x, 8 C_y, 9 C_z, 10 Z */
#pragma omp parallel num_threads(o->nthreads)
  {
    double *s = malloc(sizeof(double) * 24 * my);
    cplx *c = malloc(sizeof(cplx) * 6 * my);
    double *w1 = s, *w2 = s + my, *tt1 = s + 2 * my, *tt2 = s + 3 * my, *sc = s + 4 * my;
    cplx *vo = c, *ph = c + my, *mv = c + 2 * my, *dmv = c + 3 * my, *d1 = c + 4 * my, *d2 = c + 5 * my;
#pragma omp for schedule(static)
    for (int m = 0; m < o->nmode; m++) {
      int i = m / mz, k = m % mz;
      double kx = o->kxv[i], kz = o->kzv[k], rK = kx * kx + kz * kz;
      size_t b = (size_t)m * my;
      for (int j = 0; j < my; j++) { vo[j] = o->vor[b + j]; ph[j] = o->phi[b + j]; f[3][b + j] = o->scal[b + j]; }
      vo[0] = vo[1]; vo[my - 1] = vo[my - 2];           /* cross.f:315-327 */
      ph[0] = 0; ph[my - 1] = 0;                        /* cross.f:329-335 */
      lapvdvhom_c(o, ph, mv, dmv, rK, sc);              /* cross.f:365-372 */
      deryr2_c(o, o->psi + b, d1, w1, w2, tt1, tt2);    /* cross.f:434-437 */
      cplx ta = 0, tb = 0;
      if (rK != 0.0) { ta = I * kx / rK; tb = I * kz / rK; }
      for (int j = 0; j < my; j++) {                    /* cross.f:395-407, 463-482 */
        f[0][b + j] = dmv[j] * ta - vo[j] * tb + I * kx * o->psi[b + j];
        f[2][b + j] = dmv[j] * tb + vo[j] * ta + I * kz * o->psi[b + j];
        f[1][b + j] = mv[j] + d1[j];
      }
      if (m == 0)                                        /* cross.f:486-491 */
        for (int j = 0; j < my; j++) { f[0][j] = o->u00wk[j]; f[1][j] = o->v00wk[j]; f[2][j] = o->w00wk[j]; }
      deryr2_c(o, f[3] + b, f[5] + b, w1, w2, tt1, tt2);
      deryr2_c(o, f[0] + b, d1, w1, w2, tt1, tt2);
      deryr2_c(o, f[2] + b, d2, w1, w2, tt1, tt2);
      for (int j = 0; j < my; j++) {
        f[4][b + j] = I * kx * f[3][b + j];
        f[6][b + j] = I * kz * f[3][b + j];
        f[7][b + j] = d2[j] - I * kz * f[1][b + j];
        f[8][b + j] = I * kz * f[0][b + j] - I * kx * f[2][b + j];
        f[9][b + j] = I * kx * f[1][b + j] - d1[j];
      }
      if (o->scalar) {
        for (int j = 0; j < my; j++) f[10][b + j] = o->zsc[b + j];
      }
    }
    free(s); free(c);
  }
#pragma omp parallel num_threads(o->nthreads)
  {
    cplx *buf = malloc(sizeof(cplx) * (mgalz > mgalx ? mgalz : mgalx)), *fo = malloc(sizeof(cplx) * (mgalz > mgalx ? mgalz : mgalx));
#pragma omp for collapse(2) schedule(static)
    for (int q = 0; q < nf; q++)
      for (int i = 0; i < nkx; i++) zinv_plane(o, i, f[q], ln[q], buf, fo);
    free(buf); free(fo);
  }
#pragma omp parallel num_threads(o->nthreads)
  {
    double *ph = malloc(sizeof(double) * mgalx * 12);
    cplx *buf = malloc(sizeof(cplx) * mgalx), *fo = malloc(sizeof(cplx) * mgalx);
#pragma omp for collapse(2) schedule(static)
    for (int p = 0; p < nplanes; p++)
      for (int z = 0; z < mgalz; z++) {
        const size_t L = (size_t)(jplanes[p] - 1) * mgalz + z;
        double *r[12];
        for (int q = 0; q < 12; q++) r[q] = ph + (size_t)q * mgalx;
        for (int q = 0; q < nf; q += 2)
          xinv2(o, ln[q] + L * nkx, q + 1 < nf ? ln[q + 1] + L * nkx : ln[q] + L * nkx, r[q], r[q + 1], buf, fo);
        for (int x = 0; x < mgalx; x++) {
          const double mu = r[0][x], mvv = r[1][x], mw = r[2][x], T = r[3][x];
          const double tx = r[4][x], ty = r[5][x], tz = r[6][x];
          double v[8];
          v[0] = mu * T; v[1] = mvv * T; v[2] = mw * T; v[3] = T;
          v[4] = T * r[7][x] + ty * mw - tz * mvv;
          v[5] = T * r[8][x] + tz * mu - tx * mw;
          v[6] = T * r[9][x] + tx * mvv - ty * mu;
          v[7] = o->scalar ? r[10][x] : 0.0;
          for (int q = 0; q < nq; q++) out[(((size_t)p * nq + q) * mgalz + z) * mgalx + x] = v[q];
        }
      }
    free(ph); free(buf); free(fo);
  }
  for (int q = 0; q < nf; q++) { free(f[q]); free(ln[q]); }
  return 0;
}

int lmo_set_variant(lmo *o, int variant) {
  if (!o || variant < 0 || variant > 1 || (variant && (o->scalar || o->vs))) return -1;
  o->variant = variant;
  return 0;
}

int lmo_set_scalar(lmo *o, int on, double schmidt) {
  if (!o || o->variant || (on && !(schmidt > 0))) return -1;
  size_t ns = (size_t)o->nmode * o->my, np = (size_t)o->mgalz * o->my * o->mgalx;
  o->scalar = on != 0;
  if (!on) return 0;
  o->pez = o->Re * schmidt;
  cplx **b[] = {&o->zsc, &o->w_zlap, &o->w_zx, &o->w_zy, &o->w_zz, &o->w_dz};
  for (size_t i = 0; i < sizeof(b) / sizeof(b[0]); i++)
    if (!*b[i]) *b[i] = xcalloc(ns, sizeof(cplx));
  if (!o->rhsz) o->rhsz = xcalloc(np, 8);
  return 0;
}

int lmo_set_viscosity(lmo *o, int on, double sigma) {
  if (!o || o->variant || (on && !(sigma >= 0.0 && sigma <= 4.0))) return -1;
  o->vs = on != 0;
  o->vsig = on ? sigma : 0.0;
  if (!on) return 0;
  size_t ns = (size_t)o->nmode * o->my, nl = (size_t)o->mgalz * o->my * o->nkx;
  for (int f = 0; f < 6; f++)
    if (!o->w_g[f]) o->w_g[f] = xcalloc(ns, sizeof(cplx));
  for (int f = 12; f < 18; f++)
    if (!o->ln[f]) o->ln[f] = xcalloc(nl, sizeof(cplx));
  return 0;
}

int lmo_set_scalar_state(lmo *o, const double *z) {
  if (!o || !o->scalar || !z) return -1;
  size_t ns = (size_t)o->nmode * o->my;
  memcpy(o->zsc, z, ns * sizeof(cplx));
  memset(o->rhsz, 0, (size_t)o->mgalz * o->my * o->mgalx * 8);
  o->zbot = creal(o->zsc[SIDX(o, 0, 0, 0)]);
  o->ztop = creal(o->zsc[SIDX(o, 0, 0, o->my - 1)]);
  return 0;
}

int lmo_get_scalar_state(const lmo *o, double *z) {
  if (!o || !o->scalar || !z) return -1;
  memcpy(z, o->zsc, (size_t)o->nmode * o->my * sizeof(cplx));
  return 0;
}

int lmo_stats_reset(lmo *o, int nsp, const int *jsp, double sigma) {
  if (!o || nsp < 0 || (nsp && !jsp) || o->variant) return -1;
  for (int i = 0; i < nsp; i++)
    if (jsp[i] < 1 || jsp[i] > o->my) return -1;
  free(o->jsp); free(o->st); free(o->sp);
  o->nsp = nsp;
  o->jsp = xcalloc(nsp, sizeof(int));
  for (int i = 0; i < nsp; i++) o->jsp[i] = jsp[i] - 1;
  o->sigma = sigma;
  o->st = xcalloc((size_t)LMO_NSTAT * o->my, 8);
  o->sp = xcalloc((size_t)o->nkx * 12 * nsp * (o->nz1 + 1), 8);
  memset(o->uner, 0, sizeof(o->uner));
  o->nacum = o->nacumsp = 0;
  return 0;
}

int lmo_stats_step(lmo *o, int nsteps) {
  if (!o || !o->st) return -1;
  o->istati = 1;
  int rc = lmo_step(o, nsteps);
  o->istati = 0;
  return rc;
}

int lmo_stats_read(lmo *o, double *prof, double *spec, double *uner, int *counts, int clear_spectra) {
  if (!o || !o->st) return -1;
  size_t nsp = (size_t)o->nkx * 12 * o->nsp * (o->nz1 + 1);
  if (prof) memcpy(prof, o->st, sizeof(double) * LMO_NSTAT * o->my);
  if (spec) memcpy(spec, o->sp, sizeof(double) * nsp);
  if (uner) memcpy(uner, o->uner, sizeof(o->uner));
  if (counts) { counts[0] = o->nacum; counts[1] = o->nacumsp; }
  if (clear_spectra) { /* escru.f:466-477 */
    memset(o->sp, 0, sizeof(double) * nsp);
    o->nacumsp = 0;
  }
  return 0;
}

/* Timing samples: from now on the parallel loops of a substep visit only
 * the units whose index is phase modulo stride (stride <= 1: all of them).
 * The state is then no longer a solution; for timing only. */
int lmo_set_sample(lmo *o, int stride, int phase) {
  if (stride < 1 || phase < 0 || (stride > 1 && phase >= stride)) return -1;
  o->smp = stride;
  o->smph = phase;
  return 0;
}

/* One substep with RK coefficient r (0..2) on the current state, without
 * the step bookkeeping: used only to time bounded CPU samples. */
int lmo_substep(lmo *o, int r) {
  if (r < 0 || r > 2) return -1;
  if (o->variant == 1) substep14(o, r, 0);
  else substep(o, r, 0);
  return 0;
}

void lmo_get_diag(const lmo *o, double *d) { memcpy(d, o->diag, sizeof(double) * LMO_NDIAG); }

void lmo_get_coefs(const lmo *o, double *prem1_lu, double *dt11, double *dt12, double *prem3_lu,
                   double *dt21, double *dt22, double *fmap) {
  size_t n7 = (size_t)7 * o->my, n5 = (size_t)5 * o->my;
  if (prem1_lu) memcpy(prem1_lu, o->prem1, n7 * 8);
  if (dt11) memcpy(dt11, o->dt11, n7 * 8);
  if (dt12) memcpy(dt12, o->dt12, n7 * 8);
  if (prem3_lu) memcpy(prem3_lu, o->prem3, n5 * 8);
  if (dt21) memcpy(dt21, o->dt21, n5 * 8);
  if (dt22) memcpy(dt22, o->dt22, n5 * 8);
  if (fmap) memcpy(fmap, o->fmap, (size_t)o->my * 8);
}
