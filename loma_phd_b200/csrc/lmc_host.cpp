// lmc_host.cpp -- host-side set-up of liblomacte_b200: compact-FD operator
// tables, per-mode Poisson factors and the seeded initial condition.
//
// Everything here runs once per case (lmc_create / lmc_make_ic); the time
// stepping itself runs only on the GPU.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "lmc_internal.h"

namespace lmc {

RK3::RK3() {
  // trunk/lomacte3/src/modulos.f:193-209 (p0 = 5/66, p1 = -1)
  const double p0 = 5.0 / 66.0, p1 = -1.0;
  xi[0] = 0.0; xi[1] = -17.0 / 60.0; xi[2] = -5.0 / 12.0;
  gama[0] = 8.0 / 15.0; gama[1] = 5.0 / 12.0; gama[2] = 3.0 / 4.0;
  const double b3 = (p1 * (gama[0] * gama[2] + gama[1] * gama[2] + xi[1] * gama[2] + gama[0] * xi[2]) -
                     gama[0] * gama[1] * gama[2] - gama[0] * gama[1] * xi[2]) /
                    (p1 - gama[0] * gama[1]);
  beta[0] = gama[0] - p0; beta[1] = p1; beta[2] = b3;
  alpha[0] = p0; alpha[1] = gama[1] + xi[1] - p1; alpha[2] = gama[2] + xi[2] - beta[2];
}

// ---------------------------------------------------------------------
// Band linear algebra (row form).  A band matrix with p sub- and q super-
// diagonals is stored as rows of p+q+1 entries, entry c <-> column i-p+c.
// band_lu performs Gaussian elimination without pivoting (the reference's
// bandec / bandec7, cfdiff.f:977-1022 and 1058-1137, eliminate the same
// way) and returns L as row multipliers L[i][d-1] (x_i -= L x_{i-d}) and U
// as [reciprocal pivot, u_{i,i+1}, ..., u_{i,i+q}].
// ---------------------------------------------------------------------
void band_lu(int n, int p, int q, const double *A, double *L, double *U, bool singular_last) {
  const int w = p + q + 1;
  std::vector<double> W(A, A + (size_t)n * w);
  auto at = [&](int i, int col) -> double & { return W[(size_t)i * w + (col - i + p)]; };
  std::memset(L, 0, sizeof(double) * (size_t)n * p);
  std::memset(U, 0, sizeof(double) * (size_t)n * (q + 1));
  for (int k = 0; k < n; k++) {
    const double piv = at(k, k);
    if (singular_last && k == n - 1) {
      U[(size_t)k * (q + 1)] = 0.0;  // x_{n-1} := 0, see build_yops (inty8)
      break;
    }
    if (piv == 0.0) throw std::runtime_error("band_lu: zero pivot");
    U[(size_t)k * (q + 1)] = 1.0 / piv;
    for (int d = 1; d <= q && k + d < n; d++) U[(size_t)k * (q + 1) + d] = at(k, k + d);
    for (int i = k + 1; i <= k + p && i < n; i++) {
      const double l = at(i, k) / piv;
      L[(size_t)i * p + (i - k - 1)] = l;
      for (int d = 1; d <= q && k + d < n; d++) at(i, k + d) -= l * at(k, k + d);
    }
  }
}

void band_solve(int n, int p, int q, const double *L, const double *U, double *x) {
  for (int i = 0; i < n; i++)
    for (int d = 1; d <= p && i - d >= 0; d++) x[i] -= L[(size_t)i * p + d - 1] * x[i - d];
  for (int i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int d = 1; d <= q && i + d < n; d++) s -= U[(size_t)i * (q + 1) + d] * x[i + d];
    x[i] = s * U[(size_t)i * (q + 1)];
  }
}

void band_matvec(int n, int h, const double *M, const double *u, double *out) {
  const int w = 2 * h + 1;
  for (int i = 0; i < n; i++) {
    double s = 0.0;
    for (int c = 0; c < w; c++) {
      const int col = i - h + c;
      if (col >= 0 && col < n) s += M[(size_t)i * w + c] * u[col];
    }
    out[i] = s;
  }
}

// Dense LU with partial pivoting for the small Taylor-matching systems.
static void dense_solve(int n, std::vector<double> &A /*row-major n x n*/, std::vector<double> &b) {
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int k = 0; k < n; k++) {
    int pr = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(A[(size_t)i * n + k]) > std::fabs(A[(size_t)pr * n + k])) pr = i;
    if (pr != k) {
      for (int c = 0; c < n; c++) std::swap(A[(size_t)k * n + c], A[(size_t)pr * n + c]);
      std::swap(b[k], b[pr]);
    }
    const double piv = A[(size_t)k * n + k];
    if (piv == 0.0) throw std::runtime_error("dense_solve: singular");
    for (int i = k + 1; i < n; i++) {
      const double l = A[(size_t)i * n + k] / piv;
      if (l == 0.0) continue;
      for (int c = k; c < n; c++) A[(size_t)i * n + c] -= l * A[(size_t)k * n + c];
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int c = i + 1; c < n; c++) s -= A[(size_t)i * n + c] * b[c];
    b[i] = s / A[(size_t)i * n + i];
  }
}

// Second-derivative compact scheme on the actual mesh (the scheme of
// prederiv2, cfdiff.f:196-501): for row j, unknown LHS weights beta_m at
// offsets lo (the centre weight is 1) and RHS weights a_m at offsets ro,
// matched on the monomials (x-x_j)^n, n = 0..N-1:
//   sum_lhs beta_m n(n-1) h_m^(n-2) + [n==2]*2 = sum_rhs a_m h_m^n.
static void d2_row(const double *x, int j, const std::vector<int> &lo, const std::vector<int> &ro,
                   double *lhs5, double *rhs5) {
  const int nl = (int)lo.size(), nr = (int)ro.size(), N = nl + nr;
  std::vector<double> A((size_t)N * N, 0.0), b(N, 0.0);
  for (int n = 0; n < N; n++) {
    for (int m = 0; m < nl; m++) {
      const double h = x[j + lo[m]] - x[j];
      A[(size_t)n * N + m] = (n >= 2) ? (double)(n * (n - 1)) * std::pow(h, n - 2) : 0.0;
    }
    for (int m = 0; m < nr; m++) {
      const double h = x[j + ro[m]] - x[j];
      A[(size_t)n * N + nl + m] = -((n == 0) ? 1.0 : std::pow(h, n));
    }
    b[n] = (n == 2) ? -2.0 : 0.0;
  }
  dense_solve(N, A, b);
  for (int c = 0; c < 5; c++) { lhs5[c] = 0.0; rhs5[c] = 0.0; }
  lhs5[2] = 1.0;
  for (int m = 0; m < nl; m++) lhs5[lo[m] + 2] = b[m];
  for (int m = 0; m < nr; m++) rhs5[ro[m] + 2] = b[nl + m];
}

void build_yops(int my, const double *y, YOps &o) {
  if (my < 9) throw std::runtime_error("my too small");
  o.my = my;
  o.y.assign(y, y + my);
  o.hy.assign(my, 0.0); o.trp.assign(my, 0.0); o.fmap.assign(my, 0.0);
  // trapezoid / mesh weights: main.f:689-696
  for (int j = 1; j < my - 1; j++) {
    o.trp[j] = 0.25 * (y[j + 1] - y[j - 1]);
    o.hy[j] = 0.5 * (y[j + 1] - y[j - 1]);
  }
  o.trp[0] = 0.25 * (y[1] - y[0]); o.trp[my - 1] = 0.25 * (y[my - 1] - y[my - 2]);
  o.hy[0] = 0.5 * (y[1] - y[0]); o.hy[my - 1] = 0.5 * (y[my - 1] - y[my - 2]);

  // First derivative on uniform eta in [-1,1] (the scheme of pred1m6o,
  // cfdiff.f:24-182): interior 7/7-point compact stencil with the
  // spectral-like constants aaa,bbb,ccc; reduced stencils in rows 1-3 and
  // their mirror images at the other end.
  const double h = 2.0 / (double)(my - 1);
  const double aaa = 0.56926818603810, bbb = 0.31997939759919, ccc = 0.03751544855390;
  const double al = -3.0 / 4.0 + (33.0 / 20.0) * ccc + (239.0 / 180.0) * aaa + (82.0 / 45.0) * bbb;
  const double be = 3.0 / 10.0 + (24.0 / 25.0) * ccc - (88.0 / 225.0) * aaa + (34.0 / 225.0) * bbb;
  const double de = -1.0 / 20.0 + (39.0 / 100.0) * ccc + (19.0 / 300.0) * aaa + (2.0 / 75.0) * bbb;
  std::vector<double> lhs1((size_t)my * 7, 0.0);
  o.dt12.assign((size_t)my * 7, 0.0);
  auto setrow = [&](int j, const double l[7], const double r[7]) {
    for (int c = 0; c < 7; c++) { lhs1[(size_t)j * 7 + c] = l[c]; o.dt12[(size_t)j * 7 + c] = r[c]; }
  };
  {
    const double l0[7] = {0, 0, 0, 1, 1, 0, 0}, r0[7] = {0, 0, 0, -2.0 / h, 2.0 / h, 0, 0};
    const double l1[7] = {0, 0, 0.25, 1, 0.25, 0, 0}, r1[7] = {0, 0, -0.75 / h, 0, 0.75 / h, 0, 0};
    const double l2[7] = {0, 1.0 / 36.0, 4.0 / 9.0, 1, 4.0 / 9.0, 1.0 / 36.0, 0};
    const double r2[7] = {0, -25.0 / 216.0 / h, -20.0 / 27.0 / h, 0, 20.0 / 27.0 / h, 25.0 / 216.0 / h, 0};
    const double li[7] = {de, be, al, 1, al, be, de};
    const double ri[7] = {-ccc / h, -bbb / h, -aaa / h, 0, aaa / h, bbb / h, ccc / h};
    for (int j = 3; j < my - 3; j++) setrow(j, li, ri);
    const double *ls[3] = {l0, l1, l2}, *rs[3] = {r0, r1, r2};
    for (int e = 0; e < 3; e++) {
      setrow(e, ls[e], rs[e]);
      double lm[7], rm[7];
      for (int c = 0; c < 7; c++) { lm[c] = ls[e][6 - c]; rm[c] = -rs[e][6 - c]; }
      setrow(my - 1 - e, lm, rm);
    }
  }
  o.dt11 = lhs1;
  o.p1L.assign((size_t)my * 3, 0.0); o.p1U.assign((size_t)my * 4, 0.0);
  band_lu(my, 3, 3, lhs1.data(), o.p1L.data(), o.p1U.data());

  // Second derivative (prederiv2 scheme) and its LHS LU.
  std::vector<double> lhs2((size_t)my * 5, 0.0);
  o.dt22.assign((size_t)my * 5, 0.0);
  for (int j = 0; j < my; j++) {
    std::vector<int> lo, ro;
    if (j == 0) { lo = {1, 2}; ro = {0, 1, 2}; }
    else if (j == 1) { lo = {-1, 1, 2}; ro = {-1, 0, 1, 2}; }
    else if (j == my - 2) { lo = {-2, -1, 1}; ro = {-2, -1, 0, 1}; }
    else if (j == my - 1) { lo = {-1, -2}; ro = {0, -1, -2}; }
    else { lo = {-2, -1, 1, 2}; ro = {-2, -1, 0, 1, 2}; }
    d2_row(y, j, lo, ro, &lhs2[(size_t)j * 5], &o.dt22[(size_t)j * 5]);
  }
  o.dt21 = lhs2;
  o.p3L.assign((size_t)my * 2, 0.0); o.p3U.assign((size_t)my * 3, 0.0);
  band_lu(my, 2, 2, lhs2.data(), o.p3L.data(), o.p3U.data());

  // fmap = 1/(dy/deta) by the first-derivative scheme (cfdiff.f:912-937).
  std::vector<double> t(my);
  band_matvec(my, 3, o.dt12.data(), y, t.data());
  band_solve(my, 3, 3, o.p1L.data(), o.p1U.data(), t.data());
  for (int j = 0; j < my; j++) o.fmap[j] = 1.0 / t[j];

  // inty8 integration matrix: LU of dt12 (laps.f:509-523).  dt12 maps
  // constants to zero, so its last pivot vanishes in exact arithmetic and
  // the computed one is round-off.  inty8 only uses g - g(1), which does not
  // depend on the last unknown; taking the reciprocal last pivot as 0 (last
  // unknown = 0) gives that difference without the round-off blow-up.
  o.i8L.assign((size_t)my * 3, 0.0); o.i8U.assign((size_t)my * 4, 0.0);
  band_lu(my, 3, 3, o.dt12.data(), o.i8L.data(), o.i8U.data(), true);

  // Wall derivatives as linear functionals: dv/dy(wall) = sum_j e(j) v(j)
  // with e = fmap(wall) * row(wall) of prem1^-1 dt12 (the role endderiv,
  // cfdiff.f:819-860, plays for the bottom wall).
  o.ebot.assign(my, 0.0); o.etop.assign(my, 0.0);
  std::vector<double> col(my);
  for (int c = 0; c < my; c++) {
    std::fill(col.begin(), col.end(), 0.0);
    for (int r = std::max(0, c - 3); r <= std::min(my - 1, c + 3); r++) col[r] = o.dt12[(size_t)r * 7 + (c - r + 3)];
    band_solve(my, 3, 3, o.p1L.data(), o.p1U.data(), col.data());
    o.ebot[c] = o.fmap[0] * col[0];
    o.etop[c] = o.fmap[my - 1] * col[my - 1];
  }
}

// Chunk transfer matrices and Kogge-Stone tables.  The device solves run
// each lane's chunk of rows with an incoming state S (the last B solution
// values, most recent first); the chunk maps S_in to S_out = M S_in + p.
// At scan step s (offset 2^s) lane l composes with lane l -/+ 2^s, using
// the map of the lanes already folded into it: the table holds that map.
static std::vector<double> scan_table(int my, int B, const std::vector<double> &T, bool upper, int lpm, int base,
                                      int extra) {
  const int W = upper ? B + 1 : B;
  std::vector<std::vector<double>> M(32, std::vector<double>(B * B, 0.0));
  for (int l = 0; l < 32; l++) {
    const int n = (l < lpm) ? base + (l < extra ? 1 : 0) : 0;
    const int s0 = (l < lpm) ? l * base + (l < extra ? l : extra) : 0;
    for (int q = 0; q < B; q++) {
      std::vector<double> S(B, 0.0);
      S[q] = 1.0;
      for (int tt = 0; tt < n; tt++) {
        const int row = upper ? s0 + n - 1 - tt : s0 + tt;
        if (row >= my) break;
        double v = 0.0;
        for (int d = 0; d < B; d++) v -= T[(size_t)row * W + (upper ? 1 + d : d)] * S[d];
        if (upper) v *= T[(size_t)row * W];
        for (int d = B - 1; d > 0; d--) S[d] = S[d - 1];
        S[0] = v;
      }
      for (int r = 0; r < B; r++) M[l][r * B + q] = S[r];
    }
  }
  std::vector<double> tab((size_t)5 * 32 * B * B, 0.0);
  for (int s = 0; s < 5; s++) {
    const int off = 1 << s;
    std::vector<std::vector<double>> nM = M;
    for (int l = 0; l < 32; l++) {
      const int o = upper ? l + off : l - off;
      if (o < 0 || o >= 32) continue;
      for (int i = 0; i < B * B; i++) tab[((size_t)s * 32 + l) * B * B + i] = M[l][i];
      for (int r = 0; r < B; r++)
        for (int q = 0; q < B; q++) {
          double a = 0.0;
          for (int k = 0; k < B; k++) a += M[l][r * B + k] * M[o][k * B + q];
          nM[l][r * B + q] = a;
        }
    }
    M = nM;
  }
  return tab;
}

std::vector<double> chunk_major(const std::vector<double> &T, int my, int W, int C, int lpm, int base, int extra) {
  std::vector<double> out((size_t)C * W * 32, 0.0);
  for (int l = 0; l < lpm && l < 32; l++) {
    const int n = base + (l < extra ? 1 : 0), s0 = l * base + (l < extra ? l : extra);
    for (int t = 0; t < n && t < C; t++)
      for (int c = 0; c < W; c++)
        if (s0 + t < my) out[((size_t)t * W + c) * 32 + l] = T[(size_t)(s0 + t) * W + c];
  }
  return out;
}

void build_scans(YOps &o, int lpm, int base, int extra) {
  const int my = o.my;
  o.k1L = scan_table(my, 3, o.p1L, false, lpm, base, extra);
  o.k1U = scan_table(my, 3, o.p1U, true, lpm, base, extra);
  o.k3L = scan_table(my, 2, o.p3L, false, lpm, base, extra);
  o.k3U = scan_table(my, 2, o.p3U, true, lpm, base, extra);
  o.k8L = scan_table(my, 3, o.i8L, false, lpm, base, extra);
  o.k8U = scan_table(my, 3, o.i8U, true, lpm, base, extra);
}

// Per-mode data of the Poisson operator dt22 - k^2 dt21 with Dirichlet
// (identity) wall rows: laps.f:349-366 (Lapvdvhom) and laps.f:648-728
// (solvepsi, whose homogeneous solutions and 2x2 Neumann matrix depend on
// the mode only and are therefore built once here).
void build_poisson(const Grid &g, const YOps &o, const double *kx, const double *kz, PoissonTables &pt) {
  const int my = g.my, nm = g.nmode;
  pt.L.assign((size_t)nm * my * 2, 0.0);
  pt.U.assign((size_t)nm * my * 3, 0.0);
  pt.V12.assign((size_t)nm * my * 2, 0.0);
  pt.AAinv.assign((size_t)nm * 4, 0.0);
  pt.k2.assign(nm, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int m = 0; m < nm; m++) {
    const int i = m / g.mz, k = m % g.mz;
    const double k2 = kx[i] * kx[i] + kz[k] * kz[k];
    pt.k2[m] = k2;
    if (k2 == 0.0) continue;
    std::vector<double> A((size_t)my * 5, 0.0), L((size_t)my * 2), U((size_t)my * 3), v1(my, 0.0), v2(my, 0.0);
    for (int j = 1; j < my - 1; j++)
      for (int c = 0; c < 5; c++) A[(size_t)j * 5 + c] = o.dt22[(size_t)j * 5 + c] - k2 * o.dt21[(size_t)j * 5 + c];
    A[2] = 1.0;
    A[(size_t)(my - 1) * 5 + 2] = 1.0;
    band_lu(my, 2, 2, A.data(), L.data(), U.data());
    v1[0] = 1.0;
    v2[my - 1] = 1.0;
    band_solve(my, 2, 2, L.data(), U.data(), v1.data());
    band_solve(my, 2, 2, L.data(), U.data(), v2.data());
    double a11 = 0, a12 = 0, a21 = 0, a22 = 0;
    for (int j = 0; j < my; j++) {
      a11 += o.ebot[j] * v1[j]; a12 += o.ebot[j] * v2[j];
      a21 += o.etop[j] * v1[j]; a22 += o.etop[j] * v2[j];
    }
    const double det = a11 * a22 - a12 * a21;
    double *ai = &pt.AAinv[(size_t)m * 4];
    ai[0] = a22 / det; ai[1] = -a12 / det; ai[2] = -a21 / det; ai[3] = a11 / det;
    std::memcpy(&pt.L[(size_t)m * my * 2], L.data(), sizeof(double) * my * 2);
    std::memcpy(&pt.U[(size_t)m * my * 3], U.data(), sizeof(double) * my * 3);
    for (int j = 0; j < my; j++) {
      pt.V12[((size_t)m * my + j) * 2 + 0] = v1[j];
      pt.V12[((size_t)m * my + j) * 2 + 1] = v2[j];
    }
  }
}

}  // namespace lmc

// ---------------------------------------------------------------------
// Seeded initial condition (host only).
// ---------------------------------------------------------------------
namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Counter-based uniform in [0,1): independent of loop order and threads.
inline double urand(uint64_t seed, uint64_t a, uint64_t b, uint64_t c, uint64_t d) {
  uint64_t h = splitmix64(seed);
  h = splitmix64(h ^ (a * 0x100000001B3ull));
  h = splitmix64(h ^ (b * 0xC2B2AE3D27D4EB4Full));
  h = splitmix64(h ^ (c * 0x165667B19E3779F9ull));
  h = splitmix64(h ^ (d * 0x27D4EB2F165667C5ull));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

typedef std::complex<double> cd;

void cderiv1(const lmc::YOps &o, const cd *u, cd *du) {
  const int my = o.my;
  std::vector<double> re(my), im(my), a(my), b(my);
  for (int j = 0; j < my; j++) { re[j] = u[j].real(); im[j] = u[j].imag(); }
  lmc::band_matvec(my, 3, o.dt12.data(), re.data(), a.data());
  lmc::band_matvec(my, 3, o.dt12.data(), im.data(), b.data());
  lmc::band_solve(my, 3, 3, o.p1L.data(), o.p1U.data(), a.data());
  lmc::band_solve(my, 3, 3, o.p1L.data(), o.p1U.data(), b.data());
  for (int j = 0; j < my; j++) du[j] = cd(a[j] * o.fmap[j], b[j] * o.fmap[j]);
}
void cderiv2(const lmc::YOps &o, const cd *u, cd *du) {
  const int my = o.my;
  std::vector<double> re(my), im(my), a(my), b(my);
  for (int j = 0; j < my; j++) { re[j] = u[j].real(); im[j] = u[j].imag(); }
  lmc::band_matvec(my, 2, o.dt22.data(), re.data(), a.data());
  lmc::band_matvec(my, 2, o.dt22.data(), im.data(), b.data());
  lmc::band_solve(my, 2, 2, o.p3L.data(), o.p3U.data(), a.data());
  lmc::band_solve(my, 2, 2, o.p3L.data(), o.p3U.data(), b.data());
  for (int j = 0; j < my; j++) du[j] = cd(a[j], b[j]);
}
// Dirichlet Poisson solve v'' - k2 v = f, v = 0 at the walls (Lapvdvhom).
void cpoisson(const lmc::YOps &o, double k2, const cd *f, cd *v) {
  const int my = o.my;
  std::vector<double> A((size_t)my * 5, 0.0), L((size_t)my * 2), U((size_t)my * 3);
  for (int j = 1; j < my - 1; j++)
    for (int c = 0; c < 5; c++) A[(size_t)j * 5 + c] = o.dt22[(size_t)j * 5 + c] - k2 * o.dt21[(size_t)j * 5 + c];
  A[2] = 1.0; A[(size_t)(my - 1) * 5 + 2] = 1.0;
  lmc::band_lu(my, 2, 2, A.data(), L.data(), U.data());
  std::vector<double> re(my), im(my), a(my), b(my);
  for (int j = 0; j < my; j++) { re[j] = f[j].real(); im[j] = f[j].imag(); }
  lmc::band_matvec(my, 2, o.dt21.data(), re.data(), a.data());
  lmc::band_matvec(my, 2, o.dt21.data(), im.data(), b.data());
  a[0] = b[0] = a[my - 1] = b[my - 1] = 0.0;
  lmc::band_solve(my, 2, 2, L.data(), U.data(), a.data());
  lmc::band_solve(my, 2, 2, L.data(), U.data(), b.data());
  for (int j = 0; j < my; j++) v[j] = cd(a[j], b[j]);
}

}  // namespace

extern "C" int lmc_make_ic(const lmc_params *p, const double *y, const lmc_ic_params *ic, double *vor,
                           double *phi, double *psi, double *scal, double *u00, double *v00, double *w00) {
  if (!p || !y || !ic || !vor || !phi || !psi || !scal || !u00 || !v00 || !w00) return LMC_EINVAL;
  try {
    lmc::Grid g;
    g.set(p->mgalx, p->mgalz, p->my);
    if (g.my < 9 || g.nkx < 1 || g.mz < 1) return LMC_EINVAL;
    lmc::YOps o;
    lmc::build_yops(g.my, y, o);
    const int my = g.my, nkx = g.nkx, mz = g.mz;
    const size_t ns = (size_t)g.nmode * my;
    std::vector<double> kxv(nkx), kzv(mz);
    std::vector<int> kzi(mz);
    for (int i = 0; i < nkx; i++) kxv[i] = p->alp * i;
    for (int k = 0; k < mz; k++) {
      kzi[k] = (k <= g.nz1) ? k : k - mz;
      kzv[k] = p->bet * kzi[k];
    }
    std::vector<double> win(my);
    for (int j = 0; j < my; j++) win[j] = std::exp(-(y[j] / ic->swin) * (y[j] / ic->swin));
    // Only the modes with 1 <= |k| <= nkmax (mode-index units) carry noise,
    // and every step below works on one mode at a time, so every other mode
    // is zero in all outputs (the 00 mode gets the mean profiles).  The
    // band's modes are listed in increasing mode order.
    std::vector<int> band, slot(g.nmode, -1);
    for (int m = 0; m < g.nmode; m++) {
      const int i = m / mz, kz = kzi[m % mz];
      const double nh = std::sqrt((double)(i * i + kz * kz));
      if (nh >= 1.0 && nh <= (double)ic->nkmax) {
        slot[m] = (int)band.size();
        band.push_back(m);
      }
    }
    const int nb = (int)band.size();
    const size_t nbs = (size_t)nb * my;
    // 1) random velocity per mode (initloma3/src/main.f:128-226); modes are
    // independent (counter-based random numbers), so the loops over the band
    // run in parallel and the result does not depend on the threads
    std::vector<cd> uf(nbs, 0.0), vf(nbs, 0.0), wf(nbs, 0.0);
    cd *fld[3] = {uf.data(), vf.data(), wf.data()};
    const int nym = ic->nymax > 0 ? ic->nymax : 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int bi = 0; bi < nb; bi++) {
      const int m = band[bi], i = m / mz, k = m % mz, kz = kzi[k];
      if (i == 0 && kz < 0) continue;  // filled by Hermitian symmetry below
      const double kh = std::sqrt(kxv[i] * kxv[i] + kzv[k] * kzv[k]);
      for (int c = 0; c < 3; c++) {
        cd *f = fld[c] + (size_t)bi * my;
        for (int jj = 1; jj <= nym; jj++) {
          const double a = 2.0 * (0.5 - urand(ic->seed, i, (uint64_t)(kz + 100000), c, 2 * jj));
          const double ph = urand(ic->seed, i, (uint64_t)(kz + 100000), c, 2 * jj + 1);
          const double ky = 2.0 * kh / nym * jj;
          for (int j = 0; j < my; j++) f[j] += a * std::exp(cd(0.0, ky * y[j] + 2.0 * M_PI * ph)) * win[j];
        }
      }
    }
    for (int bi = 0; bi < nb; bi++) {
      const int m = band[bi];
      if (m / mz != 0 || kzi[m % mz] >= 0) continue;
      const int src_slot = slot[-kzi[m % mz]];  // kx = 0, kz > 0 partner (same |k|, in the band)
      for (int c = 0; c < 3; c++) {
        const cd *src = fld[c] + (size_t)src_slot * my;
        cd *dst = fld[c] + (size_t)bi * my;
        for (int j = 0; j < my; j++) dst[j] = std::conj(src[j]);
      }
    }
    // 2) solenoidal: curl (initloma3/src/main.f:231-256)
    std::vector<cd> cu(nbs), cv(nbs), cw(nbs);
#pragma omp parallel for schedule(dynamic, 1)
    for (int bi = 0; bi < nb; bi++) {
      std::vector<cd> t1(my), t2(my);
      const int m = band[bi], i = m / mz, k = m % mz;
      const cd ikx(0.0, kxv[i]), ikz(0.0, kzv[k]);
      const size_t b = (size_t)bi * my;
      cderiv1(o, &wf[b], t1.data());
      cderiv1(o, &uf[b], t2.data());
      for (int j = 0; j < my; j++) {
        cu[b + j] = t1[j] - ikz * vf[b + j];
        cv[b + j] = ikz * uf[b + j] - ikx * wf[b + j];
        cw[b + j] = ikx * vf[b + j] - t2[j];
      }
    }
    // 3) scale to rms amp at the mid plane (initloma3/src/main.f:291-356),
    // summed over the band in mode order (the other modes add zeros)
    int jm = 0;
    for (int j = 1; j < my; j++)
      if (std::fabs(y[j]) < std::fabs(y[jm])) jm = j;
    double e = 0.0;
    for (int bi = 0; bi < nb; bi++) {
      const int i = band[bi] / mz;
      e += (i == 0 ? 1.0 : 2.0) * std::norm(cu[(size_t)bi * my + jm]);
    }
    const double fac = (e > 0.0) ? ic->amp / std::sqrt(e) : 0.0;
    // 4) mean profiles and rho u_i (initloma3/src/main.f:362-374, 572-600)
    std::vector<double> rho00(my);
    for (int j = 0; j < my; j++) rho00[j] = 1.0 + (ic->s - 1.0) / (ic->s + 1.0) * std::tanh(-y[j] / (2.0 * ic->dm0));
    // 5) psi, Omega_y, phi (initloma3/src/main.f:473-561); zero outside the band
    cd *VOR = reinterpret_cast<cd *>(vor), *PHI = reinterpret_cast<cd *>(phi);
    cd *PSI = reinterpret_cast<cd *>(psi), *SCA = reinterpret_cast<cd *>(scal);
    std::fill(VOR, VOR + ns, cd(0.0));
    std::fill(PHI, PHI + ns, cd(0.0));
    std::fill(PSI, PSI + ns, cd(0.0));
    std::fill(SCA, SCA + ns, cd(0.0));
#pragma omp parallel for schedule(dynamic, 1)
    for (int bi = 0; bi < nb; bi++) {
      std::vector<cd> ru(my), rv(my), rw(my), dv(my), div(my), ps(my), dps(my), myv(my), d2(my);
      const int m = band[bi], i = m / mz, k = m % mz;
      const cd ikx(0.0, kxv[i]), ikz(0.0, kzv[k]);
      const double k2 = kxv[i] * kxv[i] + kzv[k] * kzv[k];
      const size_t bb = (size_t)bi * my, b = (size_t)m * my;
      for (int j = 0; j < my; j++) {
        ru[j] = rho00[j] * fac * cu[bb + j];
        rv[j] = rho00[j] * fac * cv[bb + j];
        rw[j] = rho00[j] * fac * cw[bb + j];
      }
      cderiv1(o, rv.data(), dv.data());
      for (int j = 0; j < my; j++) div[j] = ikx * ru[j] + ikz * rw[j] + dv[j];
      if (k2 == 0.0) std::fill(ps.begin(), ps.end(), cd(0.0));
      else cpoisson(o, k2, div.data(), ps.data());
      cderiv1(o, ps.data(), dps.data());
      for (int j = 0; j < my; j++) myv[j] = rv[j] - dps[j];
      cderiv2(o, myv.data(), d2.data());
      for (int j = 0; j < my; j++) {
        PSI[b + j] = ps[j];
        VOR[b + j] = -ikx * rw[j] + ikz * ru[j];
        PHI[b + j] = -k2 * myv[j] + d2[j];
      }
    }
    for (int j = 0; j < my; j++) {
      SCA[j] = cd(1.0 / rho00[j], 0.0);
      u00[j] = rho00[j] * ic->u0 * std::tanh(y[j] / (2.0 * ic->dm0));
      v00[j] = 0.0;
      w00[j] = 0.0;
    }
  } catch (...) {
    return LMC_EINVAL;
  }
  return LMC_OK;
}

extern "C" int lmc_y_metrics(int my, const double *y, double *fmap, double *hy, double *trp) {
  if (!y || my < 9) return LMC_EINVAL;
  lmc::YOps o;
  try {
    lmc::build_yops(my, y, o);
  } catch (...) {
    return LMC_EINVAL;
  }
  for (int j = 0; j < my; j++) {
    if (fmap) fmap[j] = o.fmap[j];
    if (hy) hy[j] = o.hy[j];
    if (trp) trp[j] = o.trp[j];
  }
  return LMC_OK;
}
