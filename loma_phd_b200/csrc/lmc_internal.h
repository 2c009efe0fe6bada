// lmc_internal.h -- shared host/device definitions of liblomacte_b200.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/lomacte_b200.h"

namespace lmc {

// Grid sizes derived as in trunk/lomacte3/src/ctes3D:24-33.
struct Grid {
  int mgalx, mgalz, my;
  int mx, nkx, mz, nz1, nz2, nmode;
  void set(int gx, int gz, int ny) {
    mgalx = gx; mgalz = gz; my = ny;
    mx = 2 * (gx / 3); nkx = mx / 2;
    mz = 2 * (gz / 3) - 1; nz1 = (mz - 1) / 2; nz2 = gz - nz1;
    nmode = nkx * mz;
  }
};

// Host-side y-operator tables (all FP64).
//   D1 = first derivative: rows of the RHS band dt12 (7 per row), the LU of
//        the LHS prem1 in row form (L: 3 multipliers, U: reciprocal pivot +
//        3 super-diagonals), fmap = 1/(dy/deta).
//   D2 = second derivative: dt22 (5), LU of prem3 (L: 2, U: 1+2), dt21 (5).
//   I8 = integration of inty8 (laps.f:484-575): dt11 (7) and the LU of
//        dt12 (L: 3, U: 1+3).
struct YOps {
  int my = 0;
  std::vector<double> y, hy, trp, fmap;
  std::vector<double> dt12, dt11, dt22, dt21;     // [my][7] / [my][5]
  std::vector<double> p1L, p1U;                   // [my][3], [my][4]
  std::vector<double> p3L, p3U;                   // [my][2], [my][3]
  std::vector<double> i8L, i8U;                   // [my][3], [my][4]
  std::vector<double> ebot, etop;                 // dv/dy at the walls as linear functionals
  // Kogge-Stone scan tables of the chunked device solves ([5][32][B][B])
  std::vector<double> k1L, k1U, k3L, k3U, k8L, k8U;
};

// Per-mode Poisson data (operator dt22 - k^2 dt21 with identity wall rows).
struct PoissonTables {
  std::vector<double> L;     // [nmode][my][2]
  std::vector<double> U;     // [nmode][my][3]
  std::vector<double> V12;   // [nmode][my][2]  homogeneous solutions v1, v2
  std::vector<double> AAinv; // [nmode][4]      inverse of the 2x2 Neumann matrix
  std::vector<double> k2;    // [nmode]
};

void build_yops(int my, const double *y, YOps &ops);
// Chunk-major copy of a row table T[my][W] for the lane split of a pencil:
// out[(t*W + c)*32 + l] = T[s_l + t][c] (zero where lane l has no row t).
std::vector<double> chunk_major(const std::vector<double> &T, int my, int W, int C, int lpm, int base, int extra);
// Scan tables of the constant band solves for the chunk split of a pencil
// over the lanes of a warp (lane l owns n_l rows starting at s_l).
void build_scans(YOps &ops, int lpm, int base, int extra);
void build_poisson(const Grid &g, const YOps &ops, const double *kx,
                   const double *kz, PoissonTables &pt);
// Band helpers used by the host code (row-form LU, see build_yops).
void band_lu(int n, int p, int q, const double *A /*[n][p+q+1]*/, double *L /*[n][p]*/,
             double *U /*[n][q+1]*/, bool singular_last = false);
void band_solve(int n, int p, int q, const double *L, const double *U, double *x);
void band_matvec(int n, int h, const double *M /*[n][2h+1]*/, const double *u, double *out);

// The RK3 coefficients of trunk/lomacte3/src/modulos.f:193-209.
struct RK3 {
  double gama[3], xi[3], alpha[3], beta[3];
  RK3();
};

}  // namespace lmc
