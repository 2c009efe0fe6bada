/*
 * lomacte_oracle.h -- CPU FP64 oracle for the lomacte RK3 substep.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load this library, always as the
 * checker or as the timed CPU baseline; the product (loma_phd_b200) never
 * links, imports or executes it.
 *
 * What it is: a statement-by-statement FP64 restatement of the reference
 * Fortran lomacte3 substep (Beovulfo/LoMa_phD trunk/lomacte3/src):
 *   cross.f:307-1141 (cross1 RK3 substep), cross.f:1282-1430 (foup2),
 *   cross.f:1440-1828 (phys2), laps.f:17-129,319-764 (Poisson solvers),
 *   cfdiff.f:24-1223 (compact FD coefficients, band LU), fou3D.f:29-189
 *   (transform wrappers, padding/truncation, kz ordering), main.f:689-800
 *   (hy/trp weights, wavenumbers), modulos.f:193-209 (RK3 coefficients).
 * The reference computes in FP32 with FP64 work vectors; this oracle keeps
 * every quantity in FP64.  Its FFT is written from the DFT definition and
 * pinned against the reference's own benchmark_fft golden vectors
 * (branches/reactml/benchmark_fft/{cft,rfft}test_double.txt).  Parity of the
 * full substep is pinned by restatement (the Fortran cannot be compiled in
 * this environment: no Fortran compiler, no MPI).
 *
 * Field layout ("reference layout"): complex values interleaved re,im, in
 * the order of the Fortran arrays vor(0:my-1,0:mz1,1:nplanes):
 *   index(kx, kz, j) = ((kx*mz + kz)*my + j), y fastest.
 */
#ifndef LOMACTE_ORACLE_H
#define LOMACTE_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct lmo lmo;

/* dtmode: 0 = reference CFL mode (Deltat starts at dt0 and is replaced by
 * the CFL value computed every ncfl steps, rounded to FP32 as the
 * reference's real*4 Deltat), 1 = fixed Deltat = dt0. */
lmo *lmo_create(int mgalx, int mgalz, int my, const double *y, double Re,
                double alp, double bet, double peclet, double cfl, int ncfl,
                int dtmode, double dt0, int nthreads);
void lmo_destroy(lmo *o);

int lmo_set_state(lmo *o, const double *vor, const double *phi,
                  const double *psi, const double *scal, const double *u00,
                  const double *v00, const double *w00, double time);
int lmo_get_state(const lmo *o, double *vor, double *phi, double *psi,
                  double *scal, double *u00, double *v00, double *w00,
                  double *time);
/* Advance nsteps full RK3 steps (3 substeps each). */
int lmo_step(lmo *o, int nsteps);
/* 0: trunk/lomacte3 (2017, default); 1: the 2014 variant trunk/lomacte
 * (spectral T, d(rho) transform round trip, Dirichlet psi). */
int lmo_set_variant(lmo *o, int variant);

/* One substep with RK coefficient r on the current state (timing samples). */
int lmo_substep(lmo *o, int r);
/* Timing samples: the parallel loops of later substeps visit only the
 * units (modes, kx planes of a field, physical lines) whose index is phase
 * modulo stride, i.e. 1/stride of a substep's work; stride 1 restores the
 * full substep.  The state is then no longer a solution (timing only). */
int lmo_set_sample(lmo *o, int stride, int phase);

/* Diagnostics of the last step, in this order:
 * 0 time (before the step), 1 Deltat used, 2 dm, 3 dw, 4 Re*dw, 5 trapz,
 * 6 masst, 7 massu, 8 massv, 9 massw, 10 H00u, 11 H00w, 12 next Deltat */
#define LMO_NDIAG 13
void lmo_get_diag(const lmo *o, double *d);

/* Statistics (addstats1 cross.f:1981-2064, addstats2 cross.f:2070-2290,
 * the physical sums of phys2 cross.f:1583-1607, writestats
 * escru.f:276-484, resetstats escru.f:485-580).  Profiles are kept raw
 * (without the 1/(mgalx*mgalz) of writestats) in the order of the .sta
 * record; spectra as [kx plane][field 0..11][spectra plane][|kz|].
 * reset: zero everything, set the 1-based spectra rows and the exponent of
 * mu/mu0 = T^sigma; step: nsteps RK3 steps with istati = 1; read: copy
 * out (NULL skips), counts = {nacum, nacumsp}; clear_spectra zeroes the
 * spectra and nacumsp as writestats does. */
#define LMO_NSTAT 33
enum {
  LMO_S_UM, LMO_S_VM, LMO_S_WM, LMO_S_RUM, LMO_S_RVM, LMO_S_RWM, LMO_S_TM, LMO_S_W1M, LMO_S_W2M,
  LMO_S_W3M, LMO_S_THEM, LMO_S_UP, LMO_S_VP, LMO_S_WP, LMO_S_UVR, LMO_S_UWR, LMO_S_VWR, LMO_S_W1P,
  LMO_S_W2P, LMO_S_W3P, LMO_S_TP, LMO_S_EP, LMO_S_RUU, LMO_S_RUV, LMO_S_RUW, LMO_S_RVV, LMO_S_RVW,
  LMO_S_RWW, LMO_S_RHOM, LMO_S_THEP, LMO_S_THEUP, LMO_S_MUM, LMO_S_NUM
};
int lmo_stats_reset(lmo *o, int nsp, const int *jsp, double sigma);
int lmo_stats_step(lmo *o, int nsteps);
int lmo_stats_read(lmo *o, double *prof, double *spec, double *uner, int *counts, int clear_spectra);

/* Passive scalar Z (an extension: no lomacte code carries one).  Z is
 * advanced exactly as the lomacte3 substep advances T (cross.f:336-349,
 * 521-554, 619-627, 1625-1647): zero at the walls except its mean, held at
 * the wall values it was loaded with; its derivatives go through the same
 * transforms; in physical space RHS(Z) = -u.grad Z + T lap Z / (Re Sc) with
 * the FP64 RK3 accumulator; the increment Delta Z is transformed back and
 * added to the spectral Z.  The diffusive CFL limit takes the larger of
 * 1/Pe and 1/(Re Sc).  Not for the 2014 variant.  set_scalar allocates;
 * set_scalar_state loads Z (reference layout) and clears its RK3 memory. */
int lmo_set_scalar(lmo *o, int on, double schmidt);
int lmo_set_scalar_state(lmo *o, const double *z);
int lmo_get_scalar_state(const lmo *o, double *z);

/* Variable viscosity (an extension restated from branches/loma/src/cross.f:
 * 1591-1596, 2177-2196): mu = k = rho D = T^sigma.  In physical space
 *   RHS(T) = -u.grad T + T^sigma (T lap T + sigma |grad T|^2) / Pe,
 *   RHS(Z) = -u.grad Z + T^sigma (T lap Z + sigma grad T.grad Z) / (Re Sc),
 * and the products rho u_i u_j lose the variable part of the stress,
 * 2 (T^sigma - 1) S_ij / Re, with S_ij from d(u_i)/dx_j = T d(rho u_i)/dx_j
 * + rho u_i dT/dx_j (six more transform inputs); lomacte3's constant-
 * viscosity terms stay as they are, so that the total viscous force is the
 * divergence of 2 T^sigma S_ij / Re up to a gradient (which the Omega_y and
 * phi equations do not see).  The diffusive CFL limit takes T_max^(1+sigma).
 * sigma in [0, 4]; sigma = 0 reproduces the constant-viscosity substep.
 * Not for the 2014 variant. */
int lmo_set_viscosity(lmo *o, int on, double sigma);

/* Physical fields of the current state on chosen y planes (the quantities
 * of tofis_loma's escrphys, trunk/tofis_loma/src/escru.f:11-314, from the
 * solver's own rho u_i): out[p][q][z][x] with q = u, v, w, T, omega_x,
 * omega_y, omega_z (and Z with the scalar); jplanes 1-based. */
int lmo_physical(const lmo *o, int nplanes, const int *jplanes, double *out);

/* Coefficient access for tests (band storage row-major [row][band]). */
void lmo_get_coefs(const lmo *o, double *prem1_lu, double *dt11, double *dt12,
                   double *prem3_lu, double *dt21, double *dt22, double *fmap);
/* 1-D FP64 y-operators on one real vector (deryr / deryyr / inty8). */
void lmo_deryr(const lmo *o, const double *u, double *du);
void lmo_deryyr(const lmo *o, const double *u, double *du);
void lmo_inty8(const lmo *o, const double *du, double *u);
/* One (kx,kz) mode: Lapvdvhom / solvepsi on complex vectors (re,im). */
void lmo_lapvdvhom(const lmo *o, const double *phi, double *v, double *dvdy,
                   double rk);
void lmo_solvepsi(const lmo *o, const double *phi, double *v, double *dvdy,
                  double rk);

/* FFT conventions of rftsingle.f / cftsingle.f (forward scaled by 1/n).
 * c2c: in-place on n complex (re,im interleaved), sign<0 forward.
 * rft forward: x[n] real -> packed[n+2] = (Re X0, 0, Re X1, Im X1, ...,
 *   Re X_{n/2}, 0); rft inverse: packed -> x[n]. */
void lmo_cft(int n, double *c, int iopt);
void lmo_rft(int n, double *c, int iopt);

#ifdef __cplusplus
}
#endif
#endif
