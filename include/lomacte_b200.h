/*
 * lomacte_b200.h -- C ABI of the B200-native lomacte substep library
 * (liblomacte_b200.so).
 *
 * The library replaces the time loop of the reference Fortran subroutine
 * cross1 (Beovulfo/LoMa_phD trunk/lomacte3/src/cross.f:24-45, called once
 * from trunk/lomacte3/src/main.f:215) with a device-resident RK3 stepper.
 * Every entry point returns an int status (LMC_OK = 0, < 0 on error); no
 * C++ exception crosses this boundary.  Arrays are plain host or device
 * pointers with sizes implied by the grid; no torch types appear here.
 *
 * Grid conventions follow trunk/lomacte3/src/ctes3D:18-36:
 *   mx = 2*(mgalx/3), nplanes = mx/2 (kx planes), mz = 2*(mgalz/3)-1 (kz
 *   modes, kz = 0..nz1, -nz1..-1 with nz1 = (mz-1)/2), my points in y.
 * Spectral fields use the reference layout vor(0:my-1, 0:mz-1, 1:nplanes):
 *   complex values (re, im interleaved), y fastest, then kz, then kx plane.
 * One handle = one case = one CUDA stream; calls on one handle must come
 * from one host thread at a time.
 */
#ifndef LOMACTE_B200_H
#define LOMACTE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  LMC_OK = 0,
  LMC_EINVAL = -1,   /* bad argument or grid */
  LMC_ENOMEM = -2,   /* device allocation failed */
  LMC_ENAN = -3,     /* non-finite value in the step's diagnostics (the
                        run blew up); lmc_get_diag / lmc_status report it */
  LMC_ETIMEOUT = -4, /* a bounded device wait gave up */
  LMC_ECUDA = -5,    /* CUDA runtime error */
  LMC_ENODEV = -6    /* no CUDA device (the library has no CPU path) */
};

/* Run parameters: the hre.dat records parsed by initcr
 * (trunk/lomacte3/src/main.f:502-570) plus the build's own switches. */
typedef struct lmc_params {
  int mgalx, mgalz, my; /* physical grid (ctes3D:18-20) */
  double Re, alp, bet;  /* hre.dat line 1 (main.f:506,555-557) */
  double peclet;        /* <= 0: Re*0.7f as main.f:569 */
  double cfl;           /* hre.dat CFL (main.f:517,560) */
  int ncfl;             /* steps between CFL updates (main.f:564) */
  int dt_mode;          /* 0: reference CFL mode, 1: fixed Deltat */
  double dt;            /* initial Deltat (reference: 1e-4, main.f:559) or the fixed Deltat */
  int precision;        /* 0: FP64 (the plain path)
                           1: mixed: FP32 work buffers and FP32 FFTs; FP64
                              state, RK3 accumulators, y solves, 00 modes
                              and pointwise EOS / d(rho)/dt math
                           2: as 1 with FP64 FFT arithmetic (FP32 storage)
                           With precision 1, LMC_FFT64=<mask> in the
                           environment at lmc_create gives chosen stages FP64
                           butterflies (1 inverse z, 2 x stage, 4 direct z),
                           for attributing the mixed form's error. */
  int device;           /* CUDA device ordinal */
  int variant;          /* 0: trunk/lomacte3 (2017); 1: the 2014 code
                           trunk/lomacte (spectral T, d(rho) by a transform
                           round trip, Dirichlet psi; FP64 only) */
  int scalar;           /* 1: carry a passive scalar Z (an extension with no
                           counterpart in the lomacte codes, see
                           lmc_load_scalar_f64); not with variant 1 */
  double schmidt;       /* Schmidt number Sc of Z; <= 0: Sc = Pr = 0.7f */
  int visc;             /* 1: variable viscosity mu = k = rho D = T^sigma (an
                           extension after branches/loma/src/cross.f:
                           1591-1596, 2177-2196); 0: the constant viscosity
                           of lomacte3.  Not with variant 1; the x stage
                           then needs mgalx <= 1152 with the scalar for
                           its shared memory */
  double sigma;         /* exponent sigma in [0, 4] (0.7 for air;
                           branches/loma reads it as hre.dat's fourth
                           value, main.f:543) */
} lmc_params;

/* Per-step diagnostics (the .cf record of cross.f:1172-1176 without the
 * stats-only energies). */
typedef struct lmc_diag {
  double time;        /* time at the start of the step */
  double Deltat;      /* Deltat used by the step */
  double dm;          /* momentum thickness (cross.f:1416-1429) */
  double dw;          /* vorticity thickness (cross.f:692-699) */
  double Redw;        /* Re*dw */
  double trapz;       /* -int d(rho)/dt dy (cross.f:1046) */
  double masst;       /* int <rho>_xz dy (escru.f:372-376) */
  double massu, massv, massw; /* int rho u_i,00 dy (cross.f:1013-1020) */
  double H00u, H00w;  /* 0.25 int RHS(u00), RHS(w00) dy (cross.f:713-722) */
  double Deltat_next; /* Deltat of the next step */
  int step;           /* steps taken by the handle */
  int status;         /* device status word (0 ok) */
} lmc_diag;

typedef struct lmc_handle lmc_handle;

/* Create a case: coefficients (cfdiff.f derivadas), wavenumbers, per-mode
 * Poisson factors, device buffers and the stream.  y has my entries.
 * Replaces initcr's grid set-up (main.f:461-800) and cross1's set-up
 * (cross.f:125-220). */
int lmc_create(const lmc_params *p, const double *y, lmc_handle **out);
int lmc_destroy(lmc_handle *h);

/* Load the state (getfil, main.f:329-455, then cross.f:211-215,276-280).
 * FP64 variant: complex*16 fields in the reference layout.  FP32 variant:
 * complex*8 fields exactly as the restart file stores them.  Both zero
 * the RK3 memory (main.f:171-174). */
int lmc_load_state_f64(lmc_handle *h, const double *vor, const double *phi,
                       const double *psi, const double *scal,
                       const double *u00, const double *v00,
                       const double *w00, double time);
int lmc_load_state_f32(lmc_handle *h, const float *vor, const float *phi,
                       const float *psi, const float *scal, const double *u00,
                       const double *v00, const double *w00, double time);
/* Read the state back (for escru, escru.f:11-193).  NULL pointers skip. */
int lmc_get_state_f64(lmc_handle *h, double *vor, double *phi, double *psi,
                      double *scal, double *u00, double *v00, double *w00,
                      double *time);
int lmc_get_state_f32(lmc_handle *h, float *vor, float *phi, float *psi,
                      float *scal, double *u00, double *v00, double *w00,
                      double *time);

/* Passive scalar Z (lmc_params.scalar = 1).  No lomacte code carries a
 * scalar; Z is advanced exactly as the lomacte3 substep advances T
 * (cross.f:336-349, 521-554, 619-627, 1625-1647): zero at the walls except
 * its 00 mode, held at the wall values it was loaded with; dZ/dy and lap Z
 * by the compact schemes; in physical space RHS(Z) = -u.grad Z +
 * T lap Z / (Re Sc) with its own FP64 RK3 accumulator; Delta Z transformed
 * back and added to the spectral Z.  The diffusive CFL limit takes the
 * larger of 1/Pe and 1/(Re Sc).  Load Z after lmc_load_state_*: the layout
 * is that of the other fields (reference layout, complex*16); loading
 * clears Z's RK3 memory.  LMC_EINVAL without the scalar. */
int lmc_load_scalar_f64(lmc_handle *h, const double *z);
int lmc_get_scalar_f64(lmc_handle *h, double *z);

/* Physical fields of the current state on chosen y planes: the quantities
 * tofis_loma writes (escrphys, trunk/tofis_loma/src/escru.f:11-314; y work
 * of uvw.f:7-94), formed from the solver's own rho u_i, i.e. Lapvdvhom with
 * the substep's wall conditions of Omega_y and phi (cross.f:315-335,
 * 365-499) rather than tofis_loma's own Robin-condition solve for rho v,
 * and T, Z as stored (as tofis_loma reads them): for each 1-based row
 * jplanes[p] the mgalz x mgalx planes (x fastest, natural order) of u, v, w,
 * T, omega_x, omega_y, omega_z and, with the scalar, Z, in that order:
 * out[p][q][z][x], q < 7 (8).  omega = curl(T rho u) = T curl(rho u) +
 * grad T x rho u, per point.  Computed in FP64 whatever the precision form,
 * on device buffers of its own (about 11 spectral and 10 z-padded fields,
 * freed before returning); the state and its RK3 memory are not changed.
 * Not for the 2014 variant.  Replaces tofis_loma's main program
 * (trunk/tofis_loma/src/main.f:14) for a restart the library holds. */
int lmc_physical_f64(lmc_handle *h, int nplanes, const int *jplanes, double *out);

/* Variable viscosity (lmc_params.visc = 1): mu = k = rho D = T^sigma.  The
 * lomacte3 substep keeps its constant-viscosity terms; in physical space
 *   RHS(T) = -u.grad T + T^sigma (T lap T + sigma |grad T|^2) / Pe
 *   RHS(Z) = -u.grad Z + T^sigma (T lap Z + sigma grad T.grad Z) / (Re Sc)
 * (branches/loma/src/cross.f:1591-1596), and the products rho u_i u_j that
 * the substep differentiates lose 2 (T^sigma - 1) S_ij / Re, with S_ij from
 * d(u_i)/dx_j = T d(rho u_i)/dx_j + rho u_i dT/dx_j (six more transform
 * inputs).  The total viscous force is then the divergence of
 * 2 T^sigma S_ij / Re up to a gradient, which the Omega_y and phi
 * equations do not see, as branches/loma/src/cross.f:2177-2196 forms it
 * (tau_ij = 2 T^sigma S_ij, the isotropic part left in the pressure).  The
 * diffusive CFL limit takes T_max^(1+sigma).  sigma = 0 reproduces the
 * constant-viscosity substep. */

/* Advance nsteps full RK3 steps (the body of cross.f:225-1226, 3
 * substeps of cross.f:307-1141 each).  Asynchronous on the handle's
 * stream; Deltat is computed on the device. */
int lmc_step(lmc_handle *h, int nsteps);
/* lmc_step with the transform stage decomposed as the reference's slab
 * decomposition (chpl2ln / chln2pl and pointers_calc,
 * trunk/lomacte3/src/change.f:1-211) over nblocks blocks on this device:
 * block r's inverse and direct z transforms cover its contiguous kx planes,
 * its x stage covers its contiguous (z, y) lines (the first n mod nblocks
 * blocks one longer), and the plane -> line and line -> plane exchanges
 * between the blocks' buffers are device copies -- the data path of a run
 * whose blocks sit on several GPUs, where the copies become the all-to-all.
 * The y work is per mode and runs over all modes at once.  Results are
 * those of lmc_step (FP64: to round-off).  nblocks in [1, nplanes], fixed
 * for the handle after the first call (its block buffers are kept);
 * mgalx >= 144 (one z line per x-stage tile); not with the 2014 variant;
 * no CUDA graphs.  LMC_EINVAL otherwise. */
int lmc_step_split(lmc_handle *h, int nblocks, int nsteps);
int lmc_sync(lmc_handle *h);
/* Diagnostics of the last completed step (synchronises). */
int lmc_get_diag(lmc_handle *h, lmc_diag *d);
/* Device status word (0 ok, else an LMC_E* code); synchronises.  A bounded
 * device wait that gave up reads LMC_ETIMEOUT; non-finite diagnostics read
 * LMC_ENAN. */
int lmc_status(lmc_handle *h);
/* Failure-path check: runs on the handle's stream one bounded mbarrier wait
 * that nothing completes, with at most `polls` polls (1 .. 2^24, the limit
 * of the transform kernels' waits), as when a kernel's bulk copy never
 * lands; afterwards lmc_status reads LMC_ETIMEOUT (the handle's status word
 * stays set: use a handle made for the check).  No counterpart in the
 * reference, which has no device waits. */
int lmc_wait_selftest(lmc_handle *h, unsigned polls);
const char *lmc_strerror(int code);

/* The handle's CUDA stream (cudaStream_t as void*) and device pointers of
 * the state, for zero-copy use by a host framework. */
void *lmc_stream(lmc_handle *h);
int lmc_state_device_ptrs(lmc_handle *h, double **vor, double **phi,
                          double **psi, double **scal);

/* Per-kernel timing with CUDA events on the handle's stream.  After
 * lmc_profile_start every lmc_step records an event before each kernel;
 * lmc_profile_read synchronises, returns the summed milliseconds and the
 * launch counts per kernel id and stops recording.  Kernel ids:
 *   0 lapv (Lapvdvhom), 1 assemble (rho u_i), 2 tder (T derivatives),
 *   3 zinv (inverse z transforms), 4 xphys (x transforms + products),
 *   5 zfwd (direct z transforms), 6 post1 (N_i), 7 post2 (vorticity,
 *   RHS, RK3 update), 8 psi (solvepsi + 00 modes), 9 memsets,
 *   10 statistics (lmc_stats_step). */
int lmc_profile_start(lmc_handle *h);
int lmc_profile_read(lmc_handle *h, int nk, double *ms, int *count);

/* Serving helpers (no counterpart in the reference, which runs one case per
 * MPI job).
 * lmc_use_graphs: lmc_step replays one CUDA graph per RK3 step (the default,
 *   on) or enqueues the kernels one by one (off).  The first step after a
 *   load and steps run while profiling always enqueue directly.
 * lmc_query: 1 when all work enqueued on the handle's stream has finished,
 *   0 while it runs, < 0 on error (never blocks).
 * lmc_device_bytes: device memory held by the handle.
 * lmc_footprint: device bytes lmc_create would allocate for p (0 for an
 *   unsupported grid), for admission control before creating a case. */
/* lmc_launches_per_step: kernels one RK3 step launches on this handle.
 * lmc_y_family: 1 when the handle runs the mode-parallel y kernels (one
 *   thread per (kx,kz) mode; chosen for grids with >= 16384 modes, or by
 *   LMC_YPATH=mode|warp in the environment at lmc_create), 0 for the
 *   warp-per-mode kernels. */
int lmc_launches_per_step(lmc_handle *h);
int lmc_y_family(lmc_handle *h);
int lmc_use_graphs(lmc_handle *h, int on);
int lmc_query(lmc_handle *h);
size_t lmc_device_bytes(lmc_handle *h);
size_t lmc_footprint(const lmc_params *p);

/* Statistics and spectra on the device: what the reference accumulates
 * while istati = 1 (addstats1 cross.f:1981-2064 and addstats2
 * cross.f:2070-2290 at the first substep, cross.f:578-585 and 794-812; the
 * physical sums of phys2 cross.f:1583-1607), with resetstats
 * (escru.f:485-580) and the data writestats writes (escru.f:276-484).
 * lmc_stats_reset: zero every accumulator, nacum and nacumsp, and set the
 *   nsp spectra planes jsp (1-based y indices: the reference's jsptot,
 *   main.f:698-703) and the exponent sigma of mu/mu0 = T^sigma (main.f:570
 *   sets 0).  Allocates the statistics buffers on first use (3 spectral
 *   FP64 fields and the accumulators).  LMC_EINVAL for the 2014 variant.
 * lmc_stats_step: nsteps RK3 steps like lmc_step that also accumulate at
 *   their first substep (five extra kernels); nacum and nacumsp grow by one
 *   per step (cross.f:800-801).  Steps taken with lmc_step accumulate
 *   nothing, as with istati = 0.
 * lmc_stats_read: synchronises and copies out (NULL skips)
 *   prof[33*my]  profile q of row j at prof[q*my + j], raw (writestats
 *                multiplies the last eleven by 1/(mgalx*mgalz)), in the
 *                order of the .sta record (escru.f:381-402): um vm wm rum
 *                rvm rwm Tm w1m w2m w3m them up vp wp uvr uwr vwr w1p w2p
 *                w3p Tp ep ruu ruv ruw rvv rvw rww rhom thep theup mum num
 *   spec[nplanes*12*nsp*(nz1+1)] the spectra in the order of the .spe plane
 *                records (escru.f:445-448): kx plane, then field (u v w
 *                uv_re uv_im o1 o2 o3 rhou rhov rhow T), then spectra
 *                plane, then |kz| = 0..nz1 fastest (FP64 sums; the
 *                reference sums in real*4)
 *   uner[9]      the nine hy-weighted energies of the last accumulating
 *                step (cross.f:2207-2210; the .cf writes their square roots)
 *   counts[2]    nacum, nacumsp
 *   clear_spectra != 0 then zeroes the spectra and nacumsp, as writestats
 *   does after writing them (escru.f:466-477). */
int lmc_stats_reset(lmc_handle *h, int nsp, const int *jsp, double sigma);
int lmc_stats_step(lmc_handle *h, int nsteps);
int lmc_stats_read(lmc_handle *h, double *prof, double *spec, double *uner,
                   int *counts, int clear_spectra);

/* Seeded initial condition (host only, no GPU): the structure of the
 * reference generator trunk/initloma3/src/main.f:95-609 with a
 * counter-based PRNG keyed by seed.  Mean profiles rho00 = 1 +
 * (s-1)/(s+1) tanh(-y/(2 dm0)), T00 = 1/rho00, rho u00 = rho00 u0
 * tanh(y/(2 dm0)); solenoidal noise on 1 <= |k| <= nkmax (mode-index
 * units) windowed by exp(-(y/swin)^2), scaled to rms amp at y = 0. */
typedef struct lmc_ic_params {
  double s;     /* density ratio rho_bot/rho_top = T_top/T_bot */
  double u0;    /* mean velocity amplitude (reference sign: negative) */
  double dm0;   /* initial thickness scale */
  double amp;   /* rms of the perturbation velocity at y = 0 */
  double swin;  /* y window width */
  int nkmax;    /* largest |k| (mode-index units) carrying noise */
  int nymax;    /* number of random y-harmonics per mode */
  unsigned long long seed;
} lmc_ic_params;
int lmc_make_ic(const lmc_params *p, const double *y, const lmc_ic_params *ic,
                double *vor, double *phi, double *psi, double *scal,
                double *u00, double *v00, double *w00);

/* Single-operator entry points on device buffers in the reference layout
 * (all nplanes*mz modes at once), on the handle's stream:
 *   op 1: deryr2   (cfdiff.f:518-601)   out = d in/dy
 *   op 2: deryyr2  (cfdiff.f:735-797)   out = d2 in/dy2
 *   op 3: Lapvdvhom (laps.f:319-477)    out = v, out2 = dv/dy
 *   op 4: solvepsi  (laps.f:580-730)    out = psi
 * Used by the parity tests of the y-kernels. */
int lmc_op_y(lmc_handle *h, int op, const double *in_dev, double *out_dev,
             double *out2_dev);
/* The same operators as dense my x my matrices (column j = the operator
 * applied to e_j; d/dy and d2/dy2 do not depend on the mode) applied to all
 * modes as one GEMM on the tensor cores (cuBLAS): op 1 (deryr2) or 2
 * (deryyr2); method 1 FP64 (DGEMM), method 2 3xTF32 (hi/lo split of both
 * operands, three TF32 products accumulated in FP32).  Reference layout as
 * lmc_op_y.  The dense matrices and the GEMM workspace (about 3 x 4 bytes
 * per point) are made on first use and freed with the handle.  An
 * alternative to the banded solves, no counterpart in the reference. */
int lmc_op_y_dense(lmc_handle *h, int op, int method, const double *in_dev, double *out_dev);
/* Autotuner of the y operator op (1 or 2) on this grid: times, on the
 * handle's stream with CUDA events (best of three), the banded solve of the
 * substep (as lmc_op_y) and both dense methods on the current Omega_y, and
 * their relative L2 difference from the banded result.  out[6]: banded ms,
 * FP64-GEMM ms, 3xTF32 ms, FP64-GEMM error, 3xTF32 error, choice (0 banded,
 * 1 FP64 GEMM, 2 3xTF32: the fastest within 1e-12 for the FP64 path, 1e-6
 * for the mixed forms).  Uses the FP64 staging buffers of the handle; run
 * between steps. */
int lmc_yop_tune(lmc_handle *h, int op, double *out);
/* Compact first y-derivative (the operator of op 1 above) for callers that
 * may not allocate device memory: drivers with a fixed device-memory
 * budget, or time loops that cannot afford the device-wide synchronisation
 * of cudaFree.  It has no counterpart in the reference.  It takes npencil
 * complex pencils of my points each (y fastest, re/im interleaved) at
 * in_dev and writes d/dy to out_dev on `stream` (a cudaStream_t; NULL for
 * the default stream).  in_dev and out_dev must be 16-byte aligned and must
 * not overlap.  Its operator tables live in one fixed 256 KiB device array
 * per device (no cudaMalloc/cudaFree): my <= 544, larger returns
 * LMC_EINVAL.  The array is shared by all calls and overwritten by each;
 * calls that overlap on the GPU race on it.  The first call in a CUDA
 * context takes the array's address and should precede any stream capture;
 * while `stream` is being captured the call returns LMC_EINVAL (its table
 * upload reads a host buffer that is released on return). */
int lmc_deryr2_noalloc(int my, const double *y, int npencil,
                       const double *in_dev, double *out_dev, void *stream);

/* y-metrics of a mesh, host only (no device needed): fmap = 1/(dy/deta)
 * by the compact first-derivative scheme (cfdiff.f:912-937, the fmap the
 * reference writes into restart record 1, escru.f:130-132), and the mesh
 * weights hy and trp of main.f:689-696.  Any output pointer may be NULL.
 * Returns LMC_EINVAL for my < 9. */
int lmc_y_metrics(int my, const double *y, double *fmap, double *hy, double *trp);
#ifdef __cplusplus
}
#endif
#endif
