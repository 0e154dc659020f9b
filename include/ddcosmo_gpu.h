/*
 * ddcosmo_gpu.h -- C ABI of the B200 ddCOSMO solver.
 *
 * Every entry point is a drop-in for one routine of the Fortran reference
 * (filippolipparini/ddPCM).  The reference keeps its state in module globals
 * (ddcosmo.f90:87-127); here that state lives in an opaque context, so several
 * molecules can be set up side by side.  Arrays cross the boundary as FP64 in
 * exactly the reference's column-major shapes (X(nylm,nsph) is
 * X[isph*nylm + lm], ccav(3,ncav) is ccav[3*ic + k], ...), by plain pointer.
 * By default the pointers are host memory and each call is synchronous, like
 * the reference; with ddc_params.device_pointers = 1 they are device memory of
 * the context's GPU and no host<->device copy happens.
 *
 * Every function returns a status (DDC_OK = 0).  Where the reference prints
 * and calls `stop`, the library returns an error code instead.
 */
#ifndef DDCOSMO_GPU_H
#define DDCOSMO_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DDC_OK 0
#define DDC_ERR_PARAM 1        /* invalid argument or parameter */
#define DDC_ERR_STATE 2        /* call order (e.g. cosmo before init) */
#define DDC_ERR_CUDA 3         /* CUDA runtime error */
#define DDC_ERR_NOMEM 4        /* device allocation failed */
#define DDC_ERR_NOCONV 5       /* Jacobi/DIIS hit max_iter (cosmo.f90:188-200) */
#define DDC_ERR_UNSUPPORTED 6  /* lmax outside the compiled range, or a problem beyond
                                * 32-bit indexing (nsph*ngrid or the triple count
                                * at or above 2^31) */
#define DDC_ERR_NUMERIC 7      /* NaN/Inf in a stage output */
#define DDC_ERR_CAPACITY 8     /* problem larger than the fixed scratch of ddc_efld_noalloc */

/* precision modes */
#define DDC_PREC_FP64 0   /* every stage in FP64 */
#define DDC_PREC_MIXED 1  /* FP32 operator inside FP64 iterative refinement */

/* initial guess for the solves */
#define DDC_GUESS_REFERENCE 0 /* facl * rhs, as cosmo.f90:136-138 / 174-176 */
#define DDC_GUESS_ZERO 1      /* zero vector */
#define DDC_GUESS_USER 2      /* the caller's sigma on entry */
#define DDC_GUESS_LEARNED 3   /* facl * rhs plus the correction predicted by the
                               * context's guess model (ddc_set_guess_model);
                               * ddc_energy_forces and ddc_batch_energy_forces */

#define DDC_MAX_LMAX 12

typedef struct ddc_ctx ddc_ctx;
typedef struct ddc_guess ddc_guess;

/* Control parameters: the reference's Input.txt scalars (main.f90:129-136,
 * ddcosmo.f90:106-107) plus solver knobs that the reference hard-codes
 * (ndiis=25 ddcosmo.f90:87, n_iter=200 cosmo.f90:81). */
typedef struct {
  int lmax;            /* max angular momentum, 0..DDC_MAX_LMAX */
  int ngrid;           /* requested Lebedev size; snapped like ddinit */
  int iconv;           /* tolerance 10^-iconv on the increment H-norm */
  int igrad;           /* 1: prepare the force intermediates (zi) */
  double eps;          /* solvent dielectric constant */
  double eta;          /* switch-function regularisation */
  int iprint;          /* >0: print the iteration log like jacobi_diis */
  int max_iter;        /* 200 in the reference */
  int ndiis;           /* 25 in the reference; 0 disables DIIS (the FP32 inner
                        * solves of DDC_PREC_MIXED keep at most 15) */
  int precision;       /* DDC_PREC_* */
  int guess;           /* DDC_GUESS_* */
  int device;          /* CUDA device ordinal */
  int device_pointers; /* 0: host arrays, 1: device arrays */
  void* stream;        /* cudaStream_t to run on; NULL: the context's own */
  int timing;          /* 1: time each stage with CUDA events (ddc_stage_times) */
  int pair_solves;     /* 1 (default): ddc_energy_forces solves the direct and
                        * adjoint systems together, one fused pass over the
                        * (sphere, point, neighbour) triples giving both L x
                        * and L* s per iteration; 0: one after the other as in
                        * the reference.  Same iterates either way. */
} ddc_params;

/* Solver report of one cosmo call (replaces the iprint log and the
 * non-convergence stop of cosmo.f90:188-221). */
typedef struct {
  int iterations;      /* Jacobi iterations taken (n_iter on return) */
  int converged;       /* 1 if the increment norm fell below 10^-iconv */
  int diis_restarts;   /* singular DIIS systems that reset the history */
  int refinements;     /* outer FP64 refinement steps (mixed precision) */
  double final_norm;   /* last increment norm */
  double seconds;      /* wall time of the solve */
  double norms[256];   /* increment norm of each iteration (first 256) */
} ddc_solve_info;

/* Report of the fused energy+forces flow. */
typedef struct {
  ddc_solve_info direct, adjoint;
  /* seconds; in ddc_energy_forces t_forces covers forces_dd and both field
   * contractions (run side by side on two streams) and t_efld is 0 */
  double t_init, t_mkrhs, t_direct, t_adjoint, t_forces, t_efld;
  int nsph, ncav, nylm, ngrid;
  long long ntriples;  /* (sphere, point, neighbour) triples with t < 1 */
  int npairs;          /* neighbour pairs in the CSR list */
} ddc_run_info;

/* Defaults: lmax 6, ngrid 110, iconv 7, igrad 1, eps 78.3553, eta 0.2,
 * max_iter 200, ndiis 25, FP64, reference guess, device 0, host pointers,
 * paired solves. */
int ddc_default_params(ddc_params* p);

/* Create / destroy a context (module state; memfree ddcosmo.f90:491). */
int ddc_create(const ddc_params* p, ddc_ctx** ctx);
int ddc_destroy(ddc_ctx* ctx);

/* Last error message of this context (static storage, never NULL). */
const char* ddc_last_error(ddc_ctx* ctx);
const char* ddc_status_string(int status);

/* ddinit(n, x, y, z, rvdw)  ddcosmo.f90:159-483.  Coordinates and radii in
 * bohr.  Builds the grid, basis, neighbour list, fi/ui/zi and the cavity. */
int ddc_init(ddc_ctx* ctx, int n, const double* x, const double* y, const double* z,
             const double* rvdw);

/* Module sizes after init: nsph, ncav, nylm and the snapped ngrid. */
int ddc_sizes(ddc_ctx* ctx, int* nsph, int* ncav, int* nylm, int* ngrid);

/* Module arrays read by the host code (main.f90:184-265):
 * ccav(3,ncav), ui(ngrid,nsph), csph(3,nsph), grid(3,ngrid), w(ngrid). */
int ddc_get_ccav(ddc_ctx* ctx, double* ccav);
int ddc_get_ui(ddc_ctx* ctx, double* ui);
int ddc_get_csph(ddc_ctx* ctx, double* csph);
int ddc_get_grid(ddc_ctx* ctx, double* grid, double* w);

/* mkrhs(n, charge, x, y, z, ncav, ccav, phi, nylm, psi)  mkrhs.f90:1-123.
 * phi(ncav) = sum_j q_j / |ccav - x_j|; psi(nylm,n) with psi(1,i)=sqrt(4pi)q_i.
 * ccav may be NULL: the context's own cavity points are used (no copy). */
int ddc_mkrhs(ddc_ctx* ctx, int n, const double* charge, const double* x, const double* y,
              const double* z, int ncav, const double* ccav, double* phi, int nylm, double* psi);

/* cosmo(star, cart, phi, glm, psi, sigma, esolv)  cosmo.f90:1-226.
 * star=0: solve L X = g (g from phi if cart, else glm); returns sigma = X and
 * esolv = 1/2 (eps-1)/eps <X, psi>.  star=1: solve L* S = psi; sigma = S.
 * info may be NULL.  Returns DDC_ERR_NOCONV (with sigma holding the last
 * iterate) where the reference stops. */
int ddc_cosmo(ddc_ctx* ctx, int star, int cart, const double* phi, const double* glm,
              const double* psi, double* sigma, double* esolv, ddc_solve_info* info);

/* forces_dd(n, phi, sigma, s, fx)  forces_dd.f90:1-164: fep * (fdoka + fdokb
 * + fdoga) into fx(3,n) (overwritten). */
int ddc_forces_dd(ddc_ctx* ctx, const double* phi, const double* sigma, const double* s,
                  double* fx);

/* ddmkzeta(s, zeta) ddcosmo.f90:1787-1806 and ddmkxi(s, xi) 1758-1781. */
int ddc_mkzeta(ddc_ctx* ctx, const double* s, double* zeta);
int ddc_mkxi(ddc_ctx* ctx, const double* s, double* xi);

/* efld(nsrc, src, csrc, ntrg, ctrg, ef)  efld.f90:1-116: field of point
 * sources at the targets.  csrc/ctrg may be NULL to mean the context's
 * cavity points (ccav) when the count equals ncav, or its sphere centres
 * (csph) when the count equals nsph. */
int ddc_efld(ddc_ctx* ctx, int nsrc, const double* src, const double* csrc, int ntrg,
             const double* ctrg, double* ef);

/* The main.f90 energy+forces flow in one call (main.f90:164-265): ddinit,
 * mkrhs, direct solve, energy, adjoint solve, forces_dd, ddmkzeta and the two
 * efld contractions.  Inputs: charges and bohr coordinates/radii; outputs
 * esolv (Hartree), sigma = X and s = S (nylm,n), fx(3,n) total forces
 * (Hartree/bohr; any of sigma, s, fx may be NULL).  info may be NULL.
 * With guess = DDC_GUESS_USER, sigma and s are in/out: on entry they hold the
 * initial guesses of the direct and adjoint solves (e.g. the previous
 * frame's solutions of a trajectory) and must not be NULL. */
int ddc_energy_forces(ddc_ctx* ctx, int n, const double* charge, const double* x,
                      const double* y, const double* z, const double* rvdw, double* esolv,
                      double* sigma, double* s, double* fx, ddc_run_info* info);

/* Batched energy+forces for nmol independent molecules in one call.  No
 * counterpart in the reference, which solves one molecule per process; the
 * result for each molecule is that of ddc_energy_forces on it alone.  The
 * spheres of all molecules are concatenated: molecule k owns spheres
 * [off[k], off[k+1]) (off is a host array of nmol+1 offsets, off[0] = 0).
 * Each molecule runs the reference's Jacobi/DIIS with its own history and
 * convergence test; all molecules share each kernel launch.  Outputs:
 * esolv[nmol] (host), fx(3, off[nmol]) (may be NULL), iters[2*nmol]
 * (direct, adjoint per molecule; host, may be NULL).  With precision
 * DDC_PREC_MIXED each molecule runs the mixed refinement of ddc_cosmo (FP64
 * residual and stop test, FP32 inner solves); iters then counts each
 * molecule's inner iterations. */
int ddc_batch_energy_forces(ddc_ctx* ctx, int nmol, const int* off, const double* charge,
                            const double* x, const double* y, const double* z,
                            const double* rvdw, double* esolv, double* fx, int* iters,
                            ddc_run_info* info);

/* The operators the solver iterates (matvec.f90): y = off-diagonal L x
 * (lx, :94), y = off-diagonal L* x (lstarx, :161), y = D^-1 x (ldm1x, :246)
 * and the increment norm hnorm (:281).  x, y are (nylm,nsph).  In a
 * DDC_PREC_MIXED context lx, lstarx and lx_lstarx apply the FP32 operators of
 * the inner solves (FP32 sums, tensor-core split-TF32 projection and
 * expansion), read and written as FP64; otherwise everything is FP64. */
int ddc_lx(ddc_ctx* ctx, const double* x, double* y);
int ddc_lstarx(ddc_ctx* ctx, const double* x, double* y);
int ddc_ldm1x(ddc_ctx* ctx, const double* x, double* y);
int ddc_hnorm(ddc_ctx* ctx, const double* x, double* norm);

/* y = off-diagonal L x and z = off-diagonal L* s from one fused pass over the
 * (sphere, point, neighbour) triples (the operator step of the paired
 * solves).  No reference counterpart: it equals ddc_lx(x) and ddc_lstarx(s)
 * (matvec.f90:94, :161) up to rounding, in the context's precision. */
int ddc_lx_lstarx(ddc_ctx* ctx, const double* x, double* y, const double* s, double* z);

/* RHS of the direct equation from phi (wghpot + intrhs, cosmo.f90:104-117). */
int ddc_rhs(ddc_ctx* ctx, const double* phi, double* g);

/* Number of kernel launches issued by this context since creation. */
long long ddc_launch_count(ddc_ctx* ctx);

/* Per-stage device time, measured with CUDA events on the context's stream
 * when ddc_params.timing = 1.  No reference counterpart (the reference only
 * times whole solves, cosmo.f90:84-85, 202).  ms/calls have
 * ddc_stage_count() entries; ddc_stage_name(k) names stage k. */
int ddc_stage_count(void);
const char* ddc_stage_name(int k);
int ddc_stage_times(ddc_ctx* ctx, double* ms, long long* calls);
int ddc_reset_stage_times(ddc_ctx* ctx);
/* Restrict the stage timers to the stages whose bit (1 << k) is set in mask
 * (default: every stage).  Each timed stage records two events per call, so
 * timing only the stage of interest keeps the host work between a solver
 * step's reductions and its next launches small. */
int ddc_set_timed_stages(ddc_ctx* ctx, unsigned int mask);

/* Measured FP64 FMA throughput of the device (GFLOP/s, 2 flops per FMA),
 * from a register-resident FMA kernel timed with CUDA events.  No
 * reference counterpart: it is the roofline denominator of the FP64-bound
 * kernels. */
int ddc_fp64_peak(int device, double* gflops);
/* The same for FP32 FMA: the denominator of the FP32 operator kernels of the
 * mixed-precision path. */
int ddc_fp32_peak(int device, double* gflops);

/* Learned initial guess.  No counterpart in the reference, which always
 * starts from facl * rhs (cosmo.f90:136-138, 174-176); the model only moves
 * the start, the Jacobi/DIIS solve and its stop test are unchanged.  A model
 * is a per-sphere network (features -> `hidden` x 3 ReLU layers -> the
 * corrections of X0 and S0), BF16 weights with FP32 accumulation, on one GPU.
 * Features and targets are DEVICE arrays of the model's GPU, one row per
 * sphere: feat[n][nfeat], target[n][nout] (FP32). */
int ddc_guess_create(int lmax, int hidden, int device, ddc_guess** m);
int ddc_guess_destroy(ddc_guess* m);
const char* ddc_guess_last_error(ddc_guess* m);
/* row widths and the length of the parameter vector of get/set_params */
int ddc_guess_sizes(ddc_guess* m, int* nfeat, int* nout, long long* nparams);
/* parameters as one FP32 host vector: weights, biases, then the feature
 * means, the feature inverse deviations and the output scales */
int ddc_guess_get_params(ddc_guess* m, float* host);
int ddc_guess_set_params(ddc_guess* m, const float* host);
int ddc_guess_init_random(ddc_guess* m, unsigned long long seed);
/* standardisation statistics from a training set of n rows */
int ddc_guess_fit_scaling(ddc_guess* m, const float* feat, const float* target, long long n);
/* one pass over n rows (in the order of the device int array `order`, or
 * as stored if NULL) in mini-batches of `batch`, Adam with step lr; *loss is
 * the mean squared error of the scaled outputs over the pass */
int ddc_guess_train_epoch(ddc_guess* m, const float* feat, const float* target, const int* order,
                          long long n, int batch, float lr, double* loss);
/* scaled outputs out[n][nout] (multiply by the output scales for the
 * corrections) */
int ddc_guess_predict(ddc_guess* m, const float* feat, float* out, long long n);
/* training rows from the context's last ddc_energy_forces or
 * ddc_batch_energy_forces call: features (rhs, psi, radii, distance
 * histogram) and targets (solution minus facl * rhs, for X then S) of every
 * sphere, written to device arrays of the context's GPU */
int ddc_guess_features(ddc_ctx* ctx, float* feat);
int ddc_guess_targets(ddc_ctx* ctx, float* target);
/* the model used by DDC_GUESS_LEARNED (same lmax and device; NULL detaches) */
int ddc_set_guess_model(ddc_ctx* ctx, ddc_guess* m);

/* efld without any device allocation.  No counterpart in the reference: it
 * serves host programs that own all of the GPU's memory (a QM/MM or MD code
 * that reserves the HBM for its own pool at start-up), for which a cudaMalloc
 * issued by the library mid-step would fail or stall the device.  Same
 * result as ddc_efld (efld.f90:1-116); every pointer is DEVICE memory of
 * `device`: src(nsrc), csrc(3,nsrc), ctrg(3,ntrg), ef(3,ntrg).  The kernels
 * are queued on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * the call returns without waiting; ef is valid once that stream reaches it.
 * Scratch is a fixed 8 MiB array compiled into the library (held on every GPU
 * that loads it until exit): ntrg is limited to 349,525 targets, larger
 * problems return DDC_ERR_CAPACITY (use ddc_efld).  `stream` must belong to
 * `device` (else DDC_ERR_PARAM).  The first call on a device does a one-time
 * set-up: CUDA loads this library's device code (the array included) lazily,
 * so that call may allocate module memory on the device, and it resolves the
 * array's device address.  Callers whose pool will take the whole GPU make
 * that first call with ntrg = 0 at start-up, before the pool claims the
 * memory and outside any stream capture; it does the set-up and nothing
 * else.  All calls share the array, so calls whose work overlaps on the GPU
 * race; order them on one stream. */
int ddc_efld_noalloc(int device, int nsrc, const double* src, const double* csrc, int ntrg,
                     const double* ctrg, double* ef, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DDCOSMO_GPU_H */
