/*
 * pincflow_poisson.h -- C ABI of the B200 (sm_100a) semi-implicit pressure
 * Poisson solver that replaces PinCFlow.jl's PoissonSolver hot path.
 *
 * The entry points mirror the reference's Julia functions so that a Julia
 * method (the package extension ext/PinCFlowGPUExt.jl of the binding) can
 * `ccall` them with the arrays it already owns:
 *
 *   pcf_solve              <- solve_poisson!(state, dt, rayleigh_factor, tolref)
 *                             src/PoissonSolver/solve_poisson!.jl:39-75
 *                             (operator assembly + BiCGSTAB + unscaling into dpip)
 *   pcf_compute_operator   <- compute_operator!(state, dt, rayleigh_factor)
 *                             src/PoissonSolver/compute_operator!.jl:40-1606
 *   pcf_apply_operator     <- apply_operator!(sin, ls, Total() | Horizontal(), state)
 *                             src/PoissonSolver/apply_operator!.jl:48-479
 *   pcf_apply_preconditioner <- apply_preconditioner!(sin, sout, state)
 *                             src/PoissonSolver/apply_preconditioner!.jl:40-124
 *   pcf_bicgstab           <- apply_bicgstab!(state, tolref)
 *                             src/PoissonSolver/apply_bicgstab!.jl:24-150
 *   pcf_global_dot         <- compute_global_dot_product(a, b, state)
 *                             src/MPIOperations/compute_global_dot_product.jl:22-36
 *   pcf_compute_lhs        <- compute_lhs!(state)
 *                             src/PoissonSolver/compute_lhs!.jl:68-223
 *   pcf_correct            <- correct!(state, dt, rayleigh_factor) after the dpip fill
 *                             src/PoissonSolver/correct!.jl:164-385
 *   pcf_implicit_predictor_device
 *                          <- update!(state, dt, U/V/W/RhoP, RHS(), Implicit(), rf)
 *                             src/Update/update!.jl:632-1336 (Implicit methods)
 *   pcf_implicit_step      <- implicit_integration!(state, dtstage, ...) without output
 *                             src/Integration/implicit_integration!.jl:40-80
 *   pcf_set_grid / pcf_set_background
 *                          <- the State fields these read: Grid.jac, Grid.met
 *                             (src/Types/FoundationalTypes/Grid.jl:243-313) and
 *                             Atmosphere.pbar/rhobar/thetabar/n2
 *                             (src/Types/FoundationalTypes/Atmosphere.jl:278-323)
 *   pcf_params             <- PoissonNamelist
 *                             (src/Types/NamelistTypes/PoissonNamelist.jl:38-66)
 *                             plus SpongeNamelist.damp_horizontal_wind_on_rhs
 *
 * Array conventions are the reference's: FP64, column-major (x fastest, then
 * y, then z).  "Haloed" arrays have (nx + 2 nbx, ny + 2 nby, nz + 2 nbz)
 * elements like every PinCFlow field; "interior" arrays have (nx, ny, nz)
 * elements like Poisson.rhs / Poisson.solution.  The 25 operator planes are
 * stored one after another (plane stride nx*ny*nz) in the field order of the
 * reference Tensor struct (src/Types/PoissonTypes/Tensor.jl:70-96), given by
 * enum pcf_coef below.  `met` is passed as its three used planes, met[:,:,:,1,3],
 * met[:,:,:,2,3] and met[:,:,:,3,3], which are contiguous blocks of the
 * reference's 5-D array.
 *
 * Single GPU, single MPI rank: x and y are periodic, z has solid walls.
 *
 * Host pointers are read during the call only and never retained.  Entry
 * points whose name ends in _device take device pointers (resident in the
 * handle's GPU memory) and run on the handle's stream.
 *
 * Return codes: 0 on success, a negative PCF_E* code otherwise.
 * Non-convergence is not an error code: it sets result->errflag = 1 and
 * result->niter = poisson_iterations, as the reference returns
 * (true, niter) (apply_bicgstab!.jl:146-149).
 */
#ifndef PINCFLOW_POISSON_H
#define PINCFLOW_POISSON_H

#ifdef __cplusplus
extern "C" {
#endif

#define PCF_ABI_VERSION 1

enum pcf_status {
    PCF_OK = 0,
    PCF_EINVAL = -1,      /* bad argument (dt == 0: solve_poisson!.jl:52-54 raises) */
    PCF_ENOMEM = -2,      /* device allocation failed */
    PCF_ECUDA = -3,       /* CUDA runtime error */
    PCF_ENOTREADY = -4,   /* grid or background not set */
    PCF_EBREAKDOWN = -5,  /* BiCGSTAB breakdown: a zero or non-finite scalar */
    PCF_ENONFINITE = -6,  /* non-finite value in the inputs or the residual */
    PCF_ENODEVICE = -7,   /* no usable sm_100 device */
    PCF_ERANGE = -8       /* size beyond a documented limit */
};

enum pcf_model {
    PCF_MODEL_BOUSSINESQ = 0,
    PCF_MODEL_PSEUDO_INCOMPRESSIBLE = 1,
    PCF_MODEL_COMPRESSIBLE = 2
};

/* Operator plane order = field order of the reference Tensor struct. */
enum pcf_coef {
    PCF_AC = 0, PCF_AL, PCF_AR, PCF_AB, PCF_AF, PCF_AD, PCF_AU,
    PCF_ALD, PCF_ALU, PCF_ARD, PCF_ARU, PCF_ABD, PCF_ABU, PCF_AFD, PCF_AFU,
    PCF_ADD, PCF_AUU, PCF_ALDD, PCF_ALUU, PCF_ARDD, PCF_ARUU, PCF_ABDD, PCF_ABUU,
    PCF_AFDD, PCF_AFUU, PCF_NCOEF
};

enum pcf_precision {
    PCF_PRECISION_FP64 = 0,   /* the reference's arithmetic: FP64 everywhere */
    PCF_PRECISION_MIXED = 1,  /* FP32 inner BiCGSTAB inside FP64 iterative refinement */
    PCF_PRECISION_FP32 = 2    /* component entry points only: FP32 operator copy */
};

enum pcf_residual {
    PCF_RESIDUAL_RECURSIVE = 0, /* reference test: RMS of the recursive residual */
    PCF_RESIDUAL_TRUE = 1       /* FP64 true residual b - A x decides convergence */
};

enum pcf_operator_mode { PCF_TOTAL = 0, PCF_HORIZONTAL = 1 };

typedef struct {
    int nx, ny, nz;      /* interior sizes (x_size, y_size, z_size on one rank) */
    int nbx, nby, nbz;   /* halo widths of the caller's haloed arrays (reference: 3) */
    int model;           /* enum pcf_model (AtmosphereNamelist.model) */
    int device;          /* CUDA device ordinal */
} pcf_dims;

typedef struct {
    /* PoissonNamelist (PoissonNamelist.jl:48-66 defaults) */
    double tolerance;              /* 1e-8 */
    int poisson_iterations;        /* 1000 */
    int preconditioner;            /* 1 */
    double dtau;                   /* 1.0 */
    int preconditioner_iterations; /* 2 */
    int tolerance_is_relative;     /* 0 */
    /* SpongeNamelist */
    int damp_horizontal_wind_on_rhs; /* 0 */
    /* Additions without a reference counterpart; defaults reproduce the reference. */
    int precision;                 /* PCF_PRECISION_FP64 */
    int residual;                  /* PCF_RESIDUAL_RECURSIVE */
    double inner_tolerance;        /* mixed: FP64 reliable update each time the FP32 residual fell by this factor (1e-2) */
    int max_refinements;           /* mixed: cap on restarts of the FP32 iteration after a breakdown (5) */
    int learned;                   /* mixed, bit set: 1 learned warm start, 2 learned preconditioner stage (0) */
    int check_interval;            /* iterations per graph batch between host checks of the status word (4) */
    int restart_interval;          /* mixed: restart the Krylov recurrences at every n-th reliable update (1; 0: never) */
    int multigrid;                 /* mixed: 0: the reference preconditioner; 1: horizontal aggregation multigrid
                                      V-cycle with the reference line relaxation as smoother on every level (0) */
    double mg_dtau;                /* multigrid: pseudo-time step of the smoother, all levels (2.5) */
    int mg_coarse_iterations;      /* multigrid: smoothing steps on the coarsest level (4) */
    int mg_min_columns;            /* multigrid: a level with at most this many columns is the coarsest (16) */
    int autotune;                  /* 1: time the stencil tile shapes of every new grid size on first use and keep
                                      the fastest (process-wide table, pcf_autotune_entries); 0: fixed heuristic (0) */
    int mg_operator_bf16;          /* multigrid: 1: the V-cycle's residual and smoothing stencils on the finest and
                                      the first coarse level read BF16 copies of their operators (half their bytes;
                                      the Krylov operator, the coarser levels and the FP64 true residual are
                                      unchanged); 0: the FP32 copies.  On levels 128 or more cells wide with nx a
                                      multiple of 8 those stencils load the BF16 tiles into shared memory by TMA
                                      (same arithmetic, same results); the learned preconditioner stage
                                      (learned & 2) runs the same V-cycle, which its training pairs come from (1) */
    int mg_fused_coarse;           /* multigrid: the levels of at most 1024 columns (nz <= 256) as ONE launch
                                      per cycle: a cluster of 16 thread blocks with the hardware cluster barrier
                                      between the steps (column solves by warp scans).  1: on; 0: one kernel per
                                      step as on the finer levels; -1 (default): on in pcf_ensemble_solve_device
                                      (whose members' launches then leave the other SMs to one another), off in
                                      single solves (measured slower there) */
    int mg_smoother_fp8;           /* multigrid with mg_operator_bf16: the finest level's pseudo-time steps read
                                      an FP8 E4M3 copy of their 22 planes (each plane scaled by a power of 2 so
                                      that its largest value lands in [64, 128)), a quarter of the FP32 planes'
                                      bytes; the residual keeps the BF16 copy.  Off by default (0): measured
                                      slower at 512 x 512 x 192, where widening FP8 to FP32 runs on the
                                      conversion pipe and takes about as long as the launch itself */
} pcf_params;

typedef struct {
    int errflag;           /* 1 when not converged, as the reference's errflag */
    int niter;             /* BiCGSTAB iterations (summed over refinement sweeps) */
    int nrefine;           /* FP64 refinement sweeps (mixed precision) */
    int status;            /* PCF_OK or PCF_EBREAKDOWN / PCF_ENONFINITE */
    double residual;       /* final relative residual as tested (recursive or true) */
    double true_residual;  /* FP64 RMS(b - A x) / RMS(b) */
    double b_norm;         /* RMS of the initial residual */
    double ms_upload;      /* host -> device copies of rho, betar, p (the right-hand side's runs on a second
                              stream, concurrent with the assembly) */
    double ms_assemble;    /* operator assembly + preconditioner factors */
    double ms_solve;       /* Krylov iterations */
    double ms_download;    /* device -> host copies */
    double ms_total;
} pcf_result;

typedef struct pcf_handle pcf_handle;

/* Grids of at most 2048 cells are solved by the reference FP64 BiCGSTAB in a
 * single thread block (all vectors in shared memory), whatever precision,
 * multigrid and learned say: the solve is launch-latency bound there.
 * Fills *p with the reference defaults. */
int pcf_params_default(pcf_params *p);

/* Allocates all device memory of one solver instance (one `State`).
 * PCF_EINVAL unless nx, ny >= 1, nz >= 4, nbx, nby >= 1, nbz >= 2;
 * PCF_ERANGE for 2^31 or more haloed cells. */
int pcf_create(pcf_handle **h, const pcf_dims *dims);
int pcf_destroy(pcf_handle *h);
const char *pcf_strerror(int code);

/* Grid: non-dimensional spacings and haloed jac, met13, met23, met33. */
int pcf_set_grid(pcf_handle *h, double dx, double dy, double dz, const double *jac,
                 const double *met13, const double *met23, const double *met33);

/* Background: haloed pbar, rhobar, n2; thetabar is read for the Compressible
 * model only (may be NULL otherwise). */
int pcf_set_background(pcf_handle *h, const double *pbar, const double *rhobar,
                       const double *thetabar, const double *n2);

/* solve_poisson!: assembles the operator from the haloed predictand rho, the
 * haloed sponge coefficient betar and (Compressible only, else NULL) the
 * haloed predictand p, solves A s = rhs (interior rhs from compute_lhs!) and
 * writes dpip = s / sqrt(pbar^2/rhobar) / dt into the interior of the haloed
 * array dpip (halo cells untouched).  tolref is compute_lhs!'s return value. */
int pcf_solve(pcf_handle *h, const double *rhs, const double *rho, const double *betar,
              const double *p, double dt, double rayleigh_factor, double tolref,
              const pcf_params *prm, double *dpip, pcf_result *res);

/* Same with device-resident inputs and output (haloed layouts as above). */
int pcf_solve_device(pcf_handle *h, const double *d_rhs, const double *d_rho,
                     const double *d_betar, const double *d_p, double dt,
                     double rayleigh_factor, double tolref, const pcf_params *prm,
                     double *d_dpip, pcf_result *res);

/* compute_operator!: fills the handle's operator; if coef is not NULL the 25
 * FP64 planes are also copied to the host (25 * nx*ny*nz doubles). */
int pcf_compute_operator(pcf_handle *h, const double *rho, const double *betar, const double *p,
                         double dt, double rayleigh_factor, int damp_horizontal_wind_on_rhs,
                         double *coef);

/* Loads 25 FP64 operator planes (Tensor order) instead of assembling them,
 * as if compute_operator! had produced them. */
int pcf_set_operator(pcf_handle *h, const double *coef);

/* apply_operator!: ls = A sin (mode PCF_TOTAL) or its horizontal part
 * (PCF_HORIZONTAL); interior arrays.  precision PCF_PRECISION_FP64 uses the
 * FP64 planes, PCF_PRECISION_FP32 the FP32 copy (inputs rounded to FP32). */
int pcf_apply_operator(pcf_handle *h, const double *sin_, double *ls, int mode, int precision);

/* apply_preconditioner!: sout = M sin with prm->dtau and
 * prm->preconditioner_iterations; interior arrays. */
/* compute_lhs! (src/PoissonSolver/compute_lhs!.jl:68-160 Boussinesq /
 * PseudoIncompressible, :162-223 Compressible): rhs (interior, nx*ny*nz) =
 * the scaled divergence of the staggered winds u, v, w (haloed arrays of the
 * reference's predictands; mass fluxes in the Compressible model) and tolref
 * = RMS(rhs) / RMS(bu, bv, bw).  heating (interior, or NULL for zero) is the
 * Compressible model's compute_volume_force(state, i, j, k, P()); the other
 * models ignore it.  A zero divergence gives tolref = 1.  Needs the grid and
 * background.  Returns PCF_ENONFINITE where the reference raises (or on
 * non-finite sums).  The _device variant takes device pointers (rhs may be
 * the input of pcf_solve_device). */
int pcf_compute_lhs(pcf_handle *h, const double *u, const double *v, const double *w,
                    const double *heating, double *rhs, double *tolref);
int pcf_compute_lhs_device(pcf_handle *h, const double *d_u, const double *d_v, const double *d_w,
                           const double *d_heating, double *d_rhs, double *tolref);

/* The corrector after the solve (apply_corrector!.jl:58-61): fills the halo
 * of dpip (periodic x/y, mirrored z: set_*_boundaries_of_field!) and applies
 * correct!(state, dt, rayleigh_factor) (correct!.jl:164-385, with
 * compute_pressure_gradient.jl:108-297): u, v, w, rhop corrected in place,
 * pip += dpip on the interior and one ghost layer.  All arrays haloed; rho,
 * betar and p are those of the handle's last solve.  The _device variant
 * takes device pointers.  pcf_apply_corrector_device runs the whole
 * apply_corrector!(state, dt, rayleigh_factor) (:44-61) on device arrays:
 * compute_lhs!, solve_poisson! (into d_dpip), then the corrector; like the
 * reference it leaves the fields uncorrected when res->errflag is set. */
int pcf_correct(pcf_handle *h, double dt, double rayleigh_factor, int damp_horizontal_wind_on_rhs, double *dpip,
                double *u, double *v, double *w, double *rhop, double *pip);
int pcf_correct_device(pcf_handle *h, double dt, double rayleigh_factor, int damp_horizontal_wind_on_rhs,
                       double *d_dpip, double *d_u, double *d_v, double *d_w, double *d_rhop, double *d_pip);
int pcf_apply_corrector_device(pcf_handle *h, double *d_u, double *d_v, double *d_w, const double *d_rho,
                               double *d_rhop, const double *d_betar, const double *d_p, double *d_pip,
                               const double *d_heating, double dt, double rayleigh_factor, const pcf_params *prm,
                               double *d_dpip, pcf_result *res);

/* The implicit half step around the solve (src/Integration/
 * implicit_integration!.jl:49-77, one rank, no tracers).  All arrays are the
 * reference's haloed FP64 predictands and need nz > nbz.
 *
 * pcf_set_predictand_boundaries_device replaces set_boundaries!(state,
 * BoundaryPredictands()) (src/Boundaries/set_boundaries!.jl:46-60): x and y
 * periodic; in z rho and rhop point-reflected, u, v, pip and p
 * line-reflected, w zero on both walls and point-reflected
 * (set_vertical_boundaries!.jl:185-240).  rho is filled for the
 * PseudoIncompressible and Compressible models (NULL allowed for
 * Boussinesq), p for Compressible (else NULL allowed).
 *
 * pcf_modify_compressible_wind_device replaces modify_compressible_wind!(
 * state, *) (divide = 0) and (state, /) (divide = 1)
 * (src/Integration/modify_compressible_wind!.jl:38-80); a no-op unless the
 * model is Compressible.
 *
 * pcf_implicit_predictor_device replaces implicit_integration!.jl:53-63:
 * save_backups!(state, :w) into d_wold (NULL: handle scratch), the implicit
 * predictor update!(state, dt, U() / V() / W(), RHS(), Implicit(),
 * rayleigh_factor) (src/Update/update!.jl:837-882, :988-1033, :1248-1336),
 * set_boundaries!, update!(..., RhoP(), ...) (:632-728), set_boundaries!.
 * d_dudt, d_dvdt are the WKB momentum tendencies (state.wkb.tendencies) of
 * compute_volume_force.jl:159-206, or both NULL for wkb_mode = NoWKB.
 *
 * pcf_implicit_step_device runs the whole implicit_integration!.jl:49-77
 * without output: modify_compressible_wind!(*), set_boundaries!, the
 * predictor, apply_corrector! (as pcf_apply_corrector_device, d_heating as
 * there), modify_compressible_wind!(/), set_boundaries!.  On res->errflag
 * it returns PCF_OK with the predicted, uncorrected fields (where the
 * reference writes output and raises).  dt == 0 returns PCF_EINVAL.
 * res->ms_total is the device time of the whole step (CUDA events on the
 * handle's stream); the other timings are the solve's.
 * pcf_implicit_step is the same with host arrays (heating interior, wold
 * may be NULL; u, v, w, rho, rhop, pip, p, dpip and wold are written
 * back). */
int pcf_set_predictand_boundaries_device(pcf_handle *h, double *d_rho, double *d_rhop, double *d_u, double *d_v,
                                         double *d_w, double *d_pip, double *d_p);
int pcf_modify_compressible_wind_device(pcf_handle *h, const double *d_p, double *d_u, double *d_v, double *d_w,
                                        int divide);
int pcf_implicit_predictor_device(pcf_handle *h, double dt, double rayleigh_factor, int damp_horizontal_wind_on_rhs,
                                  double *d_u, double *d_v, double *d_w, double *d_rho, double *d_rhop,
                                  double *d_pip, double *d_p, const double *d_betar, const double *d_dudt,
                                  const double *d_dvdt, double *d_wold);
int pcf_implicit_step_device(pcf_handle *h, double dt, double rayleigh_factor, const pcf_params *prm, double *d_u,
                             double *d_v, double *d_w, double *d_rho, double *d_rhop, double *d_pip, double *d_p,
                             const double *d_betar, const double *d_dudt, const double *d_dvdt,
                             const double *d_heating, double *d_wold, double *d_dpip, pcf_result *res);
int pcf_implicit_step(pcf_handle *h, double dt, double rayleigh_factor, const pcf_params *prm, double *u, double *v,
                      double *w, double *rho, double *rhop, double *pip, double *p, const double *betar,
                      const double *dudt, const double *dvdt, const double *heating, double *wold, double *dpip,
                      pcf_result *res);

int pcf_apply_preconditioner(pcf_handle *h, const double *sin_, double *sout,
                             const pcf_params *prm, int precision);

/* Horizontal aggregation multigrid preconditioner of the mixed solve (no
 * reference counterpart; it wraps the reference line relaxation of
 * apply_preconditioner!.jl:40-124 as the smoother of every level).
 * pcf_multigrid_levels builds the hierarchy for the current operator with
 * prm's mg_* settings and returns the level count and (nx, ny, nz) per level
 * (up to cap levels); pcf_multigrid_operator copies the 25 planes of a level
 * (level 0: the assembled FP64 operator); pcf_apply_multigrid applies one
 * V-cycle z = MG(sin) in FP32 (host FP64 arrays, nx*ny*nz). */
int pcf_multigrid_levels(pcf_handle *h, const pcf_params *prm, int cap, int *nlevels, int *dims);
int pcf_multigrid_operator(pcf_handle *h, int level, double *coef);
int pcf_apply_multigrid(pcf_handle *h, const double *sin, double *sout, const pcf_params *prm);

/* Stencil tile autotuner (no reference counterpart).  One entry per device,
 * kernel family and grid size that a solve with pcf_params.autotune = 1 has
 * tuned: the chosen tile (tile_x threads along x, 128 threads per block, vec
 * values per thread) and z-levels per block, with the measured time per
 * launch of the chosen and of the heuristic shape. */
enum {
    PCF_TUNE_TOTAL32 = 0,       /* Total apply, FP32, plain form (multigrid residuals) */
    PCF_TUNE_TOTAL32_DIFF = 1,  /* Total apply, FP32, difference form (Krylov loop) */
    PCF_TUNE_HORIZ32 = 2,       /* Horizontal apply + pseudo-time step, FP32 */
    PCF_TUNE_TOTAL64 = 3,
    PCF_TUNE_HORIZ64 = 4
};
typedef struct {
    int kernel, nx, ny, nz;
    int tile_x, vec, levels;
    double ms_best, ms_default;
} pcf_tune_entry;
int pcf_autotune_entries(pcf_tune_entry *out, int cap, int *count);
int pcf_autotune_clear(void);

/* Ensemble of solver handles (no reference counterpart; the reference runs
 * ensemble members as separate MPI sub-communicators, src/ensemble.jl:40-43).
 * Members are handles on one device with grid and background set; their
 * sizes may differ.  pcf_ensemble_solve_device runs solve_poisson! for every
 * member (arrays of per-member device pointers and scalars, as
 * pcf_solve_device) with the mixed-precision iteration only: after each
 * member's setup on its own stream, every batch of check_interval
 * iterations of all members is one CUDA graph launch.  res has one entry
 * per member.  A handle may belong to one ensemble at a time and must not be
 * used by another thread while the ensemble solves. */
typedef struct pcf_ensemble pcf_ensemble;
int pcf_ensemble_create(pcf_ensemble **e, pcf_handle *const *members, int count);
int pcf_ensemble_destroy(pcf_ensemble *e);
int pcf_ensemble_solve_device(pcf_ensemble *e, const double *const *d_rhs, const double *const *d_rho,
                              const double *const *d_betar, const double *const *d_p, const double *dt,
                              const double *rayleigh_factor, const double *tolref, const pcf_params *prm,
                              double *const *d_dpip, pcf_result *res);
long long pcf_ensemble_launch_count(const pcf_ensemble *e);


/* apply_bicgstab!: solves A s = rhs with the handle's current operator;
 * interior arrays. */
int pcf_bicgstab(pcf_handle *h, const double *rhs, double tolref, const pcf_params *prm,
                 double *solution, pcf_result *res);

/* compute_global_dot_product: deterministic FP64 sum of a[i]*b[i] over the
 * interior (n = nx*ny*nz elements); result in *out. */
int pcf_global_dot(pcf_handle *h, const double *a, const double *b, double *out);

/* Device memory held by the handle, in bytes. */
long long pcf_device_bytes(const pcf_handle *h);

/* Instrumentation (no reference counterpart).  Kernels launched by the handle
 * since creation; per-kernel-class device time measured with CUDA events on
 * the handle's stream while profiling is on.  Launches issued after a
 * BiCGSTAB run converged (which return at once) are not counted.
 * `bytes` is the algorithmic traffic of the counted launches. */
enum pcf_prof_tag {
    PCF_PROF_APPLY32 = 0,   /* Total operator apply, FP32, fused dots */
    PCF_PROF_APPLY64 = 1,   /* Total operator apply, FP64, fused dots / residual */
    PCF_PROF_PSEUDO32 = 2,  /* Horizontal apply + pseudo-time step, FP32 */
    PCF_PROF_PSEUDO64 = 3,
    PCF_PROF_THOMAS32 = 4,  /* column tridiagonal sweeps, FP32 */
    PCF_PROF_THOMAS64 = 5,
    PCF_PROF_UPDATE32 = 6,  /* BiCGSTAB vector updates, FP32 */
    PCF_PROF_UPDATE64 = 7,
    PCF_PROF_ASSEMBLE = 8,  /* operator assembly + factors */
    PCF_PROF_RELIABLE = 9,  /* FP64 true-residual applies of reliable updates: every guarded launch's time,
                               the bytes of the launches that performed an update */
    PCF_PROF_MG = 10,       /* multigrid coarse levels and grid transfers, FP32 */
    PCF_PROF_LEARNED = 11,  /* learned preconditioner stage: residual, network, combination */
    PCF_PROF_PREDICT = 12,  /* implicit predictor with its predictand boundary fills (FP64) */
    PCF_PROF_CORRECT = 13,  /* corrector: dpip boundary fill and correct! (FP64) */
    PCF_PROF_MG_BF16 = 14,  /* V-cycle finest-level residual and smoothing stencils on the BF16 operator copy */
    PCF_PROF_NTAGS = 15
};
long long pcf_launch_count(const pcf_handle *h);
/* Relative recursive residual after each BiCGSTAB iteration of the last
 * solve (refinement sweeps concatenated, relative to the original b); the
 * reference prints only the final value (apply_bicgstab!.jl:124-127).
 * Copies min(cap, *n) entries; *n receives the total count. */
int pcf_residual_history(pcf_handle *h, double *out, int cap, int *n);

/* Test entry point of the learned part's tensor-core GEMM (no reference
 * counterpart): D[M][N] = sum_k A(m,k) B(n,k), BF16 inputs as uint16 bit
 * patterns with A(m,k) = A[m*a_rs + k*a_ks] (one of the two strides 1), FP32
 * output, optional split-K.  Host arrays, current device.  N <= 256. */
int pcf_gemm_bf16(const unsigned short *A, long long a_len, long long a_rs, long long a_ks,
                  const unsigned short *B, long long b_len, long long b_rs, long long b_ks, int M, int N, int K,
                  int ksplit, float *D);

/* ---- learned warm start / preconditioner (no reference counterpart) ------
 * A per-column MLP fused with full 3x3 horizontal convolutions.  The column
 * of a field is resampled to 64 levels (x); with im2col(v)[c] the periodic
 * 3x3 window of columns around c (tap t = (dj+1)*3 + (di+1)):
 *   a = relu(C1 im2col(x) + c1), h1 = relu(W1 a + b1), h2 = relu(W2 h1 + b2),
 *   z = W3 h2 + b3, y = z + C2 im2col(z) + c2 (64 -> 256 -> 256 -> 64),
 * resampled back.  172,736 parameters; BF16 weights and activations, FP32
 * accumulation on the tensor cores (tcgen05); FP32 master weights trained
 * with Adam on the residual-weighted loss sum (N(b) - x)^2 / sum x^2.  An
 * application (pcf_net_apply_device, pcf_net_forward) is one cooperative
 * kernel; training keeps the activations and runs the layers as GEMMs.
 * Parameter order: C1[64][9][64] ([out][tap][in]), c1[64], W1[256][64],
 * b1[256], W2[256][256], b2[256], W3[64][256], b3[64], C2[64][9][64], c2[64].
 * A new network outputs zero (W3, C2 and the biases start at zero). */
typedef struct pcf_net pcf_net;
int pcf_net_num_params(void);
int pcf_net_create(pcf_net **net, int device, long long max_columns, unsigned seed);
int pcf_net_destroy(pcf_net *net);
int pcf_net_get_params(pcf_net *net, float *params);
int pcf_net_set_params(pcf_net *net, const float *params);
int pcf_net_save(pcf_net *net, const char *path);
int pcf_net_load(pcf_net *net, const char *path);
/* out = N(in) for host arrays of nz*ny*nx doubles */
int pcf_net_forward(pcf_net *net, const double *in, int nx, int ny, int nz, double *out);
/* out = beta * out + scale_out * N(scale_in * in) on device fields (doubles if fp64, else
 * floats), on `stream` (a cudaStream_t, NULL: the network's own stream) */
int pcf_net_apply_device(pcf_net *net, const void *in, int nx, int ny, int nz, double scale_in,
                         double scale_out, double beta, void *out, int fp64, void *stream);
/* one step on device FP32 fields b, x (normalised): loss before the step, gradients
 * (nullable host buffer), Adam update when lr > 0 */
int pcf_net_train_step(pcf_net *net, const float *b, const float *x, int nx, int ny, int nz, double lr,
                       double *loss, float *grad);
/* Adam over `count` samples given as host arrays b, x (each nz*ny*nx FP32,
 * normalised; sample q at offset q*nz*ny*nx), uploaded once for the call:
 * `epochs` passes in an order drawn from `seed`; losses (nullable,
 * count*epochs doubles) receives every step's loss before its update. */
int pcf_net_train(pcf_net *net, const float *b, const float *x, int count, int nx, int ny, int nz, int epochs,
                  double lr, unsigned seed, double *losses);
/* loss and gradients for host arrays, no update (gradient check) */
int pcf_net_gradients(pcf_net *net, const double *b, const double *x, int nx, int ny, int nz, double *loss,
                      float *grad);
/* Hold the biases at zero (zeroed now, skipped by Adam): the network is then
 * positively homogeneous, N(a x) = a N(x) for a > 0, and applies to a
 * residual of any size without normalisation (the preconditioner stage). */
int pcf_net_set_bias_free(pcf_net *net, int on);
/* Attach a trained network to a solver for the mixed-precision solve.
 * prm->learned is a bit set: 1, warm start x0 = RMS(b) N(b / RMS(b)) instead
 * of 0; 2, a learned stage in the right preconditioner of the flexible FP32
 * BiCGSTAB, z = M(r) + N(r - A M(r)) with M the reference or multigrid
 * preconditioner (for a bias-free network).  NULL detaches. */
int pcf_set_network(pcf_handle *h, pcf_net *net);

/* Allocation-free global dot product.  No counterpart in the reference: a
 * deterministic, run-to-run reproducible sum that agrees with pcf_global_dot
 * to rounding (it adds fixed chunks of 32768 elements per block, not
 * pcf_global_dot's blocking), for callers that cannot let the library
 * allocate device memory -- a host model whose GPU memory belongs to
 * its own pool allocator (such as Julia's CUDA.jl pool), or a time step being
 * captured into a CUDA graph, where cudaMalloc/cudaFree are not allowed.
 * a, b: device arrays of n doubles; *result: a device double, written
 * asynchronously on `stream` (a cudaStream_t; NULL = the legacy default
 * stream).  No handle is needed and nothing is allocated: the scratch is a
 * fixed 64 KB __device__ array that every GPU loading the library holds until
 * the process exits.  n must not exceed 268,435,456 (PCF_ERANGE otherwise).
 * The first call on a device (and the first after the device's context was
 * re-created, e.g. by cudaDeviceReset) looks up the scratch address; make that
 * call before any stream capture.  All calls share the scratch, so calls that
 * may overlap on the GPU (on different streams) race and must be serialised. */
int pcf_global_dot_noalloc(const double *a, const double *b, long long n, double *result, void *stream);
/* Test hook of the failure path (no reference counterpart): in the stencils
 * that stage their BF16 coefficient tiles by TMA, the copy of z-level `level`
 * is not issued, and every wait for a copy gives up after wait_limit_s
 * seconds (at most 10).  The wait for the missing copy then runs out, the
 * kernel records PCF_ECUDA in the solve's status and leaves, and the solve
 * returns errflag = 1 with status PCF_ECUDA.  level < 0 turns the hook off
 * (waits bounded by 2 s again).  Drops the handle's captured iteration
 * batches. */
int pcf_test_stall_staged_copy(pcf_handle *h, int level, double wait_limit_s);
/* Bounds checking (no reference counterpart): in the library built with
 * -DPCF_BOUNDS_CHECK (libpincflow_poisson_checked.so) the kernels check their
 * global indices against the arrays' extents, skip an access out of range and
 * record the first one.  Sets *enabled (1 in that build, 0 otherwise) and the
 * first recorded event since the last call -- the check site (0: none) and the
 * index -- then clears the records; synchronises the current device. */
int pcf_bounds_check_status(int *enabled, long long *site, long long *index);
int pcf_profile_enable(pcf_handle *h, int on);  /* also clears the accumulators */
int pcf_profile_read(const pcf_handle *h, int tag, double *ms, long long *count, double *bytes);

#ifdef __cplusplus
}
#endif
#endif /* PINCFLOW_POISSON_H */
