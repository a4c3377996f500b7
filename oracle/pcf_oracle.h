/*
 * pcf_oracle.h -- CPU oracle for the semi-implicit pressure Poisson solve of
 * PinCFlow.jl (module PoissonSolver).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a literal FP64 restatement of the
 * reference Julia code, used as the checker for the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The
 * product (pincflow.jl_b200/) never links or calls it.
 *
 * Parity status: PARITY UNPINNED by reference golden vectors.  The reference
 * ships no known-answer data for the Poisson path in isolation (its only
 * pinned numbers are end-to-end norms of whole simulations, e.g.
 * test/test_periodic_hill.jl:2-27, which need the Julia model), and Julia is
 * not available to run it.  The oracle is instead pinned to analytic
 * known-answer tests (flat-terrain Fourier eigenpairs, dense tridiagonal
 * solves, null-vector identities) in tests/test_oracle_kat.py.
 *
 * Array conventions follow the reference (column-major, x fastest):
 *   haloed fields  (nxx, nyy, nzz), nxx = nx + 2*nbx, ...   index i + nxx*(j + nyy*k)
 *   interior arrays (nx, ny, nz)                             index i + nx*(j + ny*k)
 * The 25 operator planes are stored one after another (plane stride nx*ny*nz)
 * in the field order of the reference's Tensor struct
 * (src/Types/PoissonTypes/Tensor.jl:70-96), see enum or_coef.
 */
#ifndef PCF_ORACLE_H
#define PCF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz;    /* interior sizes of this (single) subdomain */
    int nbx, nby, nbz; /* halo widths (reference default 3) */
    int ko;            /* vertical offset of the subdomain (0 on one rank) */
    int z_size;        /* global vertical size */
} or_dims;

/* Plane order of the reference Tensor struct (Tensor.jl:70-96). */
enum or_coef {
    OR_AC = 0, OR_AL, OR_AR, OR_AB, OR_AF, OR_AD, OR_AU,
    OR_ALD, OR_ALU, OR_ARD, OR_ARU, OR_ABD, OR_ABU, OR_AFD, OR_AFU,
    OR_ADD, OR_AUU, OR_ALDD, OR_ALUU, OR_ARDD, OR_ARUU, OR_ABDD, OR_ABUU,
    OR_AFDD, OR_AFUU, OR_NCOEF
};

enum or_model { OR_BOUSSINESQ = 0, OR_PSEUDO_INCOMPRESSIBLE = 1, OR_COMPRESSIBLE = 2 };

/* ---- input generators (Constants.jl, Grid.jl, Atmosphere.jl, compute_n2!.jl,
 *      compute_sponges!.jl) ------------------------------------------------ */

/* Non-dimensionalisation constants, Constants.jl:113-155.
 * out[0..8] = gamma, kappa, rsp, g, rhoref, pref, lref, tref, thetaref,
 * out[9..11] = g_ndim, ma, sig. */
void or_constants(double *out);

/* Grid metric, Grid.jl:173-338 (npx = npy = npz = 1).
 * lx, ly, lz, dimensional [m]; stretch_exp: vertical stretching
 * z~(z^) = lz * (z^/lz)^stretch_exp (1.0 = the reference default identity);
 * hb_dim: dimensional topography at interior cells (nx*ny, x fastest).
 * Outputs (haloed, nxx*nyy*nzz): jac, met13, met23, met33, zc (non-dim).
 * Returns 0, or -1 if the stretched levels are not increasing. */
int or_grid(const or_dims *d, double lx, double ly, double lz, double stretch_exp,
            const double *hb_dim, double *jac, double *met13, double *met23,
            double *met33, double *zc, double *dxdydz_out);

/* Atmosphere backgrounds.  background 0 = Boussinesq StableStratification
 * (Atmosphere.jl:278-296, params[0] = N [1/s], params[1] = theta0 [K]);
 * background 1 = Isothermal (Atmosphere.jl:298-323, params[0] = T0 [K],
 * params[1] = p0 [Pa]) with N^2 from compute_n2!.jl:43-82.
 * Outputs (haloed): pbar, thetabar, rhobar, n2. */
int or_atmosphere(const or_dims *d, int background, const double *params,
                  const double *jac, const double *zc, double dz,
                  double *pbar, double *thetabar, double *rhobar, double *n2);

/* RHS sponge of the periodic-hill case, compute_sponges!.jl:26-65 with
 * rhs_sponge(z) = sin^2(pi/2 (z - zr)/(lz - zr))/dt for z >= zr
 * (src/Examples/periodic_hill.jl:36-37).  zr, lz dimensional [m];
 * dt non-dimensional.  Output betar (haloed). */
void or_sponge_sin2(const or_dims *d, const double *zc, double zr, double lz,
                    double dt, double *betar);

/* ---- the Poisson path ------------------------------------------------- */

/* compute_operator!, src/PoissonSolver/compute_operator!.jl:40-1606, with
 * compute_buoyancy_factor(W) inlined (src/Update/compute_buoyancy_factor.jl:
 * 135-172).  All field inputs haloed; thetabar and p are read only for the
 * Compressible model (may be NULL otherwise).  coef: 25 interior planes. */
void or_compute_operator(const or_dims *d, int model, double dx, double dy, double dz,
                         const double *jac, const double *met13, const double *met23,
                         const double *met33, const double *pbar, const double *rhobar,
                         const double *thetabar, const double *n2, const double *rho,
                         const double *betar, const double *p, double dt,
                         double rayleigh_factor, int damp_horizontal_wind_on_rhs,
                         double *coef);

/* apply_operator!, src/PoissonSolver/apply_operator!.jl:48-273 (Total,
 * horizontal = 0) and :275-479 (Horizontal, horizontal = 1); periodic x/y,
 * zero vertical ghosts (single rank). */
void or_apply_operator(const or_dims *d, const double *coef, const double *sin_,
                       double *ls, int horizontal);

/* apply_preconditioner!, src/PoissonSolver/apply_preconditioner!.jl:40-124. */
void or_apply_preconditioner(const or_dims *d, const double *coef, double dx, double dy,
                             double dtau, int preconditioner_iterations,
                             const double *sin_, double *sout);

/* apply_bicgstab!, src/PoissonSolver/apply_bicgstab!.jl:24-150.
 * Writes solution; out[0] = errflag, out[1] = niter, out[2] = final
 * recursive relative residual, out[3] = b_norm. */
void or_bicgstab(const or_dims *d, const double *coef, double dx, double dy,
                 double tolerance, int poisson_iterations, int preconditioner,
                 double dtau, int preconditioner_iterations, int tolerance_is_relative,
                 double tolref, const double *rhs, double *solution, double *out);

/* solve_poisson!, src/PoissonSolver/solve_poisson!.jl:39-75: operator
 * assembly + BiCGSTAB + unscaling; dpip haloed, interior written.
 * Returns -1 for dt == 0 (the reference raises), else 0. */
int or_solve_poisson(const or_dims *d, int model, double dx, double dy, double dz,
                     const double *jac, const double *met13, const double *met23,
                     const double *met33, const double *pbar, const double *rhobar,
                     const double *thetabar, const double *n2, const double *rho,
                     const double *betar, const double *p, double dt,
                     double rayleigh_factor, int damp_horizontal_wind_on_rhs,
                     double tolerance, int poisson_iterations, int preconditioner,
                     double dtau, int preconditioner_iterations,
                     int tolerance_is_relative, double tolref, const double *rhs,
                     double *dpip, double *out);

/* compute_lhs! (Boussinesq / PseudoIncompressible),
 * src/PoissonSolver/compute_lhs!.jl:68-160.  u, v, w haloed staggered
 * velocities.  Writes rhs (interior); returns tolref (NaN where the
 * reference raises). */
double or_compute_lhs(const or_dims *d, double dx, double dy, double dz, double ma,
                      double kappa, const double *jac, const double *pbar,
                      const double *rhobar, const double *u, const double *v,
                      const double *w, double *rhs);

/* compute_lhs! (Compressible), src/PoissonSolver/compute_lhs!.jl:162-223.
 * u, v, w are the staggered mass fluxes; heating (interior, may be NULL for
 * zero) is compute_volume_force(state, i, j, k, P()), which the caller
 * supplies.  Returns tolref as or_compute_lhs. */
double or_compute_lhs_compressible(const or_dims *d, double dx, double dy, double dz, double ma,
                                   double kappa, const double *jac, const double *pbar,
                                   const double *rhobar, const double *u, const double *v,
                                   const double *w, const double *heating, double *rhs);

/* The corrector after the solve (apply_corrector!.jl:58-61): dpip's halo
 * fill (periodic x/y, mirrored z; in place) then correct!.jl:164-385
 * (u, v, w, rhop corrected in place, pip += dpip on one ghost layer
 * around the interior).  All arrays haloed; model 0/1/2 as
 * or_compute_operator; kappainv = 1/kappa, mainv2 = 1/Ma^2, g_ndim the
 * non-dimensional gravity (Constants.jl:116, :131, :150). */
void or_fill_dpip(const or_dims *d, double *dpip);
void or_correct(const or_dims *d, int model, double dx, double dy, double dz, const double *jac,
                const double *met13, const double *met23, const double *met33, const double *rhobar,
                const double *pbar, const double *thetabar, const double *n2, const double *betar,
                const double *rho, const double *p, double dt, double rayleigh_factor, int damp_h,
                double kappainv, double mainv2, double g_ndim, double *dpip, double *u, double *v,
                double *w, double *rhop, double *pip);

/* The implicit half step around the corrector (implicit_integration!.jl:
 * 49-77 without output), one rank, no tracers.
 * or_set_predictand_boundaries: set_boundaries!(state, BoundaryPredictands())
 * (periodic x/y; in z rho, rhop point-reflected, u, v, pip, p
 * line-reflected, w zero on the walls and point-reflected); rho is filled
 * for models 1 and 2, p for model 2.  or_modify_compressible_wind:
 * modify_compressible_wind!(state, * or /) (Compressible only; divide = 1
 * for /).  or_implicit_predictor: save_backups!(state, :w) into wold, then
 * update!(U, V, W; Implicit()), set_boundaries!, update!(RhoP; Implicit()),
 * set_boundaries! (:53-63); dudt, dvdt are the WKB momentum tendencies or
 * NULL (NoWKB).  All arrays haloed. */
void or_set_predictand_boundaries(const or_dims *d, int model, double *rho, double *rhop, double *u, double *v,
                                  double *w, double *pip, double *p);
void or_modify_compressible_wind(const or_dims *d, int model, const double *jac, const double *p, double *u,
                                 double *v, double *w, int divide);
void or_implicit_predictor(const or_dims *d, int model, double dx, double dy, double dz, const double *jac,
                           const double *met13, const double *met23, const double *met33, const double *rhobar,
                           const double *pbar, const double *thetabar, const double *n2, const double *betar,
                           double *rho, double *p, double dt, double rayleigh_factor, int damp_h, double kappainv,
                           double mainv2, double g_ndim, const double *dudt, const double *dvdt, double *u,
                           double *v, double *w, double *rhop, double *pip, double *wold);

/* Helpers for tests and the CPU baseline. */
double or_dot(long n, const double *a, const double *b); /* pairwise FP64 sum */
void or_set_threads(int n);
int or_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
