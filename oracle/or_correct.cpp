// or_correct.cpp -- CPU oracle (test infrastructure only): the corrector
// step after the Poisson solve, single MPI rank, literal FP64 restatements of
//   the dpip boundary fill of apply_corrector!.jl:58-60
//     (set_zonal_boundaries_of_field!.jl:78-104, the meridional twin,
//      set_vertical_boundaries_of_field!.jl:52-101 with mode = +)
//   correct!.jl:164-385 (U, V, W, RhoP, PiP)
//   compute_pressure_gradient.jl:108-297 (U, V, W)
//   compute_compressible_wind_factor.jl:102-157
//   compute_buoyancy_factor.jl:108-172 (RhoP, W)
// Indices are 0-based: i0 = nbx, i1 = nbx + nx - 1 (likewise j, k), ko = 0.
#include "or_terms.h"

#include <cmath>
#include <cstddef>
#include <vector>

using namespace or_terms;

extern "C" {

void or_fill_dpip(const or_dims *d, double *f) {
    const int nxx = d->nx + 2 * d->nbx, nyy = d->ny + 2 * d->nby, nzz = d->nz + 2 * d->nbz;
    auto at = [&](int i, int j, int k) { return (size_t)i + (size_t)nxx * ((size_t)j + (size_t)nyy * (size_t)k); };
    const int i0 = d->nbx, i1 = d->nbx + d->nx - 1, j0 = d->nby, j1 = d->nby + d->ny - 1;
    const int k0 = d->nbz, k1 = d->nbz + d->nz - 1;
    // zonal (:91-101; one rank: the halo exchange is the periodic copy)
    for (int k = 0; k < nzz; ++k)
        for (int j = 0; j < nyy; ++j)
            for (int i = 1; i <= d->nbx; ++i) {
                f[at(i0 - i, j, k)] = f[at(i1 - i + 1, j, k)];
                f[at(i1 + i, j, k)] = f[at(i0 + i - 1, j, k)];
            }
    // meridional
    for (int k = 0; k < nzz; ++k)
        for (int j = 1; j <= d->nby; ++j)
            for (int i = 0; i < nxx; ++i) {
                f[at(i, j0 - j, k)] = f[at(i, j1 - j + 1, k)];
                f[at(i, j1 + j, k)] = f[at(i, j0 + j - 1, k)];
            }
    // vertical, mode = + (:74-98, not staggered)
    for (int k = 1; k <= d->nbz; ++k)
        for (int j = 0; j < nyy; ++j)
            for (int i = 0; i < nxx; ++i) {
                f[at(i, j, k0 - k)] = f[at(i, j, k0 + k - 1)];
                f[at(i, j, k1 + k)] = f[at(i, j, k1 - k + 1)];
            }
}

void or_correct(const or_dims *d, int model, double dx, double dy, double dz, const double *jac,
                const double *met13, const double *met23, const double *met33, const double *rhobar,
                const double *pbar, const double *thetabar, const double *n2, const double *betar,
                const double *rho, const double *p, double dt, double rayleigh_factor, int damp_h,
                double kappainv, double mainv2, double g_ndim, double *dpip, double *u, double *v, double *w,
                double *rhop, double *pip) {
    const int nxx = d->nx + 2 * d->nbx, nyy = d->ny + 2 * d->nby, nzz = d->nz + 2 * d->nbz;
    Ctx c{d, model, dx, dy, dz, kappainv, mainv2, jac, met13, met23, met33, rhobar, pbar, thetabar, rho, p,
          nxx, nyy};
    const int i0 = d->nbx, i1 = d->nbx + d->nx - 1, j0 = d->nby, j1 = d->nby + d->ny - 1;
    const int k0 = d->nbz, k1 = d->nbz + d->nz - 1;
    const size_t nh = (size_t)nxx * nyy * nzz;
    or_fill_dpip(d, dpip);
    std::vector<double> corx(nh, 0.0), cory(nh, 0.0);
    // U (:177-210): k0..k1 (single rank), i0-1..i1
    for (int k = k0; k <= k1; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0 - 1; i <= i1; ++i) {
                double factor = 1.0;
                if (damp_h) factor += dt * 0.5 * (betar[c.at(i, j, k)] + betar[c.at(i + 1, j, k)]) * rayleigh_factor;
                const double gradient = grad_u(c, dpip, i, j, k);
                corx[c.at(i, j, k)] = dt / factor * gradient;
                u[c.at(i, j, k)] -= wind_u(c, i, j, k) * corx[c.at(i, j, k)];
            }
    // V (:212-245)
    for (int k = k0; k <= k1; ++k)
        for (int j = j0 - 1; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                double factor = 1.0;
                if (damp_h) factor += dt * 0.5 * (betar[c.at(i, j, k)] + betar[c.at(i, j + 1, k)]) * rayleigh_factor;
                const double gradient = grad_v(c, dpip, i, j, k);
                cory[c.at(i, j, k)] = dt / factor * gradient;
                v[c.at(i, j, k)] -= wind_v(c, i, j, k) * cory[c.at(i, j, k)];
            }
    // W (:247-305): k0..k1-1 (single rank)
    for (int k = k0; k <= k1 - 1; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                auto J = [&](int a, int b, int e) { return jac[c.at(a, b, e)]; };
                double factor = 1.0;
                factor += dt * (J(i, j, k + 1) * betar[c.at(i, j, k)] + J(i, j, k) * betar[c.at(i, j, k + 1)]) /
                          (J(i, j, k) + J(i, j, k + 1)) * rayleigh_factor;
                const double n2edgeu = (J(i, j, k + 1) * n2[c.at(i, j, k)] + J(i, j, k) * n2[c.at(i, j, k + 1)]) /
                                       (J(i, j, k) + J(i, j, k + 1));
                const double gradient = grad_w(c, dpip, i, j, k);
                const double jpedgeu = wind_w(c, i, j, k);
                const double fw = buoy_w(c, i, j, k);
                w[c.at(i, j, k)] +=
                    -dt / (factor + fw * n2edgeu * std::pow(dt, 2.0)) * jpedgeu * gradient -
                    1.0 / (factor + fw * n2edgeu * std::pow(dt, 2.0)) * fw * n2edgeu * std::pow(dt, 2.0) * jpedgeu *
                        0.5 *
                        (J(i, j, k + 1) * (met13[c.at(i, j, k)] * (corx[c.at(i, j, k)] + corx[c.at(i - 1, j, k)]) +
                                           met23[c.at(i, j, k)] * (cory[c.at(i, j, k)] + cory[c.at(i, j - 1, k)])) +
                         J(i, j, k) *
                             (met13[c.at(i, j, k + 1)] * (corx[c.at(i, j, k + 1)] + corx[c.at(i - 1, j, k + 1)]) +
                              met23[c.at(i, j, k + 1)] * (cory[c.at(i, j, k + 1)] + cory[c.at(i, j - 1, k + 1)]))) /
                        (J(i, j, k) + J(i, j, k + 1));
            }
    // RhoP (:307-360)
    for (int k = k0; k <= k1; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                const size_t n = c.at(i, j, k);
                double factor = 1.0;
                factor += dt * betar[n] * rayleigh_factor;
                double lower_gradient = grad_w(c, dpip, i, j, k - 1);
                double upper_gradient = grad_w(c, dpip, i, j, k);
                if (d->ko + k == k0)
                    lower_gradient = 0.0;
                else if (d->ko + k == d->z_size + d->nbz - 1)
                    upper_gradient = 0.0;
                const double gradient = 0.5 * (lower_gradient + upper_gradient);
                const double fb = buoy_rhop(c, i, j, k);
                const double db =
                    -1.0 / (factor + fb * n2[n] * std::pow(dt, 2.0)) *
                    (-fb * n2[n] * std::pow(dt, 2.0) * jac[n] * gradient +
                     fb * n2[n] * dt * jac[n] * factor * 0.5 *
                         (met13[n] * (corx[n] + corx[c.at(i - 1, j, k)]) +
                          met23[n] * (cory[n] + cory[c.at(i, j - 1, k)])));
                rhop[n] -= (rho[n] + rhobar[n]) / g_ndim * db;
            }
    // PiP (:375-385)
    for (int k = k0 - 1; k <= k1 + 1; ++k)
        for (int j = j0 - 1; j <= j1 + 1; ++j)
            for (int i = i0 - 1; i <= i1 + 1; ++i) pip[c.at(i, j, k)] += dpip[c.at(i, j, k)];
}

}  // extern "C"
