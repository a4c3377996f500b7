// or_terms.h -- CPU oracle (test infrastructure only): the pointwise terms
// shared by the corrector (correct!.jl) and the implicit predictor
// (update!.jl, Implicit()): compute_pressure_gradient.jl:108-297 for any
// pressure field, compute_compressible_wind_factor.jl:102-157 and
// compute_buoyancy_factor.jl:108-172.  Literal FP64 restatements; indices
// 0-based (i0 = nbx, k0 = nbz), one rank.
#pragma once

#include "pcf_oracle.h"

#include <cstddef>

namespace or_terms {

struct Ctx {
    const or_dims *d;
    int model;
    double dx, dy, dz, kappainv, mainv2;
    const double *jac, *met13, *met23, *met33, *rhobar, *pbar, *thetabar, *rho, *p;
    int nxx, nyy;
    size_t at(int i, int j, int k) const {
        return (size_t)i + (size_t)nxx * ((size_t)j + (size_t)nyy * (size_t)k);
    }
};

// compute_pressure_gradient(state, pip, i, j, k, U()), :108-158
inline double grad_u(const Ctx &c, const double *pip, int i, int j, int k) {
    const or_dims *d = c.d;
    const int k0 = d->nbz;
    auto P = [&](int a, int b, int e) { return pip[c.at(a, b, e)]; };
    double rhoedger = 0.5 * (c.rho[c.at(i, j, k)] + c.rho[c.at(i + 1, j, k)]);
    const double rhobaredger = 0.5 * (c.rhobar[c.at(i, j, k)] + c.rhobar[c.at(i + 1, j, k)]);
    rhoedger += rhobaredger;
    const double pedger = 0.5 * (c.pbar[c.at(i, j, k)] + c.pbar[c.at(i + 1, j, k)]);
    const double met13edger = 0.5 * (c.met13[c.at(i, j, k)] + c.met13[c.at(i + 1, j, k)]);
    double gradient;
    if (d->ko + k == k0) {
        const double pipuuedger = 0.5 * (P(i, j, k + 2) + P(i + 1, j, k + 2));
        const double pipuedger = 0.5 * (P(i, j, k + 1) + P(i + 1, j, k + 1));
        const double pipedger = 0.5 * (P(i, j, k) + P(i + 1, j, k));
        gradient = c.kappainv * c.mainv2 * pedger / rhoedger *
                   ((P(i + 1, j, k) - P(i, j, k)) / c.dx +
                    met13edger * (-pipuuedger + 4.0 * pipuedger - 3.0 * pipedger) * 0.5 / c.dz);
    } else if (d->ko + k == d->z_size + d->nbz - 1) {
        const double pipddedger = 0.5 * (P(i, j, k - 2) + P(i + 1, j, k - 2));
        const double pipdedger = 0.5 * (P(i, j, k - 1) + P(i + 1, j, k - 1));
        const double pipedger = 0.5 * (P(i, j, k) + P(i + 1, j, k));
        gradient = c.kappainv * c.mainv2 * pedger / rhoedger *
                   ((P(i + 1, j, k) - P(i, j, k)) / c.dx +
                    met13edger * (pipddedger - 4.0 * pipdedger + 3.0 * pipedger) * 0.5 / c.dz);
    } else {
        const double pipuedger = 0.5 * (P(i, j, k + 1) + P(i + 1, j, k + 1));
        const double pipdedger = 0.5 * (P(i, j, k - 1) + P(i + 1, j, k - 1));
        gradient = c.kappainv * c.mainv2 * pedger / rhoedger *
                   ((P(i + 1, j, k) - P(i, j, k)) / c.dx + met13edger * (pipuedger - pipdedger) * 0.5 / c.dz);
    }
    return gradient;
}

// compute_pressure_gradient(state, pip, i, j, k, V()), :160-210
inline double grad_v(const Ctx &c, const double *pip, int i, int j, int k) {
    const or_dims *d = c.d;
    const int k0 = d->nbz;
    auto P = [&](int a, int b, int e) { return pip[c.at(a, b, e)]; };
    double rhoedgef = 0.5 * (c.rho[c.at(i, j, k)] + c.rho[c.at(i, j + 1, k)]);
    const double rhobaredgef = 0.5 * (c.rhobar[c.at(i, j, k)] + c.rhobar[c.at(i, j + 1, k)]);
    rhoedgef += rhobaredgef;
    const double pedgef = 0.5 * (c.pbar[c.at(i, j, k)] + c.pbar[c.at(i, j + 1, k)]);
    const double met23edgef = 0.5 * (c.met23[c.at(i, j, k)] + c.met23[c.at(i, j + 1, k)]);
    double gradient;
    if (d->ko + k == k0) {
        const double pipuuedgef = 0.5 * (P(i, j, k + 2) + P(i, j + 1, k + 2));
        const double pipuedgef = 0.5 * (P(i, j, k + 1) + P(i, j + 1, k + 1));
        const double pipedgef = 0.5 * (P(i, j, k) + P(i, j + 1, k));
        gradient = c.kappainv * c.mainv2 * pedgef / rhoedgef *
                   ((P(i, j + 1, k) - P(i, j, k)) / c.dy +
                    met23edgef * (-pipuuedgef + 4.0 * pipuedgef - 3.0 * pipedgef) * 0.5 / c.dz);
    } else if (d->ko + k == d->z_size + d->nbz - 1) {
        const double pipddedgef = 0.5 * (P(i, j, k - 2) + P(i, j + 1, k - 2));
        const double pipdedgef = 0.5 * (P(i, j, k - 1) + P(i, j + 1, k - 1));
        const double pipedgef = 0.5 * (P(i, j, k) + P(i, j + 1, k));
        gradient = c.kappainv * c.mainv2 * pedgef / rhoedgef *
                   ((P(i, j + 1, k) - P(i, j, k)) / c.dy +
                    met23edgef * (pipddedgef - 4.0 * pipdedgef + 3.0 * pipedgef) * 0.5 / c.dz);
    } else {
        const double pipuedgef = 0.5 * (P(i, j, k + 1) + P(i, j + 1, k + 1));
        const double pipdedgef = 0.5 * (P(i, j, k - 1) + P(i, j + 1, k - 1));
        gradient = c.kappainv * c.mainv2 * pedgef / rhoedgef *
                   ((P(i, j + 1, k) - P(i, j, k)) / c.dy + met23edgef * (pipuedgef - pipdedgef) * 0.5 / c.dz);
    }
    return gradient;
}

// compute_pressure_gradient(state, pip, i, j, k, W()), :212-297
inline double grad_w(const Ctx &c, const double *pip, int i, int j, int k) {
    auto J = [&](int a, int b, int e) { return c.jac[c.at(a, b, e)]; };
    auto P = [&](int a, int b, int e) { return pip[c.at(a, b, e)]; };
    const double jk = J(i, j, k), jk1 = J(i, j, k + 1);
    double rhoedgeu = (jk1 * c.rho[c.at(i, j, k)] + jk * c.rho[c.at(i, j, k + 1)]) / (jk + jk1);
    rhoedgeu += (jk1 * c.rhobar[c.at(i, j, k)] + jk * c.rhobar[c.at(i, j, k + 1)]) / (jk + jk1);
    const double pedgeu = (jk1 * c.pbar[c.at(i, j, k)] + jk * c.pbar[c.at(i, j, k + 1)]) / (jk + jk1);
    const double met13edgeu = (jk1 * c.met13[c.at(i, j, k)] + jk * c.met13[c.at(i, j, k + 1)]) / (jk + jk1);
    const double met23edgeu = (jk1 * c.met23[c.at(i, j, k)] + jk * c.met23[c.at(i, j, k + 1)]) / (jk + jk1);
    const double met33edgeu = (jk1 * c.met33[c.at(i, j, k)] + jk * c.met33[c.at(i, j, k + 1)]) / (jk + jk1);
    const double pipredgeu = (J(i + 1, j, k + 1) * P(i + 1, j, k) + J(i + 1, j, k) * P(i + 1, j, k + 1)) /
                             (J(i + 1, j, k) + J(i + 1, j, k + 1));
    const double pipledgeu = (J(i - 1, j, k + 1) * P(i - 1, j, k) + J(i - 1, j, k) * P(i - 1, j, k + 1)) /
                             (J(i - 1, j, k) + J(i - 1, j, k + 1));
    const double pipfedgeu = (J(i, j + 1, k + 1) * P(i, j + 1, k) + J(i, j + 1, k) * P(i, j + 1, k + 1)) /
                             (J(i, j + 1, k) + J(i, j + 1, k + 1));
    const double pipbedgeu = (J(i, j - 1, k + 1) * P(i, j - 1, k) + J(i, j - 1, k) * P(i, j - 1, k + 1)) /
                             (J(i, j - 1, k) + J(i, j - 1, k + 1));
    return c.kappainv * c.mainv2 * pedgeu / rhoedgeu *
           (met13edgeu * (pipredgeu - pipledgeu) * 0.5 / c.dx + met23edgeu * (pipfedgeu - pipbedgeu) * 0.5 / c.dy +
            met33edgeu * (P(i, j, k + 1) - P(i, j, k)) / c.dz);
}

// compute_compressible_wind_factor, :102-157 (1 unless Compressible)
inline double wind_u(const Ctx &c, int i, int j, int k) {
    if (c.model != 2) return 1.0;
    return (c.jac[c.at(i, j, k)] * c.p[c.at(i, j, k)] + c.jac[c.at(i + 1, j, k)] * c.p[c.at(i + 1, j, k)]) / 2;
}
inline double wind_v(const Ctx &c, int i, int j, int k) {
    if (c.model != 2) return 1.0;
    return (c.jac[c.at(i, j, k)] * c.p[c.at(i, j, k)] + c.jac[c.at(i, j + 1, k)] * c.p[c.at(i, j + 1, k)]) / 2;
}
inline double wind_w(const Ctx &c, int i, int j, int k) {
    if (c.model != 2) return 1.0;
    const double jk = c.jac[c.at(i, j, k)], jk1 = c.jac[c.at(i, j, k + 1)];
    return jk * jk1 * (c.p[c.at(i, j, k)] + c.p[c.at(i, j, k + 1)]) / (jk + jk1);
}

// compute_buoyancy_factor(W) :135-172 and (RhoP) :108-133
inline double buoy_w(const Ctx &c, int i, int j, int k) {
    const double jk = c.jac[c.at(i, j, k)], jk1 = c.jac[c.at(i, j, k + 1)];
    const double den = jk1 * (c.rho[c.at(i, j, k)] + c.rhobar[c.at(i, j, k)]) +
                       jk * (c.rho[c.at(i, j, k + 1)] + c.rhobar[c.at(i, j, k + 1)]);
    if (c.model == 2)
        return (jk1 * c.pbar[c.at(i, j, k)] / c.thetabar[c.at(i, j, k)] +
                jk * c.pbar[c.at(i, j, k + 1)] / c.thetabar[c.at(i, j, k + 1)]) /
               den;
    return (jk1 * c.rhobar[c.at(i, j, k)] + jk * c.rhobar[c.at(i, j, k + 1)]) / den;
}
inline double buoy_rhop(const Ctx &c, int i, int j, int k) {
    const size_t n = c.at(i, j, k);
    if (c.model == 2) return c.pbar[n] / c.thetabar[n] / (c.rho[n] + c.rhobar[n]);
    return c.rhobar[n] / (c.rho[n] + c.rhobar[n]);
}

}  // namespace or_terms
