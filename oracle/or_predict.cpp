// or_predict.cpp -- CPU oracle (test infrastructure only): the implicit half
// step around the corrector, single MPI rank, no tracers, literal FP64
// restatements of
//   set_boundaries!(state, BoundaryPredictands()) (set_boundaries!.jl:46-60):
//     set_zonal_boundaries!.jl:127-176 and set_zonal_boundaries_of_field!.jl:
//     78-104, the meridional twins (set_meridional_boundaries_of_field!.jl:
//     84-104), set_vertical_boundaries!.jl:185-240 with
//     set_vertical_boundaries_of_field!.jl:52-101 (one rank: the vertical
//     halo exchange has no neighbour, the wall conditions set both ends)
//   modify_compressible_wind!.jl:38-80
//   save_backups!.jl:16-24 (wold = w)
//   update!(state, dt, U() / V() / W() / RhoP(), RHS(), Implicit(), rf)
//     (update!.jl:837-882, :988-1033, :1248-1336, :632-728)
//   compute_volume_force.jl:148-206 for U, V, W (NoWKB: zero; otherwise the
//     averaged WKB momentum tendencies dudt, dvdt)
// The pointwise terms are those of or_terms.h.  Indices are 0-based:
// i0 = nbx, i1 = nbx + nx - 1 (likewise j, k), ko = 0, z_size = nz.
#include "or_terms.h"

#include <cmath>
#include <cstddef>
#include <vector>

using namespace or_terms;

namespace {

struct Box {
    int nxx, nyy, nzz, i0, i1, j0, j1, k0, k1;
    explicit Box(const or_dims *d)
        : nxx(d->nx + 2 * d->nbx), nyy(d->ny + 2 * d->nby), nzz(d->nz + 2 * d->nbz), i0(d->nbx),
          i1(d->nbx + d->nx - 1), j0(d->nby), j1(d->nby + d->ny - 1), k0(d->nbz), k1(d->nbz + d->nz - 1) {}
    size_t at(int i, int j, int k) const {
        return (size_t)i + (size_t)nxx * ((size_t)j + (size_t)nyy * (size_t)k);
    }
};

// set_zonal_boundaries_of_field!.jl:91-101 (x_size > 1 on one rank: the
// periodic halo exchange with itself; x_size = 1: the same copy)
void zonal(const or_dims *d, const Box &b, double *f) {
    for (int k = 0; k < b.nzz; ++k)
        for (int j = 0; j < b.nyy; ++j)
            for (int i = 1; i <= d->nbx; ++i) {
                f[b.at(b.i0 - i, j, k)] = f[b.at(b.i1 - i + 1, j, k)];
                f[b.at(b.i1 + i, j, k)] = f[b.at(b.i0 + i - 1, j, k)];
            }
}

// set_meridional_boundaries_of_field!.jl:91-101
void meridional(const or_dims *d, const Box &b, double *f) {
    for (int k = 0; k < b.nzz; ++k)
        for (int j = 1; j <= d->nby; ++j)
            for (int i = 0; i < b.nxx; ++i) {
                f[b.at(i, b.j0 - j, k)] = f[b.at(i, b.j1 - j + 1, k)];
                f[b.at(i, b.j1 + j, k)] = f[b.at(i, b.j0 + j - 1, k)];
            }
}

// set_vertical_boundaries_of_field!.jl:74-98; sign = +1 (line reflection) or
// -1 (point reflection)
void vertical(const or_dims *d, const Box &b, double *f, double sign, bool staggered) {
    for (int j = 0; j < b.nyy; ++j)
        for (int i = 0; i < b.nxx; ++i) {
            if (staggered) {
                f[b.at(i, j, b.k0 - 1)] = 0.0;
                for (int k = 1; k <= d->nbz; ++k) f[b.at(i, j, b.k0 - k)] = sign * f[b.at(i, j, b.k0 + k - 2)];
            } else {
                for (int k = 1; k <= d->nbz; ++k) f[b.at(i, j, b.k0 - k)] = sign * f[b.at(i, j, b.k0 + k - 1)];
            }
        }
    for (int j = 0; j < b.nyy; ++j)
        for (int i = 0; i < b.nxx; ++i) {
            if (staggered) {
                f[b.at(i, j, b.k1)] = 0.0;
                for (int k = 1; k <= d->nbz; ++k) f[b.at(i, j, b.k1 + k)] = sign * f[b.at(i, j, b.k1 - k)];
            } else {
                for (int k = 1; k <= d->nbz; ++k) f[b.at(i, j, b.k1 + k)] = sign * f[b.at(i, j, b.k1 - k + 1)];
            }
        }
}

// compute_volume_force(state, i, j, k, W()), :185-206 (zero without WKB)
double force_w(const Ctx &c, const double *dudt, const double *dvdt, int i, int j, int k) {
    if (!dudt) return 0.0;
    auto J = [&](int a, int b, int e) { return c.jac[c.at(a, b, e)]; };
    return (J(i, j, k + 1) * (c.met13[c.at(i, j, k)] * dudt[c.at(i, j, k)] +
                              c.met23[c.at(i, j, k)] * dvdt[c.at(i, j, k)]) +
            J(i, j, k) * (c.met13[c.at(i, j, k + 1)] * dudt[c.at(i, j, k + 1)] +
                          c.met23[c.at(i, j, k + 1)] * dvdt[c.at(i, j, k + 1)])) /
           (J(i, j, k) + J(i, j, k + 1));
}

}  // namespace

extern "C" {

void or_set_predictand_boundaries(const or_dims *d, int model, double *rho, double *rhop, double *u, double *v,
                                  double *w, double *pip, double *p) {
    const Box b(d);
    // set_zonal_boundaries!.jl:127-176: (rhop, u, v, w, pip), plus rho
    // (PseudoIncompressible) and p (Compressible: every predictand)
    std::vector<double *> all;
    if (model >= 1) all.push_back(rho);
    all.push_back(rhop);
    all.push_back(u);
    all.push_back(v);
    all.push_back(w);
    all.push_back(pip);
    if (model == 2) all.push_back(p);
    for (double *f : all) zonal(d, b, f);
    for (double *f : all) meridional(d, b, f);
    // set_vertical_boundaries!.jl:185-240
    if (model >= 1) vertical(d, b, rho, -1.0, false);
    vertical(d, b, rhop, -1.0, false);
    vertical(d, b, u, 1.0, false);
    vertical(d, b, v, 1.0, false);
    vertical(d, b, w, -1.0, true);
    vertical(d, b, pip, 1.0, false);
    if (model == 2) vertical(d, b, p, 1.0, false);
}

// modify_compressible_wind!.jl:52-80: divide = 0 multiplies, 1 divides
void or_modify_compressible_wind(const or_dims *d, int model, const double *jac, const double *p, double *u,
                                 double *v, double *w, int divide) {
    if (model != 2) return;
    const Box b(d);
    auto op = [&](double x, double y) { return divide ? x / y : x * y; };
    for (int k = b.k0; k <= b.k1; ++k)
        for (int j = b.j0; j <= b.j1; ++j)
            for (int i = b.i0; i <= b.i1; ++i) {
                const size_t c = b.at(i, j, k), r = b.at(i + 1, j, k), f = b.at(i, j + 1, k), t = b.at(i, j, k + 1);
                u[c] = op(u[c], (jac[c] * p[c] + jac[r] * p[r]) / 2);
                v[c] = op(v[c], (jac[c] * p[c] + jac[f] * p[f]) / 2);
                w[c] = op(w[c], jac[c] * jac[t] * (p[c] + p[t]) / (jac[c] + jac[t]));
            }
}

// implicit_integration!.jl:53-63: save_backups!(state, :w); update! of U, V,
// W (Implicit); set_boundaries!; update! of RhoP (Implicit); set_boundaries!.
// dudt, dvdt: WKB tendencies (haloed) or NULL for wkb_mode = NoWKB.
void or_implicit_predictor(const or_dims *d, int model, double dx, double dy, double dz, const double *jac,
                           const double *met13, const double *met23, const double *met33, const double *rhobar,
                           const double *pbar, const double *thetabar, const double *n2, const double *betar,
                           double *rho, double *p, double dt, double rayleigh_factor, int damp_h, double kappainv,
                           double mainv2, double g_ndim, const double *dudt, const double *dvdt, double *u,
                           double *v, double *w, double *rhop, double *pip, double *wold) {
    const Box b(d);
    Ctx c{d, model, dx, dy, dz, kappainv, mainv2, jac, met13, met23, met33, rhobar, pbar, thetabar, rho, p,
          b.nxx, b.nyy};
    const size_t nh = (size_t)b.nxx * b.nyy * b.nzz;
    const int i0 = b.i0, i1 = b.i1, j0 = b.j0, j1 = b.j1, k0 = b.k0, k1 = b.k1;
    auto J = [&](int a, int e, int f) { return jac[c.at(a, e, f)]; };
    auto R = [&](const double *f, int a, int e, int g) { return f[c.at(a, e, g)]; };
    for (size_t q = 0; q < nh; ++q) wold[q] = w[q];
    // U (update!.jl:837-882): k0..k1 (one rank), i0-1..i1
    for (int k = k0; k <= k1; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0 - 1; i <= i1; ++i) {
                double rhoedger = 0.5 * (R(rho, i, j, k) + R(rho, i + 1, j, k));
                const double rhobaredger = 0.5 * (R(rhobar, i, j, k) + R(rhobar, i + 1, j, k));
                rhoedger += rhobaredger;
                const double gradient = grad_u(c, pip, i, j, k);
                const double force = dudt ? (R(dudt, i, j, k) + R(dudt, i + 1, j, k)) / 2 : 0.0;
                double factor = 1.0;
                if (damp_h)
                    factor += dt * 0.5 * (R(betar, i, j, k) + R(betar, i + 1, j, k)) * rayleigh_factor;
                const double jpedger = wind_u(c, i, j, k);
                double &uc = u[c.at(i, j, k)];
                uc = 1.0 / factor * (uc + dt * (-gradient + force / rhoedger) * jpedger);
            }
    // V (:988-1033)
    for (int k = k0; k <= k1; ++k)
        for (int j = j0 - 1; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                double rhoedgef = 0.5 * (R(rho, i, j, k) + R(rho, i, j + 1, k));
                const double rhobaredgef = 0.5 * (R(rhobar, i, j, k) + R(rhobar, i, j + 1, k));
                rhoedgef += rhobaredgef;
                const double gradient = grad_v(c, pip, i, j, k);
                const double force = dvdt ? (R(dvdt, i, j, k) + R(dvdt, i, j + 1, k)) / 2 : 0.0;
                double factor = 1.0;
                if (damp_h)
                    factor += dt * 0.5 * (R(betar, i, j, k) + R(betar, i, j + 1, k)) * rayleigh_factor;
                const double jpedgef = wind_v(c, i, j, k);
                double &vc = v[c.at(i, j, k)];
                vc = 1.0 / factor * (vc + dt * (-gradient + force / rhoedgef) * jpedgef);
            }
    // W (:1248-1336): k0..k1-1 (one rank)
    for (int k = k0; k <= k1 - 1; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                double rhoc = R(rho, i, j, k);
                double rhou = R(rho, i, j, k + 1);
                double rhoedgeu = (J(i, j, k + 1) * R(rho, i, j, k) + J(i, j, k) * R(rho, i, j, k + 1)) /
                                  (J(i, j, k) + J(i, j, k + 1));
                rhoc += R(rhobar, i, j, k);
                rhou += R(rhobar, i, j, k + 1);
                rhoedgeu += (J(i, j, k + 1) * R(rhobar, i, j, k) + J(i, j, k) * R(rhobar, i, j, k + 1)) /
                            (J(i, j, k) + J(i, j, k + 1));
                const double gradient = grad_w(c, pip, i, j, k);
                const double force = force_w(c, dudt, dvdt, i, j, k);
                const double n2edgeu = (J(i, j, k + 1) * R(n2, i, j, k) + J(i, j, k) * R(n2, i, j, k + 1)) /
                                       (J(i, j, k) + J(i, j, k + 1));
                double factor = 1.0;
                factor += dt * (J(i, j, k + 1) * R(betar, i, j, k) + J(i, j, k) * R(betar, i, j, k + 1)) /
                          (J(i, j, k) + J(i, j, k + 1)) * rayleigh_factor;
                const double bb = -g_ndim *
                                  (J(i, j, k + 1) * R(rhop, i, j, k) / rhoc / J(i, j, k) +
                                   J(i, j, k) * R(rhop, i, j, k + 1) / rhou / J(i, j, k + 1)) /
                                  (J(i, j, k) + J(i, j, k + 1));
                const double jpedger = wind_u(c, i, j, k), jpedgel = wind_u(c, i - 1, j, k);
                const double jpedgef = wind_v(c, i, j, k), jpedgeb = wind_v(c, i, j - 1, k);
                const double jpuedger = wind_u(c, i, j, k + 1), jpuedgel = wind_u(c, i - 1, j, k + 1);
                const double jpuedgef = wind_v(c, i, j, k + 1), jpuedgeb = wind_v(c, i, j - 1, k + 1);
                const double uc = 0.5 * (R(u, i, j, k) / jpedger + R(u, i - 1, j, k) / jpedgel);
                const double uu = 0.5 * (R(u, i, j, k + 1) / jpuedger + R(u, i - 1, j, k + 1) / jpuedgel);
                const double vc = 0.5 * (R(v, i, j, k) / jpedgef + R(v, i, j - 1, k) / jpedgeb);
                const double vu = 0.5 * (R(v, i, j, k + 1) / jpuedgef + R(v, i, j - 1, k + 1) / jpuedgeb);
                const double jpedgeu = wind_w(c, i, j, k);
                const double fw = buoy_w(c, i, j, k);
                const double dt2 = std::pow(dt, 2.0);
                double &wc = w[c.at(i, j, k)];
                wc = 1.0 / (factor + fw * n2edgeu * dt2) *
                     (wc - dt * gradient * jpedgeu + dt * bb * jpedgeu + dt * force / rhoedgeu * jpedgeu +
                      jpedgeu * fw * n2edgeu * dt2 *
                          (J(i, j, k + 1) * (R(met13, i, j, k) * uc + R(met23, i, j, k) * vc) +
                           J(i, j, k) * (R(met13, i, j, k + 1) * uu + R(met23, i, j, k + 1) * vu)) /
                          (J(i, j, k) + J(i, j, k + 1)));
            }
    or_set_predictand_boundaries(d, model, rho, rhop, u, v, w, pip, p);
    // RhoP (:632-728)
    for (int k = k0; k <= k1; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                const double rhoc = R(rho, i, j, k) + R(rhobar, i, j, k);
                double rhoedgeu = (J(i, j, k + 1) * R(rho, i, j, k) + J(i, j, k) * R(rho, i, j, k + 1)) /
                                  (J(i, j, k) + J(i, j, k + 1));
                rhoedgeu += (J(i, j, k + 1) * R(rhobar, i, j, k) + J(i, j, k) * R(rhobar, i, j, k + 1)) /
                            (J(i, j, k) + J(i, j, k + 1));
                double rhoedged = (J(i, j, k - 1) * R(rho, i, j, k) + J(i, j, k) * R(rho, i, j, k - 1)) /
                                  (J(i, j, k) + J(i, j, k - 1));
                rhoedged += (J(i, j, k - 1) * R(rhobar, i, j, k) + J(i, j, k) * R(rhobar, i, j, k - 1)) /
                            (J(i, j, k) + J(i, j, k - 1));
                const double jpedgeu = wind_w(c, i, j, k);
                const double jpedged = wind_w(c, i, j, k - 1);
                const double wv = 0.5 * (R(wold, i, j, k) / jpedgeu + R(wold, i, j, k - 1) / jpedged);
                double lower_gradient = grad_w(c, pip, i, j, k - 1);
                double lower_force = force_w(c, dudt, dvdt, i, j, k - 1);
                double upper_gradient = grad_w(c, pip, i, j, k);
                double upper_force = force_w(c, dudt, dvdt, i, j, k);
                if (d->ko + k == k0) {
                    lower_gradient = 0.0;
                    lower_force = 0.0;
                } else if (d->ko + k == d->z_size + d->nbz - 1) {
                    upper_gradient = 0.0;
                    upper_force = 0.0;
                }
                const double gradient = 0.5 * (lower_gradient + upper_gradient);
                const double force = 0.5 * (lower_force / rhoedged + upper_force / rhoedgeu) * rhoc;
                double factor = 1.0;
                factor += dt * R(betar, i, j, k) * rayleigh_factor;
                double bb = -g_ndim * R(rhop, i, j, k) / (R(rho, i, j, k) + R(rhobar, i, j, k));
                const double jpedger = wind_u(c, i, j, k), jpedgel = wind_u(c, i - 1, j, k);
                const double jpedgef = wind_v(c, i, j, k), jpedgeb = wind_v(c, i, j - 1, k);
                const double fb = buoy_rhop(c, i, j, k);
                const double n2c = R(n2, i, j, k), jc = J(i, j, k);
                bb = 1.0 / (factor + fb * n2c * std::pow(dt, 2.0)) *
                     (-fb * n2c * dt * jc * (wv + dt * (-gradient + force / rhoc)) + factor * bb +
                      fb * n2c * dt * jc * factor * 0.5 *
                          (R(met13, i, j, k) * (R(u, i, j, k) / jpedger + R(u, i - 1, j, k) / jpedgel) +
                           R(met23, i, j, k) * (R(v, i, j, k) / jpedgef + R(v, i, j - 1, k) / jpedgeb)));
                rhop[c.at(i, j, k)] = -bb * (R(rho, i, j, k) + R(rhobar, i, j, k)) / g_ndim;
            }
    or_set_predictand_boundaries(d, model, rho, rhop, u, v, w, pip, p);
}

}  // extern "C"
