// or_operator.cpp -- CPU oracle (test infrastructure only): operator assembly.
//
// Literal FP64 restatement of compute_operator!
// (src/PoissonSolver/compute_operator!.jl:40-1606) with
// compute_buoyancy_factor(..., W()) (src/Update/compute_buoyancy_factor.jl:135-172)
// inlined.  The statement order and the branch order of every
// `if ko + k == ...` chain follow the reference, so that rounding matches a
// non-contracting (-ffp-contract=off) evaluation of the Julia expressions.
#include "pcf_oracle.h"

#include <cmath>
#include <cstddef>

extern "C" void or_compute_operator(const or_dims *d, int model, double dx, double dy,
                                    double dz, const double *jac, const double *met13,
                                    const double *met23, const double *met33,
                                    const double *pbar, const double *rhobar,
                                    const double *thetabar, const double *n2,
                                    const double *rho, const double *betar, const double *p,
                                    double dt, double rayleigh_factor,
                                    int damp_horizontal_wind_on_rhs, double *coef) {
    const int nbx = d->nbx, nby = d->nby, nbz = d->nbz;
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    const int nxx = nx + 2 * nbx, nyy = ny + 2 * nby;
    const int ko = d->ko, z_size = d->z_size;
    const size_t vol = (size_t)nx * ny * nz;
    double cst[12];
    or_constants(cst);
    const double gamma = cst[0], kappa = cst[1], rsp = cst[2], pref = cst[5];

#pragma omp parallel for collapse(2) schedule(static)
    for (int k = nbz; k < nbz + nz; ++k)
        for (int j = nby; j < nby + ny; ++j)
            for (int i = nbx; i < nbx + nx; ++i) {
                auto H = [&](int a, int b, int c) {
                    return (size_t)a + (size_t)nxx * ((size_t)b + (size_t)nyy * (size_t)c);
                };
                auto PB = [&](int a, int b, int c) { return pbar[H(a, b, c)]; };
                auto RB = [&](int a, int b, int c) { return rhobar[H(a, b, c)]; };
                auto J = [&](int a, int b, int c) { return jac[H(a, b, c)]; };
                auto R = [&](int a, int b, int c) { return rho[H(a, b, c)]; };
                auto BR = [&](int a, int b, int c) { return betar[H(a, b, c)]; };
                auto N2 = [&](int a, int b, int c) { return n2[H(a, b, c)]; };
                auto M13 = [&](int a, int b, int c) { return met13[H(a, b, c)]; };
                auto M23 = [&](int a, int b, int c) { return met23[H(a, b, c)]; };
                auto M33 = [&](int a, int b, int c) { return met33[H(a, b, c)]; };
                auto fc = [&](int a, int b, int c) {
                    return std::sqrt(std::pow(PB(a, b, c), 2.0) / RB(a, b, c));
                };
                // compute_buoyancy_factor(state, i, j, k, W()) at (i, j, kk)
                auto fw = [&](int kk) {
                    if (model == OR_COMPRESSIBLE)
                        return (J(i, j, kk + 1) * PB(i, j, kk) / thetabar[H(i, j, kk)] +
                                J(i, j, kk) * PB(i, j, kk + 1) / thetabar[H(i, j, kk + 1)]) /
                               (J(i, j, kk + 1) * (R(i, j, kk) + RB(i, j, kk)) +
                                J(i, j, kk) * (R(i, j, kk + 1) + RB(i, j, kk + 1)));
                    return (J(i, j, kk + 1) * RB(i, j, kk) + J(i, j, kk) * RB(i, j, kk + 1)) /
                           (J(i, j, kk + 1) * (R(i, j, kk) + RB(i, j, kk)) +
                            J(i, j, kk) * (R(i, j, kk + 1) + RB(i, j, kk + 1)));
                };

                // compute_operator!.jl:85-109
                const double fcscal = fc(i, j, k);
                const double fcscal_r = fc(i + 1, j, k), fcscal_l = fc(i - 1, j, k);
                const double fcscal_f = fc(i, j + 1, k), fcscal_b = fc(i, j - 1, k);
                const double fcscal_u = fc(i, j, k + 1), fcscal_d = fc(i, j, k - 1);
                const double fcscal_ru = fc(i + 1, j, k + 1), fcscal_rd = fc(i + 1, j, k - 1);
                const double fcscal_lu = fc(i - 1, j, k + 1), fcscal_ld = fc(i - 1, j, k - 1);
                const double fcscal_fu = fc(i, j + 1, k + 1), fcscal_fd = fc(i, j + 1, k - 1);
                const double fcscal_bu = fc(i, j - 1, k + 1), fcscal_bd = fc(i, j - 1, k - 1);
                const double fcscal_uu = fc(i, j, k + 2), fcscal_dd = fc(i, j, k - 2);
                const double fcscal_ruu = fc(i + 1, j, k + 2), fcscal_rdd = fc(i + 1, j, k - 2);
                const double fcscal_luu = fc(i - 1, j, k + 2), fcscal_ldd = fc(i - 1, j, k - 2);
                const double fcscal_fuu = fc(i, j + 1, k + 2), fcscal_fdd = fc(i, j + 1, k - 2);
                const double fcscal_buu = fc(i, j - 1, k + 2), fcscal_bdd = fc(i, j - 1, k - 2);

                // :112
                const double jacinv = 1.0 / J(i, j, k);

                // :115-138
                const double pedgerdiv = 0.5 * (J(i, j, k) * PB(i, j, k) + J(i + 1, j, k) * PB(i + 1, j, k));
                const double pedgeldiv = 0.5 * (J(i, j, k) * PB(i, j, k) + J(i - 1, j, k) * PB(i - 1, j, k));
                const double pedgefdiv = 0.5 * (J(i, j, k) * PB(i, j, k) + J(i, j + 1, k) * PB(i, j + 1, k));
                const double pedgebdiv = 0.5 * (J(i, j, k) * PB(i, j, k) + J(i, j - 1, k) * PB(i, j - 1, k));
                const double pedgeudiv = J(i, j, k) * J(i, j, k + 1) * (PB(i, j, k) + PB(i, j, k + 1)) /
                                         (J(i, j, k) + J(i, j, k + 1));
                const double pedgeddiv = J(i, j, k) * J(i, j, k - 1) * (PB(i, j, k) + PB(i, j, k - 1)) /
                                         (J(i, j, k) + J(i, j, k - 1));

                // :141-161
                const double pedgergra = 0.5 * (PB(i, j, k) + PB(i + 1, j, k));
                const double pedgelgra = 0.5 * (PB(i, j, k) + PB(i - 1, j, k));
                const double pedgefgra = 0.5 * (PB(i, j, k) + PB(i, j + 1, k));
                const double pedgebgra = 0.5 * (PB(i, j, k) + PB(i, j - 1, k));
                const double pedgeugra = (J(i, j, k + 1) * PB(i, j, k) + J(i, j, k) * PB(i, j, k + 1)) /
                                         (J(i, j, k) + J(i, j, k + 1));
                const double pedgedgra = (J(i, j, k - 1) * PB(i, j, k) + J(i, j, k) * PB(i, j, k - 1)) /
                                         (J(i, j, k) + J(i, j, k - 1));
                const double puedgergra = 0.5 * (PB(i, j, k + 1) + PB(i + 1, j, k + 1));
                const double puedgelgra = 0.5 * (PB(i, j, k + 1) + PB(i - 1, j, k + 1));
                const double puedgefgra = 0.5 * (PB(i, j, k + 1) + PB(i, j + 1, k + 1));
                const double puedgebgra = 0.5 * (PB(i, j, k + 1) + PB(i, j - 1, k + 1));
                const double pdedgergra = 0.5 * (PB(i, j, k - 1) + PB(i + 1, j, k - 1));
                const double pdedgelgra = 0.5 * (PB(i, j, k - 1) + PB(i - 1, j, k - 1));
                const double pdedgefgra = 0.5 * (PB(i, j, k - 1) + PB(i, j + 1, k - 1));
                const double pdedgebgra = 0.5 * (PB(i, j, k - 1) + PB(i, j - 1, k - 1));

                // :164-195
                const double rhobaredger = 0.5 * (RB(i, j, k) + RB(i + 1, j, k));
                const double rhobaredgel = 0.5 * (RB(i, j, k) + RB(i - 1, j, k));
                const double rhobaredgef = 0.5 * (RB(i, j, k) + RB(i, j + 1, k));
                const double rhobaredgeb = 0.5 * (RB(i, j, k) + RB(i, j - 1, k));
                const double rhobaredgeu = (J(i, j, k + 1) * RB(i, j, k) + J(i, j, k) * RB(i, j, k + 1)) /
                                           (J(i, j, k) + J(i, j, k + 1));
                const double rhobaredged = (J(i, j, k - 1) * RB(i, j, k) + J(i, j, k) * RB(i, j, k - 1)) /
                                           (J(i, j, k) + J(i, j, k - 1));
                const double rhoedger = 0.5 * (R(i, j, k) + R(i + 1, j, k)) + rhobaredger;
                const double rhoedgel = 0.5 * (R(i, j, k) + R(i - 1, j, k)) + rhobaredgel;
                const double rhoedgef = 0.5 * (R(i, j, k) + R(i, j + 1, k)) + rhobaredgef;
                const double rhoedgeb = 0.5 * (R(i, j, k) + R(i, j - 1, k)) + rhobaredgeb;
                const double rhoedgeu = (J(i, j, k + 1) * R(i, j, k) + J(i, j, k) * R(i, j, k + 1)) /
                                            (J(i, j, k) + J(i, j, k + 1)) + rhobaredgeu;
                const double rhoedged = (J(i, j, k - 1) * R(i, j, k) + J(i, j, k) * R(i, j, k - 1)) /
                                            (J(i, j, k) + J(i, j, k - 1)) + rhobaredged;

                // :200-201
                const double fwu = fw(k);
                const double fwd = fw(k - 1);

                // :203-258
                const double rhouedger = 0.5 * (R(i, j, k + 1) + R(i + 1, j, k + 1) + RB(i, j, k + 1) + RB(i + 1, j, k + 1));
                const double rhouedgel = 0.5 * (R(i, j, k + 1) + R(i - 1, j, k + 1) + RB(i, j, k + 1) + RB(i - 1, j, k + 1));
                const double rhouedgef = 0.5 * (R(i, j, k + 1) + R(i, j + 1, k + 1) + RB(i, j, k + 1) + RB(i, j + 1, k + 1));
                const double rhouedgeb = 0.5 * (R(i, j, k + 1) + R(i, j - 1, k + 1) + RB(i, j, k + 1) + RB(i, j - 1, k + 1));
                const double rhodedger = 0.5 * (R(i, j, k - 1) + R(i + 1, j, k - 1) + RB(i, j, k - 1) + RB(i + 1, j, k - 1));
                const double rhodedgel = 0.5 * (R(i, j, k - 1) + R(i - 1, j, k - 1) + RB(i, j, k - 1) + RB(i - 1, j, k - 1));
                const double rhodedgef = 0.5 * (R(i, j, k - 1) + R(i, j + 1, k - 1) + RB(i, j, k - 1) + RB(i, j + 1, k - 1));
                const double rhodedgeb = 0.5 * (R(i, j, k - 1) + R(i, j - 1, k - 1) + RB(i, j, k - 1) + RB(i, j - 1, k - 1));

                // :261-266
                const double n2edgeu = (J(i, j, k + 1) * N2(i, j, k) + J(i, j, k) * N2(i, j, k + 1)) /
                                       (J(i, j, k) + J(i, j, k + 1));
                const double n2edged = (J(i, j, k - 1) * N2(i, j, k) + J(i, j, k) * N2(i, j, k - 1)) /
                                       (J(i, j, k) + J(i, j, k - 1));

                // :269-318
                const double met13edger = 0.5 * (M13(i, j, k) + M13(i + 1, j, k));
                const double met13edgel = 0.5 * (M13(i, j, k) + M13(i - 1, j, k));
                const double met23edgef = 0.5 * (M23(i, j, k) + M23(i, j + 1, k));
                const double met23edgeb = 0.5 * (M23(i, j, k) + M23(i, j - 1, k));
                const double met13edgeu = (J(i, j, k + 1) * M13(i, j, k) + J(i, j, k) * M13(i, j, k + 1)) /
                                          (J(i, j, k) + J(i, j, k + 1));
                const double met23edgeu = (J(i, j, k + 1) * M23(i, j, k) + J(i, j, k) * M23(i, j, k + 1)) /
                                          (J(i, j, k) + J(i, j, k + 1));
                const double met33edgeu = (J(i, j, k + 1) * M33(i, j, k) + J(i, j, k) * M33(i, j, k + 1)) /
                                          (J(i, j, k) + J(i, j, k + 1));
                const double met13edged = (J(i, j, k - 1) * M13(i, j, k) + J(i, j, k) * M13(i, j, k - 1)) /
                                          (J(i, j, k) + J(i, j, k - 1));
                const double met23edged = (J(i, j, k - 1) * M23(i, j, k) + J(i, j, k) * M23(i, j, k - 1)) /
                                          (J(i, j, k) + J(i, j, k - 1));
                const double met33edged = (J(i, j, k - 1) * M33(i, j, k) + J(i, j, k) * M33(i, j, k - 1)) /
                                          (J(i, j, k) + J(i, j, k - 1));
                const double met13uedger = 0.5 * (M13(i, j, k + 1) + M13(i + 1, j, k + 1));
                const double met13uedgel = 0.5 * (M13(i, j, k + 1) + M13(i - 1, j, k + 1));
                const double met23uedgef = 0.5 * (M23(i, j, k + 1) + M23(i, j + 1, k + 1));
                const double met23uedgeb = 0.5 * (M23(i, j, k + 1) + M23(i, j - 1, k + 1));
                const double met13dedger = 0.5 * (M13(i, j, k - 1) + M13(i + 1, j, k - 1));
                const double met13dedgel = 0.5 * (M13(i, j, k - 1) + M13(i - 1, j, k - 1));
                const double met23dedgef = 0.5 * (M23(i, j, k - 1) + M23(i, j + 1, k - 1));
                const double met23dedgeb = 0.5 * (M23(i, j, k - 1) + M23(i, j - 1, k - 1));

                // :321-406 Rayleigh damping
                double facedger = 1.0, facedgel = 1.0, facedgef = 1.0, facedgeb = 1.0;
                double facuedger = 1.0, facuedgel = 1.0, facuedgef = 1.0, facuedgeb = 1.0;
                double facdedger = 1.0, facdedgel = 1.0, facdedgef = 1.0, facdedgeb = 1.0;
                double facedgeu = 1.0, facedged = 1.0;
                if (damp_horizontal_wind_on_rhs) {
                    facedger += dt * 0.5 * (BR(i, j, k) + BR(i + 1, j, k)) * rayleigh_factor;
                    facedgel += dt * 0.5 * (BR(i, j, k) + BR(i - 1, j, k)) * rayleigh_factor;
                    facedgef += dt * 0.5 * (BR(i, j, k) + BR(i, j + 1, k)) * rayleigh_factor;
                    facedgeb += dt * 0.5 * (BR(i, j, k) + BR(i, j - 1, k)) * rayleigh_factor;
                    facuedger += dt * 0.5 * (BR(i, j, k + 1) + BR(i + 1, j, k + 1)) * rayleigh_factor;
                    facuedgel += dt * 0.5 * (BR(i, j, k + 1) + BR(i - 1, j, k + 1)) * rayleigh_factor;
                    facuedgef += dt * 0.5 * (BR(i, j, k + 1) + BR(i, j + 1, k + 1)) * rayleigh_factor;
                    facuedgeb += dt * 0.5 * (BR(i, j, k + 1) + BR(i, j - 1, k + 1)) * rayleigh_factor;
                    facdedger += dt * 0.5 * (BR(i, j, k - 1) + BR(i + 1, j, k - 1)) * rayleigh_factor;
                    facdedgel += dt * 0.5 * (BR(i, j, k - 1) + BR(i - 1, j, k - 1)) * rayleigh_factor;
                    facdedgef += dt * 0.5 * (BR(i, j, k - 1) + BR(i, j + 1, k - 1)) * rayleigh_factor;
                    facdedgeb += dt * 0.5 * (BR(i, j, k - 1) + BR(i, j - 1, k - 1)) * rayleigh_factor;
                }
                facedgeu += dt * (J(i, j, k + 1) * BR(i, j, k) + J(i, j, k) * BR(i, j, k + 1)) /
                            (J(i, j, k) + J(i, j, k + 1)) * rayleigh_factor;
                facedged += dt * (J(i, j, k - 1) * BR(i, j, k) + J(i, j, k) * BR(i, j, k - 1)) /
                            (J(i, j, k) + J(i, j, k - 1)) * rayleigh_factor;

                // :409-422
                const double imphoredger = 1.0 / facedger, imphoredgel = 1.0 / facedgel;
                const double imphoredgef = 1.0 / facedgef, imphoredgeb = 1.0 / facedgeb;
                const double imphoruedger = 1.0 / facuedger, imphoruedgel = 1.0 / facuedgel;
                const double imphoruedgef = 1.0 / facuedgef, imphoruedgeb = 1.0 / facuedgeb;
                const double imphordedger = 1.0 / facdedger, imphordedgel = 1.0 / facdedgel;
                const double imphordedgef = 1.0 / facdedgef, imphordedgeb = 1.0 / facdedgeb;
                const double dt2 = std::pow(dt, 2.0);
                const double impveredgeu = 1.0 / (facedgeu + fwu * n2edgeu * dt2);
                const double impveredged = 1.0 / (facedged + fwd * n2edged * dt2);

                // Branch selectors (Julia: ko + k == k0, k0 + 1, z_size + nbz - 1, z_size + nbz)
                const int kg = ko + k;  // 0-based global haloed level
                const bool BOT = kg == nbz, BOT1 = kg == nbz + 1;
                const bool TOP1 = kg == z_size + nbz - 2, TOP = kg == z_size + nbz - 1;

                // Shared sub-expressions of the G terms, written as in the reference.
                auto up_term = [&](double met) {  // jacinv/dz*pedgeudiv*impveredgeu*fwu*n2edgeu*dt^2*0.5*met*jac(k+1)/(jac+jac(k+1))
                    return jacinv / dz * pedgeudiv * impveredgeu * fwu * n2edgeu * dt2 * 0.5 * met *
                           J(i, j, k + 1) / (J(i, j, k) + J(i, j, k + 1));
                };
                auto dn_term = [&](double met) {
                    return jacinv / dz * pedgeddiv * impveredged * fwd * n2edged * dt2 * 0.5 * met *
                           J(i, j, k - 1) / (J(i, j, k) + J(i, j, k - 1));
                };

                // :426-477 G(i + 1/2)
                double gedger, gedgel, gedgef, gedgeb;
                if (BOT)
                    gedger = jacinv / dx * pedgerdiv * imphoredger / rhoedger +
                             up_term(M13(i, j, k)) * imphoredger / rhoedger;
                else if (TOP)
                    gedger = jacinv / dx * pedgerdiv * imphoredger / rhoedger -
                             dn_term(M13(i, j, k)) * imphoredger / rhoedger;
                else
                    gedger = jacinv / dx * pedgerdiv * imphoredger / rhoedger +
                             up_term(M13(i, j, k)) * imphoredger / rhoedger -
                             dn_term(M13(i, j, k)) * imphoredger / rhoedger;
                // :480-531 G(i - 1/2)
                if (BOT)
                    gedgel = -jacinv / dx * pedgeldiv * imphoredgel / rhoedgel +
                             up_term(M13(i, j, k)) * imphoredgel / rhoedgel;
                else if (TOP)
                    gedgel = -jacinv / dx * pedgeldiv * imphoredgel / rhoedgel -
                             dn_term(M13(i, j, k)) * imphoredgel / rhoedgel;
                else
                    gedgel = -jacinv / dx * pedgeldiv * imphoredgel / rhoedgel +
                             up_term(M13(i, j, k)) * imphoredgel / rhoedgel -
                             dn_term(M13(i, j, k)) * imphoredgel / rhoedgel;
                // :534-585 G(j + 1/2)
                if (BOT)
                    gedgef = jacinv / dy * pedgefdiv * imphoredgef / rhoedgef +
                             up_term(M23(i, j, k)) * imphoredgef / rhoedgef;
                else if (TOP)
                    gedgef = jacinv / dy * pedgefdiv * imphoredgef / rhoedgef -
                             dn_term(M23(i, j, k)) * imphoredgef / rhoedgef;
                else
                    gedgef = jacinv / dy * pedgefdiv * imphoredgef / rhoedgef +
                             up_term(M23(i, j, k)) * imphoredgef / rhoedgef -
                             dn_term(M23(i, j, k)) * imphoredgef / rhoedgef;
                // :588-639 G(j - 1/2)
                if (BOT)
                    gedgeb = -jacinv / dy * pedgebdiv * imphoredgeb / rhoedgeb +
                             up_term(M23(i, j, k)) * imphoredgeb / rhoedgeb;
                else if (TOP)
                    gedgeb = -jacinv / dy * pedgebdiv * imphoredgeb / rhoedgeb -
                             dn_term(M23(i, j, k)) * imphoredgeb / rhoedgeb;
                else
                    gedgeb = -jacinv / dy * pedgebdiv * imphoredgeb / rhoedgeb +
                             up_term(M23(i, j, k)) * imphoredgeb / rhoedgeb -
                             dn_term(M23(i, j, k)) * imphoredgeb / rhoedgeb;

                // :642-653
                const double gedgeu = TOP ? 0.0 : jacinv / dz * pedgeudiv * impveredgeu / rhoedgeu;
                const double gedged = BOT ? 0.0 : -jacinv / dz * pedgeddiv * impveredged / rhoedged;

                // :656-722 G(., k + 1)
                auto uk_term = [&](double met) {  // ... * met(k+1) * jac / (jac + jac(k+1))
                    return jacinv / dz * pedgeudiv * impveredgeu * fwu * n2edgeu * dt2 * 0.5 * met *
                           J(i, j, k) / (J(i, j, k) + J(i, j, k + 1));
                };
                auto dk_term = [&](double met) {
                    return -jacinv / dz * pedgeddiv * impveredged * fwd * n2edged * dt2 * 0.5 * met *
                           J(i, j, k) / (J(i, j, k) + J(i, j, k - 1));
                };
                const double guedger = TOP ? 0.0 : uk_term(M13(i, j, k + 1)) * imphoruedger / rhouedger;
                const double guedgel = TOP ? 0.0 : uk_term(M13(i, j, k + 1)) * imphoruedgel / rhouedgel;
                const double guedgef = TOP ? 0.0 : uk_term(M23(i, j, k + 1)) * imphoruedgef / rhouedgef;
                const double guedgeb = TOP ? 0.0 : uk_term(M23(i, j, k + 1)) * imphoruedgeb / rhouedgeb;
                // :725-791 G(., k - 1)
                const double gdedger = BOT ? 0.0 : dk_term(M13(i, j, k - 1)) * imphordedger / rhodedger;
                const double gdedgel = BOT ? 0.0 : dk_term(M13(i, j, k - 1)) * imphordedgel / rhodedgel;
                const double gdedgef = BOT ? 0.0 : dk_term(M23(i, j, k - 1)) * imphordedgef / rhodedgef;
                const double gdedgeb = BOT ? 0.0 : dk_term(M23(i, j, k - 1)) * imphordedgeb / rhodedgeb;

                // Frequently used jac ratios of the neighbour columns.
                auto jr = [&](double x, int a, int b, int kn) {  // x * jac(a,b,kn) / (jac(a,b,k) + jac(a,b,kn))
                    return x * J(a, b, kn) / (J(a, b, k) + J(a, b, kn));
                };

                // :795-853 A(i,j,k)
                double ac;
                if (BOT)
                    ac = -gedger * pedgergra * (1.0 / dx + 0.75 * met13edger / dz) +
                         gedgel * pedgelgra * (1.0 / dx - 0.75 * met13edgel / dz) -
                         gedgef * pedgefgra * (1.0 / dy + 0.75 * met23edgef / dz) +
                         gedgeb * pedgebgra * (1.0 / dy - 0.75 * met23edgeb / dz) -
                         gedgeu * pedgeugra * met33edgeu / dz -
                         guedger * puedgergra * 0.25 * met13uedger / dz -
                         guedgel * puedgelgra * 0.25 * met13uedgel / dz -
                         guedgef * puedgefgra * 0.25 * met23uedgef / dz -
                         guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;
                else if (BOT1)
                    ac = -gedger * pedgergra / dx + gedgel * pedgelgra / dx -
                         gedgef * pedgefgra / dy + gedgeb * pedgebgra / dy -
                         gedgeu * pedgeugra * met33edgeu / dz +
                         gedged * pedgedgra * met33edged / dz -
                         guedger * puedgergra * 0.25 * met13uedger / dz -
                         guedgel * puedgelgra * 0.25 * met13uedgel / dz -
                         guedgef * puedgefgra * 0.25 * met23uedgef / dz -
                         guedgeb * puedgebgra * 0.25 * met23uedgeb / dz +
                         gdedger * pdedgergra * met13dedger / dz +
                         gdedgel * pdedgelgra * met13dedgel / dz +
                         gdedgef * pdedgefgra * met23dedgef / dz +
                         gdedgeb * pdedgebgra * met23dedgeb / dz;
                else if (TOP1)
                    ac = -gedger * pedgergra / dx + gedgel * pedgelgra / dx -
                         gedgef * pedgefgra / dy + gedgeb * pedgebgra / dy -
                         gedgeu * pedgeugra * met33edgeu / dz +
                         gedged * pedgedgra * met33edged / dz -
                         guedger * puedgergra * met13uedger / dz -
                         guedgel * puedgelgra * met13uedgel / dz -
                         guedgef * puedgefgra * met23uedgef / dz -
                         guedgeb * puedgebgra * met23uedgeb / dz +
                         gdedger * pdedgergra * 0.25 * met13dedger / dz +
                         gdedgel * pdedgelgra * 0.25 * met13dedgel / dz +
                         gdedgef * pdedgefgra * 0.25 * met23dedgef / dz +
                         gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else if (TOP)
                    ac = -gedger * pedgergra * (1.0 / dx - 0.75 * met13edger / dz) +
                         gedgel * pedgelgra * (1.0 / dx + 0.75 * met13edgel / dz) -
                         gedgef * pedgefgra * (1.0 / dy - 0.75 * met23edgef / dz) +
                         gedgeb * pedgebgra * (1.0 / dy + 0.75 * met23edgeb / dz) +
                         gedged * pedgedgra * met33edged / dz +
                         gdedger * pdedgergra * 0.25 * met13dedger / dz +
                         gdedgel * pdedgelgra * 0.25 * met13dedgel / dz +
                         gdedgef * pdedgefgra * 0.25 * met23dedgef / dz +
                         gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else
                    ac = -gedger * pedgergra / dx + gedgel * pedgelgra / dx -
                         gedgef * pedgefgra / dy + gedgeb * pedgebgra / dy -
                         gedgeu * pedgeugra * met33edgeu / dz +
                         gedged * pedgedgra * met33edged / dz -
                         guedger * puedgergra * 0.25 * met13uedger / dz -
                         guedgel * puedgelgra * 0.25 * met13uedgel / dz -
                         guedgef * puedgefgra * 0.25 * met23uedgef / dz -
                         guedgeb * puedgebgra * 0.25 * met23uedgeb / dz +
                         gdedger * pdedgergra * 0.25 * met13dedger / dz +
                         gdedgel * pdedgelgra * 0.25 * met13dedgel / dz +
                         gdedgef * pdedgefgra * 0.25 * met23dedgef / dz +
                         gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;

                // :855-860 Compressible correction
                if (model == OR_COMPRESSIBLE) {
                    const double dpdpi = 1 / (gamma - 1) * std::pow(rsp / pref, 1 - gamma) *
                                         std::pow(p[H(i, j, k)], 2 - gamma);
                    ac -= (dpdpi / dt) / (dt * rsp / kappa);
                }

                // :864-907 A(i+1,j,k)
                double ar;
                if (BOT)
                    ar = gedger * pedgergra * (1.0 / dx - 0.75 * met13edger / dz) +
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i + 1, j, k + 1) -
                         guedger * puedgergra * 0.25 * met13uedger / dz;
                else if (BOT1)
                    ar = gedger * pedgergra / dx +
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i + 1, j, k + 1) +
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i + 1, j, k - 1) -
                         guedger * puedgergra * 0.25 * met13uedger / dz +
                         gdedger * pdedgergra * met13dedger / dz;
                else if (TOP1)
                    ar = gedger * pedgergra / dx +
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i + 1, j, k + 1) +
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i + 1, j, k - 1) -
                         guedger * puedgergra * met13uedger / dz +
                         gdedger * pdedgergra * 0.25 * met13dedger / dz;
                else if (TOP)
                    ar = gedger * pedgergra * (1.0 / dx + 0.75 * met13edger / dz) +
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i + 1, j, k - 1) +
                         gdedger * pdedgergra * 0.25 * met13dedger / dz;
                else
                    ar = gedger * pedgergra / dx +
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i + 1, j, k + 1) +
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i + 1, j, k - 1) -
                         guedger * puedgergra * 0.25 * met13uedger / dz +
                         gdedger * pdedgergra * 0.25 * met13dedger / dz;

                // :911-957 A(i-1,j,k)
                double al;
                if (BOT)
                    al = -gedgel * pedgelgra * (1.0 / dx + 0.75 * met13edgel / dz) -
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i - 1, j, k + 1) -
                         guedgel * puedgelgra * 0.25 * met13uedgel / dz;
                else if (BOT1)
                    al = -gedgel * pedgelgra / dx -
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i - 1, j, k + 1) -
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i - 1, j, k - 1) -
                         guedgel * puedgelgra * 0.25 * met13uedgel / dz +
                         gdedgel * pdedgelgra * met13dedgel / dz;
                else if (TOP1)
                    al = -gedgel * pedgelgra / dx -
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i - 1, j, k + 1) -
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i - 1, j, k - 1) -
                         guedgel * puedgelgra * met13uedgel / dz +
                         gdedgel * pdedgelgra * 0.25 * met13dedgel / dz;
                else if (TOP)
                    al = -gedgel * pedgelgra * (1.0 / dx - 0.75 * met13edgel / dz) -
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i - 1, j, k - 1) +
                         gdedgel * pdedgelgra * 0.25 * met13dedgel / dz;
                else
                    al = -gedgel * pedgelgra / dx -
                         jr(gedgeu * pedgeugra * 0.5 * met13edgeu / dx, i - 1, j, k + 1) -
                         jr(gedged * pedgedgra * 0.5 * met13edged / dx, i - 1, j, k - 1) -
                         guedgel * puedgelgra * 0.25 * met13uedgel / dz +
                         gdedgel * pdedgelgra * 0.25 * met13dedgel / dz;

                // :961-1004 A(i,j+1,k)
                double af;
                if (BOT)
                    af = gedgef * pedgefgra * (1.0 / dy - 0.75 * met23edgef / dz) +
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j + 1, k + 1) -
                         guedgef * puedgefgra * 0.25 * met23uedgef / dz;
                else if (BOT1)
                    af = gedgef * pedgefgra / dy +
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j + 1, k + 1) +
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j + 1, k - 1) -
                         guedgef * puedgefgra * 0.25 * met23uedgef / dz +
                         gdedgef * pdedgefgra * met23dedgef / dz;
                else if (TOP1)
                    af = gedgef * pedgefgra / dy +
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j + 1, k + 1) +
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j + 1, k - 1) -
                         guedgef * puedgefgra * met23uedgef / dz +
                         gdedgef * pdedgefgra * 0.25 * met23dedgef / dz;
                else if (TOP)
                    af = gedgef * pedgefgra * (1.0 / dy + 0.75 * met23edgef / dz) +
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j + 1, k - 1) +
                         gdedgef * pdedgefgra * 0.25 * met23dedgef / dz;
                else
                    af = gedgef * pedgefgra / dy +
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j + 1, k + 1) +
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j + 1, k - 1) -
                         guedgef * puedgefgra * 0.25 * met23uedgef / dz +
                         gdedgef * pdedgefgra * 0.25 * met23dedgef / dz;

                // :1008-1054 A(i,j-1,k)
                double ab;
                if (BOT)
                    ab = -gedgeb * pedgebgra * (1.0 / dy + 0.75 * met23edgeb / dz) -
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j - 1, k + 1) -
                         guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;
                else if (BOT1)
                    ab = -gedgeb * pedgebgra / dy -
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j - 1, k + 1) -
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j - 1, k - 1) -
                         guedgeb * puedgebgra * 0.25 * met23uedgeb / dz +
                         gdedgeb * pdedgebgra * met23dedgeb / dz;
                else if (TOP1)
                    ab = -gedgeb * pedgebgra / dy -
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j - 1, k + 1) -
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j - 1, k - 1) -
                         guedgeb * puedgebgra * met23uedgeb / dz +
                         gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else if (TOP)
                    ab = -gedgeb * pedgebgra * (1.0 / dy - 0.75 * met23edgeb / dz) -
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j - 1, k - 1) +
                         gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else
                    ab = -gedgeb * pedgebgra / dy -
                         jr(gedgeu * pedgeugra * 0.5 * met23edgeu / dy, i, j - 1, k + 1) -
                         jr(gedged * pedgedgra * 0.5 * met23edged / dy, i, j - 1, k - 1) -
                         guedgeb * puedgebgra * 0.25 * met23uedgeb / dz +
                         gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;

                // :1058-1096 A(i,j,k+1)
                double au;
                if (BOT)
                    au = gedger * pedgergra * met13edger / dz + gedgel * pedgelgra * met13edgel / dz +
                         gedgef * pedgefgra * met23edgef / dz + gedgeb * pedgebgra * met23edgeb / dz +
                         gedgeu * pedgeugra * met33edgeu / dz - guedger * puedgergra / dx +
                         guedgel * puedgelgra / dx - guedgef * puedgefgra / dy +
                         guedgeb * puedgebgra / dy;
                else if (BOT1)
                    au = gedger * pedgergra * 0.25 * met13edger / dz +
                         gedgel * pedgelgra * 0.25 * met13edgel / dz +
                         gedgef * pedgefgra * 0.25 * met23edgef / dz +
                         gedgeb * pedgebgra * 0.25 * met23edgeb / dz +
                         gedgeu * pedgeugra * met33edgeu / dz - guedger * puedgergra / dx +
                         guedgel * puedgelgra / dx - guedgef * puedgefgra / dy +
                         guedgeb * puedgebgra / dy -
                         gdedger * pdedgergra * 0.25 * met13dedger / dz -
                         gdedgel * pdedgelgra * 0.25 * met13dedgel / dz -
                         gdedgef * pdedgefgra * 0.25 * met23dedgef / dz -
                         gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else if (TOP1)
                    au = gedger * pedgergra * 0.25 * met13edger / dz +
                         gedgel * pedgelgra * 0.25 * met13edgel / dz +
                         gedgef * pedgefgra * 0.25 * met23edgef / dz +
                         gedgeb * pedgebgra * 0.25 * met23edgeb / dz +
                         gedgeu * pedgeugra * met33edgeu / dz -
                         guedger * puedgergra * (1.0 / dx - 0.75 * met13uedger / dz) +
                         guedgel * puedgelgra * (1.0 / dx + 0.75 * met13uedgel / dz) -
                         guedgef * puedgefgra * (1.0 / dy - 0.75 * met23uedgef / dz) +
                         guedgeb * puedgebgra * (1.0 / dy + 0.75 * met23uedgeb / dz);
                else if (TOP)
                    au = 0.0;
                else
                    au = gedger * pedgergra * 0.25 * met13edger / dz +
                         gedgel * pedgelgra * 0.25 * met13edgel / dz +
                         gedgef * pedgefgra * 0.25 * met23edgef / dz +
                         gedgeb * pedgebgra * 0.25 * met23edgeb / dz +
                         gedgeu * pedgeugra * met33edgeu / dz - guedger * puedgergra / dx +
                         guedgel * puedgelgra / dx - guedgef * puedgefgra / dy +
                         guedgeb * puedgebgra / dy;

                // :1100-1141 A(i,j,k-1)
                double ad;
                if (BOT)
                    ad = 0.0;
                else if (BOT1)
                    ad = -gedger * pedgergra * 0.25 * met13edger / dz -
                         gedgel * pedgelgra * 0.25 * met13edgel / dz -
                         gedgef * pedgefgra * 0.25 * met23edgef / dz -
                         gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                         gedged * pedgedgra * met33edged / dz -
                         gdedger * pdedgergra * (1.0 / dx + 0.75 * met13dedger / dz) +
                         gdedgel * pdedgelgra * (1.0 / dx - 0.75 * met13dedgel / dz) -
                         gdedgef * pdedgefgra * (1.0 / dy + 0.75 * met23dedgef / dz) +
                         gdedgeb * pdedgebgra * (1.0 / dy - 0.75 * met23dedgeb / dz);
                else if (TOP1)
                    ad = -gedger * pedgergra * 0.25 * met13edger / dz -
                         gedgel * pedgelgra * 0.25 * met13edgel / dz -
                         gedgef * pedgefgra * 0.25 * met23edgef / dz -
                         gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                         gedged * pedgedgra * met33edged / dz - gdedger * pdedgergra / dx +
                         gdedgel * pdedgelgra / dx - gdedgef * pdedgefgra / dy +
                         gdedgeb * pdedgebgra / dy +
                         guedger * puedgergra * 0.25 * met13uedger / dz +
                         guedgel * puedgelgra * 0.25 * met13uedgel / dz +
                         guedgef * puedgefgra * 0.25 * met23uedgef / dz +
                         guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;
                else if (TOP)
                    ad = -gedger * pedgergra * met13edger / dz - gedgel * pedgelgra * met13edgel / dz -
                         gedgef * pedgefgra * met23edgef / dz - gedgeb * pedgebgra * met23edgeb / dz -
                         gedged * pedgedgra * met33edged / dz - gdedger * pdedgergra / dx +
                         gdedgel * pdedgelgra / dx - gdedgef * pdedgefgra / dy +
                         gdedgeb * pdedgebgra / dy;
                else
                    ad = -gedger * pedgergra * 0.25 * met13edger / dz -
                         gedgel * pedgelgra * 0.25 * met13edgel / dz -
                         gedgef * pedgefgra * 0.25 * met23edgef / dz -
                         gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                         gedged * pedgedgra * met33edged / dz - gdedger * pdedgergra / dx +
                         gdedgel * pdedgelgra / dx - gdedgef * pdedgefgra / dy +
                         gdedgeb * pdedgebgra / dy;

                // :1145-1174 A(i+1,j,k+1)
                double aru;
                if (BOT)
                    aru = gedger * pedgergra * met13edger / dz +
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k + 1)) +
                          guedger * puedgergra / dx;
                else if (BOT1)
                    aru = gedger * pedgergra * 0.25 * met13edger / dz +
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k + 1)) +
                          guedger * puedgergra / dx - gdedger * pdedgergra * 0.25 * met13dedger / dz;
                else if (TOP1)
                    aru = gedger * pedgergra * 0.25 * met13edger / dz +
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k + 1)) +
                          guedger * puedgergra * (1.0 / dx + 0.75 * met13uedger / dz);
                else if (TOP)
                    aru = 0.0;
                else
                    aru = gedger * pedgergra * 0.25 * met13edger / dz +
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k + 1)) +
                          guedger * puedgergra / dx;

                // :1178-1206 A(i+1,j,k-1)
                double ard;
                if (BOT)
                    ard = 0.0;
                else if (BOT1)
                    ard = -gedger * pedgergra * 0.25 * met13edger / dz +
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k - 1)) +
                          gdedger * pdedgergra * (1.0 / dx - 0.75 * met13dedger / dz);
                else if (TOP1)
                    ard = -gedger * pedgergra * 0.25 * met13edger / dz +
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k - 1)) +
                          gdedger * pdedgergra / dx + guedger * puedgergra * 0.25 * met13uedger / dz;
                else if (TOP)
                    ard = -gedger * pedgergra * met13edger / dz +
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k - 1)) +
                          gdedger * pdedgergra / dx;
                else
                    ard = -gedger * pedgergra * 0.25 * met13edger / dz +
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i + 1, j, k) /
                              (J(i + 1, j, k) + J(i + 1, j, k - 1)) +
                          gdedger * pdedgergra / dx;

                // :1210-1237 A(i-1,j,k+1)
                double alu;
                if (BOT)
                    alu = gedgel * pedgelgra * met13edgel / dz -
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k + 1)) -
                          guedgel * puedgelgra / dx;
                else if (BOT1)
                    alu = gedgel * pedgelgra * 0.25 * met13edgel / dz -
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k + 1)) -
                          guedgel * puedgelgra / dx - gdedgel * pdedgelgra * 0.25 * met13dedgel / dz;
                else if (TOP1)
                    alu = gedgel * pedgelgra * 0.25 * met13edgel / dz -
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k + 1)) -
                          guedgel * puedgelgra * (1.0 / dx - 0.75 * met13uedgel / dz);
                else if (TOP)
                    alu = 0.0;
                else
                    alu = gedgel * pedgelgra * 0.25 * met13edgel / dz -
                          gedgeu * pedgeugra * 0.5 * met13edgeu / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k + 1)) -
                          guedgel * puedgelgra / dx;

                // :1252-1278 A(i-1,j,k-1)
                double ald;
                if (BOT)
                    ald = 0.0;
                else if (BOT1)
                    ald = -gedgel * pedgelgra * 0.25 * met13edgel / dz -
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k - 1)) -
                          gdedgel * pdedgelgra * (1.0 / dx + 0.75 * met13dedgel / dz);
                else if (TOP1)
                    ald = -gedgel * pedgelgra * 0.25 * met13edgel / dz -
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k - 1)) -
                          gdedgel * pdedgelgra / dx + guedgel * puedgelgra * 0.25 * met13uedgel / dz;
                else if (TOP)
                    ald = -gedgel * pedgelgra * met13edgel / dz -
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k - 1)) -
                          gdedgel * pdedgelgra / dx;
                else
                    ald = -gedgel * pedgelgra * 0.25 * met13edgel / dz -
                          gedged * pedgedgra * 0.5 * met13edged / dx * J(i - 1, j, k) /
                              (J(i - 1, j, k) + J(i - 1, j, k - 1)) -
                          gdedgel * pdedgelgra / dx;

                // :1282-1309 A(i,j+1,k+1)
                double afu;
                if (BOT)
                    afu = gedgef * pedgefgra * met23edgef / dz +
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k + 1)) +
                          guedgef * puedgefgra / dy;
                else if (BOT1)
                    afu = gedgef * pedgefgra * 0.25 * met23edgef / dz +
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k + 1)) +
                          guedgef * puedgefgra / dy - gdedgef * pdedgefgra * 0.25 * met23dedgef / dz;
                else if (TOP1)
                    afu = gedgef * pedgefgra * 0.25 * met23edgef / dz +
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k + 1)) +
                          guedgef * puedgefgra * (1.0 / dy + 0.75 * met23uedgef / dz);
                else if (TOP)
                    afu = 0.0;
                else
                    afu = gedgef * pedgefgra * 0.25 * met23edgef / dz +
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k + 1)) +
                          guedgef * puedgefgra / dy;

                // :1313-1341 A(i,j+1,k-1)
                double afd;
                if (BOT)
                    afd = 0.0;
                else if (BOT1)
                    afd = -gedgef * pedgefgra * 0.25 * met23edgef / dz +
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k - 1)) +
                          gdedgef * pdedgefgra * (1.0 / dy - 0.75 * met23dedgef / dz);
                else if (TOP1)
                    afd = -gedgef * pedgefgra * 0.25 * met23edgef / dz +
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k - 1)) +
                          gdedgef * pdedgefgra / dy + guedgef * puedgefgra * 0.25 * met23uedgef / dz;
                else if (TOP)
                    afd = -gedgef * pedgefgra * met23edgef / dz +
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k - 1)) +
                          gdedgef * pdedgefgra / dy;
                else
                    afd = -gedgef * pedgefgra * 0.25 * met23edgef / dz +
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j + 1, k) /
                              (J(i, j + 1, k) + J(i, j + 1, k - 1)) +
                          gdedgef * pdedgefgra / dy;

                // :1345-1372 A(i,j-1,k+1)
                double abu;
                if (BOT)
                    abu = gedgeb * pedgebgra * met23edgeb / dz -
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k + 1)) -
                          guedgeb * puedgebgra / dy;
                else if (BOT1)
                    abu = gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k + 1)) -
                          guedgeb * puedgebgra / dy - gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else if (TOP1)
                    abu = gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k + 1)) -
                          guedgeb * puedgebgra * (1.0 / dy - 0.75 * met23uedgeb / dz);
                else if (TOP)
                    abu = 0.0;
                else
                    abu = gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                          gedgeu * pedgeugra * 0.5 * met23edgeu / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k + 1)) -
                          guedgeb * puedgebgra / dy;

                // :1376-1404 A(i,j-1,k-1)
                double abd;
                if (BOT)
                    abd = 0.0;
                else if (BOT1)
                    abd = -gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k - 1)) -
                          gdedgeb * pdedgebgra * (1.0 / dy + 0.75 * met23dedgeb / dz);
                else if (TOP1)
                    abd = -gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k - 1)) -
                          gdedgeb * pdedgebgra / dy + guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;
                else if (TOP)
                    abd = -gedgeb * pedgebgra * met23edgeb / dz -
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k - 1)) -
                          gdedgeb * pdedgebgra / dy;
                else
                    abd = -gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                          gedged * pedgedgra * 0.5 * met23edged / dy * J(i, j - 1, k) /
                              (J(i, j - 1, k) + J(i, j - 1, k - 1)) -
                          gdedgeb * pdedgebgra / dy;

                // :1408-1425 A(i,j,k+2)
                double auu;
                if (BOT)
                    auu = -gedger * pedgergra * 0.25 * met13edger / dz -
                          gedgel * pedgelgra * 0.25 * met13edgel / dz -
                          gedgef * pedgefgra * 0.25 * met23edgef / dz -
                          gedgeb * pedgebgra * 0.25 * met23edgeb / dz +
                          guedger * puedgergra * 0.25 * met13uedger / dz +
                          guedgel * puedgelgra * 0.25 * met13uedgel / dz +
                          guedgef * puedgefgra * 0.25 * met23uedgef / dz +
                          guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;
                else if (kg >= z_size + nbz - 2)
                    auu = 0.0;
                else
                    auu = guedger * puedgergra * 0.25 * met13uedger / dz +
                          guedgel * puedgelgra * 0.25 * met13uedgel / dz +
                          guedgef * puedgefgra * 0.25 * met23uedgef / dz +
                          guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;

                // :1429-1446 A(i,j,k-2)
                double add;
                if (kg <= nbz + 1)
                    add = 0.0;
                else if (TOP)
                    add = gedger * pedgergra * 0.25 * met13edger / dz +
                          gedgel * pedgelgra * 0.25 * met13edgel / dz +
                          gedgef * pedgefgra * 0.25 * met23edgef / dz +
                          gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                          gdedger * pdedgergra * 0.25 * met13dedger / dz -
                          gdedgel * pdedgelgra * 0.25 * met13dedgel / dz -
                          gdedgef * pdedgefgra * 0.25 * met23dedgef / dz -
                          gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else
                    add = -gdedger * pdedgergra * 0.25 * met13dedger / dz -
                          gdedgel * pdedgelgra * 0.25 * met13dedgel / dz -
                          gdedgef * pdedgefgra * 0.25 * met23dedgef / dz -
                          gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;

                // :1450-1543 corner k+-2 elements
                double aruu, ardd, aluu, aldd, afuu, afdd, abuu, abdd;
                const bool UUZ = kg >= z_size + nbz - 2, DDZ = kg <= nbz + 1;
                if (BOT)
                    aruu = -gedger * pedgergra * 0.25 * met13edger / dz +
                           guedger * puedgergra * 0.25 * met13uedger / dz;
                else if (UUZ)
                    aruu = 0.0;
                else
                    aruu = guedger * puedgergra * 0.25 * met13uedger / dz;
                if (DDZ)
                    ardd = 0.0;
                else if (TOP)
                    ardd = gedger * pedgergra * 0.25 * met13edger / dz -
                           gdedger * pdedgergra * 0.25 * met13dedger / dz;
                else
                    ardd = -gdedger * pdedgergra * 0.25 * met13dedger / dz;
                if (BOT)
                    aluu = -gedgel * pedgelgra * 0.25 * met13edgel / dz +
                           guedgel * puedgelgra * 0.25 * met13uedgel / dz;
                else if (UUZ)
                    aluu = 0.0;
                else
                    aluu = guedgel * puedgelgra * 0.25 * met13uedgel / dz;
                if (DDZ)
                    aldd = 0.0;
                else if (TOP)
                    aldd = gedgel * pedgelgra * 0.25 * met13edgel / dz -
                           gdedgel * pdedgelgra * 0.25 * met13dedgel / dz;
                else
                    aldd = -gdedgel * pdedgelgra * 0.25 * met13dedgel / dz;
                if (BOT)
                    afuu = -gedgef * pedgefgra * 0.25 * met23edgef / dz +
                           guedgef * puedgefgra * 0.25 * met23uedgef / dz;
                else if (UUZ)
                    afuu = 0.0;
                else
                    afuu = guedgef * puedgefgra * 0.25 * met23uedgef / dz;
                if (DDZ)
                    afdd = 0.0;
                else if (TOP)
                    afdd = gedgef * pedgefgra * 0.25 * met23edgef / dz -
                           gdedgef * pdedgefgra * 0.25 * met23dedgef / dz;
                else
                    afdd = -gdedgef * pdedgefgra * 0.25 * met23dedgef / dz;
                if (BOT)
                    abuu = -gedgeb * pedgebgra * 0.25 * met23edgeb / dz +
                           guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;
                else if (UUZ)
                    abuu = 0.0;
                else
                    abuu = guedgeb * puedgebgra * 0.25 * met23uedgeb / dz;
                if (DDZ)
                    abdd = 0.0;
                else if (TOP)
                    abdd = gedgeb * pedgebgra * 0.25 * met23edgeb / dz -
                           gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;
                else
                    abdd = -gdedgeb * pdedgebgra * 0.25 * met23dedgeb / dz;

                // :1546-1570 scaling
                ac = ac / std::pow(fcscal, 2.0);
                ar = ar / fcscal / fcscal_r;
                al = al / fcscal / fcscal_l;
                af = af / fcscal / fcscal_f;
                ab = ab / fcscal / fcscal_b;
                au = au / fcscal / fcscal_u;
                ad = ad / fcscal / fcscal_d;
                aru = aru / fcscal / fcscal_ru;
                ard = ard / fcscal / fcscal_rd;
                alu = alu / fcscal / fcscal_lu;
                ald = ald / fcscal / fcscal_ld;
                afu = afu / fcscal / fcscal_fu;
                afd = afd / fcscal / fcscal_fd;
                abu = abu / fcscal / fcscal_bu;
                abd = abd / fcscal / fcscal_bd;
                auu = auu / fcscal / fcscal_uu;
                add = add / fcscal / fcscal_dd;
                aruu = aruu / fcscal / fcscal_ruu;
                ardd = ardd / fcscal / fcscal_rdd;
                aluu = aluu / fcscal / fcscal_luu;
                aldd = aldd / fcscal / fcscal_ldd;
                afuu = afuu / fcscal / fcscal_fuu;
                afdd = afdd / fcscal / fcscal_fdd;
                abuu = abuu / fcscal / fcscal_buu;
                abdd = abdd / fcscal / fcscal_bdd;

                // :1573-1603 store
                const size_t n = (size_t)(i - nbx) + (size_t)nx * ((size_t)(j - nby) + (size_t)ny * (size_t)(k - nbz));
                double *c = coef;
                c[OR_AC * vol + n] = ac;     c[OR_AL * vol + n] = al;     c[OR_AR * vol + n] = ar;
                c[OR_AB * vol + n] = ab;     c[OR_AF * vol + n] = af;     c[OR_AD * vol + n] = ad;
                c[OR_AU * vol + n] = au;     c[OR_ALD * vol + n] = ald;   c[OR_ALU * vol + n] = alu;
                c[OR_ARD * vol + n] = ard;   c[OR_ARU * vol + n] = aru;   c[OR_ABD * vol + n] = abd;
                c[OR_ABU * vol + n] = abu;   c[OR_AFD * vol + n] = afd;   c[OR_AFU * vol + n] = afu;
                c[OR_ADD * vol + n] = add;   c[OR_AUU * vol + n] = auu;   c[OR_ALDD * vol + n] = aldd;
                c[OR_ALUU * vol + n] = aluu; c[OR_ARDD * vol + n] = ardd; c[OR_ARUU * vol + n] = aruu;
                c[OR_ABDD * vol + n] = abdd; c[OR_ABUU * vol + n] = abuu; c[OR_AFDD * vol + n] = afdd;
                c[OR_AFUU * vol + n] = afuu;
            }
}
