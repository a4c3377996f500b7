// or_fields.cpp -- CPU oracle (test infrastructure only): input generators.
//
// Literal FP64 restatements of the reference's state construction for one
// MPI rank (npx = npy = npz = 1):
//   Constants.jl:113-155, Grid.jl:173-338, compute_topography.jl:145-176,
//   Atmosphere.jl:278-323, compute_n2!.jl:43-82, compute_sponges!.jl:26-65.
// Indices below are 0-based; the comments give the 1-based Julia form.
#include "pcf_oracle.h"

#include <cmath>
#include <cstddef>
#include <vector>

namespace {

struct HaloIdx {
    int nxx, nyy, nzz;
    size_t operator()(int i, int j, int k) const {
        return (size_t)i + (size_t)nxx * ((size_t)j + (size_t)nyy * (size_t)k);
    }
};

// Periodic fill of all x and y halo layers of a haloed 3-D field
// (set_zonal_boundaries_of_field!.jl:91-101 and its meridional twin, single rank).
void periodic_xy(const or_dims *d, double *f, int nzz) {
    const int nxx = d->nx + 2 * d->nbx, nyy = d->ny + 2 * d->nby;
    HaloIdx H{nxx, nyy, nzz};
    const int i0 = d->nbx, i1 = d->nbx + d->nx - 1;
    const int j0 = d->nby, j1 = d->nby + d->ny - 1;
    for (int k = 0; k < nzz; ++k)
        for (int j = 0; j < nyy; ++j)
            for (int l = 1; l <= d->nbx; ++l) {
                f[H(i0 - l, j, k)] = f[H(i1 - l + 1, j, k)];
                f[H(i1 + l, j, k)] = f[H(i0 + l - 1, j, k)];
            }
    for (int k = 0; k < nzz; ++k)
        for (int l = 1; l <= d->nby; ++l)
            for (int i = 0; i < nxx; ++i) {
                f[H(i, j0 - l, k)] = f[H(i, j1 - l + 1, k)];
                f[H(i, j1 + l, k)] = f[H(i, j0 + l - 1, k)];
            }
}

}  // namespace

extern "C" void or_constants(double *out) {
    // Constants.jl:119-155
    const double gamma = 1.4;
    const double kappa = (gamma - 1.0) / gamma;
    const double rsp = 287.0;
    const double g = 9.81;
    const double rhoref = 1.184;
    const double pref = 101325.0;
    const double aref = std::sqrt(pref / rhoref);
    const double uref = aref;
    const double lref = pref / rhoref / g;
    const double tref = lref / aref;
    const double thetaref = aref * aref / rsp;
    const double g_ndim = g / (uref * uref / lref);
    const double ma = uref / aref;
    const double fr = uref / std::sqrt(g * lref);
    const double sig = ma * ma / (fr * fr);
    out[0] = gamma; out[1] = kappa; out[2] = rsp; out[3] = g; out[4] = rhoref;
    out[5] = pref; out[6] = lref; out[7] = tref; out[8] = thetaref;
    out[9] = g_ndim; out[10] = ma; out[11] = sig;
}

extern "C" int or_grid(const or_dims *d, double lx_dim, double ly_dim, double lz_dim,
                       double stretch_exp, const double *hb_dim, double *jac,
                       double *met13, double *met23, double *met33, double *zc,
                       double *dxdydz_out) {
    double c[12];
    or_constants(c);
    const double lref = c[6];
    const int nbx = d->nbx, nby = d->nby, nbz = d->nbz;
    const int nxx = d->nx + 2 * nbx, nyy = d->ny + 2 * nby, nzz = d->nz + 2 * nbz;
    const int x_size = d->nx, y_size = d->ny, z_size = d->z_size;
    HaloIdx H{nxx, nyy, nzz};

    // Grid.jl:189-197
    const double lx = lx_dim / lref, ly = ly_dim / lref, lz = lz_dim / lref;
    const double dx = lx / x_size, dy = ly / y_size, dz = lz / z_size;
    dxdydz_out[0] = dx; dxdydz_out[1] = dy; dxdydz_out[2] = dz;

    // Grid.jl:212-216: z[k] = (k - k0) dz + dz/2
    const int nzt = z_size + 2 * nbz;
    std::vector<double> z(nzt), zt(nzt), zs(nzt);
    for (int k = 0; k < nzt; ++k) z[k] = (k - nbz) * dz + dz / 2;
    // vertical_grid_stretching(zhat) = lz_dim (zhat / lz_dim)^p  (identity for p = 1)
    auto stretch = [&](double zhat_dim) {
        return stretch_exp == 1.0 ? zhat_dim : lz_dim * std::pow(zhat_dim / lz_dim, stretch_exp);
    };
    // Grid.jl:222-233
    for (int k = 0; k < nzt; ++k) {
        const double level = z[k] + 0.5 * dz;
        if (level < 0)
            zt[k] = -stretch(-level * lref) / lref;
        else if (level > lz)
            zt[k] = 2 * lz - stretch((2 * lz - level) * lref) / lref;
        else
            zt[k] = stretch(level * lref) / lref;
    }
    // Grid.jl:234-235: ztildes[k0:k0+z_size-1] must be strictly increasing
    for (int k = nbz + 1; k < nbz + z_size; ++k)
        if (!(zt[k - 1] < zt[k])) return -1;
    // Grid.jl:236-239
    for (int k = 1; k < nzt; ++k) zs[k] = 0.5 * (zt[k] + zt[k - 1]);
    zs[0] = zt[0] - 0.5 * (zt[2 * nbz - 1] - zt[2 * nbz - 2]);

    // compute_topography.jl:167-173 plus periodic fill
    std::vector<double> hb((size_t)nxx * nyy, 0.0);
    for (int j = 0; j < d->ny; ++j)
        for (int i = 0; i < d->nx; ++i)
            hb[(size_t)(i + nbx) + (size_t)nxx * (j + nby)] = hb_dim[(size_t)i + (size_t)d->nx * j] / lref;
    for (int j = 0; j < nyy; ++j)
        for (int l = 1; l <= nbx; ++l) {
            hb[(size_t)(nbx - l) + (size_t)nxx * j] = hb[(size_t)(nbx + d->nx - l) + (size_t)nxx * j];
            hb[(size_t)(nbx + d->nx - 1 + l) + (size_t)nxx * j] = hb[(size_t)(nbx + l - 1) + (size_t)nxx * j];
        }
    for (int l = 1; l <= nby; ++l)
        for (int i = 0; i < nxx; ++i) {
            hb[(size_t)i + (size_t)nxx * (nby - l)] = hb[(size_t)i + (size_t)nxx * (nby + d->ny - l)];
            hb[(size_t)i + (size_t)nxx * (nby + d->ny - 1 + l)] = hb[(size_t)i + (size_t)nxx * (nby + l - 1)];
        }
    auto HB = [&](int i, int j) { return hb[(size_t)i + (size_t)nxx * j]; };

    const size_t nh = (size_t)nxx * nyy * nzz;
    for (size_t n = 0; n < nh; ++n) { jac[n] = 0; met13[n] = 0; met23[n] = 0; met33[n] = 0; }

    // Grid.jl:246-250 (ko = 0 -> kmin = 2 in 1-based indexing)
    for (int k = 1; k < nzz; ++k)
        for (int j = 0; j < nyy; ++j)
            for (int i = 0; i < nxx; ++i)
                jac[H(i, j, k)] = (lz - HB(i, j)) / lz * (zt[k] - zt[k - 1]) / dz;
    for (int j = 0; j < nyy; ++j)
        for (int i = 0; i < nxx; ++i) jac[H(i, j, 0)] = jac[H(i, j, 2 * nbz - 1)];

    const int i0 = nbx, i1 = nbx + d->nx - 1, j0 = nby, j1 = nby + d->ny - 1;
    // Grid.jl:259-271 (met13)
    for (int k = 1; k < nzz; ++k)
        for (int j = 0; j < nyy; ++j)
            for (int i = i0; i <= i1; ++i)
                met13[H(i, j, k)] = (HB(i + 1, j) - HB(i - 1, j)) / (2.0 * dx) * (zs[k] - lz) /
                                    (lz - HB(i, j)) * dz / (zt[k] - zt[k - 1]);
    periodic_xy(d, met13, nzz);  // x fill only matters; y rows were computed directly
    for (int j = 0; j < nyy; ++j)
        for (int i = 0; i < nxx; ++i)
            met13[H(i, j, 0)] = met13[H(i, j, 2 * nbz - 1)] * (zs[0] - lz) / (zs[2 * nbz - 1] - lz);

    // Grid.jl:274-285 (met23)
    for (int k = 1; k < nzz; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = 0; i < nxx; ++i)
                met23[H(i, j, k)] = (HB(i, j + 1) - HB(i, j - 1)) / (2.0 * dy) * (zs[k] - lz) /
                                    (lz - HB(i, j)) * dz / (zt[k] - zt[k - 1]);
    periodic_xy(d, met23, nzz);
    for (int j = 0; j < nyy; ++j)
        for (int i = 0; i < nxx; ++i)
            met23[H(i, j, 0)] = met23[H(i, j, 2 * nbz - 1)] * (zs[0] - lz) / (zs[2 * nbz - 1] - lz);

    // Grid.jl:288-313 (met33)
    for (int k = 1; k < nzz; ++k)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                const double hx = (HB(i + 1, j) - HB(i - 1, j)) / (2.0 * dx);
                const double hy = (HB(i, j + 1) - HB(i, j - 1)) / (2.0 * dy);
                const double a = lz / (lz - HB(i, j));
                const double b = (zs[k] - lz) / (lz - HB(i, j));
                const double e = dz / (zt[k] - zt[k - 1]);
                met33[H(i, j, k)] = (a * a + b * b * (hx * hx + hy * hy)) * (e * e);
            }
    for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) {
            const double hx = (HB(i + 1, j) - HB(i - 1, j)) / (2.0 * dx);
            const double hy = (HB(i, j + 1) - HB(i, j - 1)) / (2.0 * dy);
            const double a = lz / (lz - HB(i, j));
            const double b = (zs[0] - lz) / (lz - HB(i, j));
            const double e = dz / (zt[2 * nbz - 1] - zt[2 * nbz - 2]);
            met33[H(i, j, 0)] = (a * a + b * b * (hx * hx + hy * hy)) * (e * e);
        }
    periodic_xy(d, met33, nzz);

    // Grid.jl:319-323 (zc)
    for (int k = 0; k < nzz; ++k)
        for (int j = 0; j < nyy; ++j)
            for (int i = 0; i < nxx; ++i)
                zc[H(i, j, k)] = (lz - HB(i, j)) / lz * zs[k] + HB(i, j);
    (void)j1;
    return 0;
}

extern "C" int or_atmosphere(const or_dims *d, int background, const double *params,
                             const double *jac, const double *zc, double dz, double *pbar,
                             double *thetabar, double *rhobar, double *n2) {
    double c[12];
    or_constants(c);
    const double gamma = c[0], kappa = c[1], pref = c[5], tref = c[7], thetaref = c[8];
    const double g_ndim = c[9], sig = c[11];
    const int nxx = d->nx + 2 * d->nbx, nyy = d->ny + 2 * d->nby, nzz = d->nz + 2 * d->nbz;
    const size_t nh = (size_t)nxx * nyy * nzz, plane = (size_t)nxx * nyy;
    if (background == 0) {
        // Atmosphere.jl:278-296 (Boussinesq, StableStratification)
        const double nbv = params[0], theta0 = params[1];
        for (size_t n = 0; n < nh; ++n) {
            rhobar[n] = 1.0;
            thetabar[n] = theta0 / thetaref;
            pbar[n] = rhobar[n] * thetabar[n];
            n2[n] = (nbv * tref) * (nbv * tref);
        }
        return 0;
    }
    if (background != 1) return -1;
    // Atmosphere.jl:298-323 (Isothermal)
    const double t0 = params[0] / thetaref, p0 = params[1] / pref;
    for (size_t n = 0; n < nh; ++n) {
        pbar[n] = p0 * std::exp(-sig * zc[n] / gamma / t0);
        thetabar[n] = t0 * std::exp(kappa * sig / t0 * zc[n]);
        rhobar[n] = pbar[n] / thetabar[n];
    }
    // compute_n2!.jl:57-79
    const int k0 = d->nbz, k1 = d->nbz + d->nz - 1;
    for (size_t n = 0; n < nh; ++n) n2[n] = 0.0;
    for (int k = k0; k <= k1; ++k)
        for (size_t m = 0; m < plane; ++m) {
            const size_t n = m + plane * k;
            n2[n] = g_ndim / thetabar[n] / jac[n] * 0.5 *
                    (thetabar[n + plane] - thetabar[n - plane]) / dz;
        }
    for (int l = 1; l <= d->nbz; ++l)
        for (size_t m = 0; m < plane; ++m) {
            const size_t b = m + plane * (k0 - 1);
            n2[m + plane * (k0 - l)] =
                g_ndim / thetabar[b] / jac[b] * (thetabar[b + plane] - thetabar[b]) / dz;
            const size_t t = m + plane * (k1 + 1);
            n2[m + plane * (k1 + l)] =
                g_ndim / thetabar[t] / jac[t] * (thetabar[t] - thetabar[t - plane]) / dz;
        }
    return 0;
}

extern "C" void or_sponge_sin2(const or_dims *d, const double *zc, double zr, double lz,
                               double dt, double *betar) {
    double c[12];
    or_constants(c);
    const double lref = c[6], tref = c[7];
    const int nbx = d->nbx, nby = d->nby, nbz = d->nbz;
    const int nxx = d->nx + 2 * nbx, nyy = d->ny + 2 * nby, nzz = d->nz + 2 * nbz;
    HaloIdx H{nxx, nyy, nzz};
    const size_t nh = (size_t)nxx * nyy * nzz;
    for (size_t n = 0; n < nh; ++n) betar[n] = 0.0;
    const double pi = 3.14159265358979323846;
    // compute_sponges!.jl:38-49 with the periodic-hill rhs_sponge
    for (int k = nbz; k < nbz + d->nz; ++k)
        for (int j = nby; j < nby + d->ny; ++j)
            for (int i = nbx; i < nbx + d->nx; ++i) {
                const double zcdim = zc[H(i, j, k)] * lref;
                const double dtdim = dt * tref;
                double v = 0.0;
                if (zcdim >= zr) {
                    const double s = std::sin(pi / 2 * (zcdim - zr) / (lz - zr));
                    v = s * s / dtdim;
                }
                betar[H(i, j, k)] = v * tref;
            }
    periodic_xy(d, betar, nzz);
    // compute_sponges!.jl:57-64
    for (int j = 0; j < nyy; ++j)
        for (int i = 0; i < nxx; ++i) {
            betar[H(i, j, nbz - 1)] = betar[H(i, j, nbz)];
            betar[H(i, j, nbz + d->nz)] = betar[H(i, j, nbz + d->nz - 1)];
        }
}
