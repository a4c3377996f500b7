// or_solver.cpp -- CPU oracle (test infrastructure only): operator apply,
// preconditioner, BiCGSTAB, solve_poisson! and compute_lhs!.
//
// Literal FP64 restatements (single MPI rank) of
//   apply_operator!.jl:48-273 (Total) and :275-479 (Horizontal)
//   apply_preconditioner!.jl:40-124
//   apply_bicgstab!.jl:24-150 with compute_global_dot_product.jl:22-36
//   solve_poisson!.jl:39-75
//   compute_lhs!.jl:68-160
// Loops are OpenMP-parallel over cells; global sums use a fixed blocking
// (pairwise within and across blocks of 4096), so results do not depend on
// the thread count.  Julia's `sum`/`mapreduce` are pairwise too, so the
// rounding is of the same kind, though not bit-identical.
#include "pcf_oracle.h"

#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const long kBlock = 4096;

double pairwise(const double *v, long n) {
    if (n <= 128) {
        double s = 0.0;
        for (long i = 0; i < n; ++i) s += v[i];
        return s;
    }
    const long h = n / 2;
    return pairwise(v, h) + pairwise(v + h, n - h);
}

// Sum of f(n) over n in [0, len): per-block pairwise sums, then pairwise over blocks.
template <class F>
double global_sum(long len, F f) {
    const long nblk = (len + kBlock - 1) / kBlock;
    std::vector<double> part(nblk > 0 ? nblk : 1, 0.0);
#pragma omp parallel for schedule(static)
    for (long b = 0; b < nblk; ++b) {
        const long lo = b * kBlock, hi = (lo + kBlock < len) ? lo + kBlock : len;
        double tmp[kBlock];
        for (long n = lo; n < hi; ++n) tmp[n - lo] = f(n);
        part[b] = pairwise(tmp, hi - lo);
    }
    return nblk > 0 ? pairwise(part.data(), nblk) : 0.0;
}

// The operator workspace `Operator.s` (nx+2, ny+2, nz+4): interior copy,
// 1-layer periodic x/y fill over kk = k0-1:k1+1, vertical ghosts kept at 0
// (apply_operator!.jl:87-107 with npz = 1).
struct Work {
    int nx, ny, nz, sx, sy, sz;
    std::vector<double> s;
    explicit Work(const or_dims *d)
        : nx(d->nx), ny(d->ny), nz(d->nz), sx(d->nx + 2), sy(d->ny + 2), sz(d->nz + 4),
          s((size_t)(d->nx + 2) * (d->ny + 2) * (d->nz + 4), 0.0) {}
    size_t at(int i, int j, int k) const {  // i, j, k interior-relative (may be -1.. / -2..)
        return (size_t)(i + 1) + (size_t)sx * ((size_t)(j + 1) + (size_t)sy * (size_t)(k + 2));
    }
    void load(const double *in) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    s[at(i, j, k)] = in[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)];
        for (int k = -1; k <= nz; ++k) {
            for (int j = -1; j <= ny; ++j) {
                s[at(-1, j, k)] = s[at(nx - 1, j, k)];
                s[at(nx, j, k)] = s[at(0, j, k)];
            }
            for (int i = -1; i <= nx; ++i) {
                s[at(i, -1, k)] = s[at(i, ny - 1, k)];
                s[at(i, ny, k)] = s[at(i, 0, k)];
            }
        }
    }
};

void apply_impl(const or_dims *d, const double *coef, Work &w, const double *in, double *ls,
                bool horizontal) {
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    const size_t vol = (size_t)nx * ny * nz;
    w.load(in);
    const double *s = w.s.data();
    auto C = [&](int c, size_t n) { return coef[(size_t)c * vol + n]; };
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t n = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                const double sr = s[w.at(i + 1, j, k)], sl = s[w.at(i - 1, j, k)];
                const double sf = s[w.at(i, j + 1, k)], sb = s[w.at(i, j - 1, k)];
                double v;
                if (!horizontal) {
                    const double su = s[w.at(i, j, k + 1)], sd = s[w.at(i, j, k - 1)];
                    const double sc = s[w.at(i, j, k)];
                    v = C(OR_AL, n) * sl + C(OR_AR, n) * sr + C(OR_AF, n) * sf + C(OR_AB, n) * sb +
                        C(OR_AU, n) * su + C(OR_AD, n) * sd + C(OR_AC, n) * sc;
                } else {
                    v = C(OR_AL, n) * sl + C(OR_AR, n) * sr + C(OR_AF, n) * sf + C(OR_AB, n) * sb;
                }
                const double t =
                    C(OR_ARU, n) * s[w.at(i + 1, j, k + 1)] + C(OR_ARD, n) * s[w.at(i + 1, j, k - 1)] +
                    C(OR_ALU, n) * s[w.at(i - 1, j, k + 1)] + C(OR_ALD, n) * s[w.at(i - 1, j, k - 1)] +
                    C(OR_AFU, n) * s[w.at(i, j + 1, k + 1)] + C(OR_AFD, n) * s[w.at(i, j + 1, k - 1)] +
                    C(OR_ABU, n) * s[w.at(i, j - 1, k + 1)] + C(OR_ABD, n) * s[w.at(i, j - 1, k - 1)] +
                    C(OR_AUU, n) * s[w.at(i, j, k + 2)] + C(OR_ADD, n) * s[w.at(i, j, k - 2)] +
                    C(OR_ARUU, n) * s[w.at(i + 1, j, k + 2)] + C(OR_ARDD, n) * s[w.at(i + 1, j, k - 2)] +
                    C(OR_ALUU, n) * s[w.at(i - 1, j, k + 2)] + C(OR_ALDD, n) * s[w.at(i - 1, j, k - 2)] +
                    C(OR_AFUU, n) * s[w.at(i, j + 1, k + 2)] + C(OR_AFDD, n) * s[w.at(i, j + 1, k - 2)] +
                    C(OR_ABUU, n) * s[w.at(i, j - 1, k + 2)] + C(OR_ABDD, n) * s[w.at(i, j - 1, k - 2)];
                ls[n] = v + t;
            }
}

// apply_preconditioner!.jl:53-121
void precond_impl(const or_dims *d, const double *coef, double dx, double dy, double dtau,
                  int iters, Work &w, const double *sin_, double *s_pc, double *q_pc) {
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    const long plane = (long)nx * ny;
    const size_t vol = (size_t)plane * nz;
    const double *ac = coef + (size_t)OR_AC * vol;
    const double *ad = coef + (size_t)OR_AD * vol;
    const double *au = coef + (size_t)OR_AU * vol;
    std::memset(s_pc, 0, vol * sizeof(double));
    std::memset(q_pc, 0, vol * sizeof(double));
    const double deta = dtau / (2 * (1 / (dx * dx) + 1 / (dy * dy)));
    for (int it = 0; it < iters; ++it) {
        apply_impl(d, coef, w, s_pc, q_pc, true);
#pragma omp parallel for schedule(static)
        for (long n = 0; n < (long)vol; ++n) s_pc[n] += deta * (q_pc[n] - sin_[n]);
        // lower boundary (ko == 0)
#pragma omp parallel for schedule(static)
        for (long m = 0; m < plane; ++m) {
            q_pc[m] = deta * au[m] / (1 - deta * ac[m]);
            s_pc[m] /= 1 - deta * ac[m];
        }
        // upward sweep
        for (int k = 1; k < nz; ++k) {
            const size_t o = (size_t)k * plane, om = (size_t)(k - 1) * plane;
#pragma omp parallel for schedule(static)
            for (long m = 0; m < plane; ++m) {
                const double p_pc = 1 / (1 - deta * ac[o + m] - deta * ad[o + m] * q_pc[om + m]);
                q_pc[o + m] = deta * au[o + m] * p_pc;
                s_pc[o + m] = (s_pc[o + m] + deta * ad[o + m] * s_pc[om + m]) * p_pc;
            }
        }
        // downward sweep
        for (int k = nz - 2; k >= 0; --k) {
            const size_t o = (size_t)k * plane, op = (size_t)(k + 1) * plane;
#pragma omp parallel for schedule(static)
            for (long m = 0; m < plane; ++m) s_pc[o + m] += q_pc[o + m] * s_pc[op + m];
        }
    }
}

}  // namespace

extern "C" {

double or_dot(long n, const double *a, const double *b) {
    return global_sum(n, [&](long i) { return a[i] * b[i]; });
}

void or_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_apply_operator(const or_dims *d, const double *coef, const double *sin_, double *ls,
                       int horizontal) {
    Work w(d);
    apply_impl(d, coef, w, sin_, ls, horizontal != 0);
}

void or_apply_preconditioner(const or_dims *d, const double *coef, double dx, double dy,
                             double dtau, int preconditioner_iterations, const double *sin_,
                             double *sout) {
    const size_t vol = (size_t)d->nx * d->ny * d->nz;
    Work w(d);
    std::vector<double> q(vol);
    precond_impl(d, coef, dx, dy, dtau, preconditioner_iterations, w, sin_, sout, q.data());
}

void or_bicgstab(const or_dims *d, const double *coef, double dx, double dy, double tolerance,
                 int poisson_iterations, int preconditioner, double dtau,
                 int preconditioner_iterations, int tolerance_is_relative, double tolref,
                 const double *rhs, double *solution, double *out) {
    const long vol = (long)d->nx * d->ny * d->nz;
    const double ncell = (double)d->nx, ny = (double)d->ny, nz = (double)d->z_size;
    Work w(d);
    std::vector<double> p(vol), r0(vol), rold(vol), r(vol), s(vol), t(vol), v(vol),
        matvec(vol), v_pc(vol), q_pc(vol);
    auto dot = [&](const std::vector<double> &a, const std::vector<double> &b) {
        return or_dot(vol, a.data(), b.data());
    };
    auto precond = [&](const double *in, double *o) {
        precond_impl(d, coef, dx, dy, dtau, preconditioner_iterations, w, in, o, q_pc.data());
    };
    auto rms = [&](const std::vector<double> &a) {
        double res = global_sum(vol, [&](long i) { return a[i] * a[i]; });
        return std::sqrt(res / ncell / ny / nz);
    };

    // apply_bicgstab!.jl:44-67
    std::memset(solution, 0, vol * sizeof(double));
    const int maxit = poisson_iterations;
    const double tol = tolerance_is_relative ? tolerance : tolerance / tolref;
    apply_impl(d, coef, w, solution, matvec.data(), false);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < vol; ++n) {
        r0[n] = rhs[n] - matvec[n];
        p[n] = r0[n];
        r[n] = r0[n];
    }
    double res = rms(r);
    const double b_norm = res;
    out[0] = 0; out[1] = 0; out[2] = 0; out[3] = b_norm;
    // :69-76
    if (res == 0.0 || res / b_norm <= tol) return;

    int j_b = 0;
    while (j_b < maxit) {
        j_b += 1;
        // :84-91
        if (preconditioner) precond(p.data(), v_pc.data());
        else std::memcpy(v_pc.data(), p.data(), vol * sizeof(double));
        apply_impl(d, coef, w, v_pc.data(), matvec.data(), false);
        std::memcpy(v.data(), matvec.data(), vol * sizeof(double));
        // :93-96
        const double alpha = dot(r, r0) / dot(v, r0);
#pragma omp parallel for schedule(static)
        for (long n = 0; n < vol; ++n) s[n] = r[n] - alpha * v[n];
        // :98-105
        if (preconditioner) precond(s.data(), v_pc.data());
        else std::memcpy(v_pc.data(), s.data(), vol * sizeof(double));
        apply_impl(d, coef, w, v_pc.data(), matvec.data(), false);
        std::memcpy(t.data(), matvec.data(), vol * sizeof(double));
        // :107-113
        const double omega = dot(t, s) / dot(t, t);
#pragma omp parallel for schedule(static)
        for (long n = 0; n < vol; ++n) {
            solution[n] += alpha * p[n] + omega * s[n];
            rold[n] = r[n];
            r[n] = s[n] - omega * t[n];
        }
        // :119-138
        res = rms(r);
        if (res / b_norm <= tol) {
            out[1] = j_b;
            out[2] = res / b_norm;
            if (preconditioner) {
                std::memcpy(s.data(), solution, vol * sizeof(double));
                precond(s.data(), solution);
            }
            return;
        }
        // :140-143
        const double beta = alpha / omega * dot(r, r0) / dot(rold, r0);
#pragma omp parallel for schedule(static)
        for (long n = 0; n < vol; ++n) p[n] = r[n] + beta * (p[n] - omega * v[n]);
    }
    // :146-149
    out[0] = 1;
    out[1] = j_b;
    out[2] = res / b_norm;
}

int or_solve_poisson(const or_dims *d, int model, double dx, double dy, double dz,
                     const double *jac, const double *met13, const double *met23,
                     const double *met33, const double *pbar, const double *rhobar,
                     const double *thetabar, const double *n2, const double *rho,
                     const double *betar, const double *p, double dt, double rayleigh_factor,
                     int damp_horizontal_wind_on_rhs, double tolerance, int poisson_iterations,
                     int preconditioner, double dtau, int preconditioner_iterations,
                     int tolerance_is_relative, double tolref, const double *rhs, double *dpip,
                     double *out) {
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    const int nxx = nx + 2 * d->nbx, nyy = ny + 2 * d->nby;
    const long vol = (long)nx * ny * nz;
    // solve_poisson!.jl:50-54
    if (dt == 0.0) return -1;
    const double dtinv = 1.0 / dt;
    std::vector<double> coef((size_t)OR_NCOEF * vol), solution(vol);
    or_compute_operator(d, model, dx, dy, dz, jac, met13, met23, met33, pbar, rhobar, thetabar,
                        n2, rho, betar, p, dt, rayleigh_factor, damp_horizontal_wind_on_rhs,
                        coef.data());
    or_bicgstab(d, coef.data(), dx, dy, tolerance, poisson_iterations, preconditioner, dtau,
                preconditioner_iterations, tolerance_is_relative, tolref, rhs, solution.data(),
                out);
    if (out[0] != 0) return 0;
    // :65-72
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t h = (size_t)(i + d->nbx) +
                                 (size_t)nxx * ((size_t)(j + d->nby) + (size_t)nyy * (k + d->nbz));
                const size_t n = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                const double pb = pbar[h];
                double sol = solution[n] / std::sqrt(pb * pb / rhobar[h]);
                dpip[h] = dtinv * sol;
            }
    return 0;
}

double or_compute_lhs(const or_dims *d, double dx, double dy, double dz, double ma, double kappa,
                      const double *jac, const double *pbar, const double *rhobar,
                      const double *u, const double *v, const double *w, double *rhs) {
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    const int nxx = nx + 2 * d->nbx, nyy = ny + 2 * d->nby;
    const long vol = (long)nx * ny * nz;
    std::vector<double> norm2(vol);
    auto H = [&](int a, int b, int c) {
        return (size_t)a + (size_t)nxx * ((size_t)b + (size_t)nyy * (size_t)c);
    };
    // compute_lhs!.jl:85-136
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = d->nbz; k < d->nbz + nz; ++k)
        for (int j = d->nby; j < d->nby + ny; ++j)
            for (int i = d->nbx; i < d->nbx + nx; ++i) {
                const double fcscal = std::sqrt(std::pow(pbar[H(i, j, k)], 2.0) / rhobar[H(i, j, k)]);
                const double ur = u[H(i, j, k)], ul = u[H(i - 1, j, k)];
                const double vf = v[H(i, j, k)], vb = v[H(i, j - 1, k)];
                const double wu = w[H(i, j, k)], wd = w[H(i, j, k - 1)];
                const double JP = jac[H(i, j, k)] * pbar[H(i, j, k)];
                const double pedger = 0.5 * (JP + jac[H(i + 1, j, k)] * pbar[H(i + 1, j, k)]);
                const double pedgel = 0.5 * (JP + jac[H(i - 1, j, k)] * pbar[H(i - 1, j, k)]);
                const double pedgef = 0.5 * (JP + jac[H(i, j + 1, k)] * pbar[H(i, j + 1, k)]);
                const double pedgeb = 0.5 * (JP + jac[H(i, j - 1, k)] * pbar[H(i, j - 1, k)]);
                const double pedgeu = jac[H(i, j, k)] * jac[H(i, j, k + 1)] *
                                      (pbar[H(i, j, k)] + pbar[H(i, j, k + 1)]) /
                                      (jac[H(i, j, k)] + jac[H(i, j, k + 1)]);
                const double pedged = jac[H(i, j, k)] * jac[H(i, j, k - 1)] *
                                      (pbar[H(i, j, k)] + pbar[H(i, j, k - 1)]) /
                                      (jac[H(i, j, k)] + jac[H(i, j, k - 1)]);
                const double ma2 = std::pow(ma, 2.0);
                double bu = (pedger * ur - pedgel * ul) / dx / jac[H(i, j, k)] * ma2 * kappa;
                double bv = (pedgef * vf - pedgeb * vb) / dy / jac[H(i, j, k)] * ma2 * kappa;
                double bw = (pedgeu * wu - pedged * wd) / dz / jac[H(i, j, k)] * ma2 * kappa;
                bu /= fcscal;
                bv /= fcscal;
                bw /= fcscal;
                const size_t n = (size_t)(i - d->nbx) +
                                 (size_t)nx * ((size_t)(j - d->nby) + (size_t)ny * (k - d->nbz));
                rhs[n] = bu + bv + bw;
                norm2[n] = bu * bu + bv * bv + bw * bw;
            }
    // :138-159
    const double nn = (double)nx * ny * d->z_size;
    double divl2 = global_sum(vol, [&](long i) { return rhs[i] * rhs[i]; });
    divl2 = std::sqrt(divl2 / nn);
    double divl2_norm = global_sum(vol, [&](long i) { return norm2[i]; });
    divl2_norm = std::sqrt(divl2_norm / nn);
    if (divl2_norm != 0.0) return divl2 / divl2_norm;
    if (divl2 == 0.0) return 1.0;
    return NAN;  // the reference raises here
}

double or_compute_lhs_compressible(const or_dims *d, double dx, double dy, double dz, double ma,
                                   double kappa, const double *jac, const double *pbar,
                                   const double *rhobar, const double *u, const double *v,
                                   const double *w, const double *heating, double *rhs) {
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    const int nxx = nx + 2 * d->nbx, nyy = ny + 2 * d->nby;
    const long vol = (long)nx * ny * nz;
    std::vector<double> norm2(vol);
    auto H = [&](int a, int b, int c) {
        return (size_t)a + (size_t)nxx * ((size_t)b + (size_t)nyy * (size_t)c);
    };
    // compute_lhs!.jl:177-203
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = d->nbz; k < d->nbz + nz; ++k)
        for (int j = d->nby; j < d->nby + ny; ++j)
            for (int i = d->nbx; i < d->nbx + nx; ++i) {
                const double fcscal = std::sqrt(std::pow(pbar[H(i, j, k)], 2.0) / rhobar[H(i, j, k)]);
                const double ur = u[H(i, j, k)], ul = u[H(i - 1, j, k)];
                const double vf = v[H(i, j, k)], vb = v[H(i, j - 1, k)];
                const double wu = w[H(i, j, k)], wd = w[H(i, j, k - 1)];
                const size_t n = (size_t)(i - d->nbx) +
                                 (size_t)nx * ((size_t)(j - d->nby) + (size_t)ny * (k - d->nbz));
                const double ma2 = std::pow(ma, 2.0);
                double heat = (heating ? heating[n] : 0.0) * ma2 * kappa;
                double bu = (ur - ul) / dx / jac[H(i, j, k)] * ma2 * kappa;
                double bv = (vf - vb) / dy / jac[H(i, j, k)] * ma2 * kappa;
                double bw = (wu - wd) / dz / jac[H(i, j, k)] * ma2 * kappa;
                bu /= fcscal;
                bv /= fcscal;
                bw /= fcscal;
                heat /= fcscal;
                rhs[n] = bu + bv + bw - heat;
                norm2[n] = bu * bu + bv * bv + bw * bw + heat * heat;
            }
    // :205-222
    const double nn = (double)nx * ny * d->z_size;
    double divl2 = global_sum(vol, [&](long i) { return rhs[i] * rhs[i]; });
    divl2 = std::sqrt(divl2 / nn);
    double divl2_norm = global_sum(vol, [&](long i) { return norm2[i]; });
    divl2_norm = std::sqrt(divl2_norm / nn);
    if (divl2_norm != 0.0) return divl2 / divl2_norm;
    if (divl2 == 0.0) return 1.0;
    return NAN;  // the reference raises here
}

}  // extern "C"
