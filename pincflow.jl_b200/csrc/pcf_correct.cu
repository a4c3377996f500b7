// pcf_correct.cu -- the corrector after the Poisson solve (apply_corrector!.jl:
// 58-61) on the device: the boundary fill of dpip, then correct!.jl:164-385
// with compute_pressure_gradient.jl:108-297, compute_compressible_wind_factor
// .jl:102-157 and compute_buoyancy_factor.jl:108-172.  FP64 throughout, one
// thread per (staggered) cell; each kernel reads a few haloed fields and
// writes one or two, so they are memory-bound and run once per solve.
//
// Index conventions as in pcf_assemble.cu: interior cell (ii, jj, kk) is the
// haloed cell (ii + nbx, jj + nby, kk + nbz); one rank (ko = 0, z_size = nz).
#include "pcf_internal.cuh"

namespace pcf {

struct CorrectArgs {
    int nx, ny, nz, nxx, nyy, nbx, nby, nbz, model, damp_h;
    double dt, rf, rdx, rdy, rdz;
    double kappainv, mainv2, g_ndim;
    const double *jac, *met13, *met23, *met33, *rhobar, *pbar, *thetabar, *n2, *betar, *rho, *p;
    double *dpip, *u, *v, *w, *rhop, *pip, *corx, *cory;
};

struct Ix {
    long long sy, sz;
    __device__ long long operator()(int i, int j, int k) const { return i + sy * j + sz * k; }
};

// dpip halo: periodic in x and y, mirrored in z (set_zonal/meridional/
// vertical_boundaries_of_field!, mode +).  Every ghost value is an interior
// value, so one pass over the haloed grid suffices.
__global__ void __launch_bounds__(256) k_fill_dpip(CorrectArgs a) {
    const int nzz = a.nz + 2 * a.nbz;
    const long long nh = (long long)a.nxx * a.nyy * nzz;
    const Ix at{a.nxx, (long long)a.nxx * a.nyy};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nh; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % a.nxx), j = (int)((q / a.nxx) % a.nyy), k = (int)(q / ((long long)a.nxx * a.nyy));
        const int ii = i - a.nbx, jj = j - a.nby, kk = k - a.nbz;
        if (ii >= 0 && ii < a.nx && jj >= 0 && jj < a.ny && kk >= 0 && kk < a.nz) continue;
        int si = ii % a.nx;
        if (si < 0) si += a.nx;
        int sj = jj % a.ny;
        if (sj < 0) sj += a.ny;
        const int sk = kk < 0 ? -kk - 1 : (kk >= a.nz ? 2 * a.nz - 1 - kk : kk);
        a.dpip[q] = a.dpip[at(si + a.nbx, sj + a.nby, sk + a.nbz)];
    }
}

// compute_pressure_gradient for U (dir 0) or V (dir 1) at the face (i+1/2, j, k) or (i, j+1/2, k)
__device__ double grad_h(const CorrectArgs &a, const Ix &at, int i, int j, int k, int dir) {
    const long long c = at(i, j, k), o = dir == 0 ? 1 : at.sy, n = c + o;
    const double *met = dir == 0 ? a.met13 : a.met23;
    const double rh = dir == 0 ? a.rdx : a.rdy;
    const double rhoe = 0.5 * (a.rho[c] + a.rho[n]) + 0.5 * (a.rhobar[c] + a.rhobar[n]);
    const double pe = 0.5 * (a.pbar[c] + a.pbar[n]);
    const double mete = 0.5 * (met[c] + met[n]);
    const double *P = a.dpip;
    const long long z = at.sz;
    double dz;
    if (k == a.nbz) {  // bottom: one-sided
        const double puu = 0.5 * (P[c + 2 * z] + P[n + 2 * z]), pu = 0.5 * (P[c + z] + P[n + z]),
                     p0 = 0.5 * (P[c] + P[n]);
        dz = -puu + 4.0 * pu - 3.0 * p0;
    } else if (k == a.nbz + a.nz - 1) {  // top: one-sided
        const double pdd = 0.5 * (P[c - 2 * z] + P[n - 2 * z]), pd = 0.5 * (P[c - z] + P[n - z]),
                     p0 = 0.5 * (P[c] + P[n]);
        dz = pdd - 4.0 * pd + 3.0 * p0;
    } else {
        dz = 0.5 * (P[c + z] + P[n + z]) - 0.5 * (P[c - z] + P[n - z]);
    }
    return a.kappainv * a.mainv2 * pe / rhoe * ((P[n] - P[c]) * rh + mete * dz * 0.5 * a.rdz);
}

// compute_pressure_gradient for W at (i, j, k+1/2)
__device__ double grad_w(const CorrectArgs &a, const Ix &at, int i, int j, int k) {
    const long long c = at(i, j, k), u = c + at.sz;
    const double *J = a.jac, *P = a.dpip;
    const double jk = J[c], jk1 = J[u], rj = 1.0 / (jk + jk1);
    const double rhoe = (jk1 * a.rho[c] + jk * a.rho[u]) * rj + (jk1 * a.rhobar[c] + jk * a.rhobar[u]) * rj;
    const double pe = (jk1 * a.pbar[c] + jk * a.pbar[u]) * rj;
    const double m13 = (jk1 * a.met13[c] + jk * a.met13[u]) * rj;
    const double m23 = (jk1 * a.met23[c] + jk * a.met23[u]) * rj;
    const double m33 = (jk1 * a.met33[c] + jk * a.met33[u]) * rj;
    auto edge = [&](long long q) {  // Jacobian-weighted dpip at the w-level of column q
        return (J[q + at.sz] * P[q] + J[q] * P[q + at.sz]) / (J[q] + J[q + at.sz]);
    };
    const double pr = edge(c + 1), pl = edge(c - 1), pf = edge(c + at.sy), pb = edge(c - at.sy);
    return a.kappainv * a.mainv2 * pe / rhoe *
           (m13 * (pr - pl) * 0.5 * a.rdx + m23 * (pf - pb) * 0.5 * a.rdy + m33 * (P[u] - P[c]) * a.rdz);
}

// U and V corrections (correct!.jl:177-245) with corx, cory: thread (x, y, k)
// over (nx + 1) x (ny + 1) x nz staggered positions; x = 0 is the face i0 - 1/2.
__global__ void __launch_bounds__(256) k_correct_uv(CorrectArgs a) {
    const long long m = (long long)(a.nx + 1) * (a.ny + 1) * a.nz;
    const Ix at{a.nxx, (long long)a.nxx * a.nyy};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < m; q += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(q % (a.nx + 1)), y = (int)((q / (a.nx + 1)) % (a.ny + 1)),
                  kk = (int)(q / ((long long)(a.nx + 1) * (a.ny + 1)));
        const int i = a.nbx - 1 + x, j = a.nby - 1 + y, k = a.nbz + kk;
        const long long c = at(i, j, k);
        if (y >= 1) {  // U at i + 1/2 for i in i0-1 .. i1
            double factor = 1.0;
            if (a.damp_h) factor += a.dt * 0.5 * (a.betar[c] + a.betar[c + 1]) * a.rf;
            const double cor = a.dt / factor * grad_h(a, at, i, j, k, 0);
            a.corx[c] = cor;
            const double wf = a.model == PCF_MODEL_COMPRESSIBLE ? (a.jac[c] * a.p[c] + a.jac[c + 1] * a.p[c + 1]) / 2 : 1.0;
            a.u[c] -= wf * cor;
        }
        if (x >= 1) {  // V at j + 1/2 for j in j0-1 .. j1
            const long long n = c + at.sy;
            double factor = 1.0;
            if (a.damp_h) factor += a.dt * 0.5 * (a.betar[c] + a.betar[n]) * a.rf;
            const double cor = a.dt / factor * grad_h(a, at, i, j, k, 1);
            a.cory[c] = cor;
            const double wf = a.model == PCF_MODEL_COMPRESSIBLE ? (a.jac[c] * a.p[c] + a.jac[n] * a.p[n]) / 2 : 1.0;
            a.v[c] -= wf * cor;
        }
    }
}

// W and rho' corrections (correct!.jl:247-360) on the interior, and
// pip += dpip (:375-385) on the interior plus one ghost layer: thread per
// cell of the (nx + 2) x (ny + 2) x (nz + 2) box.
__global__ void __launch_bounds__(256) k_correct_w_rhop_pip(CorrectArgs a) {
    const int bx = a.nx + 2, by = a.ny + 2;
    const long long m = (long long)bx * by * (a.nz + 2);
    const Ix at{a.nxx, (long long)a.nxx * a.nyy};
    const double dt2 = a.dt * a.dt;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < m; q += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(q % bx), y = (int)((q / bx) % by), z = (int)(q / ((long long)bx * by));
        const int i = a.nbx - 1 + x, j = a.nby - 1 + y, k = a.nbz - 1 + z;
        const long long c = at(i, j, k);
        a.pip[c] += a.dpip[c];
        const bool interior = x >= 1 && x <= a.nx && y >= 1 && y <= a.ny && z >= 1 && z <= a.nz;
        if (!interior) continue;
        const double *J = a.jac;
        const long long u = c + at.sz, l = c - 1, b = c - at.sy;
        const bool top = k == a.nbz + a.nz - 1, bot = k == a.nbz;
        const double gu = top ? 0.0 : grad_w(a, at, i, j, k);
        if (!top) {  // W at k + 1/2 for k in k0 .. k1-1
            const double rj = 1.0 / (J[c] + J[u]);
            const double factor = 1.0 + a.dt * (J[u] * a.betar[c] + J[c] * a.betar[u]) * rj * a.rf;
            const double n2e = (J[u] * a.n2[c] + J[c] * a.n2[u]) * rj;
            double jp = 1.0, fw;
            const double den = J[u] * (a.rho[c] + a.rhobar[c]) + J[c] * (a.rho[u] + a.rhobar[u]);
            if (a.model == PCF_MODEL_COMPRESSIBLE) {
                jp = J[c] * J[u] * (a.p[c] + a.p[u]) * rj;
                fw = (J[u] * a.pbar[c] / a.thetabar[c] + J[c] * a.pbar[u] / a.thetabar[u]) / den;
            } else {
                fw = (J[u] * a.rhobar[c] + J[c] * a.rhobar[u]) / den;
            }
            const double inv = 1.0 / (factor + fw * n2e * dt2);
            const double cross = (J[u] * (a.met13[c] * (a.corx[c] + a.corx[l]) + a.met23[c] * (a.cory[c] + a.cory[b])) +
                                  J[c] * (a.met13[u] * (a.corx[u] + a.corx[l + at.sz]) +
                                          a.met23[u] * (a.cory[u] + a.cory[b + at.sz]))) * rj;
            a.w[c] += -a.dt * inv * jp * gu - inv * fw * n2e * dt2 * jp * 0.5 * cross;
        }
        // rho'
        const double gl = bot ? 0.0 : grad_w(a, at, i, j, k - 1);
        const double gradient = 0.5 * (gl + gu);
        const double factor = 1.0 + a.dt * a.betar[c] * a.rf;
        const double fb = a.model == PCF_MODEL_COMPRESSIBLE ? a.pbar[c] / a.thetabar[c] / (a.rho[c] + a.rhobar[c])
                                                            : a.rhobar[c] / (a.rho[c] + a.rhobar[c]);
        const double n2c = a.n2[c];
        const double db = -1.0 / (factor + fb * n2c * dt2) *
                          (-fb * n2c * dt2 * J[c] * gradient +
                           fb * n2c * a.dt * J[c] * factor * 0.5 *
                               (a.met13[c] * (a.corx[c] + a.corx[l]) + a.met23[c] * (a.cory[c] + a.cory[b])));
        a.rhop[c] -= (a.rho[c] + a.rhobar[c]) / a.g_ndim * db;
    }
}

}  // namespace pcf

// dpip (haloed, interior from the solve) -> halo fill and the corrections of
// u, v, w, rho', pip (haloed, in place); rho, betar, p are the handle's (the
// last solve's inputs).  corx, cory: haloed scratch.
int pcf_launch_correct(pcf_handle *h, double dt, double rf, int damp_h, double *dpip, double *u, double *v,
                       double *w, double *rhop, double *pip, double *corx, double *cory) {
    pcf::CorrectArgs a;
    a.nx = h->d.nx; a.ny = h->d.ny; a.nz = h->d.nz;
    a.nxx = h->nxx; a.nyy = h->nyy;
    a.nbx = h->dims.nbx; a.nby = h->dims.nby; a.nbz = h->dims.nbz;
    a.model = h->dims.model; a.damp_h = damp_h;
    a.dt = dt; a.rf = rf;
    a.rdx = 1.0 / h->dx; a.rdy = 1.0 / h->dy; a.rdz = 1.0 / h->dz;
    // Constants.jl:116, :150 (Ma = 1), :131 (g_ndim = g lref / uref^2, uref = aref = sqrt(pref / rhoref))
    const double kappa = (1.4 - 1.0) / 1.4, g = 9.81, pref = 101325.0, rhoref = 1.184;
    const double lref = pref / rhoref / g, uref = std::sqrt(pref / rhoref);
    a.kappainv = 1.0 / kappa;
    a.mainv2 = 1.0;
    a.g_ndim = g / (uref * uref / lref);
    a.jac = h->jac; a.met13 = h->met13; a.met23 = h->met23; a.met33 = h->met33;
    a.rhobar = h->rhobar; a.pbar = h->pbar; a.thetabar = h->thetabar; a.n2 = h->n2;
    a.betar = h->betar; a.rho = h->rho; a.p = h->p;
    a.dpip = dpip; a.u = u; a.v = v; a.w = w; a.rhop = rhop; a.pip = pip; a.corx = corx; a.cory = cory;
    auto grid = [](long long n) {
        long long g2 = (n + 255) / 256;
        return (unsigned)(g2 < 1 ? 1 : (g2 > 4096 ? 4096 : g2));
    };
    h->launches += 3;
    pcf::k_fill_dpip<<<grid(h->nh), 256, 0, h->stream>>>(a);
    pcf::k_correct_uv<<<grid((long long)(a.nx + 1) * (a.ny + 1) * a.nz), 256, 0, h->stream>>>(a);
    pcf::k_correct_w_rhop_pip<<<grid((long long)(a.nx + 2) * (a.ny + 2) * (a.nz + 2)), 256, 0, h->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
}
