// pcf_correct.cu -- the implicit half step around the Poisson solve on the
// device.  Before the solve (implicit_integration!.jl:49-63): the implicit
// predictor update!(..., U/V/W/RhoP, RHS(), Implicit(), rf) (update!.jl:
// 632-728, :837-882, :988-1033, :1248-1336), set_boundaries!(state,
// BoundaryPredictands()) and modify_compressible_wind!.jl:38-80.  After it
// (apply_corrector!.jl:58-61): the boundary fill of dpip, then
// correct!.jl:164-385.  Both use compute_pressure_gradient.jl:108-297,
// compute_compressible_wind_factor.jl:102-157 and compute_buoyancy_factor.jl:
// 108-172.  FP64 throughout, one thread per (staggered) cell; each kernel
// reads a few haloed fields and writes one or two, so they are memory-bound
// and run once per solve.
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
    // predictor only: WKB momentum tendencies (NULL: NoWKB) and the w backup
    const double *dudt, *dvdt;
    double *wold;
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
    const Ix at{a.nxx, (long long)a.nxx * a.nyy};
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
        if (i >= a.nxx || j >= a.nyy || k >= nzz) return;
        const long long q = at(i, j, k);
        const int ii = i - a.nbx, jj = j - a.nby, kk = k - a.nbz;
        if (ii >= 0 && ii < a.nx && jj >= 0 && jj < a.ny && kk >= 0 && kk < a.nz) return;
        int si = ii % a.nx;
        if (si < 0) si += a.nx;
        int sj = jj % a.ny;
        if (sj < 0) sj += a.ny;
        const int sk = kk < 0 ? -kk - 1 : (kk >= a.nz ? 2 * a.nz - 1 - kk : kk);
        a.dpip[q] = a.dpip[at(si + a.nbx, sj + a.nby, sk + a.nbz)];
    }
}

// compute_pressure_gradient of the field P for U (dir 0) or V (dir 1) at the
// face (i+1/2, j, k) or (i, j+1/2, k)
__device__ double grad_h(const CorrectArgs &a, const double *P, const Ix &at, int i, int j, int k, int dir) {
    const long long c = at(i, j, k), o = dir == 0 ? 1 : at.sy, n = c + o;
    const double *met = dir == 0 ? a.met13 : a.met23;
    const double rh = dir == 0 ? a.rdx : a.rdy;
    const double rhoe = 0.5 * (a.rho[c] + a.rho[n]) + 0.5 * (a.rhobar[c] + a.rhobar[n]);
    const double pe = 0.5 * (a.pbar[c] + a.pbar[n]);
    const double mete = 0.5 * (met[c] + met[n]);
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

// compute_pressure_gradient of the field P for W at (i, j, k+1/2)
// (compute_pressure_gradient.jl:212-297) for the point c at level k.  The
// halo (nbx, nby >= 1, nbz >= 2) keeps the levels k0-1 and k1+1 in bounds.
__device__ __forceinline__ double grad_w_at(const CorrectArgs &a, const double *P, long long c, long long sy,
                                            long long sz) {
    const long long u = c + sz;
    const double *J = a.jac;
    const double jk = J[c], jk1 = J[u], rj = 1.0 / (jk + jk1);
    const double rhoe = (jk1 * a.rho[c] + jk * a.rho[u]) * rj + (jk1 * a.rhobar[c] + jk * a.rhobar[u]) * rj;
    const double pe = (jk1 * a.pbar[c] + jk * a.pbar[u]) * rj;
    const double m13 = (jk1 * a.met13[c] + jk * a.met13[u]) * rj;
    const double m23 = (jk1 * a.met23[c] + jk * a.met23[u]) * rj;
    const double m33 = (jk1 * a.met33[c] + jk * a.met33[u]) * rj;
    auto edge = [&](long long q) {  // Jacobian-weighted P at the w-level of column q
        return (J[q + sz] * P[q] + J[q] * P[q + sz]) / (J[q] + J[q + sz]);
    };
    const double pr = edge(c + 1), pl = edge(c - 1), pf = edge(c + sy), pb = edge(c - sy);
    return a.kappainv * a.mainv2 * pe / rhoe *
           (m13 * (pr - pl) * 0.5 * a.rdx + m23 * (pf - pb) * 0.5 * a.rdy + m33 * (P[u] - P[c]) * a.rdz);
}

// The pointwise kernels below are chains of dependent FP64 divisions and
// products: they run at as many resident warps as 64 registers a thread
// allow (4 blocks of 256 per SM), which hides those latencies better than
// fewer threads with more loads in flight each.
#define PCF_POINTWISE_BOUNDS __launch_bounds__(256, 4)

// U and V corrections (correct!.jl:177-245) with corx, cory: thread (x, y, k)
// over (nx + 1) x (ny + 1) x nz staggered positions; x = 0 is the face i0 - 1/2.
__global__ void PCF_POINTWISE_BOUNDS k_correct_uv(CorrectArgs a) {
    const Ix at{a.nxx, (long long)a.nxx * a.nyy};
    {
        const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, kk = blockIdx.z;
        if (x > a.nx || y > a.ny) return;
        const int i = a.nbx - 1 + x, j = a.nby - 1 + y, k = a.nbz + kk;
        const long long c = at(i, j, k);
        // the gradients reach one cell around (i, j, k) and the faces beyond it
        const long long nh = at.sz * (a.nz + 2 * a.nbz);
        if (!PCF_IN(c - at.sz - at.sy - 1, nh, 501) || !PCF_IN(c + at.sz + 2 * at.sy + 2, nh, 502)) return;
        if (y >= 1) {  // U at i + 1/2 for i in i0-1 .. i1
            double factor = 1.0;
            if (a.damp_h) factor += a.dt * 0.5 * (a.betar[c] + a.betar[c + 1]) * a.rf;
            const double cor = a.dt / factor * grad_h(a, a.dpip, at, i, j, k, 0);
            a.corx[c] = cor;
            const double wf = a.model == PCF_MODEL_COMPRESSIBLE ? (a.jac[c] * a.p[c] + a.jac[c + 1] * a.p[c + 1]) / 2 : 1.0;
            a.u[c] -= wf * cor;
        }
        if (x >= 1) {  // V at j + 1/2 for j in j0-1 .. j1
            const long long n = c + at.sy;
            double factor = 1.0;
            if (a.damp_h) factor += a.dt * 0.5 * (a.betar[c] + a.betar[n]) * a.rf;
            const double cor = a.dt / factor * grad_h(a, a.dpip, at, i, j, k, 1);
            a.cory[c] = cor;
            const double wf = a.model == PCF_MODEL_COMPRESSIBLE ? (a.jac[c] * a.p[c] + a.jac[n] * a.p[n]) / 2 : 1.0;
            a.v[c] -= wf * cor;
        }
    }
}

// W and rho' corrections (correct!.jl:247-360) on the interior, and
// pip += dpip (:375-385) on the interior plus one ghost layer: thread per
// cell of the (nx + 2) x (ny + 2) x (nz + 2) box.  COMP: the Compressible
// model's wind and buoyancy factors (1 and rhobar / rho in the others).
template <bool COMP>
__global__ void PCF_POINTWISE_BOUNDS k_correct_w_rhop_pip(CorrectArgs a) {
    const int bx = a.nx + 2, by = a.ny + 2;
    const long long sy = a.nxx, sz = (long long)a.nxx * a.nyy;
    const double dt2 = a.dt * a.dt;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= bx || y >= by) return;
    const int i = a.nbx - 1 + x, j = a.nby - 1 + y, k = a.nbz - 1 + z;
    const long long c = i + sy * j + sz * k;
    if (!PCF_IN(c, sz * (a.nz + 2 * a.nbz), 503)) return;
    a.pip[c] += a.dpip[c];
    const bool interior = x >= 1 && x <= a.nx && y >= 1 && y <= a.ny && z >= 1 && z <= a.nz;
    if (!interior) return;
    const double *J = a.jac;
    const long long u = c + sz, l = c - 1, b = c - sy;
    const bool top = k == a.nbz + a.nz - 1, bot = k == a.nbz;
    const double gu = top ? 0.0 : grad_w_at(a, a.dpip, c, sy, sz);
    if (!top) {  // W at k + 1/2 for k in k0 .. k1-1
        const double rj = 1.0 / (J[c] + J[u]);
        const double factor = 1.0 + a.dt * (J[u] * a.betar[c] + J[c] * a.betar[u]) * rj * a.rf;
        const double n2e = (J[u] * a.n2[c] + J[c] * a.n2[u]) * rj;
        double jp = 1.0, fw;
        const double den = J[u] * (a.rho[c] + a.rhobar[c]) + J[c] * (a.rho[u] + a.rhobar[u]);
        if (COMP) {
            jp = J[c] * J[u] * (a.p[c] + a.p[u]) * rj;
            fw = (J[u] * a.pbar[c] / a.thetabar[c] + J[c] * a.pbar[u] / a.thetabar[u]) / den;
        } else {
            fw = (J[u] * a.rhobar[c] + J[c] * a.rhobar[u]) / den;
        }
        const double inv = 1.0 / (factor + fw * n2e * dt2);
        const double cross = (J[u] * (a.met13[c] * (a.corx[c] + a.corx[l]) + a.met23[c] * (a.cory[c] + a.cory[b])) +
                              J[c] * (a.met13[u] * (a.corx[u] + a.corx[l + sz]) +
                                      a.met23[u] * (a.cory[u] + a.cory[b + sz]))) * rj;
        a.w[c] += -a.dt * inv * jp * gu - inv * fw * n2e * dt2 * jp * 0.5 * cross;
    }
    // rho'
    const double gl = bot ? 0.0 : grad_w_at(a, a.dpip, c - sz, sy, sz);
    const double gradient = 0.5 * (gl + gu);
    const double factor = 1.0 + a.dt * a.betar[c] * a.rf;
    const double fb = COMP ? a.pbar[c] / a.thetabar[c] / (a.rho[c] + a.rhobar[c])
                           : a.rhobar[c] / (a.rho[c] + a.rhobar[c]);
    const double n2c = a.n2[c];
    const double db = -1.0 / (factor + fb * n2c * dt2) *
                      (-fb * n2c * dt2 * J[c] * gradient +
                       fb * n2c * a.dt * J[c] * factor * 0.5 *
                           (a.met13[c] * (a.corx[c] + a.corx[l]) + a.met23[c] * (a.cory[c] + a.cory[b])));
    a.rhop[c] -= (a.rho[c] + a.rhobar[c]) / a.g_ndim * db;
}

// ------------------------------------------------------------ predictor --

// set_boundaries!(state, BoundaryPredictands()) on one rank: x and y
// periodic (the zonal, then the meridional pass over the full haloed range),
// then the wall conditions in z over the full horizontal range, mode + (line
// reflection) or - (point reflection); the staggered w is zero on both walls
// (the haloed level k0 - 1 and the interior level k1) and point-reflected
// about them.  With nz > nbz every ghost value is a function of interior
// values alone, so one pass over the haloed grid fills all fields without
// ordering.
constexpr int kMaxFillFields = 7;
struct FillArgs {
    int nx, ny, nz, nxx, nyy, nbx, nby, nbz, nf;
    double *f[kMaxFillFields];
    double sign[kMaxFillFields];
    int staggered[kMaxFillFields];
};

// One thread per ghost cell (plus, for the staggered w, per interior cell
// of the top level, which the wall condition zeroes), numbered as
//   [0, 2 nbz P)            the z-ghost levels, P = nxx nyy cells each,
//   [.., + nz R)            the x/y ghost ring of each interior level,
//                           R = P - nx ny (nby full rows below, nby above,
//                           then 2 nbx ghost cells per interior row),
//   [.., + nx ny)           the interior of level k1 (w only).
__global__ void __launch_bounds__(256) k_fill_predictands(FillArgs a) {
    const int P = a.nxx * a.nyy, R = P - a.nx * a.ny, S = a.nx * a.ny;
    const int tA = 2 * a.nbz * P, tB = tA + a.nz * R, tC = tB + S;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tC) return;
    int i, j, k;
    bool top_interior = false;
    if (t < tA) {
        const int L = t / P, p = t - L * P;
        k = L < a.nbz ? L : L + a.nz;
        j = p / a.nxx;
        i = p - j * a.nxx;
    } else if (t < tB) {
        const int kk = (t - tA) / R;
        int r = (t - tA) - kk * R;
        k = a.nbz + kk;
        const int rows = a.nby * a.nxx;
        if (r < rows) {
            j = r / a.nxx;
            i = r - j * a.nxx;
        } else if (r < 2 * rows) {
            r -= rows;
            j = a.nby + a.ny + r / a.nxx;
            i = r % a.nxx;
        } else {
            r -= 2 * rows;
            const int w2 = 2 * a.nbx, row = r / w2, c = r - row * w2;
            j = a.nby + row;
            i = c < a.nbx ? c : a.nx + c;
        }
    } else {
        const int p = t - tB, jj = p / a.nx;
        i = a.nbx + (p - jj * a.nx);
        j = a.nby + jj;
        k = a.nbz + a.nz - 1;
        top_interior = true;
    }
    const long long sy = a.nxx, sz = (long long)a.nxx * a.nyy;
    const long long q = i + sy * j + sz * k;
    const int ii = i - a.nbx, jj = j - a.nby, kk = k - a.nbz;
    const bool zin = kk >= 0 && kk < a.nz;
    int si = ii % a.nx;
    if (si < 0) si += a.nx;
    int sj = jj % a.ny;
    if (sj < 0) sj += a.ny;
    const long long col = (si + a.nbx) + sy * (sj + a.nby);
    for (int m = 0; m < a.nf; ++m) {
        double *f = a.f[m];
        if (a.staggered[m]) {
            if (kk == -1 || kk == a.nz - 1) f[q] = 0.0;
            else if (kk < -1) f[q] = a.sign[m] * f[col + sz * (-kk - 2 + a.nbz)];
            else if (kk >= a.nz) f[q] = a.sign[m] * f[col + sz * (2 * (a.nz - 1) - kk + a.nbz)];
            else f[q] = f[col + sz * k];
        } else if (!top_interior) {
            if (zin) f[q] = f[col + sz * k];
            else if (kk < 0) f[q] = a.sign[m] * f[col + sz * (-kk - 1 + a.nbz)];
            else f[q] = a.sign[m] * f[col + sz * (2 * a.nz - 1 - kk + a.nbz)];
        }
    }
}

// modify_compressible_wind!.jl:52-80 on the interior: u, v, w multiplied
// (divide = 0) or divided (divide = 1) by the compressible wind factors.
__global__ void __launch_bounds__(256) k_modify_wind(CorrectArgs a, int divide) {
    const Ix at{a.nxx, (long long)a.nxx * a.nyy};
    const double *J = a.jac, *P = a.p;
    {
        const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
        if (x >= a.nx || y >= a.ny) return;
        const long long c = at(x + a.nbx, y + a.nby, z + a.nbz), r = c + 1, f = c + at.sy, t = c + at.sz;
        // explicitly rounded products and sums (no FMA contraction), so the
        // factors and hence u, v, w round exactly as in the reference
        const double jpc = __dmul_rn(J[c], P[c]);
        const double fu = __dadd_rn(jpc, __dmul_rn(J[r], P[r])) / 2;
        const double fv = __dadd_rn(jpc, __dmul_rn(J[f], P[f])) / 2;
        const double fw = __dmul_rn(__dmul_rn(J[c], J[t]), __dadd_rn(P[c], P[t])) / __dadd_rn(J[c], J[t]);
        if (divide) {
            a.u[c] = a.u[c] / fu;
            a.v[c] = a.v[c] / fv;
            a.w[c] = a.w[c] / fw;
        } else {
            a.u[c] = __dmul_rn(a.u[c], fu);
            a.v[c] = __dmul_rn(a.v[c], fv);
            a.w[c] = __dmul_rn(a.w[c], fw);
        }
    }
}

__device__ __forceinline__ double wind_factor_u(const CorrectArgs &a, long long c, long long o) {
    return a.model == PCF_MODEL_COMPRESSIBLE ? (a.jac[c] * a.p[c] + a.jac[c + o] * a.p[c + o]) / 2 : 1.0;
}
// update!(U / V, RHS(), Implicit()) (update!.jl:837-882, :988-1033) over the
// (nx + 1) x (ny + 1) x nz staggered positions of k_correct_uv.
__global__ void PCF_POINTWISE_BOUNDS k_predict_uv(CorrectArgs a) {
    const Ix at{a.nxx, (long long)a.nxx * a.nyy};
    {
        const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, kk = blockIdx.z;
        if (x > a.nx || y > a.ny) return;
        const int i = a.nbx - 1 + x, j = a.nby - 1 + y, k = a.nbz + kk;
        const long long c = at(i, j, k);
        if (y >= 1) {  // U at i + 1/2 for i in i0-1 .. i1
            const long long n = c + 1;
            double rhoe = 0.5 * (a.rho[c] + a.rho[n]);
            rhoe += 0.5 * (a.rhobar[c] + a.rhobar[n]);
            const double gradient = grad_h(a, a.pip, at, i, j, k, 0);
            const double force = a.dudt ? (a.dudt[c] + a.dudt[n]) / 2 : 0.0;
            double factor = 1.0;
            if (a.damp_h) factor += a.dt * 0.5 * (a.betar[c] + a.betar[n]) * a.rf;
            const double jp = wind_factor_u(a, c, 1);
            a.u[c] = 1.0 / factor * (a.u[c] + a.dt * (-gradient + force / rhoe) * jp);
        }
        if (x >= 1) {  // V at j + 1/2 for j in j0-1 .. j1
            const long long n = c + at.sy;
            double rhoe = 0.5 * (a.rho[c] + a.rho[n]);
            rhoe += 0.5 * (a.rhobar[c] + a.rhobar[n]);
            const double gradient = grad_h(a, a.pip, at, i, j, k, 1);
            const double force = a.dvdt ? (a.dvdt[c] + a.dvdt[n]) / 2 : 0.0;
            double factor = 1.0;
            if (a.damp_h) factor += a.dt * 0.5 * (a.betar[c] + a.betar[n]) * a.rf;
            const double jp = wind_factor_u(a, c, at.sy);
            a.v[c] = 1.0 / factor * (a.v[c] + a.dt * (-gradient + force / rhoe) * jp);
        }
    }
}

// compute_compressible_wind_factor (compute_compressible_wind_factor.jl:
// 102-157) of U (o = 1) or V (o = sy) at the face after c, and of W
// (o = sz) at c's upper face; 1 outside the Compressible model.
template <bool COMP>
__device__ __forceinline__ double jp_uv(const CorrectArgs &a, long long c, long long o) {
    return COMP ? (a.jac[c] * a.p[c] + a.jac[c + o] * a.p[c + o]) / 2 : 1.0;
}
template <bool COMP>
__device__ __forceinline__ double jp_w(const CorrectArgs &a, long long c, long long sz) {
    if (!COMP) return 1.0;
    const double jk = a.jac[c], jk1 = a.jac[c + sz];
    return jk * jk1 * (a.p[c] + a.p[c + sz]) / (jk + jk1);
}

// compute_volume_force(state, i, j, k, W()) (compute_volume_force.jl:185-206)
__device__ __forceinline__ double force_w(const CorrectArgs &a, long long c, long long sz) {
    if (!a.dudt) return 0.0;
    const double *J = a.jac;
    const long long u = c + sz;
    return (J[u] * (a.met13[c] * a.dudt[c] + a.met23[c] * a.dvdt[c]) +
            J[c] * (a.met13[u] * a.dudt[u] + a.met23[u] * a.dvdt[u])) /
           (J[c] + J[u]);
}

// x / y, or x when y is the non-compressible wind factor 1 (exact either way)
template <bool COMP>
__device__ __forceinline__ double over(double x, double y) {
    return COMP ? x / y : x;
}

// update!(W, RHS(), Implicit()) (update!.jl:1248-1336) for k in k0 .. k1-1,
// with the u and v of k_predict_uv and the rho' before its own update.
template <bool COMP>
__global__ void PCF_POINTWISE_BOUNDS k_predict_w(CorrectArgs a) {
    const long long sy = a.nxx, sz = (long long)a.nxx * a.nyy;
    const double dt2 = a.dt * a.dt;
    const double *J = a.jac;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long c = (a.nbx + x) + sy * (a.nby + y) + sz * (a.nbz + z), u = c + sz, l = c - 1, b = c - sy;
    const double rj = J[c] + J[u];
    double rhoc = a.rho[c];
    double rhou = a.rho[u];
    double rhoedgeu = (J[u] * a.rho[c] + J[c] * a.rho[u]) / rj;
    rhoc += a.rhobar[c];
    rhou += a.rhobar[u];
    rhoedgeu += (J[u] * a.rhobar[c] + J[c] * a.rhobar[u]) / rj;
    const double gradient = grad_w_at(a, a.pip, c, sy, sz);
    const double force = force_w(a, c, sz);
    const double n2edgeu = (J[u] * a.n2[c] + J[c] * a.n2[u]) / rj;
    double factor = 1.0;
    factor += a.dt * (J[u] * a.betar[c] + J[c] * a.betar[u]) / rj * a.rf;
    const double bb = -a.g_ndim * (J[u] * a.rhop[c] / rhoc / J[c] + J[c] * a.rhop[u] / rhou / J[u]) / rj;
    const double uc = 0.5 * (over<COMP>(a.u[c], jp_uv<COMP>(a, c, 1)) + over<COMP>(a.u[l], jp_uv<COMP>(a, l, 1)));
    const double uu = 0.5 * (over<COMP>(a.u[u], jp_uv<COMP>(a, u, 1)) +
                             over<COMP>(a.u[l + sz], jp_uv<COMP>(a, l + sz, 1)));
    const double vc = 0.5 * (over<COMP>(a.v[c], jp_uv<COMP>(a, c, sy)) + over<COMP>(a.v[b], jp_uv<COMP>(a, b, sy)));
    const double vu = 0.5 * (over<COMP>(a.v[u], jp_uv<COMP>(a, u, sy)) +
                             over<COMP>(a.v[b + sz], jp_uv<COMP>(a, b + sz, sy)));
    const double jpedgeu = jp_w<COMP>(a, c, sz);
    double fw;
    const double den = J[u] * (a.rho[c] + a.rhobar[c]) + J[c] * (a.rho[u] + a.rhobar[u]);
    if (COMP)
        fw = (J[u] * a.pbar[c] / a.thetabar[c] + J[c] * a.pbar[u] / a.thetabar[u]) / den;
    else
        fw = (J[u] * a.rhobar[c] + J[c] * a.rhobar[u]) / den;
    a.w[c] = 1.0 / (factor + fw * n2edgeu * dt2) *
             (a.w[c] - a.dt * gradient * jpedgeu + a.dt * bb * jpedgeu + a.dt * force / rhoedgeu * jpedgeu +
              jpedgeu * fw * n2edgeu * dt2 *
                  (J[u] * (a.met13[c] * uc + a.met23[c] * vc) + J[c] * (a.met13[u] * uu + a.met23[u] * vu)) / rj);
}

// update!(RhoP, RHS(), Implicit()) (update!.jl:632-728) on the interior,
// after the boundary fill of u, v, w.
template <bool COMP>
__global__ void PCF_POINTWISE_BOUNDS k_predict_rhop(CorrectArgs a) {
    const long long sy = a.nxx, sz = (long long)a.nxx * a.nyy;
    const double dt2 = a.dt * a.dt;
    const double *J = a.jac;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long c = (a.nbx + x) + sy * (a.nby + y) + sz * (a.nbz + z), u = c + sz, d = c - sz, l = c - 1,
                    b = c - sy;
    const double rhoc = a.rho[c] + a.rhobar[c];
    double rhoedgeu = (J[u] * a.rho[c] + J[c] * a.rho[u]) / (J[c] + J[u]);
    rhoedgeu += (J[u] * a.rhobar[c] + J[c] * a.rhobar[u]) / (J[c] + J[u]);
    double rhoedged = (J[d] * a.rho[c] + J[c] * a.rho[d]) / (J[c] + J[d]);
    rhoedged += (J[d] * a.rhobar[c] + J[c] * a.rhobar[d]) / (J[c] + J[d]);
    const double wv = 0.5 * (over<COMP>(a.wold[c], jp_w<COMP>(a, c, sz)) + over<COMP>(a.wold[d], jp_w<COMP>(a, d, sz)));
    const bool bot = z == 0, top = z == a.nz - 1 && !bot;
    const double lower_gradient = bot ? 0.0 : grad_w_at(a, a.pip, d, sy, sz);
    const double lower_force = bot ? 0.0 : force_w(a, d, sz);
    const double upper_gradient = top ? 0.0 : grad_w_at(a, a.pip, c, sy, sz);
    const double upper_force = top ? 0.0 : force_w(a, c, sz);
    const double gradient = 0.5 * (lower_gradient + upper_gradient);
    const double force = 0.5 * (lower_force / rhoedged + upper_force / rhoedgeu) * rhoc;
    double factor = 1.0;
    factor += a.dt * a.betar[c] * a.rf;
    double bb = -a.g_ndim * a.rhop[c] / (a.rho[c] + a.rhobar[c]);
    const double fb = COMP ? a.pbar[c] / a.thetabar[c] / (a.rho[c] + a.rhobar[c])
                           : a.rhobar[c] / (a.rho[c] + a.rhobar[c]);
    const double n2c = a.n2[c], jc = J[c];
    bb = 1.0 / (factor + fb * n2c * dt2) *
         (-fb * n2c * a.dt * jc * (wv + a.dt * (-gradient + force / rhoc)) + factor * bb +
          fb * n2c * a.dt * jc * factor * 0.5 *
              (a.met13[c] * (over<COMP>(a.u[c], jp_uv<COMP>(a, c, 1)) + over<COMP>(a.u[l], jp_uv<COMP>(a, l, 1))) +
               a.met23[c] * (over<COMP>(a.v[c], jp_uv<COMP>(a, c, sy)) + over<COMP>(a.v[b], jp_uv<COMP>(a, b, sy)))));
    a.rhop[c] = -bb * (a.rho[c] + a.rhobar[c]) / a.g_ndim;
}

}  // namespace pcf

// One thread per point of an X x Y x Z box: 64 x 4 threads per block in the
// x-y plane (coalesced along x), one z level per block row of the grid.
struct Box3 {
    dim3 grid, block;
};
static Box3 box3(long long X, long long Y, long long Z) {
    Box3 b;
    b.block = dim3(64, 4, 1);
    b.grid = dim3((unsigned)((X + 63) / 64), (unsigned)((Y + 3) / 4), (unsigned)Z);
    return b;
}

// The handle's grid, background and constants in a CorrectArgs; rho, p,
// betar are the handle's copies of the last solve's inputs.
static pcf::CorrectArgs correct_args(pcf_handle *h, double dt, double rf, int damp_h) {
    pcf::CorrectArgs a{};
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
    return a;
}

// dpip (haloed, interior from the solve) -> halo fill and the corrections of
// u, v, w, rho', pip (haloed, in place); rho, betar, p are the handle's (the
// last solve's inputs).  corx, cory: haloed scratch.
int pcf_launch_correct(pcf_handle *h, double dt, double rf, int damp_h, double *dpip, double *u, double *v,
                       double *w, double *rhop, double *pip, double *corx, double *cory) {
    pcf::CorrectArgs a = correct_args(h, dt, rf, damp_h);
    a.dpip = dpip; a.u = u; a.v = v; a.w = w; a.rhop = rhop; a.pip = pip; a.corx = corx; a.cory = cory;
    h->launches += 3;
    const Box3 bf = box3(a.nxx, a.nyy, a.nz + 2 * a.nbz), buv = box3(a.nx + 1, a.ny + 1, a.nz),
               bw = box3(a.nx + 2, a.ny + 2, a.nz + 2);
    pcf::k_fill_dpip<<<bf.grid, bf.block, 0, h->stream>>>(a);
    pcf::k_correct_uv<<<buv.grid, buv.block, 0, h->stream>>>(a);
    if (a.model == PCF_MODEL_COMPRESSIBLE)
        pcf::k_correct_w_rhop_pip<true><<<bw.grid, bw.block, 0, h->stream>>>(a);
    else
        pcf::k_correct_w_rhop_pip<false><<<bw.grid, bw.block, 0, h->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
}

// set_boundaries!(state, BoundaryPredictands()): the model's predictands
// (rhop, u, v, w, pip; rho for PseudoIncompressible and Compressible; p for
// Compressible), haloed, in place.  Needs nz > nbz.
int pcf_launch_fill_predictands(pcf_handle *h, double *rho, double *rhop, double *u, double *v, double *w,
                                double *pip, double *p) {
    pcf::FillArgs a{};
    a.nx = h->d.nx; a.ny = h->d.ny; a.nz = h->d.nz;
    a.nxx = h->nxx; a.nyy = h->nyy;
    a.nbx = h->dims.nbx; a.nby = h->dims.nby; a.nbz = h->dims.nbz;
    auto add = [&](double *f, double sign, int stag) {
        a.f[a.nf] = f;
        a.sign[a.nf] = sign;
        a.staggered[a.nf] = stag;
        ++a.nf;
    };
    const int model = h->dims.model;
    if (model != PCF_MODEL_BOUSSINESQ) add(rho, -1.0, 0);
    add(rhop, -1.0, 0);
    add(u, 1.0, 0);
    add(v, 1.0, 0);
    add(w, -1.0, 1);
    add(pip, 1.0, 0);
    if (model == PCF_MODEL_COMPRESSIBLE) add(p, 1.0, 0);
    h->launches += 1;
    const long long plane = (long long)a.nxx * a.nyy, ring = plane - (long long)a.nx * a.ny;
    const long long cells = 2LL * a.nbz * plane + (long long)a.nz * ring + (long long)a.nx * a.ny;
    if (cells >= (1LL << 31)) return PCF_ERANGE;
    pcf::k_fill_predictands<<<(unsigned)((cells + 255) / 256), 256, 0, h->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
}

// modify_compressible_wind!(state, * or /) (Compressible only; no-op otherwise).
int pcf_launch_modify_wind(pcf_handle *h, const double *p, double *u, double *v, double *w, int divide) {
    if (h->dims.model != PCF_MODEL_COMPRESSIBLE) return PCF_OK;
    pcf::CorrectArgs a = correct_args(h, 0.0, 0.0, 0);
    a.p = p; a.u = u; a.v = v; a.w = w;
    h->launches += 1;
    const Box3 b = box3(a.nx, a.ny, a.nz);
    pcf::k_modify_wind<<<b.grid, b.block, 0, h->stream>>>(a, divide);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
}

// implicit_integration!.jl:53-63: wold = w, the implicit U, V, W updates,
// the predictand boundaries, the implicit RhoP update, the boundaries again.
// All arrays haloed device pointers of the caller (rho, p, betar: the
// current state; p only read in the Compressible model; dudt, dvdt: NULL for
// NoWKB).
int pcf_launch_predictor(pcf_handle *h, double dt, double rf, int damp_h, double *u, double *v, double *w,
                         double *rho, double *rhop, double *pip, double *p, const double *betar, const double *dudt,
                         const double *dvdt, double *wold) {
    pcf::CorrectArgs a = correct_args(h, dt, rf, damp_h);
    a.u = u; a.v = v; a.w = w; a.rhop = rhop; a.pip = pip; a.rho = rho; a.p = p; a.betar = betar;
    a.dudt = dudt; a.dvdt = dvdt; a.wold = wold;
    h->launches += 3;
    // save_backups!(state, :w) (save_backups!.jl:16-24): the whole haloed array
    cudaError_t e0 = cudaMemcpyAsync(wold, w, sizeof(double) * (size_t)h->nh, cudaMemcpyDeviceToDevice, h->stream);
    if (e0 != cudaSuccess) return pcf_set_cuda_error(e0);
    const Box3 buv = box3(a.nx + 1, a.ny + 1, a.nz), bw = box3(a.nx, a.ny, a.nz - 1), br = box3(a.nx, a.ny, a.nz);
    pcf::k_predict_uv<<<buv.grid, buv.block, 0, h->stream>>>(a);
    const bool comp = a.model == PCF_MODEL_COMPRESSIBLE;
    if (comp) pcf::k_predict_w<true><<<bw.grid, bw.block, 0, h->stream>>>(a);
    else pcf::k_predict_w<false><<<bw.grid, bw.block, 0, h->stream>>>(a);
    int rc = pcf_launch_fill_predictands(h, rho, rhop, u, v, w, pip, p);
    if (rc) return rc;
    if (comp) pcf::k_predict_rhop<true><<<br.grid, br.block, 0, h->stream>>>(a);
    else pcf::k_predict_rhop<false><<<br.grid, br.block, 0, h->stream>>>(a);
    if ((rc = pcf_launch_fill_predictands(h, rho, rhop, u, v, w, pip, p))) return rc;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
}

unsigned long long pcf_bounds_take_correct() { return pcf_bounds_take_local(); }
