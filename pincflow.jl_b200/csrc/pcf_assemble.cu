// pcf_assemble.cu -- operator assembly (compute_operator!) and the
// preconditioner's Thomas factors, sm_100a.
//
// Formulation.  The reference writes each of the 25 tensor elements as a
// long per-element expression with five vertical cases
// (src/PoissonSolver/compute_operator!.jl:795-1543).  All of them follow from
// one rule, which this kernel evaluates instead: the scaled operator is a sum
// over 14 faces of the cell,
//     A s = sum_F  flux_F * grad_F(s),   flux_F = g_F * P_F,
// where g_F are the gradient coefficients of :426-791 (gedger ... gdedgeb)
// and P_F the face-interpolated P of :141-161.  The 12 horizontal faces
// (i+-1/2 and j+-1/2 at levels k-1, k, k+1) carry
//     grad = (s_hi - s_lo) / dx  +  met_F * d/dz(s) on both adjacent columns,
// with d/dz one-sided at the walls (weights -3/4, 1, -1/4 at the bottom level,
// +3/4, -1, +1/4 at the top level, +-1/4 centred elsewhere, all / dz).  The 2
// vertical faces (k+-1/2) carry
//     grad = met33_F (s_k+1 - s_k)/dz + met13_F/(2dx) (s~_i+1 - s~_i-1) + met23_F/(2dy) (...)
// with s~ the Jacobian-weighted vertical interpolation of :261-266.  Each
// coefficient is finally scaled by 1/(fcscal * fcscal_neighbour) (:1546-1570).
// The Compressible model subtracts dpdpi / dt / (dt rsp / kappa) from A_c
// (:855-860).  compute_buoyancy_factor(W) (src/Update/compute_buoyancy_factor.jl:
// 135-172) is evaluated inline.
//
// One thread per cell, FP64 throughout; the FP32 copy is rounded from the
// FP64 result.  Assembly runs once per solve, so this kernel favours clarity
// over bandwidth (about 34 words per cell, L2-resident neighbour reads).
#include "pcf_internal.cuh"

namespace pcf {

struct AssembleArgs {
    int nx, ny, nz, nxx, nyy, nbx, nby, nbz;
    int z_size, ko, model, damp_h;
    double dx, dy, dz, dt, rf;
    double rdx, rdy, rdz;  // 1 / dx, 1 / dy, 1 / dz
    double gamma, kappa, rsp, pref;
    const double *jac, *met13, *met23, *met33, *pbar, *rhobar, *thetabar, *n2, *rho, *betar, *p;
    const double *fch;   // fcscal = sqrt(pbar^2 / rhobar) on the haloed grid (computed with the background)
    const double *rfch;  // 1 / fcscal, same grid
    double *coef64;
    float *coef32;
    __nv_bfloat16 *coef16;  // BF16 copy (when the handle holds one)
};

// Column offsets of the 5 columns that carry coefficients.
enum Col { CC = 0, CR = 1, CL = 2, CF = 3, CB = 4 };

// Plane index of (column, vertical offset -2..2) in Tensor order.
__device__ __constant__ int kPlane[5][5] = {
    {PCF_ADD, PCF_AD, PCF_AC, PCF_AU, PCF_AUU},
    {PCF_ARDD, PCF_ARD, PCF_AR, PCF_ARU, PCF_ARUU},
    {PCF_ALDD, PCF_ALD, PCF_AL, PCF_ALU, PCF_ALUU},
    {PCF_AFDD, PCF_AFD, PCF_AF, PCF_AFU, PCF_AFUU},
    {PCF_ABDD, PCF_ABD, PCF_AB, PCF_ABU, PCF_ABUU},
};

// Vertical case of a level, first match of the reference's chain
// (ko + k == k0, k0 + 1, z_size + nbz - 1, z_size + nbz).
enum Case { K_BOT = 0, K_BOT1 = 1, K_TOP1 = 2, K_TOP = 3, K_IN = 4 };

__device__ __forceinline__ int level_case(int kg, int nbz, int z_size) {
    if (kg == nbz) return K_BOT;
    if (kg == nbz + 1) return K_BOT1;
    if (kg == z_size + nbz - 2) return K_TOP1;
    if (kg == z_size + nbz - 1) return K_TOP;
    return K_IN;
}

__global__ void __launch_bounds__(128) k_assemble(AssembleArgs a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    // 32-bit decomposition: pcf_create admits fewer than 2^31 cells
    const unsigned ucell = (unsigned)cell, ux = (unsigned)a.nx, uy = (unsigned)a.ny;
    const int ii = (int)(ucell % ux);
    const int jj = (int)((ucell / ux) % uy);
    const int kk = (int)(ucell / (ux * uy));
    const int i = ii + a.nbx, j = jj + a.nby, k = kk + a.nbz;
    const long long sx = 1, sy = a.nxx, sz = (long long)a.nxx * a.nyy;
    const long long h = i * sx + j * sy + k * sz;
    // the reads below reach one cell in x and y and two in z around h
    const long long nh = sz * (a.nz + 2 * a.nbz);
    if (!PCF_IN(h - 2 * sz - sy - 1, nh, 401) || !PCF_IN(h + 2 * sz + sy + 1, nh, 402)) return;

    auto J = [&](int di, int dj, int dk) { return __ldg(a.jac + h + di * sx + dj * sy + dk * sz); };
    auto PB = [&](int di, int dj, int dk) { return __ldg(a.pbar + h + di * sx + dj * sy + dk * sz); };
    auto RB = [&](int di, int dj, int dk) { return __ldg(a.rhobar + h + di * sx + dj * sy + dk * sz); };
    auto RO = [&](int di, int dj, int dk) { return __ldg(a.rho + h + di * sx + dj * sy + dk * sz); };
    auto BR = [&](int di, int dj, int dk) { return __ldg(a.betar + h + di * sx + dj * sy + dk * sz); };
    auto M13 = [&](int di, int dj, int dk) { return __ldg(a.met13 + h + di * sx + dj * sy + dk * sz); };
    auto M23 = [&](int di, int dj, int dk) { return __ldg(a.met23 + h + di * sx + dj * sy + dk * sz); };
    auto M33 = [&](int di, int dj, int dk) { return __ldg(a.met33 + h + di * sx + dj * sy + dk * sz); };
    auto N2 = [&](int dk) { return __ldg(a.n2 + h + dk * sz); };
    auto RFC = [&](int di, int dj, int dk) { return __ldg(a.rfch + h + di * sx + dj * sy + dk * sz); };
    // Jacobian-weighted value at the w-level between dk and dk + up (up = +-1):
    // (J(dk+up) X(dk) + J(dk) X(dk+up)) / (J(dk) + J(dk+up)); rj = 1 / (J(dk) + J(dk+up)).
    // Divisions are the kernel's main cost in FP64, so every repeated
    // denominator is inverted once.
    auto zint = [&](double xk, double xn, double jk, double jn, double rj) { return (jn * xk + jk * xn) * rj; };

    const double dt2 = a.dt * a.dt;
    const double jc = J(0, 0, 0), ju = J(0, 0, 1), jd = J(0, 0, -1);
    const double rju = 1.0 / (jc + ju), rjd = 1.0 / (jc + jd);
    const double jacinv = 1.0 / jc;
    const double pc = PB(0, 0, 0);
    const double jpc = jc * pc;

    // buoyancy factor at k+1/2 (up = +1) and k-1/2 (up = -1)
    auto fw = [&](int lo) {  // W() factor between levels lo and lo + 1
        const double jl = J(0, 0, lo), jh = J(0, 0, lo + 1);
        const double rl = RB(0, 0, lo), rh = RB(0, 0, lo + 1);
        const double den = jh * (RO(0, 0, lo) + rl) + jl * (RO(0, 0, lo + 1) + rh);
        if (a.model == PCF_MODEL_COMPRESSIBLE)
            return (jh * PB(0, 0, lo) / __ldg(a.thetabar + h + lo * sz) +
                    jl * PB(0, 0, lo + 1) / __ldg(a.thetabar + h + (lo + 1) * sz)) / den;
        return (jh * rl + jl * rh) / den;
    };
    const double fwu = fw(0), fwd = fw(-1);

    // vertical face quantities
    const double pudiv = jc * ju * (pc + PB(0, 0, 1)) * rju;
    const double pddiv = jc * jd * (pc + PB(0, 0, -1)) * rjd;
    const double n2u = zint(N2(0), N2(1), jc, ju, rju), n2d = zint(N2(0), N2(-1), jc, jd, rjd);
    const double facu = 1.0 + a.dt * zint(BR(0, 0, 0), BR(0, 0, 1), jc, ju, rju) * a.rf;
    const double facd = 1.0 + a.dt * zint(BR(0, 0, 0), BR(0, 0, -1), jc, jd, rjd) * a.rf;
    const double impu = 1.0 / (facu + fwu * n2u * dt2);
    const double impd = 1.0 / (facd + fwd * n2d * dt2);
    // buoyancy-coupling factors shared by every horizontal face
    const double cu = jacinv * a.rdz * pudiv * impu * fwu * n2u * dt2 * 0.5;
    const double cd = jacinv * a.rdz * pddiv * impd * fwd * n2d * dt2 * 0.5;

    const int kg = a.ko + k;
    const bool bot = kg == a.nbz, top = kg == a.z_size + a.nbz - 1;
    const int case_k = level_case(kg, a.nbz, a.z_size);

    double A[5][5];
#pragma unroll
    for (int c = 0; c < 5; ++c)
#pragma unroll
        for (int z = 0; z < 5; ++z) A[c][z] = 0.0;

    // Adds flux * (one-sided or centred d/dz at level L = k + dl) * met / dz to
    // the two columns c0, c1 adjacent to a horizontal face.
    auto add_vz = [&](int c0, int c1, int dl, double w) {
        const int cs = level_case(kg + dl, a.nbz, a.z_size);
        const int z0 = dl + 2;  // index of level L in the -2..2 window
        if (cs == K_BOT) {
            A[c0][z0] += -0.75 * w; A[c0][z0 + 1] += w; A[c0][z0 + 2] += -0.25 * w;
            A[c1][z0] += -0.75 * w; A[c1][z0 + 1] += w; A[c1][z0 + 2] += -0.25 * w;
        } else if (cs == K_TOP) {
            A[c0][z0] += 0.75 * w; A[c0][z0 - 1] += -w; A[c0][z0 - 2] += 0.25 * w;
            A[c1][z0] += 0.75 * w; A[c1][z0 - 1] += -w; A[c1][z0 - 2] += 0.25 * w;
        } else {
            A[c0][z0 + 1] += 0.25 * w; A[c0][z0 - 1] += -0.25 * w;
            A[c1][z0 + 1] += 0.25 * w; A[c1][z0 - 1] += -0.25 * w;
        }
    };

    // ---- the 12 horizontal faces -------------------------------------------
    // dir: 0 = r (i+1/2), 1 = l (i-1/2), 2 = f (j+1/2), 3 = b (j-1/2)
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        const int di = dir == 0 ? 1 : (dir == 1 ? -1 : 0);
        const int dj = dir == 2 ? 1 : (dir == 3 ? -1 : 0);
        const int cn = dir == 0 ? CR : (dir == 1 ? CL : (dir == 2 ? CF : CB));
        const double sgn = (dir == 0 || dir == 2) ? 1.0 : -1.0;  // outward normal
        const double rdh = dir < 2 ? a.rdx : a.rdy;
        const double *met = dir < 2 ? a.met13 : a.met23;
        auto MH = [&](int dk) { return __ldg(met + h + dk * sz); };
        auto MHn = [&](int dk) { return __ldg(met + h + di * sx + dj * sy + dk * sz); };
#pragma unroll
        for (int dl = -1; dl <= 1; ++dl) {
            // skip the faces whose g vanishes: level k+1 at the top, k-1 at the bottom
            if ((dl == 1 && top) || (dl == -1 && bot)) continue;
            const double pgra = 0.5 * (PB(0, 0, dl) + PB(di, dj, dl));
            const double rho_e = 0.5 * (RO(0, 0, dl) + RO(di, dj, dl) + RB(0, 0, dl) + RB(di, dj, dl));
            const double fac = a.damp_h ? 1.0 + a.dt * 0.5 * (BR(0, 0, dl) + BR(di, dj, dl)) * a.rf : 1.0;
            const double imp_over_rho = 1.0 / (fac * rho_e);
            double g;
            if (dl == 0) {
                // gedge{r,l,f,b} (:426-639): horizontal gradient plus the two vertical couplings
                const double pdiv = 0.5 * (jpc + J(di, dj, 0) * PB(di, dj, 0));
                g = sgn * jacinv * rdh * pdiv;
                if (!top) g += cu * MH(0) * ju * rju;
                if (!bot) g -= cd * MH(0) * jd * rjd;
                g *= imp_over_rho;
            } else if (dl == 1) {
                // guedge{r,l,f,b} (:656-722)
                g = cu * MH(1) * jc * rju * imp_over_rho;
            } else {
                // gdedge{r,l,f,b} (:725-791)
                g = -cd * MH(-1) * jc * rjd * imp_over_rho;
            }
            const double flux = g * pgra;
            const double metf = 0.5 * (MH(dl) + MHn(dl));
            // horizontal difference (s_hi - s_lo)/dh, hi = neighbour for r/f, cell for l/b
            const double wh = flux * rdh;
            A[cn][dl + 2] += sgn * wh;
            A[CC][dl + 2] -= sgn * wh;
            add_vz(CC, cn, dl, flux * metf * a.rdz);
        }
    }

    // ---- the 2 vertical faces ------------------------------------------------
    if (!top) {  // G(k + 1/2) (:642-646)
        const double rho_u =
            zint(RO(0, 0, 0), RO(0, 0, 1), jc, ju, rju) + zint(RB(0, 0, 0), RB(0, 0, 1), jc, ju, rju);
        const double g = jacinv * a.rdz * pudiv * impu / rho_u;
        const double flux = g * zint(pc, PB(0, 0, 1), jc, ju, rju);
        const double w33 = flux * zint(M33(0, 0, 0), M33(0, 0, 1), jc, ju, rju) * a.rdz;
        A[CC][3] += w33;
        A[CC][2] -= w33;
        const double w13 = flux * zint(M13(0, 0, 0), M13(0, 0, 1), jc, ju, rju) * 0.5 * a.rdx;
        const double w23 = flux * zint(M23(0, 0, 0), M23(0, 0, 1), jc, ju, rju) * 0.5 * a.rdy;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int di = q == 0 ? 1 : (q == 1 ? -1 : 0), dj = q == 2 ? 1 : (q == 3 ? -1 : 0);
            const int cn = q == 0 ? CR : (q == 1 ? CL : (q == 2 ? CF : CB));
            const double w = (q < 2 ? w13 : w23) * ((q == 0 || q == 2) ? 1.0 : -1.0);
            const double j0 = J(di, dj, 0), j1 = J(di, dj, 1);
            const double r01 = w / (j0 + j1);
            A[cn][2] += j1 * r01;
            A[cn][3] += j0 * r01;
        }
    }
    if (!bot) {  // G(k - 1/2) (:649-653)
        const double rho_d =
            zint(RO(0, 0, 0), RO(0, 0, -1), jc, jd, rjd) + zint(RB(0, 0, 0), RB(0, 0, -1), jc, jd, rjd);
        const double g = -jacinv * a.rdz * pddiv * impd / rho_d;
        const double flux = g * zint(pc, PB(0, 0, -1), jc, jd, rjd);
        const double w33 = flux * zint(M33(0, 0, 0), M33(0, 0, -1), jc, jd, rjd) * a.rdz;
        A[CC][2] += w33;
        A[CC][1] -= w33;
        const double w13 = flux * zint(M13(0, 0, 0), M13(0, 0, -1), jc, jd, rjd) * 0.5 * a.rdx;
        const double w23 = flux * zint(M23(0, 0, 0), M23(0, 0, -1), jc, jd, rjd) * 0.5 * a.rdy;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int di = q == 0 ? 1 : (q == 1 ? -1 : 0), dj = q == 2 ? 1 : (q == 3 ? -1 : 0);
            const int cn = q == 0 ? CR : (q == 1 ? CL : (q == 2 ? CF : CB));
            const double w = (q < 2 ? w13 : w23) * ((q == 0 || q == 2) ? 1.0 : -1.0);
            const double j0 = J(di, dj, 0), j1 = J(di, dj, -1);
            const double r01 = w / (j0 + j1);
            A[cn][2] += j1 * r01;
            A[cn][1] += j0 * r01;
        }
    }

    if (a.model == PCF_MODEL_COMPRESSIBLE) {
        const double dpdpi = 1.0 / (a.gamma - 1.0) * pow(a.rsp / a.pref, 1.0 - a.gamma) *
                             pow(__ldg(a.p + h), 2.0 - a.gamma);
        A[CC][2] -= (dpdpi / a.dt) / (a.dt * a.rsp / a.kappa);
    }
    (void)case_k;

    // ---- scaling by 1 / (fcscal fcscal_neighbour) and store ----------------
    const double rfcc = RFC(0, 0, 0);
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const int di = c == CR ? 1 : (c == CL ? -1 : 0);
        const int dj = c == CF ? 1 : (c == CB ? -1 : 0);
#pragma unroll
        for (int z = 0; z < 5; ++z) {
            const double v = A[c][z] * rfcc * RFC(di, dj, z - 2);
            const long long o = (long long)kPlane[c][z] * n + cell;
            if (!PCF_IN(o, (long long)PCF_NCOEF * n, 403)) continue;
            a.coef64[o] = v;
            a.coef32[o] = (float)v;
            if (a.coef16) a.coef16[o] = __float2bfloat16_rn((float)v);
        }
    }
}

// Pivots of the preconditioner's tridiagonal systems
// (1 - d_eta ac) s_k - d_eta ad s_k-1 - d_eta au s_k+1 = rhs_k
// (apply_preconditioner!.jl:73-93).  Forward sweep y_k = P_k rhs_k + M_k y_k-1,
// back substitution s_k = y_k + Q_k s_k+1.  They depend on the operator and
// d_eta only, so they are built once per solve instead of once per sweep.
// The recurrence is serial in k, so the loads of each block of kFactorChunk
// levels are issued together ahead of it: one memory round trip per block
// instead of one per level (the arithmetic, and so the result, is unchanged).
constexpr int kFactorChunk = 8;

__global__ void k_factors(int plane, int nz, long long n, double deta, const double *__restrict__ coef,
                          double *__restrict__ f64, float *__restrict__ f32) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= plane) return;
    const double *ac = coef + (long long)PCF_AC * n, *ad = coef + (long long)PCF_AD * n,
                 *au = coef + (long long)PCF_AU * n;
    double qprev = 0.0;
    for (int k0 = 0; k0 < nz; k0 += kFactorChunk) {
        double vc[kFactorChunk], vd[kFactorChunk], vu[kFactorChunk];
#pragma unroll
        for (int q = 0; q < kFactorChunk; ++q) {
            const int k = k0 + q;
            const long long o = col + (long long)plane * (k < nz ? k : 0);
            vc[q] = ac[o];
            vd[q] = ad[o];
            vu[q] = au[o];
        }
#pragma unroll
        for (int q = 0; q < kFactorChunk; ++q) {
            const int k = k0 + q;
            if (k >= nz) break;
            const long long o = col + (long long)plane * k;
            if (!PCF_IN(o, n, 404)) break;
            const double piv = k == 0 ? 1.0 / (1.0 - deta * vc[q])
                                      : 1.0 / (1.0 - deta * vc[q] - deta * vd[q] * qprev);
            const double m = k == 0 ? 0.0 : deta * vd[q] * piv;
            const double qv = deta * vu[q] * piv;
            f64[o] = piv;
            f64[n + o] = m;
            f64[2 * n + o] = qv;
            f32[o] = (float)piv;
            f32[n + o] = (float)m;
            f32[2 * n + o] = (float)qv;
            qprev = qv;
        }
    }
}

}  // namespace pcf

int pcf_launch_assemble(pcf_handle *h, double dt, double rf, int damp_h) {
    pcf::AssembleArgs a;
    a.nx = h->d.nx; a.ny = h->d.ny; a.nz = h->d.nz;
    a.nxx = h->nxx; a.nyy = h->nyy;
    a.nbx = h->dims.nbx; a.nby = h->dims.nby; a.nbz = h->dims.nbz;
    a.z_size = h->d.nz; a.ko = 0; a.model = h->dims.model; a.damp_h = damp_h;
    a.dx = h->dx; a.dy = h->dy; a.dz = h->dz; a.dt = dt; a.rf = rf;
    // Constants.jl:119-128
    a.gamma = 1.4; a.kappa = (1.4 - 1.0) / 1.4; a.rsp = 287.0; a.pref = 101325.0;
    a.jac = h->jac; a.met13 = h->met13; a.met23 = h->met23; a.met33 = h->met33;
    a.pbar = h->pbar; a.rhobar = h->rhobar; a.thetabar = h->thetabar; a.n2 = h->n2;
    a.rho = h->rho; a.betar = h->betar; a.p = h->p;
    a.fch = h->fch;
    a.rfch = h->rfch;
    a.rdx = 1.0 / h->dx; a.rdy = 1.0 / h->dy; a.rdz = 1.0 / h->dz;
    a.coef64 = h->coef64; a.coef32 = h->coef32; a.coef16 = h->coef16;
    const long long n = h->d.n;
    const int bs = 128;
    pcf::k_assemble<<<(unsigned)((n + bs - 1) / bs), bs, 0, h->stream>>>(a);
    PCF_CUDA_TRY(cudaGetLastError());
    h->fac_deta = __builtin_nan("");
    return PCF_OK;
}

int pcf_launch_factors(pcf_handle *h, double deta) {
    const int bs = 128;
    pcf::k_factors<<<(h->d.plane + bs - 1) / bs, bs, 0, h->stream>>>(h->d.plane, h->d.nz, h->d.n, deta,
                                                                      h->coef64, h->fac64, h->fac32);
    PCF_CUDA_TRY(cudaGetLastError());
    h->fac_deta = deta;
    return PCF_OK;
}

unsigned long long pcf_bounds_take_assemble() { return pcf_bounds_take_local(); }
