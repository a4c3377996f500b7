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
// One thread per cell, FP64 throughout; the FP32 and BF16 copies and the
// difference form are rounded from the FP64 result.  The inputs of a tile of
// columns are staged level by level in shared memory (below).
#include <atomic>

#include "pcf_internal.cuh"

namespace pcf {

struct AssembleArgs {
    int nx, ny, nz, nxx, nyy, nbx, nby, nbz;
    int z_size, ko, model, damp_h;
    int kc0;  // first z-chunk (of AKC levels) of the launch
    double dx, dy, dz, dt, rf;
    double rdx, rdy, rdz;  // 1 / dx, 1 / dy, 1 / dz
    double gamma, kappa, rsp, pref;
    const double *jac, *met13, *met23, *met33, *pbar, *rhobar, *thetabar, *n2, *rho, *betar, *p;
    const double *fch;   // fcscal = sqrt(pbar^2 / rhobar) on the haloed grid (computed with the background)
    const double *rfch;  // 1 / fcscal, same grid
    double *coef64;
    float *coef32;
    __nv_bfloat16 *coef16;  // BF16 copy (when the handle holds one)
    float *diff32;          // difference-form FP32 operator (k_build_diff's planes)
    double *fc64;           // fcscal on the interior
    float *rfc32;           // 1 / fcscal on the interior
};

// Column offsets of the 5 columns that carry coefficients.
enum Col { CC = 0, CR = 1, CL = 2, CF = 3, CB = 4 };

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

// ---- staging -------------------------------------------------------------
// A block assembles a tile of AX x AY columns over AKC levels, marching up in
// z.  Every input it reads lies within one column in x and y and two levels
// in z of the cell, so each level of each input field is copied once per block
// into a shared-memory ring (cp.async, 8 bytes per element) and every cell
// reads its neighbourhood from there.  The copy of level k + 2 (k + 3 for the
// 5-level fields) is in flight while level k is computed.
constexpr int AX = 32, AY = 4, AKC = 16;
constexpr int AHX = AX + 2, AHY = AY + 2, AT = AHX * AHY;  // the tile with its 1-column halo
// fields with a halo and a 3-level window (k-1..k+1): J, pbar, rhobar, rho', betar, met13, met23
constexpr int NH3 = 7, F_J = 0, F_PB = 1, F_RB = 2, F_RO = 3, F_BR = 4, F_M13 = 5, F_M23 = 6;
// fields with a halo and a 5-level window (k-2..k+2): 1 / fcscal, fcscal
constexpr int NH5 = 2, F_RFC = 0, F_FCH = 1;
// centre-column fields with a 3-level window, held in registers: met33, N^2, thetabar
constexpr int NC3 = 3, F_M33 = 0, F_N2 = 1, F_TH = 2;
constexpr int S3 = 4, S5 = 6;  // ring slots: the window plus the level in flight
constexpr int ASM_H3 = 0, ASM_H5 = ASM_H3 + NH3 * S3 * AT, ASM_DOUBLES = ASM_H5 + NH5 * S5 * AT;
constexpr int ASM_SMEM = ASM_DOUBLES * (int)sizeof(double);  // 65,280 bytes: three blocks per SM

// (di, dj, dk) of plane p in Tensor order (pincflow_poisson.h: AC, AL, AR, AB,
// AF, AD, AU, ...), and the column index (Col) of (di, dj).
__host__ __device__ constexpr int plane_di(int p) {
    return (p == PCF_AL || p == PCF_ALD || p == PCF_ALU || p == PCF_ALDD || p == PCF_ALUU)   ? -1
           : (p == PCF_AR || p == PCF_ARD || p == PCF_ARU || p == PCF_ARDD || p == PCF_ARUU) ? 1
                                                                                               : 0;
}
__host__ __device__ constexpr int plane_dj(int p) {
    return (p == PCF_AB || p == PCF_ABD || p == PCF_ABU || p == PCF_ABDD || p == PCF_ABUU)   ? -1
           : (p == PCF_AF || p == PCF_AFD || p == PCF_AFU || p == PCF_AFDD || p == PCF_AFUU) ? 1
                                                                                               : 0;
}
__host__ __device__ constexpr int plane_dk(int p) {
    return (p == PCF_ADD || p == PCF_ALDD || p == PCF_ARDD || p == PCF_ABDD || p == PCF_AFDD)   ? -2
           : (p == PCF_AUU || p == PCF_ALUU || p == PCF_ARUU || p == PCF_ABUU || p == PCF_AFUU) ? 2
           : (p == PCF_AD || p == PCF_ALD || p == PCF_ARD || p == PCF_ABD || p == PCF_AFD)      ? -1
           : (p == PCF_AU || p == PCF_ALU || p == PCF_ARU || p == PCF_ABU || p == PCF_AFU)      ? 1
                                                                                                 : 0;
}
__host__ __device__ constexpr int plane_col(int p) {
    return plane_di(p) == 1 ? CR : plane_di(p) == -1 ? CL : plane_dj(p) == 1 ? CF : plane_dj(p) == -1 ? CB : CC;
}

// the 25 planes are 25 distinct (column, dk) pairs
__host__ __device__ constexpr bool planes_distinct() {
    for (int p = 0; p < PCF_NCOEF; ++p)
        for (int q = p + 1; q < PCF_NCOEF; ++q)
            if (plane_col(p) == plane_col(q) && plane_dk(p) == plane_dk(q)) return false;
    return plane_col(PCF_AC) == CC && plane_col(PCF_AL) == CL && plane_col(PCF_AR) == CR &&
           plane_col(PCF_AB) == CB && plane_col(PCF_AF) == CF;
}
static_assert(planes_distinct(), "plane offsets");

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Copies level kk (interior index, -2..nz+1) of a haloed field into one ring
// slot: the tile plus its 1-column halo.
__device__ __forceinline__ void stage_level(double *dst, const double *src, const AssembleArgs &a, int i0, int j0,
                                            int kk, int tid) {
    const long long sy = a.nxx, sz = (long long)a.nxx * a.nyy;
    const long long nh = sz * (a.nz + 2 * a.nbz);
    for (int t = tid; t < AT; t += AX * AY) {
        const int ty = t / AHX, tx = t - ty * AHX;
        const int i = i0 - 1 + tx, j = j0 - 1 + ty;  // interior indices, -1..nx and -1..ny
        if (i > a.nx || j > a.ny) continue;            // beyond the halo of a partial tile
        const long long g = (i + a.nbx) + sy * (j + a.nby) + sz * (kk + a.nbz);
        if (!PCF_IN(g, nh, 401)) continue;
        cp_async8(dst + t, src + g);
    }
}

// One thread per cell, FP64 throughout, the arithmetic of compute_operator!.jl
// in the face-flux form described at the top of this file.  Besides the FP64,
// FP32 and (when the handle holds one) BF16 planes it writes the
// difference-form FP32 operator for pi = s / fcscal (the planes A_nb fcscal_nb
// and their sum in plane AC, summed in plane order in FP64), fcscal and
// 1 / fcscal on the interior.
__global__ void __launch_bounds__(AX * AY, 3) k_assemble(AssembleArgs a) {
    extern __shared__ double asm_sm[];
    const int tid = threadIdx.x + AX * threadIdx.y;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = blockIdx.x * AX, j0 = blockIdx.y * AY, k0 = (blockIdx.z + a.kc0) * AKC;
    const int k1 = min(k0 + AKC, a.nz);
    const int ii = i0 + tx, jj = j0 + ty;
    const bool live = ii < a.nx && jj < a.ny;
    const long long n = (long long)a.nx * a.ny * a.nz;
    const long long sy = a.nxx, sz = (long long)a.nxx * a.nyy;

    const double *h3src[NH3] = {a.jac, a.pbar, a.rhobar, a.rho, a.betar, a.met13, a.met23};
    const double *h5src[NH5] = {a.rfch, a.fch};
    const double *c3src[NC3] = {a.met33, a.n2, a.thetabar};
    const bool have_th = a.model == PCF_MODEL_COMPRESSIBLE && a.thetabar;
    auto slot3 = [](int kk) { return (kk + 4) & 3; };  // kk >= -2
    auto slot5 = [](int kk) { return (kk + 6) % 6; };  // kk >= -2
    auto stage3 = [&](int kk) {
#pragma unroll
        for (int f = 0; f < NH3; ++f)
            stage_level(asm_sm + ASM_H3 + (f * S3 + slot3(kk)) * AT, h3src[f], a, i0, j0, kk, tid);
    };
    auto stage5 = [&](int kk) {
#pragma unroll
        for (int f = 0; f < NH5; ++f)
            stage_level(asm_sm + ASM_H5 + (f * S5 + slot5(kk)) * AT, h5src[f], a, i0, j0, kk, tid);
    };
    // centre-column fields at level kk, straight from global memory (coalesced)
    const long long col = (ii + a.nbx) + sy * (jj + a.nby);
    const long long nh = sz * (a.nz + 2 * a.nbz);
    auto centre = [&](double (&dst)[NC3], int kk) {
        const long long g = col + sz * (kk + a.nbz);
        if (!live || !PCF_IN(g, nh, 405)) return;
#pragma unroll
        for (int f = 0; f < NC3; ++f) dst[f] = (f != F_TH || have_th) ? __ldg(c3src[f] + g) : 0.0;
    };
    // the windows of the first level
    for (int kk = k0 - 1; kk <= k0 + 1; ++kk) stage3(kk);
    for (int kk = k0 - 2; kk <= k0 + 2; ++kk) stage5(kk);
    double cw[3][NC3] = {}, cnext[NC3] = {};  // centre fields at levels kk-1, kk, kk+1; kk+2
    centre(cw[0], k0 - 1);
    centre(cw[1], k0);
    centre(cw[2], k0 + 1);
    cp_async_wait_all();
    __syncthreads();

    const double dt2 = a.dt * a.dt;
    for (int kk = k0; kk < k1; ++kk) {
        if (kk + 1 < k1) {  // the next level's new rows
            stage3(kk + 2);
            stage5(kk + 3);
            centre(cnext, kk + 2);
        }
        if (live) {
            const int k = kk + a.nbz;  // haloed level
            // ring bases of levels kk-1..kk+1 and kk-2..kk+2
            const int b3[3] = {slot3(kk - 1), slot3(kk), slot3(kk + 1)};
            const int b5[5] = {slot5(kk - 2), slot5(kk - 1), slot5(kk), slot5(kk + 1), slot5(kk + 2)};
            const int cxy = (ty + 1) * AHX + tx + 1;
            auto H3 = [&](int f, int di, int dj, int dk) {
                return asm_sm[ASM_H3 + (f * S3 + b3[dk + 1]) * AT + cxy + di + dj * AHX];
            };
            auto H5 = [&](int f, int di, int dj, int dk) {
                return asm_sm[ASM_H5 + (f * S5 + b5[dk + 2]) * AT + cxy + di + dj * AHX];
            };
            auto C3 = [&](int f, int dk) { return cw[dk + 1][f]; };
            auto J = [&](int di, int dj, int dk) { return H3(F_J, di, dj, dk); };
            auto PB = [&](int di, int dj, int dk) { return H3(F_PB, di, dj, dk); };
            auto RB = [&](int di, int dj, int dk) { return H3(F_RB, di, dj, dk); };
            auto RO = [&](int di, int dj, int dk) { return H3(F_RO, di, dj, dk); };
            auto BR = [&](int di, int dj, int dk) { return H3(F_BR, di, dj, dk); };
            auto M13 = [&](int di, int dj, int dk) { return H3(F_M13, di, dj, dk); };
            auto M23 = [&](int di, int dj, int dk) { return H3(F_M23, di, dj, dk); };
            auto M33 = [&](int dk) { return C3(F_M33, dk); };
            auto N2 = [&](int dk) { return C3(F_N2, dk); };
            auto TH = [&](int dk) { return C3(F_TH, dk); };
            // Jacobian-weighted value at the w-level between dk and dk + up (up = +-1):
            // (J(dk+up) X(dk) + J(dk) X(dk+up)) / (J(dk) + J(dk+up)); rj = 1 / (J(dk) + J(dk+up)).
            // Divisions are the kernel's main cost in FP64, so every repeated
            // denominator is inverted once.
            auto zint = [&](double xk, double xn, double jk, double jn, double rj) { return (jn * xk + jk * xn) * rj; };

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
                    return (jh * PB(0, 0, lo) / TH(lo) + jl * PB(0, 0, lo + 1) / TH(lo + 1)) / den;
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

            // ---- the 12 horizontal faces ---------------------------------------
            // dir: 0 = r (i+1/2), 1 = l (i-1/2), 2 = f (j+1/2), 3 = b (j-1/2)
#pragma unroll
            for (int dir = 0; dir < 4; ++dir) {
                const int di = dir == 0 ? 1 : (dir == 1 ? -1 : 0);
                const int dj = dir == 2 ? 1 : (dir == 3 ? -1 : 0);
                const int cn = dir == 0 ? CR : (dir == 1 ? CL : (dir == 2 ? CF : CB));
                const double sgn = (dir == 0 || dir == 2) ? 1.0 : -1.0;  // outward normal
                const double rdh = dir < 2 ? a.rdx : a.rdy;
                const int fm = dir < 2 ? F_M13 : F_M23;
                auto MH = [&](int dk) { return H3(fm, 0, 0, dk); };
                auto MHn = [&](int dk) { return H3(fm, di, dj, dk); };
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

            // ---- the 2 vertical faces ------------------------------------------
            if (!top) {  // G(k + 1/2) (:642-646)
                const double rho_u =
                    zint(RO(0, 0, 0), RO(0, 0, 1), jc, ju, rju) + zint(RB(0, 0, 0), RB(0, 0, 1), jc, ju, rju);
                const double g = jacinv * a.rdz * pudiv * impu / rho_u;
                const double flux = g * zint(pc, PB(0, 0, 1), jc, ju, rju);
                const double w33 = flux * zint(M33(0), M33(1), jc, ju, rju) * a.rdz;
                A[CC][3] += w33;
                A[CC][2] -= w33;
                const double w13 = flux * zint(M13(0, 0, 0), M13(0, 0, 1), jc, ju, rju) * 0.5 * a.rdx;
                const double w23 = flux * zint(M23(0, 0, 0), M23(0, 0, 1), jc, ju, rju) * 0.5 * a.rdy;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int di = q == 0 ? 1 : (q == 1 ? -1 : 0), dj = q == 2 ? 1 : (q == 3 ? -1 : 0);
                    const int cn = q == 0 ? CR : (q == 1 ? CL : (q == 2 ? CF : CB));
                    const double w = (q < 2 ? w13 : w23) * ((q == 0 || q == 2) ? 1.0 : -1.0);
                    const double j0v = J(di, dj, 0), j1v = J(di, dj, 1);
                    const double r01 = w / (j0v + j1v);
                    A[cn][2] += j1v * r01;
                    A[cn][3] += j0v * r01;
                }
            }
            if (!bot) {  // G(k - 1/2) (:649-653)
                const double rho_d =
                    zint(RO(0, 0, 0), RO(0, 0, -1), jc, jd, rjd) + zint(RB(0, 0, 0), RB(0, 0, -1), jc, jd, rjd);
                const double g = -jacinv * a.rdz * pddiv * impd / rho_d;
                const double flux = g * zint(pc, PB(0, 0, -1), jc, jd, rjd);
                const double w33 = flux * zint(M33(0), M33(-1), jc, jd, rjd) * a.rdz;
                A[CC][2] += w33;
                A[CC][1] -= w33;
                const double w13 = flux * zint(M13(0, 0, 0), M13(0, 0, -1), jc, jd, rjd) * 0.5 * a.rdx;
                const double w23 = flux * zint(M23(0, 0, 0), M23(0, 0, -1), jc, jd, rjd) * 0.5 * a.rdy;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int di = q == 0 ? 1 : (q == 1 ? -1 : 0), dj = q == 2 ? 1 : (q == 3 ? -1 : 0);
                    const int cn = q == 0 ? CR : (q == 1 ? CL : (q == 2 ? CF : CB));
                    const double w = (q < 2 ? w13 : w23) * ((q == 0 || q == 2) ? 1.0 : -1.0);
                    const double j0v = J(di, dj, 0), j1v = J(di, dj, -1);
                    const double r01 = w / (j0v + j1v);
                    A[cn][2] += j1v * r01;
                    A[cn][1] += j0v * r01;
                }
            }

            const long long cell = ii + (long long)a.nx * (jj + (long long)a.ny * kk);
            if (a.model == PCF_MODEL_COMPRESSIBLE) {
                const long long hp = (ii + a.nbx) + sy * (jj + a.nby) + sz * k;
                const double dpdpi = 1.0 / (a.gamma - 1.0) * pow(a.rsp / a.pref, 1.0 - a.gamma) *
                                     pow(__ldg(a.p + hp), 2.0 - a.gamma);
                A[CC][2] -= (dpdpi / a.dt) / (a.dt * a.rsp / a.kappa);
            }

            // ---- scaling by 1 / (fcscal fcscal_neighbour), stores, and the
            // difference form B_p = A_p fcscal_nb with the defect sum in plane AC
            const double rfcc = H5(F_RFC, 0, 0, 0);
            double defect = 0.0;
#pragma unroll
            for (int p = 0; p < PCF_NCOEF; ++p) {
                const int c = plane_col(p), z = plane_dk(p) + 2;
                const double v = A[c][z] * rfcc * H5(F_RFC, plane_di(p), plane_dj(p), plane_dk(p));
                const long long o = (long long)p * n + cell;
                if (!PCF_IN(o, (long long)PCF_NCOEF * n, 403)) continue;
                a.coef64[o] = v;
                a.coef32[o] = (float)v;
                if (a.coef16) a.coef16[o] = __float2bfloat16_rn((float)v);
                const double b = v * H5(F_FCH, plane_di(p), plane_dj(p), plane_dk(p));
                defect += b;
                if (p != PCF_AC) a.diff32[o] = (float)b;
            }
            if (PCF_IN(cell, n, 404)) {
                a.diff32[(long long)PCF_AC * n + cell] = (float)defect;
                const double f = H5(F_FCH, 0, 0, 0);
                a.fc64[cell] = f;
                a.rfc32[cell] = (float)(1.0 / f);
            }
        }
#pragma unroll
        for (int f = 0; f < NC3; ++f) {
            cw[0][f] = cw[1][f];
            cw[1][f] = cw[2][f];
            cw[2][f] = cnext[f];
        }
        cp_async_wait_all();
        __syncthreads();
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

int pcf_assemble_chunk_levels() { return pcf::AKC; }

// Assembles the z-chunks [c0, c1) of AKC levels each (c1 < 0: to the top).
int pcf_launch_assemble(pcf_handle *h, double dt, double rf, int damp_h, int c0, int c1) {
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
    a.diff32 = h->coefB32; a.fc64 = h->fc64; a.rfc32 = h->rfc32;
    // the dynamic shared-memory attribute is a per-device setting of the kernel
    static std::atomic<unsigned long long> attr_set{0};
    int dev = 0;
    PCF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return PCF_ENODEVICE;
    if (!(attr_set.load() >> dev & 1ull)) {
        PCF_CUDA_TRY(cudaFuncSetAttribute(pcf::k_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize, pcf::ASM_SMEM));
        attr_set.fetch_or(1ull << dev);
    }
    const int nchunks = (h->d.nz + pcf::AKC - 1) / pcf::AKC;
    if (c1 < 0 || c1 > nchunks) c1 = nchunks;
    if (c0 < 0 || c0 >= c1) return PCF_OK;
    a.kc0 = c0;
    const dim3 grid((unsigned)((h->d.nx + pcf::AX - 1) / pcf::AX), (unsigned)((h->d.ny + pcf::AY - 1) / pcf::AY),
                    (unsigned)(c1 - c0));
    pcf::k_assemble<<<grid, dim3(pcf::AX, pcf::AY), pcf::ASM_SMEM, h->stream>>>(a);
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
