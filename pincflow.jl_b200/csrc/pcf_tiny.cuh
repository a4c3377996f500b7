// pcf_tiny.cuh -- the whole reference BiCGSTAB (apply_bicgstab!.jl:24-150
// with apply_preconditioner!.jl:40-124 and apply_operator!.jl:48-479) in ONE
// thread block, FP64, for grids small enough to keep every Krylov vector in
// shared memory.  On such grids (the periodic hill is 40 x 1 x 40) each of
// the multi-kernel solver's ~40 launches per iteration moves a few kB, so the
// solve is bound by launch and dependency latency; here an iteration is a
// sequence of block-wide phases separated by __syncthreads, with the
// coefficient planes read from L2.  The arithmetic and the order of the
// steps are those of the multi-kernel FP64 path; global sums are per-thread
// partials (cells in a fixed stride order) reduced by block_sum, so the
// result is deterministic.
#pragma once

#include "pcf_kernels.cuh"

namespace pcf {

constexpr int kTinyMaxCells = 2048;  // 9 FP64 vectors + 3 pivot planes in shared memory: 192 KB
constexpr int kTinyVectors = 12;
constexpr int kTinyThreads = 512;

struct TinyArgs {
    int nx, ny, nz, n, plane;
    const double *coef;  // 25 planes
    const double *fac;   // P, M, Q for deta
    const double *b;
    double *x;           // the solution (after the final x <- M x)
    double tol;
    int maxit, precond, pc_iters;
    double deta;
    KrylovScalars *scal;  // iter, converged, status, res, b_norm
    double *hist;
    int hist_cap;
};

__device__ __forceinline__ double tiny_apply_at(const TinyArgs &a, const double *in, int c, bool horiz) {
    const int i = c % a.nx, j = (c / a.nx) % a.ny, k = c / a.plane;
    const int ip = i + 1 == a.nx ? 0 : i + 1, im = i == 0 ? a.nx - 1 : i - 1;
    const int jp = j + 1 == a.ny ? 0 : j + 1, jm = j == 0 ? a.ny - 1 : j - 1;
    auto S = [&](int ii, int jj, int kk) -> double {
        return (kk < 0 || kk >= a.nz) ? 0.0 : in[ii + a.nx * (jj + a.ny * kk)];
    };
    auto C = [&](int p) { return __ldg(a.coef + (long long)p * a.n + c); };
    double v = 0.0;
    if (!horiz) v = C(PCF_AC) * S(i, j, k) + C(PCF_AD) * S(i, j, k - 1) + C(PCF_AU) * S(i, j, k + 1);
    v += C(PCF_AL) * S(im, j, k) + C(PCF_AR) * S(ip, j, k) + C(PCF_AB) * S(i, jm, k) + C(PCF_AF) * S(i, jp, k);
    v += C(PCF_ALD) * S(im, j, k - 1) + C(PCF_ALU) * S(im, j, k + 1) + C(PCF_ARD) * S(ip, j, k - 1) +
         C(PCF_ARU) * S(ip, j, k + 1) + C(PCF_ABD) * S(i, jm, k - 1) + C(PCF_ABU) * S(i, jm, k + 1) +
         C(PCF_AFD) * S(i, jp, k - 1) + C(PCF_AFU) * S(i, jp, k + 1);
    v += C(PCF_ADD) * S(i, j, k - 2) + C(PCF_AUU) * S(i, j, k + 2) + C(PCF_ALDD) * S(im, j, k - 2) +
         C(PCF_ALUU) * S(im, j, k + 2) + C(PCF_ARDD) * S(ip, j, k - 2) + C(PCF_ARUU) * S(ip, j, k + 2) +
         C(PCF_ABDD) * S(i, jm, k - 2) + C(PCF_ABUU) * S(i, jm, k + 2) + C(PCF_AFDD) * S(i, jp, k - 2) +
         C(PCF_AFUU) * S(i, jp, k + 2);
    return v;
}

// out = A in (Total) over the block
__device__ __forceinline__ void tiny_apply(const TinyArgs &a, const double *in, double *out) {
    for (int c = threadIdx.x; c < a.n; c += blockDim.x) out[c] = tiny_apply_at(a, in, c, false);
    __syncthreads();
}

// out = M(in): pc_iters pseudo-time steps from zero, each a Thomas solve per
// column (one thread per column) after rhs = s + deta (L_h s - in).  The
// pivots P, M, Q are staged in shared memory (fac): each sweep is a chain of
// nz dependent steps, which from L2 would cost a round trip per level.
__device__ void tiny_precond(const TinyArgs &a, const double *fac, const double *in, double *out, double *tmp) {
    const double *P = fac, *M = fac + a.n, *Q = fac + 2 * a.n;
    for (int it = 0; it < a.pc_iters; ++it) {
        if (it == 0) {
            for (int c = threadIdx.x; c < a.n; c += blockDim.x) tmp[c] = -a.deta * in[c];
        } else {
            for (int c = threadIdx.x; c < a.n; c += blockDim.x)
                tmp[c] = out[c] + a.deta * (tiny_apply_at(a, out, c, true) - in[c]);
        }
        __syncthreads();
        for (int col = threadIdx.x; col < a.plane; col += blockDim.x) {
            double y = 0.0;
            for (int k = 0; k < a.nz; ++k) {
                const int o = col + a.plane * k;
                y = tmp[o] * P[o] + M[o] * y;
                out[o] = y;
            }
            double xs = y;
            for (int k = a.nz - 2; k >= 0; --k) {
                const int o = col + a.plane * k;
                xs = out[o] + Q[o] * xs;
                out[o] = xs;
            }
        }
        __syncthreads();
    }
}

// block-wide sums of up to two per-thread partials, returned to every thread
template <int NV>
__device__ __forceinline__ void tiny_sum(double (&v)[NV], double *sh, double *bc) {
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) bc[q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = bc[q];
    __syncthreads();
}

__global__ void __launch_bounds__(kTinyThreads) k_tiny_bicgstab(TinyArgs a) {
    extern __shared__ __align__(16) double tsm[];
    __shared__ double sh[64];
    __shared__ double bc[2];
    const int n = a.n;
    double *x = tsm, *r = x + n, *r0 = r + n, *p = r0 + n, *v = p + n, *s = v + n, *t = s + n, *z = t + n,
           *w = z + n, *fac = w + n;
    const int tid = threadIdx.x;
    if (a.precond)
        for (int c = tid; c < 3 * n; c += blockDim.x) fac[c] = __ldg(a.fac + c);
    // apply_bicgstab!.jl:44-67: x = 0, r = r0 = p = b
    double acc[1] = {0.0};
    for (int c = tid; c < n; c += blockDim.x) {
        const double bv = a.b[c];
        x[c] = 0.0;
        r[c] = bv;
        r0[c] = bv;
        p[c] = bv;
        acc[0] += bv * bv;
    }
    __syncthreads();
    tiny_sum<1>(acc, sh, bc);
    const double b_norm = sqrt(acc[0] / n);
    double res = b_norm, rho = acc[0];
    int iter = 0, converged = 0, status = PCF_OK;
    if (!isfinite(b_norm)) status = PCF_ENONFINITE;
    else if (b_norm == 0.0 || res / b_norm <= a.tol) converged = 1;
    while (status == PCF_OK && !converged && iter < a.maxit) {
        iter += 1;
        // v = A M p; alpha = rho / <v, r0>   (:84-96)
        const double *zp = p;
        if (a.precond) {
            tiny_precond(a, fac, p, z, w);
            zp = z;
        }
        tiny_apply(a, zp, v);
        double d1[1] = {0.0};
        for (int c = tid; c < n; c += blockDim.x) d1[0] += v[c] * r0[c];
        tiny_sum<1>(d1, sh, bc);
        const double alpha = rho / d1[0];
        if (!isfinite(alpha)) {
            status = PCF_EBREAKDOWN;
            break;
        }
        for (int c = tid; c < n; c += blockDim.x) s[c] = r[c] - alpha * v[c];
        __syncthreads();
        // t = A M s; omega = <t, s> / <t, t>   (:98-109)
        const double *zs = s;
        if (a.precond) {
            tiny_precond(a, fac, s, z, w);
            zs = z;
        }
        tiny_apply(a, zs, t);
        double d2[2] = {0.0, 0.0};
        for (int c = tid; c < n; c += blockDim.x) {
            d2[0] += t[c] * s[c];
            d2[1] += t[c] * t[c];
        }
        tiny_sum<2>(d2, sh, bc);
        const double omega = d2[0] / d2[1];
        if (!isfinite(omega) || omega == 0.0) {
            status = PCF_EBREAKDOWN;
            break;
        }
        // x += alpha p + omega s; r = s - omega t; residual test, beta   (:110-143)
        double d3[2] = {0.0, 0.0};
        for (int c = tid; c < n; c += blockDim.x) {
            x[c] += alpha * p[c] + omega * s[c];
            const double rv = s[c] - omega * t[c];
            r[c] = rv;
            d3[0] += rv * rv;
            d3[1] += rv * r0[c];
        }
        tiny_sum<2>(d3, sh, bc);
        res = sqrt(d3[0] / n);
        if (tid == 0 && a.hist && iter - 1 < a.hist_cap) a.hist[iter - 1] = res / b_norm;
        if (!isfinite(res)) {
            status = PCF_ENONFINITE;
            break;
        }
        if (res / b_norm <= a.tol) {
            converged = 1;
            break;
        }
        const double beta = alpha / omega * d3[1] / rho;
        rho = d3[1];
        if (!isfinite(beta)) {
            status = PCF_EBREAKDOWN;
            break;
        }
        for (int c = tid; c < n; c += blockDim.x) p[c] = r[c] + beta * (p[c] - omega * v[c]);
        __syncthreads();
    }
    // solution = M(solution) on convergence (:132-135)
    const double *xf = x;
    if (converged && iter > 0 && a.precond) {
        tiny_precond(a, fac, x, z, w);
        xf = z;
    }
    for (int c = tid; c < n; c += blockDim.x) a.x[c] = xf[c];
    if (tid == 0) {
        KrylovScalars *k = a.scal;
        k->iter = iter;
        k->converged = converged;
        k->status = status;
        k->res = res;
        k->b_norm = b_norm;
        k->done = 1;
    }
}

}  // namespace pcf
