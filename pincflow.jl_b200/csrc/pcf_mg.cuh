// pcf_mg.cuh -- device kernels of the horizontal aggregation multigrid
// preconditioner of the mixed-precision solve (no reference counterpart; the
// reference preconditioner, apply_preconditioner!.jl:40-124, is its smoother).
//
// Hierarchy.  Level l+1 aggregates cx x cy columns of level l (cx, cy in
// {1, 2}); levels keep every vertical level, so each column stays a line of
// the smoother's tridiagonal solves.  With piecewise-constant prolongation
// the Galerkin product of the 25-point operator has the same 25 offsets
// (no xy diagonals arise), so every level runs the same stencil and Thomas
// kernels as the finest one.
//
// Coarse operator.  The assembled operator is symmetrically scaled,
// A = F^-1 A0 F^-1 with F = diag(fcscal) and A0 the unscaled operator whose
// rows sum to (about) zero.  Level l+1 is
//     A_c = Fc^-1 [ (1 / (cx cy)) R A0_l P ]_h Fc^-1,
// R = P^T the aggregate sum, Fc the RMS of fcscal over an aggregate, and
// [.]_h scales every coupling that crosses an aggregate boundary in x by
// 1/cx (in y by 1/cy), moving the removed weight to the (0, 0, dz) entry of
// the same row so that row sums, and with them the null space, are kept.
// The 1/cx factor turns the Galerkin face couplings (cy fine faces per
// coarse face) into those of a re-discretisation on the coarse grid, which
// the pseudo-time smoother is tuned for.  Restriction and prolongation act
// on fcscal-weighted values: b_c = sum(f r) / (cx cy f_c), s += f_c e / f.
#pragma once

#include "pcf_kernels.cuh"

namespace pcf {

// index of offset (dx, dy, dz) in the Tensor order of enum pcf_coef
__host__ __device__ constexpr int coef_index(int dx, int dy, int dz) {
    return dz == 0   ? (dx == -1 ? PCF_AL : dx == 1 ? PCF_AR : dy == -1 ? PCF_AB : dy == 1 ? PCF_AF : PCF_AC)
           : dz == -1 ? (dx == -1 ? PCF_ALD : dx == 1 ? PCF_ARD : dy == -1 ? PCF_ABD : dy == 1 ? PCF_AFD : PCF_AD)
           : dz == 1  ? (dx == -1 ? PCF_ALU : dx == 1 ? PCF_ARU : dy == -1 ? PCF_ABU : dy == 1 ? PCF_AFU : PCF_AU)
           : dz == -2 ? (dx == -1 ? PCF_ALDD : dx == 1 ? PCF_ARDD : dy == -1 ? PCF_ABDD : dy == 1 ? PCF_AFDD : PCF_ADD)
                      : (dx == -1 ? PCF_ALUU : dx == 1 ? PCF_ARUU : dy == -1 ? PCF_ABUU : dy == 1 ? PCF_AFUU : PCF_AUU);
}

__host__ __device__ constexpr int off_x(int p) {
    return (p == PCF_AL || p == PCF_ALD || p == PCF_ALU || p == PCF_ALDD || p == PCF_ALUU)   ? -1
           : (p == PCF_AR || p == PCF_ARD || p == PCF_ARU || p == PCF_ARDD || p == PCF_ARUU) ? 1
                                                                                               : 0;
}
__host__ __device__ constexpr int off_y(int p) {
    return (p == PCF_AB || p == PCF_ABD || p == PCF_ABU || p == PCF_ABDD || p == PCF_ABUU)   ? -1
           : (p == PCF_AF || p == PCF_AFD || p == PCF_AFU || p == PCF_AFDD || p == PCF_AFUU) ? 1
                                                                                               : 0;
}
__host__ __device__ constexpr int off_z(int p) {
    return (p == PCF_AD || p == PCF_ALD || p == PCF_ARD || p == PCF_ABD || p == PCF_AFD)       ? -1
           : (p == PCF_AU || p == PCF_ALU || p == PCF_ARU || p == PCF_ABU || p == PCF_AFU)     ? 1
           : (p == PCF_ADD || p == PCF_ALDD || p == PCF_ARDD || p == PCF_ABDD || p == PCF_AFDD) ? -2
           : (p == PCF_AUU || p == PCF_ALUU || p == PCF_ARUU || p == PCF_ABUU || p == PCF_AFUU) ? 2
                                                                                                 : 0;
}

// floor((a + d) / c) for c in {1, 2} and a + d in [-1, 2]
__host__ __device__ constexpr int agg_off(int a, int d, int c) { return c == 1 ? d : (a + d < 0 ? -1 : (a + d) / 2); }

// fc_c = sqrt(mean over the aggregate of fc^2)
template <typename TF, int CX, int CY>
__global__ void __launch_bounds__(256) k_mg_fc(const TF *__restrict__ fc, int nx, int ny, int nz,
                                                float *__restrict__ fcc) {
    const int NX = nx / CX, NY = ny / CY;
    const long long nc = (long long)NX * NY * nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nc; q += (long long)gridDim.x * blockDim.x) {
        const unsigned qu = (unsigned)q, ux = (unsigned)NX, uy = (unsigned)NY;  // n < 2^31
        const int I = (int)(qu % ux), J = (int)((qu / ux) % uy), k = (int)(qu / (ux * uy));
        double acc = 0.0;
#pragma unroll
        for (int b = 0; b < CY; ++b)
#pragma unroll
            for (int a = 0; a < CX; ++a) {
                const double f = (double)fc[(CX * I + a) + (long long)nx * ((CY * J + b) + (long long)ny * k)];
                acc += f * f;
            }
        fcc[q] = (float)sqrt(acc / (CX * CY));
    }
}

// Coarse operator of level l+1 from level l (see the file header).  The
// aggregation is horizontal, so the fine couplings at vertical offset dz
// feed only the coarse couplings at dz (re-discretisation moves included):
// one thread per coarse cell and dz group (blockIdx.y = dz + 2) sums the 5
// planes of its group, in the plane order of the Tensor struct.  TI is the
// type of the finer level's planes and fcscal (double on the finest level,
// float below).
template <typename TI, int CX, int CY, int DZ>
__device__ __forceinline__ void coarsen_group(const TI *__restrict__ coef, const TI *__restrict__ fc, int nx, int ny,
                                              int nz, const float *__restrict__ fcc, float *__restrict__ out,
                                              __nv_bfloat16 *__restrict__ out16, long long q, int I, int J, int k) {
    const int NX = nx / CX, NY = ny / CY;
    const long long n = (long long)nx * ny * nz, nc = (long long)NX * NY * nz;
    if (k + DZ < 0 || k + DZ >= nz) {  // couplings to a zero z-ghost
#pragma unroll
        for (int p = 0; p < PCF_NCOEF; ++p)
            if (off_z(p) == DZ) {
                out[(long long)p * nc + q] = 0.0f;
                if (out16) out16[(long long)p * nc + q] = __float2bfloat16_rn(0.0f);
            }
        return;
    }
    double acc[PCF_NCOEF];
#pragma unroll
    for (int p = 0; p < PCF_NCOEF; ++p) acc[p] = 0.0;
#pragma unroll
    for (int b = 0; b < CY; ++b)
#pragma unroll
        for (int a = 0; a < CX; ++a) {
            const int i = CX * I + a, j = CY * J + b;
            const long long c = i + (long long)nx * (j + (long long)ny * k);
            const double fcv = (double)fc[c];
#pragma unroll
            for (int p = 0; p < PCF_NCOEF; ++p) {
                if (off_z(p) != DZ) continue;
                const int dx = off_x(p), dy = off_y(p);
                const long long t = wrap1(i + dx, nx) + (long long)nx * (wrap1(j + dy, ny) + (long long)ny * (k + DZ));
                const double a0 = fcv * (double)coef[(long long)p * n + c] * (double)fc[t];
                acc[coef_index(agg_off(a, dx, CX), agg_off(b, dy, CY), DZ)] += a0;
            }
        }
    // re-discretisation scaling of the couplings across aggregate faces
#pragma unroll
    for (int p = 0; p < PCF_NCOEF; ++p) {
        if (off_z(p) != DZ) continue;
        const int dx = off_x(p), dy = off_y(p);
        if (dx == 0 && dy == 0) continue;
        const double keep = dx != 0 ? 1.0 / CX : 1.0 / CY;
        const double moved = (1.0 - keep) * acc[p];
        acc[p] -= moved;
        acc[coef_index(0, 0, DZ)] += moved;
    }
    const double fcI = (double)fcc[q];
#pragma unroll
    for (int p = 0; p < PCF_NCOEF; ++p) {
        if (off_z(p) != DZ) continue;
        const long long t = wrap1(I + off_x(p), NX) + (long long)NX * (wrap1(J + off_y(p), NY) + (long long)NY * (k + DZ));
        const float v = (float)(acc[p] / ((double)(CX * CY) * fcI * (double)fcc[t]));
        out[(long long)p * nc + q] = v;
        if (out16) out16[(long long)p * nc + q] = __float2bfloat16_rn(v);
    }
}

template <typename TI, int CX, int CY>
__global__ void __launch_bounds__(128) k_mg_coarsen(const TI *__restrict__ coef, const TI *__restrict__ fc, int nx,
                                                    int ny, int nz, const float *__restrict__ fcc,
                                                    float *__restrict__ out, __nv_bfloat16 *__restrict__ out16) {
    const int NX = nx / CX, NY = ny / CY;
    const long long nc = (long long)NX * NY * nz;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nc) return;
    const unsigned qu = (unsigned)q, ux = (unsigned)NX, uy = (unsigned)NY;  // n < 2^31
    const int I = (int)(qu % ux), J = (int)((qu / ux) % uy), k = (int)(qu / (ux * uy));
    switch (blockIdx.y) {
        case 0: coarsen_group<TI, CX, CY, -2>(coef, fc, nx, ny, nz, fcc, out, out16, q, I, J, k); break;
        case 1: coarsen_group<TI, CX, CY, -1>(coef, fc, nx, ny, nz, fcc, out, out16, q, I, J, k); break;
        case 2: coarsen_group<TI, CX, CY, 0>(coef, fc, nx, ny, nz, fcc, out, out16, q, I, J, k); break;
        case 3: coarsen_group<TI, CX, CY, 1>(coef, fc, nx, ny, nz, fcc, out, out16, q, I, J, k); break;
        default: coarsen_group<TI, CX, CY, 2>(coef, fc, nx, ny, nz, fcc, out, out16, q, I, J, k); break;
    }
}

// Thomas pivots P, M, Q of a level (as k_factors, from FP32 planes; the
// loads of each block of 8 levels are issued together ahead of the serial
// recurrence).
__global__ void __launch_bounds__(128) k_mg_factors(int plane, int nz, long long n, double deta,
                                                    const float *__restrict__ coef, float *__restrict__ fac) {
    constexpr int CH = 8;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= plane) return;
    const float *ac = coef + (long long)PCF_AC * n, *ad = coef + (long long)PCF_AD * n,
                *au = coef + (long long)PCF_AU * n;
    double qprev = 0.0;
    for (int k0 = 0; k0 < nz; k0 += CH) {
        float vc[CH], vd[CH], vu[CH];
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int k = k0 + q;
            const long long o = col + (long long)plane * (k < nz ? k : 0);
            vc[q] = ac[o];
            vd[q] = ad[o];
            vu[q] = au[o];
        }
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int k = k0 + q;
            if (k >= nz) break;
            const long long o = col + (long long)plane * k;
            const double piv = k == 0 ? 1.0 / (1.0 - deta * vc[q]) : 1.0 / (1.0 - deta * vc[q] - deta * vd[q] * qprev);
            const double m = k == 0 ? 0.0 : deta * vd[q] * piv;
            const double qv = deta * vu[q] * piv;
            fac[o] = (float)piv;
            fac[n + o] = (float)m;
            fac[2 * n + o] = (float)qv;
            qprev = qv;
        }
    }
}

// b_c = sum over the aggregate of (f r) / (cx cy f_c); one thread per
// coarse point of an (NX, NY, nz) grid of blocks (32 x 8 threads in x-y, one
// level per grid row).
template <typename TF, int CX, int CY>
__global__ void __launch_bounds__(256) k_mg_restrict(const float *__restrict__ r, const TF *__restrict__ fc, int nx,
                                                      int ny, int nz, const float *__restrict__ fcc,
                                                      float *__restrict__ bc, const KrylovScalars *guard) {
    if (krylov_done(guard)) return;
    const int NX = nx / CX, NY = ny / CY;
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (I >= NX || J >= NY) return;
    const long long q = I + (long long)NX * (J + (long long)NY * k);
    float acc = 0.0f;
#pragma unroll
    for (int b = 0; b < CY; ++b)
#pragma unroll
        for (int a = 0; a < CX; ++a) {
            const long long c = (CX * I + a) + (long long)nx * ((CY * J + b) + (long long)ny * k);
            if (PCF_IN(c, (long long)nx * ny * nz, 301)) acc += (float)fc[c] * r[c];
        }
    if (PCF_IN(q, (long long)NX * NY * nz, 302)) bc[q] = acc / ((float)(CX * CY) * fcc[q]);
}

// s += f_c e / f (piecewise-constant prolongation of the coarse correction);
// one thread per fine point, 64 x 4 threads in x-y, one level per grid row.
template <typename TF, int CX, int CY>
__global__ void __launch_bounds__(256) k_mg_prolong(const float *__restrict__ e, const float *__restrict__ fcc,
                                                     const TF *__restrict__ fc, int nx, int ny, int nz, float *s,
                                                     const KrylovScalars *guard) {
    if (krylov_done(guard)) return;
    const int NX = nx / CX, NY = ny / CY;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= nx || j >= ny) return;
    const long long c = i + (long long)nx * (j + (long long)ny * k);
    const long long q = i / CX + (long long)NX * (j / CY + (long long)NY * k);
    if (PCF_IN(c, (long long)nx * ny * nz, 303) && PCF_IN(q, (long long)NX * NY * nz, 304))
        s[c] += fcc[q] * e[q] / (float)fc[c];
}

// k_mg_restrict for four consecutive fine x cells per thread (4 / CX coarse
// points) with 128-bit loads of r and fc (nx % 4 == 0); the sums run in the
// order of k_mg_restrict.
template <int CX, int CY>
__global__ void __launch_bounds__(256) k_mg_restrict4(const float *__restrict__ r, const float *__restrict__ fc,
                                                       int nx, int ny, int nz, const float *__restrict__ fcc,
                                                       float *__restrict__ bc, const KrylovScalars *guard) {
    if (krylov_done(guard)) return;
    const int NX = nx / CX, NY = ny / CY;
    const int i4 = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (4 * i4 >= nx || J >= NY) return;
    constexpr int NC = 4 / CX;  // coarse points of this thread
    float acc[NC];
#pragma unroll
    for (int m = 0; m < NC; ++m) acc[m] = 0.0f;
#pragma unroll
    for (int b = 0; b < CY; ++b) {
        const long long c = 4LL * i4 + (long long)nx * ((CY * J + b) + (long long)ny * k);
        if (!PCF_IN(c, (long long)nx * ny * nz - 3, 305)) continue;
        const float4 rv = *reinterpret_cast<const float4 *>(r + c);
        const float4 fv = *reinterpret_cast<const float4 *>(fc + c);
        const float pr[4] = {fv.x * rv.x, fv.y * rv.y, fv.z * rv.z, fv.w * rv.w};
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[a / CX] += pr[a];
    }
    const long long q = (long long)(4 / CX) * i4 + (long long)NX * (J + (long long)NY * k);
#pragma unroll
    for (int m = 0; m < NC; ++m)
        if (PCF_IN(q + m, (long long)NX * NY * nz, 306)) bc[q + m] = acc[m] / ((float)(CX * CY) * fcc[q + m]);
}

// k_mg_prolong on four consecutive x cells per thread with 128-bit loads
// and stores of s and fc (nx % 4 == 0, so every row starts 16-byte aligned).
template <int CX, int CY>
__global__ void __launch_bounds__(256) k_mg_prolong4(const float *__restrict__ e, const float *__restrict__ fcc,
                                                      const float *__restrict__ fc, int nx, int ny, int nz, float *s,
                                                      const KrylovScalars *guard) {
    if (krylov_done(guard)) return;
    const int NX = nx / CX, NY = ny / CY;
    const int i4 = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (4 * i4 >= nx || j >= ny) return;
    const long long c = 4LL * i4 + (long long)nx * (j + (long long)ny * k);
    const long long qrow = (long long)NX * (j / CY + (long long)NY * k);
    if (!PCF_IN(c, (long long)nx * ny * nz - 3, 307) || !PCF_IN(qrow + (4 * i4 + 3) / CX, (long long)NX * NY * nz, 308))
        return;
    const float4 f = *reinterpret_cast<const float4 *>(fc + c);
    float4 v = *reinterpret_cast<const float4 *>(s + c);
    const int i = 4 * i4;
    const long long q0 = qrow + i / CX, q1 = qrow + (i + 1) / CX, q2 = qrow + (i + 2) / CX, q3 = qrow + (i + 3) / CX;
    v.x += fcc[q0] * e[q0] / f.x;
    v.y += fcc[q1] * e[q1] / f.y;
    v.z += fcc[q2] * e[q2] / f.z;
    v.w += fcc[q3] * e[q3] / f.w;
    *reinterpret_cast<float4 *>(s + c) = v;
}

// ===================================== the coarse V-cycle in one launch --
//
// The coarse levels of the V-cycle (from the first level with at most
// kCoarseColumns columns down to the coarsest) are latency-bound: each of
// their ~40 kernels per cycle moves a few MB.  k_mg_coarse runs that whole
// part of the cycle -- the same steps as the per-kernel path (column solve
// from zero, residual, restriction, ..., coarsest smoothing, prolongation,
// pseudo-time step, column solve) -- as phases of ONE thread-block cluster
// of kCoarseCluster CTAs, separated by the hardware cluster barrier
// (barrier.cluster with release / acquire semantics: every global write of a
// phase is visible to the whole cluster in the next).  The coarse levels'
// data (a few MB) stay in L2.  Phases are cell-parallel (stencils and grid
// transfers, the stencil's terms summed in k_stencil's order) or
// column-parallel (the Thomas sweeps: one warp per column, each lane a run of
// at most 8 levels, the runs' affine maps chained by warp-shuffle scans).
constexpr int kCoarseColumns = 1024;   // levels of at most 32 x 32 columns
constexpr int kCoarseMaxLevels = 12;
constexpr int kCoarseThreads = 256;
constexpr int kCoarseCluster = 16;     // CTAs of the cluster (the non-portable maximum; 8 where 16 is refused)

struct CoarseLevel {
    int nx, ny, nz, cx, cy;  // cx, cy: the aggregation from the next finer level
    long long plane, n;
    float deta;
    const float *coef, *fac, *fc;
    float *s, *t, *b;
};

struct CoarseArgs {
    CoarseLevel lv[kCoarseMaxLevels];
    int nlev;          // lv[0] is the first level of the coarse part
    int coarse_iters;  // smoothing steps on the coarsest level
    const KrylovScalars *guard;
};

// Barrier of the whole cluster (every thread of every CTA arrives; the CTAs
// of a cluster are co-scheduled, so it needs no bound).
__device__ __forceinline__ void coarse_barrier() {
    __syncwarp();  // the .aligned form wants the whole warp at the same instruction
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Column solves of level L, one warp per column: mode TH_B solves from -deta b
// into out, TH_T solves t in place.  Forward y_k = rhs_k P_k + M_k y_(k-1),
// back x_k = y_k + Q_k x_(k+1) (x_(nz-1) = y_(nz-1)), as k_thomas.
template <int MODE>
__device__ void coarse_thomas(const CoarseLevel &L, const float *in, float *out) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int R = (L.nz + 31) / 32;  // levels per lane, at most 8 (nz <= 256)
    const float *P = L.fac, *M = L.fac + L.n, *Q = L.fac + 2 * L.n;
    for (long long col = warp; col < L.plane; col += nwarps) {
        float yv[8], pp[8], mm[8], qq[8];
        const int k0 = lane * R;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = k0 + q;
            const bool on = q < R && k < L.nz;
            const long long o = col + L.plane * (on ? k : 0);
            const float v = on ? in[o] : 0.f;
            yv[q] = MODE == TH_B ? -L.deta * v : v;
            pp[q] = on ? P[o] : 0.f;
            mm[q] = on ? M[o] : 1.f;
            qq[q] = (on && k != L.nz - 1) ? Q[o] : (on ? 0.f : 1.f);
        }
        // forward: this lane's run as y_out = A + B y_in, then an inclusive scan over lanes
        float A = 0.f, B = 1.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            yv[q] *= pp[q];
            A = mm[q] * A + yv[q];
            B = mm[q] * B;
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const float a2 = __shfl_up_sync(0xffffffffu, A, off), b2 = __shfl_up_sync(0xffffffffu, B, off);
            if (lane >= off) {
                A = A + B * a2;
                B = B * b2;
            }
        }
        float y = __shfl_up_sync(0xffffffffu, A, 1);
        if (lane == 0) y = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            y = mm[q] * y + yv[q];
            yv[q] = (q < R && k0 + q < L.nz) ? y : 0.f;  // levels past the run: identity maps below
        }
        // back: this lane's run as x_start = C + D x_in, then a reverse inclusive scan
        float C = 0.f, D = 1.f;
#pragma unroll
        for (int q = 7; q >= 0; --q) {
            C = yv[q] + qq[q] * C;
            D = qq[q] * D;
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const float c2 = __shfl_down_sync(0xffffffffu, C, off), d2 = __shfl_down_sync(0xffffffffu, D, off);
            if (lane + off < 32) {
                C = C + D * c2;
                D = D * d2;
            }
        }
        float x = __shfl_down_sync(0xffffffffu, C, 1);
        if (lane == 31) x = 0.f;
#pragma unroll
        for (int q = 7; q >= 0; --q) {
            const int k = k0 + q;
            x = yv[q] + qq[q] * x;
            if (q < R && k < L.nz) out[col + L.plane * k] = x;
        }
    }
}

// Stencil of level L on s (periodic in x and y, zero beyond the walls), cell
// parallel.  HORIZ: out = s + deta (L_h s - b); otherwise out = b - A s.  The
// terms are summed in the order of k_stencil.
template <bool HORIZ>
__device__ void coarse_stencil(const CoarseLevel &L, const float *s, const float *b, float *out) {
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const long long n = L.n, plane = L.plane;
    // 32-bit index arithmetic: pcf_create admits fewer than 2^31 cells
    for (unsigned c = blockIdx.x * blockDim.x + threadIdx.x; c < (unsigned)n; c += gridDim.x * blockDim.x) {
        const unsigned cx = c % (unsigned)nx, rest = c / (unsigned)nx;
        const int i = (int)cx, j = (int)(rest % (unsigned)ny), k = (int)(rest / (unsigned)ny);
        const int il = i == 0 ? nx - 1 : i - 1, ir = i == nx - 1 ? 0 : i + 1;
        const int jb = j == 0 ? ny - 1 : j - 1, jf = j == ny - 1 ? 0 : j + 1;
        auto S = [&](int ii, int jj, int kk) -> float {
            return (kk < 0 || kk >= nz) ? 0.f : s[ii + (long long)nx * (jj + (long long)ny * kk)];
        };
        const float *A = L.coef + c;
        auto K = [&](int p) { return A[(long long)p * n]; };
        float acc;
        if (HORIZ) {
            acc = K(PCF_AL) * S(il, j, k);
        } else {
            acc = K(PCF_AC) * S(i, j, k);
            acc = fmaf(K(PCF_AD), S(i, j, k - 1), acc);
            acc = fmaf(K(PCF_AU), S(i, j, k + 1), acc);
            acc = fmaf(K(PCF_AL), S(il, j, k), acc);
        }
        acc = fmaf(K(PCF_AR), S(ir, j, k), acc);
        acc = fmaf(K(PCF_AB), S(i, jb, k), acc);
        acc = fmaf(K(PCF_AF), S(i, jf, k), acc);
        acc = fmaf(K(PCF_ALD), S(il, j, k - 1), acc);
        acc = fmaf(K(PCF_ALU), S(il, j, k + 1), acc);
        acc = fmaf(K(PCF_ARD), S(ir, j, k - 1), acc);
        acc = fmaf(K(PCF_ARU), S(ir, j, k + 1), acc);
        acc = fmaf(K(PCF_ABD), S(i, jb, k - 1), acc);
        acc = fmaf(K(PCF_ABU), S(i, jb, k + 1), acc);
        acc = fmaf(K(PCF_AFD), S(i, jf, k - 1), acc);
        acc = fmaf(K(PCF_AFU), S(i, jf, k + 1), acc);
        acc = fmaf(K(PCF_ADD), S(i, j, k - 2), acc);
        acc = fmaf(K(PCF_AUU), S(i, j, k + 2), acc);
        acc = fmaf(K(PCF_ALDD), S(il, j, k - 2), acc);
        acc = fmaf(K(PCF_ALUU), S(il, j, k + 2), acc);
        acc = fmaf(K(PCF_ARDD), S(ir, j, k - 2), acc);
        acc = fmaf(K(PCF_ARUU), S(ir, j, k + 2), acc);
        acc = fmaf(K(PCF_ABDD), S(i, jb, k - 2), acc);
        acc = fmaf(K(PCF_ABUU), S(i, jb, k + 2), acc);
        acc = fmaf(K(PCF_AFDD), S(i, jf, k - 2), acc);
        acc = fmaf(K(PCF_AFUU), S(i, jf, k + 2), acc);
        out[c] = HORIZ ? S(i, j, k) + L.deta * (acc - b[c]) : b[c] - acc;
    }
}

// b of level C from the residual r of the finer level F (k_mg_restrict's sums)
__device__ void coarse_restrict(const CoarseLevel &F, const CoarseLevel &C, const float *r) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < C.n;
         q += (long long)gridDim.x * blockDim.x) {
        const int I = (int)(q % C.nx), J = (int)((q / C.nx) % C.ny), k = (int)(q / C.plane);
        float acc = 0.f;
        for (int bb = 0; bb < C.cy; ++bb)
            for (int aa = 0; aa < C.cx; ++aa) {
                const long long c = (C.cx * I + aa) + (long long)F.nx * ((C.cy * J + bb) + (long long)F.ny * k);
                acc += F.fc[c] * r[c];
            }
        C.b[q] = acc / ((float)(C.cx * C.cy) * C.fc[q]);
    }
}

// s of level F += f_c e / f (k_mg_prolong)
__device__ void coarse_prolong(const CoarseLevel &F, const CoarseLevel &C, const float *e) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < F.n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % F.nx), j = (int)((c / F.nx) % F.ny), k = (int)(c / F.plane);
        const long long q = i / C.cx + (long long)C.nx * (j / C.cy + (long long)C.ny * k);
        F.s[c] += C.fc[q] * e[q] / F.fc[c];
    }
}

__global__ void __launch_bounds__(kCoarseThreads) k_mg_coarse(const __grid_constant__ CoarseArgs a) {
    // the guard is written by earlier kernels only: every CTA takes the same branch
    if (krylov_done(a.guard)) return;
    const int top = a.nlev - 1;
    // descent: column solve from zero, residual, restriction
    for (int l = 0; l < top; ++l) {
        const CoarseLevel &L = a.lv[l];
        coarse_thomas<TH_B>(L, L.b, L.s);
        coarse_barrier();
        coarse_stencil<false>(L, L.s, L.b, L.t);
        coarse_barrier();
        coarse_restrict(L, a.lv[l + 1], L.t);
        coarse_barrier();
    }
    // the coarsest level: a column solve from zero, then pseudo-time steps
    const CoarseLevel &Z = a.lv[top];
    coarse_thomas<TH_B>(Z, Z.b, Z.s);
    coarse_barrier();
    float *cur = Z.s, *oth = Z.t;
    for (int q = 1; q < a.coarse_iters; ++q) {
        coarse_stencil<true>(Z, cur, Z.b, oth);
        coarse_barrier();
        coarse_thomas<TH_T>(Z, oth, oth);
        coarse_barrier();
        float *w = cur;
        cur = oth;
        oth = w;
    }
    // ascent: prolongation, pseudo-time step, column solve
    const float *e = cur;
    for (int l = top - 1; l >= 0; --l) {
        const CoarseLevel &L = a.lv[l];
        coarse_prolong(L, a.lv[l + 1], e);
        coarse_barrier();
        coarse_stencil<true>(L, L.s, L.b, L.t);
        coarse_barrier();
        coarse_thomas<TH_T>(L, L.t, L.t);
        if (l > 0) coarse_barrier();
        e = L.t;
    }
}

}  // namespace pcf
