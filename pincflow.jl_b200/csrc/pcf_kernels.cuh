// pcf_kernels.cuh -- device kernels of the Krylov loop, templated on the
// working precision T (double for the reference path and the true residual,
// float for the inner iterations of the mixed-precision solve).
//
//   k_stencil   25-point operator apply (apply_operator!.jl:48-479), Total or
//               Horizontal, with fused epilogues (dot products for BiCGSTAB,
//               the preconditioner's pseudo-time step, the true residual)
//   k_thomas    the preconditioner's per-column tridiagonal solve
//               (apply_preconditioner!.jl:73-111) with fused input forming
//   k_update    BiCGSTAB solution / residual updates with fused dots
//               (apply_bicgstab!.jl:110-123)
// All global sums accumulate in FP64 and are reduced deterministically: one
// partial per block, then the last block to finish sums the partials in block
// order and runs the scalar step of the iteration (KrylovScalars).
#pragma once

#include "pcf_internal.cuh"

namespace pcf {

// ---------------------------------------------------------------- helpers --

template <typename T, int V>
struct Vec;
template <>
struct Vec<float, 4> {
    using type = float4;
};
template <>
struct Vec<float, 2> {
    using type = float2;
};
template <>
struct Vec<float, 1> {
    using type = float;
};
template <>
struct Vec<double, 2> {
    using type = double2;
};
template <>
struct Vec<double, 1> {
    using type = double;
};

template <typename T, int V>
__device__ __forceinline__ void load_vec(const T *__restrict__ p, T (&v)[V]) {
    using VT = typename Vec<T, V>::type;
    const VT x = __ldg(reinterpret_cast<const VT *>(p));
    const T *e = reinterpret_cast<const T *>(&x);
#pragma unroll
    for (int q = 0; q < V; ++q) v[q] = e[q];
}

// two BF16 values packed in 4 bytes, widened to FP32
__device__ __forceinline__ void unpack_bf16x2(unsigned x, float (&v)[2]) {
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&x));
    v[0] = a.x; v[1] = a.y;
}

// four BF16 values packed in 8 bytes, widened to FP32
__device__ __forceinline__ void unpack_bf16x4(uint2 x, float (&v)[4]) {
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&x.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&x.y));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// two and four FP8 E4M3 values widened to FP32 (exact, through FP16)
__device__ __forceinline__ float2 fp8x2_to_float2(unsigned short x) {
    const __half2_raw h = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)x, __NV_E4M3);
    return __half22float2(*reinterpret_cast<const __half2 *>(&h));
}
__device__ __forceinline__ void unpack_fp8x2(unsigned short x, float scale, float (&v)[2]) {
    const float2 a = fp8x2_to_float2(x);
    v[0] = a.x * scale; v[1] = a.y * scale;
}
__device__ __forceinline__ void unpack_fp8x4(unsigned x, float scale, float (&v)[4]) {
    const float2 a = fp8x2_to_float2((unsigned short)(x & 0xffffu)), b = fp8x2_to_float2((unsigned short)(x >> 16));
    v[0] = a.x * scale; v[1] = a.y * scale; v[2] = b.x * scale; v[3] = b.y * scale;
}

// V consecutive BF16 values (2V bytes, 2V-byte aligned) widened to FP32
template <int V>
__device__ __forceinline__ void load_bf16(const __nv_bfloat16 *__restrict__ p, float (&v)[V]) {
    if constexpr (V == 4) {
        unpack_bf16x4(__ldg(reinterpret_cast<const uint2 *>(p)), v);
    } else if constexpr (V == 2) {
        const unsigned x = __ldg(reinterpret_cast<const unsigned *>(p));
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&x));
        v[0] = a.x; v[1] = a.y;
    } else {
#pragma unroll
        for (int q = 0; q < V; ++q) v[q] = __bfloat162float(p[q]);
    }
}

template <typename T, int V>
__device__ __forceinline__ void store_vec(T *__restrict__ p, const T (&v)[V]) {
    using VT = typename Vec<T, V>::type;
    VT x;
    T *e = reinterpret_cast<T *>(&x);
#pragma unroll
    for (int q = 0; q < V; ++q) e[q] = v[q];
    *reinterpret_cast<VT *>(p) = x;
}

// TMA load of one box of a 4-D tensor map (in global memory) at coordinates
// (c0, c1, c2, c3) into this CTA's shared memory (a CTA is its own cluster),
// completing on the mbarrier's transaction count.  c0 * element size must be
// a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void *map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

// one arrival on the mbarrier that also expects BYTES of bulk-copy transactions
__device__ __forceinline__ void mbar_arrive_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ int wrap(int x, int n) {
    x %= n;
    return x < 0 ? x + n : x;
}

// periodic wrap of x in [-1, n] (an in-range index plus an offset of at most
// one), without the division of wrap
__device__ __forceinline__ int wrap1(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

// Block-wide sum of NV values; the result is valid in thread 0.  The order
// of additions depends only on blockDim, so it is deterministic.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh) {
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nw = (nthreads + 31) >> 5;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[q * 32 + warp] = v[q];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            v[q] = lane < nw ? sh[q * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        }
    }
}

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

// A recursive residual this many times RMS(b) marks the FP32 iteration of the
// mixed solve as diverged (PCF_EBREAKDOWN: the solve restarts from its FP64
// residual, without a learned stage); converging runs stay below 1e2.
constexpr double kDivergedResidual = 1e3;

// Scalar step run by one thread once all partial sums of a kernel are in.
template <int NV>
__device__ void finalize(const ReduceCtx &c, const double (&s)[NV]) {
    KrylovScalars *k = c.scal;
    switch (c.op) {
        case FIN_STORE:
#pragma unroll
            for (int q = 0; q < NV; ++q) c.out[q] = s[q];
            break;
        case FIN_INIT: {  // apply_bicgstab!.jl:63-76
            const double res = sqrt(s[0] / k->ncell);
            k->res = res;
            k->b_norm = res;
            k->rho = s[0];
            k->alpha = 0.0;
            k->omega = 0.0;
            k->beta = 0.0;
            k->iter = 0;
            k->converged = 0;
            k->status = PCF_OK;
            k->done = 0;
            if (!finite(res)) {
                k->status = PCF_ENONFINITE;
                k->done = 1;
            } else if (res == 0.0 || res / res <= k->tol) {
                k->converged = 1;
                k->done = 1;
            }
            break;
        }
        case FIN_ALPHA: {  // :93-95
            k->last_dot[0] = s[0];
            const double alpha = k->rho / s[0];
            k->alpha = alpha;
            if (!finite(alpha)) {
                k->status = PCF_EBREAKDOWN;
                k->done = 1;
            }
            break;
        }
        case FIN_OMEGA: {  // :107-109
            const double omega = s[0] / s[1];
            k->omega = omega;
            if (!finite(omega) || omega == 0.0) {
                k->status = PCF_EBREAKDOWN;
                k->done = 1;
            }
            break;
        }
        case FIN_RESID: {  // :119-143
            k->iter += 1;
            const double res = sqrt(s[0] / k->ncell);
            k->res = res;
            // reliable mode: the FP32 right-hand side is b / RMS(b), so res is
            // already relative to the original b
            if (k->hist && k->hist_off + k->iter - 1 < k->hist_cap)
                k->hist[k->hist_off + k->iter - 1] = k->reliable ? res : k->hist_scale * res / k->b_norm;
            if (!finite(res)) {
                k->status = PCF_ENONFINITE;
                k->done = 1;
            } else if (k->reliable) {
                // the FP64 true residual decides; trigger a reliable update on a
                // residual drop by ru_delta, on reaching tol, or at the cap
                const double rel = res;
                if (rel > k->res_max) k->res_max = rel;
                if (rel > kDivergedResidual) {
                    // a diverging iteration (e.g. an unsuitable learned stage): stop
                    // before its correction is folded into the FP64 solution
                    k->status = PCF_EBREAKDOWN;
                    k->done = 1;
                } else if (rel <= k->tol || rel <= k->ru_delta * k->res_max || k->iter >= k->maxit) {
                    k->update = 1;
                    k->alpha_omega = k->alpha / k->omega;
                } else {
                    const double beta = k->alpha / k->omega * s[1] / k->rho;
                    k->beta = beta;
                    k->rho = s[1];
                    if (!finite(beta)) {
                        k->status = PCF_EBREAKDOWN;
                        k->done = 1;
                    }
                }
            } else if (res / k->b_norm <= k->tol) {
                k->converged = 1;
                k->done = 1;
            } else if (k->iter >= k->maxit) {
                k->done = 1;
            } else {
                const double beta = k->alpha / k->omega * s[1] / k->rho;
                k->beta = beta;
                k->rho = s[1];
                if (!finite(beta)) {
                    k->status = PCF_EBREAKDOWN;
                    k->done = 1;
                }
            }
            break;
        }
        case FIN_RU_TRUE: {  // sums[0] = |b - A x64|^2 after folding the correction
            const double rt = sqrt(s[0] / k->ncell) / k->bnorm64;
            k->res_true = rt;
            k->nupdates += 1;
            if (k->hist && k->hist_off + k->iter - 1 < k->hist_cap && k->iter > 0)
                k->hist[k->hist_off + k->iter - 1] = rt;
            if (!finite(rt)) {
                k->status = PCF_ENONFINITE;
                k->done = 1;
                k->update = 0;
            } else if (rt <= k->tol) {
                k->converged = 1;
                k->done = 1;
                k->update = 0;
            } else if (k->iter >= k->maxit) {
                k->done = 1;
                k->update = 0;
            }
            k->restart_now = k->restart_every > 0 && (k->nupdates % k->restart_every) == 0;
            break;
        }
        case FIN_RU_RHO: {  // sums[0] = <r_true, r0>: continue the recurrences on the true residual
            // (after a restart r0 = r_true, so sums[0] = <r, r> and p = r)
            const double beta = k->restart_now ? 0.0 : k->alpha_omega * s[0] / k->rho;
            k->beta = beta;
            k->rho = s[0];
            k->res_max = k->res_true;
            k->update = 0;
            k->last_update = k->iter;
            if (!finite(beta)) {
                k->status = PCF_EBREAKDOWN;
                k->done = 1;
            }
            break;
        }
        default:
            break;
    }
}

// Writes this block's partial sums; the last block sums all partials in block
// order and runs finalize().  All threads of the block must call it.
template <int NV>
__device__ void reduce_finalize(const ReduceCtx &c, double (&v)[NV]) {
    __shared__ double sh[NV * 32];
    __shared__ int is_last;
    block_sum<NV>(v, sh);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) c.partials[q * kMaxPartials + bid] = v[q];
        __threadfence();
        const unsigned t = atomicAdd(c.ticket, 1u);
        is_last = (t == nblk - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    for (unsigned b = tid; b < nblk; b += nthreads)
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += __ldcg(c.partials + q * kMaxPartials + b);
    block_sum<NV>(acc, sh);
    if (tid == 0) {
        finalize<NV>(c, acc);
        *c.ticket = 0u;
        __threadfence();
    }
}

__device__ __forceinline__ bool krylov_done(const KrylovScalars *s) {
    return s != nullptr && *((volatile const int *)&s->done) != 0;
}

// Guard of the reliable-update kernels: run only while an update is pending.
__device__ __forceinline__ bool no_update_pending(const KrylovScalars *s) {
    return *((volatile const int *)&s->done) != 0 || *((volatile const int *)&s->update) == 0;
}

// ----------------------------------------------------------- stencil apply --

enum Epi : int {
    EPI_STORE = 0,    // out = A s
    EPI_DOT1 = 1,     // out = A s;  sum out*w1                      (<v, r0>)
    EPI_DOT2 = 2,     // out = A s;  sum out*w1, sum out*out         (<t, s>, <t, t>)
    EPI_PSEUDO = 3,   // out = s + d_eta (L_h s - b)                 (pseudo-time step)
    EPI_RESID = 4,    // out = b - A s;  sum out*out                 (true residual)
    EPI_RESNR = 5     // out = b - A s                               (multigrid residual)
};

template <typename T>
struct StencilArgs {
    const T *coef;        // 25 planes
    const __nv_bfloat16 *coef16 = nullptr;  // the same planes in BF16, read by the C16 kernels
    const void *tmap16 = nullptr;           // device array of the three tensor maps of coef16 (make_coef16_maps)
    // C16 = 3: the pseudo-step's planes in FP8 E4M3, plane p scaled by 1 / inv8[p] (a power of 2)
    const void *tmap8 = nullptr;            // device array of the tensor maps of that copy (make_coef8_maps)
    const float *inv8 = nullptr;            // device array of the 25 inverse scales
    const T *s;           // input vector
    T *out;
    const T *w1;          // EPI_DOT1/2: second operand; EPI_PSEUDO/RESID: b
    int nx, ny, nz;
    long long n;
    double deta;
    ReduceCtx red{};
    const KrylovScalars *guard = nullptr;  // skip when guard->done (may be null)
    int guard_update = 0;                  // 1: run only while guard->update is pending
    // staged stencils (C16 = 2): the bound of each wait for a copy, and a test
    // hook -- the z-level whose copy is never issued, so that its wait runs out
    // (-1: none)
    unsigned long long wait_ns = 2000000000ull;
    int stall_level = -1;
};

// Shared-memory ring of z-planes of the input: NS slots of (TY+2) x (TX*V+2)
// values (one ghost ring, periodic in x and y, zero outside the walls).
// Each block marches up a z-chunk of kc levels; every level reads one new
// plane, so s is read from L2/HBM about once per apply while the 25
// coefficient planes stream through with 128-bit loads along x.
template <typename T, int V, int TX, int TY>
struct Ring {
    static constexpr int W = TX * V;
    static constexpr int RW = W + 2;
    static constexpr int NR = TY + 2;
    static constexpr int NS = 6;
    static constexpr int ROWS_PER_THREAD = (NR + TY - 1) / TY;
};

template <typename T, int V, int TX, int TY>
__device__ __forceinline__ void ring_fetch(const T *__restrict__ s, int nx, int ny, int nz, int x0, int y0,
                                           int kk, T (&rv)[Ring<T, V, TX, TY>::ROWS_PER_THREAD][V], T &hv) {
    using R = Ring<T, V, TX, TY>;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool inz = kk >= 0 && kk < nz;
    const long long zoff = (long long)nx * ny * (inz ? kk : 0);
#pragma unroll
    for (int q = 0; q < R::ROWS_PER_THREAD; ++q) {
        const int rr = ty + q * TY;
        const int y = wrap(y0 - 1 + rr, ny);
        const int x = wrap(x0 + tx * V, nx);
        const long long o = zoff + (long long)nx * y + x;
        if (rr < R::NR && inz && PCF_IN(o, (long long)nx * ny * nz - (V - 1), 101)) {
            load_vec<T, V>(s + o, rv[q]);
        } else {
#pragma unroll
            for (int e = 0; e < V; ++e) rv[q][e] = T(0);
        }
    }
    const int lt = tx + TX * ty;
    hv = T(0);
    if (lt < 2 * R::NR && inz) {
        const int rr = lt >> 1;
        const int y = wrap(y0 - 1 + rr, ny);
        const int x = (lt & 1) ? wrap(x0 + R::W, nx) : wrap(x0 - 1, nx);
        const long long o = zoff + (long long)nx * y + x;
        if (PCF_IN(o, (long long)nx * ny * nz, 102)) hv = __ldg(s + o);
    }
}

template <typename T, int V, int TX, int TY>
__device__ __forceinline__ void ring_store(T *slot, const T (&rv)[Ring<T, V, TX, TY>::ROWS_PER_THREAD][V], T hv) {
    using R = Ring<T, V, TX, TY>;
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int q = 0; q < R::ROWS_PER_THREAD; ++q) {
        const int rr = ty + q * TY;
        if (rr < R::NR)
#pragma unroll
            for (int e = 0; e < V; ++e) slot[rr * R::RW + 1 + tx * V + e] = rv[q][e];
    }
    const int lt = tx + TX * ty;
    if (lt < 2 * R::NR) {
        const int rr = lt >> 1;
        slot[rr * R::RW + ((lt & 1) ? R::W + 1 : 0)] = hv;
    }
}

// DIFF: the operator is given in zero-row-sum difference form for the
// variable pi = s / fcscal: plane AC holds the row-sum defect d (about 0) and
// every other plane B_nb = A_nb fcscal_nb, so that
//     (A s)_c = d pi_c + sum_nb B_nb (pi_nb - pi_c).
// Rounding B to FP32 then perturbs face fluxes but keeps the operator's null
// space (pi = const) exact, which a rounded A in the plain form does not:
// its smooth-mode error grows like eps32 / (k h)^2 and stalls the FP32
// Krylov iteration on large grids.
// C16: the coefficient planes are read from a.coef16 (BF16, half the bytes;
// FP32 only, for the preconditioner's stencils): 1 with a load per plane and
// level, like the FP32 planes; 2 staged through shared memory by TMA, where
// one thread loads the block's 32 V x 4 tile of every plane for level
// k + kStencilStages - 1 (one box of a 4-D tensor map over x, y, z and plane,
// two for the Horizontal operator's 22 planes) while level k is computed,
// into kStencilStages stages that complete on one mbarrier each, so no thread
// waits on DRAM for its coefficients.  C16 = 2 needs TX = 32, TY = 4, V = 4
// (128-wide tiles) or 2 (64-wide), the tensor maps a.tmap16
// (make_coef16_maps: three of box width 128, then three of box width 64)
// and stencil_bulk_smem bytes of dynamic shared memory.  A wait that gives
// up (2 s) marks the iteration failed (guard status PCF_ECUDA).  C16 = 3 is
// the same staging of the pseudo-step's 22 planes from an FP8 E4M3 copy
// (a.tmap8, make_coef8_maps), each plane widened and multiplied by its
// power-of-2 inverse scale a.inv8[p]: a quarter of the FP32 planes' bytes.
constexpr int kStencilStages = 2;  // 3 measured slower: 2 instead of 3 resident blocks per SM
template <int V, int TX, int TY, bool HORIZ, int EB = 2>
constexpr int stencil_stage_bytes() {
    return (HORIZ ? PCF_NCOEF - 3 : PCF_NCOEF) * TY * TX * V * EB;
}

// stage slot of plane p: the Horizontal operator skips AC, AD and AU
template <bool HORIZ>
__host__ __device__ constexpr int slot_of_plane(int p) {
    return HORIZ ? (p < PCF_AD ? p - 1 : p - 3) : p;
}

template <typename T, int V, int TX, int TY, bool HORIZ, int EPI, bool DIFF = false, int C16 = 0>
__global__ void __launch_bounds__(TX *TY) k_stencil(StencilArgs<T> a, int kc) {
    static_assert(C16 == 0 || sizeof(T) == 4, "BF16 planes feed the FP32 stencil only");
    static_assert(C16 < 2 || ((V == 4 || V == 2) && TX == 32 && TY == 4), "the tensor maps' boxes are 32 V x 4");
    static_assert(C16 != 3 || (HORIZ && EPI == EPI_PSEUDO && !DIFF), "the FP8 copy feeds the pseudo-time step only");
    static_assert(PCF_AC == 0 && PCF_AL == 1 && PCF_AD == 5 && PCF_AU == 6 && PCF_ALD == 7, "plane order");
    using R = Ring<T, V, TX, TY>;
    __shared__ __align__(16) T sm[R::NS][R::NR * R::RW];
    if (a.guard_update ? no_update_pending(a.guard) : krylov_done(a.guard)) return;
    // C16 >= 2: kStencilStages coefficient stages, then one mbarrier per stage
    constexpr int NST = kStencilStages;
    constexpr int NPL = HORIZ ? PCF_NCOEF - 3 : PCF_NCOEF;
    constexpr int STAGE = NPL * TY * R::W;  // values per stage
    constexpr int EB = C16 == 3 ? 1 : 2;    // bytes per value: FP8 or BF16
    extern __shared__ __align__(128) unsigned char stencil_dyn[];
    unsigned char *stg = stencil_dyn;
    uint64_t *bars = reinterpret_cast<uint64_t *>(stencil_dyn + NST * STAGE * EB);
    __shared__ float sinv[C16 == 3 ? PCF_NCOEF : 1];  // C16 == 3: the planes' inverse scales

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * R::W, y0 = blockIdx.y * TY;
    const int k0 = blockIdx.z * kc;
    const int k1 = min(k0 + kc, a.nz);
    const int x = x0 + tx * V, y = y0 + ty;
    const bool active = x < a.nx && y < a.ny;
    const long long plane = (long long)a.nx * a.ny;
    const long long n = a.n;

    double d0 = 0.0, d1 = 0.0;
    T rv[R::ROWS_PER_THREAD][V];
    T hv;
    const int lt = tx + TX * ty;
    // C16 >= 2: thread 0 loads level kk's tile of every plane into stage st.
    // BF16 maps: [0] all planes, [1] AL..AF, [2] ALD..AFUU (box width 128,
    // then the same at 64); FP8 maps: [0] AL..AF, [1] ALD..AFUU (128, then 64)
    const char *maps = C16 == 2   ? static_cast<const char *>(a.tmap16) + (V == 2 ? 3 * 128 : 0)
                       : C16 == 3 ? static_cast<const char *>(a.tmap8) + (V == 2 ? 2 * 128 : 0)
                                  : nullptr;
    const char *maps_h = C16 == 3 ? maps : C16 == 2 ? maps + 128 : nullptr;  // the Horizontal pair
    auto issue = [&](int kk, int st) {
        if (kk == a.stall_level) return;  // test hook: no copy in flight, the wait for it runs out
        const uint32_t bar = smem_u32(bars + st), dst = smem_u32(stg + st * STAGE * EB);
        mbar_arrive_expect(bar, (uint32_t)(STAGE * EB));  // whole boxes, zero-filled outside
        if (HORIZ) {
            tma_load_4d(dst, maps_h, x0, y0, kk, PCF_AL, bar);
            tma_load_4d(dst + 4 * TY * R::W * EB, maps_h + 128, x0, y0, kk, PCF_ALD, bar);
        } else {
            tma_load_4d(dst, maps, x0, y0, kk, 0, bar);
        }
    };
    if constexpr (C16 == 3) {
        if (lt < PCF_NCOEF) sinv[lt] = a.inv8[lt];  // visible after the prologue's barrier
    }
    if constexpr (C16 >= 2) {
        if (lt == 0) {
#pragma unroll
            for (int q = 0; q < NST; ++q)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars + q)));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            // the maps were written to global memory before the launch
            for (int q = 0; q < (HORIZ ? 2 : 1); ++q)
                asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((HORIZ ? maps_h : maps) + 128 * q)
                             : "memory");
            for (int q = 0; q < NST - 1 && k0 + q < k1; ++q) issue(k0 + q, q);
        }
        __syncthreads();
    }
    bool failed = false;
    // prologue: planes k0-2 .. k0+2
#pragma unroll
    for (int dz = -2; dz <= 2; ++dz) {
        const int kk = k0 + dz;
        ring_fetch<T, V, TX, TY>(a.s, a.nx, a.ny, a.nz, x0, y0, kk, rv, hv);
        ring_store<T, V, TX, TY>(sm[(kk + 12) % R::NS], rv, hv);
    }
    __syncthreads();
    // C16 >= 2: the ring's next plane and the level's b are loaded one level
    // earlier than in the other variants (registers rv / wn hold them across
    // the barrier), so that their DRAM latency overlaps a whole level
    constexpr bool AHEAD = C16 >= 2;
    T rv2[R::ROWS_PER_THREAD][V];
    T hv2;
    T wn[V];
    if constexpr (AHEAD) {
        ring_fetch<T, V, TX, TY>(a.s, a.nx, a.ny, a.nz, x0, y0, k0 + 3, rv, hv);
        if (active && k0 < k1) load_vec<T, V>(a.w1 + plane * k0 + (long long)a.nx * y + x, wn);
    }

    const int r = ty + 1;
    for (int k = k0; k < k1; ++k) {
        const int j = k - k0;
        if constexpr (C16 >= 2) {
            // stage (j + NST - 1) % NST held level k - 1, which every thread finished before the barrier below
            if (lt == 0 && k + NST - 1 < k1) issue(k + NST - 1, (j + NST - 1) % NST);
        }
        // prefetch the ring's next plane into registers while level k is
        // computed: k+3, stored at the end of this level (AHEAD: k+4, stored
        // at the end of the next)
        if constexpr (AHEAD)
            ring_fetch<T, V, TX, TY>(a.s, a.nx, a.ny, a.nz, x0, y0, k + 4, rv2, hv2);
        else
            ring_fetch<T, V, TX, TY>(a.s, a.nx, a.ny, a.nz, x0, y0, k + 3, rv, hv);
        const long long base = plane * k + (long long)a.nx * y + x;
        // every global index of this level is base (+ p n, + plane for the next level's b)
        if (active && PCF_IN(base, n - (V - 1), 103) &&
            (!AHEAD || k + 1 >= k1 || PCF_IN(base + plane, n - (V - 1), 104))) {
            T c[PCF_NCOEF][V];
            if constexpr (C16 >= 2) {
                failed = !mbar_wait(smem_u32(bars + j % NST), (uint32_t)((j / NST) & 1), a.wait_ns);
                const unsigned char *cs = stg + ((j % NST) * STAGE + ty * R::W + tx * V) * EB;
#pragma unroll
                for (int p = 0; p < PCF_NCOEF; ++p) {
                    if (HORIZ && (p == PCF_AC || p == PCF_AD || p == PCF_AU)) continue;
                    const unsigned char *cp = cs + slot_of_plane<HORIZ>(p) * TY * R::W * EB;
                    if constexpr (C16 == 3) {
                        if constexpr (V == 4)
                            unpack_fp8x4(failed ? 0u : *reinterpret_cast<const unsigned *>(cp), sinv[p], c[p]);
                        else
                            unpack_fp8x2(failed ? (unsigned short)0 : *reinterpret_cast<const unsigned short *>(cp),
                                         sinv[p], c[p]);
                    } else if constexpr (V == 4) {
                        unpack_bf16x4(failed ? make_uint2(0u, 0u) : *reinterpret_cast<const uint2 *>(cp), c[p]);
                    } else if constexpr (V == 2) {
                        unpack_bf16x2(failed ? 0u : *reinterpret_cast<const unsigned *>(cp), c[p]);
                    }
                }
            } else {
#pragma unroll
                for (int p = 0; p < PCF_NCOEF; ++p) {
                    if (HORIZ && (p == PCF_AC || p == PCF_AD || p == PCF_AU)) continue;
                    if constexpr (C16 == 1)
                        load_bf16<V>(a.coef16 + (long long)p * n + base, c[p]);
                    else
                        load_vec<T, V>(a.coef + (long long)p * n + base, c[p]);
                }
            }
            // the pseudo-step / residual operand is loaded with the coefficients, not
            // after the sum, so that the level costs one HBM round trip, not two
            // (measured 4.18 -> 4.50 TB/s); the dot-product operand is loaded after
            // the sum, which keeps those variants at 140 registers (5.31 vs 5.06 TB/s)
            T wv[V];
            if constexpr (AHEAD) {
#pragma unroll
                for (int e = 0; e < V; ++e) wv[e] = wn[e];
                if (k + 1 < k1) load_vec<T, V>(a.w1 + base + plane, wn);
            } else if (EPI == EPI_PSEUDO || EPI == EPI_RESID || EPI == EPI_RESNR) {
                load_vec<T, V>(a.w1 + base, wv);
            }
            const T *sm2 = sm[(k + 10) % R::NS], *sm1 = sm[(k + 11) % R::NS], *s0 = sm[(k + 12) % R::NS],
                    *sp1 = sm[(k + 13) % R::NS], *sp2 = sm[(k + 14) % R::NS];
            T res[V];
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const int cc = 1 + tx * V + e;
                const int ic = r * R::RW + cc;
                const int il = ic - 1, ir = ic + 1, ib = ic - R::RW, iff = ic + R::RW;
                T acc;
                if (DIFF) {
                    const T pc = s0[ic];
                    acc = c[PCF_AC][e] * pc;
                    acc = fma(c[PCF_AD][e], sm1[ic] - pc, acc);
                    acc = fma(c[PCF_AU][e], sp1[ic] - pc, acc);
                    acc = fma(c[PCF_AL][e], s0[il] - pc, acc);
                    acc = fma(c[PCF_AR][e], s0[ir] - pc, acc);
                    acc = fma(c[PCF_AB][e], s0[ib] - pc, acc);
                    acc = fma(c[PCF_AF][e], s0[iff] - pc, acc);
                    acc = fma(c[PCF_ALD][e], sm1[il] - pc, acc);
                    acc = fma(c[PCF_ALU][e], sp1[il] - pc, acc);
                    acc = fma(c[PCF_ARD][e], sm1[ir] - pc, acc);
                    acc = fma(c[PCF_ARU][e], sp1[ir] - pc, acc);
                    acc = fma(c[PCF_ABD][e], sm1[ib] - pc, acc);
                    acc = fma(c[PCF_ABU][e], sp1[ib] - pc, acc);
                    acc = fma(c[PCF_AFD][e], sm1[iff] - pc, acc);
                    acc = fma(c[PCF_AFU][e], sp1[iff] - pc, acc);
                    acc = fma(c[PCF_ADD][e], sm2[ic] - pc, acc);
                    acc = fma(c[PCF_AUU][e], sp2[ic] - pc, acc);
                    acc = fma(c[PCF_ALDD][e], sm2[il] - pc, acc);
                    acc = fma(c[PCF_ALUU][e], sp2[il] - pc, acc);
                    acc = fma(c[PCF_ARDD][e], sm2[ir] - pc, acc);
                    acc = fma(c[PCF_ARUU][e], sp2[ir] - pc, acc);
                    acc = fma(c[PCF_ABDD][e], sm2[ib] - pc, acc);
                    acc = fma(c[PCF_ABUU][e], sp2[ib] - pc, acc);
                    acc = fma(c[PCF_AFDD][e], sm2[iff] - pc, acc);
                    acc = fma(c[PCF_AFUU][e], sp2[iff] - pc, acc);
                    res[e] = acc;
                    continue;
                }
                if (HORIZ) {
                    acc = c[PCF_AL][e] * s0[il];
                } else {
                    acc = c[PCF_AC][e] * s0[ic];
                    acc = fma(c[PCF_AD][e], sm1[ic], acc);
                    acc = fma(c[PCF_AU][e], sp1[ic], acc);
                    acc = fma(c[PCF_AL][e], s0[il], acc);
                }
                acc = fma(c[PCF_AR][e], s0[ir], acc);
                acc = fma(c[PCF_AB][e], s0[ib], acc);
                acc = fma(c[PCF_AF][e], s0[iff], acc);
                acc = fma(c[PCF_ALD][e], sm1[il], acc);
                acc = fma(c[PCF_ALU][e], sp1[il], acc);
                acc = fma(c[PCF_ARD][e], sm1[ir], acc);
                acc = fma(c[PCF_ARU][e], sp1[ir], acc);
                acc = fma(c[PCF_ABD][e], sm1[ib], acc);
                acc = fma(c[PCF_ABU][e], sp1[ib], acc);
                acc = fma(c[PCF_AFD][e], sm1[iff], acc);
                acc = fma(c[PCF_AFU][e], sp1[iff], acc);
                acc = fma(c[PCF_ADD][e], sm2[ic], acc);
                acc = fma(c[PCF_AUU][e], sp2[ic], acc);
                acc = fma(c[PCF_ALDD][e], sm2[il], acc);
                acc = fma(c[PCF_ALUU][e], sp2[il], acc);
                acc = fma(c[PCF_ARDD][e], sm2[ir], acc);
                acc = fma(c[PCF_ARUU][e], sp2[ir], acc);
                acc = fma(c[PCF_ABDD][e], sm2[ib], acc);
                acc = fma(c[PCF_ABUU][e], sp2[ib], acc);
                acc = fma(c[PCF_AFDD][e], sm2[iff], acc);
                acc = fma(c[PCF_AFUU][e], sp2[iff], acc);
                res[e] = acc;
            }
            if (EPI == EPI_STORE) {
                store_vec<T, V>(a.out + base, res);
            } else if (EPI == EPI_DOT1 || EPI == EPI_DOT2) {
                load_vec<T, V>(a.w1 + base, wv);
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    d0 += (double)res[e] * (double)wv[e];
                    if (EPI == EPI_DOT2) d1 += (double)res[e] * (double)res[e];
                }
                store_vec<T, V>(a.out + base, res);
            } else if (EPI == EPI_PSEUDO) {
                const T deta = (T)a.deta;
#pragma unroll
                for (int e = 0; e < V; ++e) res[e] = s0[r * R::RW + 1 + tx * V + e] + deta * (res[e] - wv[e]);
                store_vec<T, V>(a.out + base, res);
            } else if (EPI == EPI_RESID) {
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    res[e] = wv[e] - res[e];
                    d0 += (double)res[e] * (double)res[e];
                }
                store_vec<T, V>(a.out + base, res);
            } else if (EPI == EPI_RESNR) {
#pragma unroll
                for (int e = 0; e < V; ++e) res[e] = wv[e] - res[e];
                store_vec<T, V>(a.out + base, res);
            }
        }
        ring_store<T, V, TX, TY>(sm[(k + 15) % R::NS], rv, hv);
        if constexpr (AHEAD) {
#pragma unroll
            for (int q = 0; q < R::ROWS_PER_THREAD; ++q)
#pragma unroll
                for (int e = 0; e < V; ++e) rv[q][e] = rv2[q][e];
            hv = hv2;
        }
        if constexpr (C16 >= 2) {
            if (__syncthreads_or(failed)) {
                // a stage never completed: record it, let the copies still in
                // flight land (bounded), and leave
                if (lt == 0) {
                    KrylovScalars *g = const_cast<KrylovScalars *>(a.guard);
                    if (g) {
                        g->status = PCF_ECUDA;
                        g->done = 1;
                    }
                    for (int q = j; q < j + NST && k0 + q < k1; ++q)
                        mbar_wait(smem_u32(bars + q % NST), (uint32_t)((q / NST) & 1), a.wait_ns);
                }
                return;
            }
        } else {
            __syncthreads();
        }
    }

    if (EPI == EPI_DOT1 || EPI == EPI_RESID) {
        double v[1] = {d0};
        reduce_finalize<1>(a.red, v);
    } else if (EPI == EPI_DOT2) {
        double v[2] = {d0, d1};
        reduce_finalize<2>(a.red, v);
    }
}

// --------------------------------------------------------- Thomas sweeps --

enum ThomasIn : int {
    TH_B = 0,       // rhs = -d_eta b                          (first pseudo-time step)
    TH_T = 1,       // rhs = t (in place allowed)              (later pseudo-time steps)
    TH_SUPD = 2,    // s = r - alpha v (stored); rhs = -d_eta s
    TH_PUPD = 3     // p = r + beta (p - omega v) (stored); rhs = -d_eta p
};

template <typename T>
struct ThomasArgs {
    const T *fac;   // P, M, Q planes
    const T *in;    // TH_B: b; TH_T: t
    const T *r, *v;
    T *vec;         // TH_SUPD: s (out); TH_PUPD: p (in/out)
    T *out;
    const T *post = nullptr;    // if set, the stored solution is multiplied by post (1 / fcscal)
    int plane, nz;
    long long n;
    double deta;
    const KrylovScalars *scal;  // alpha, beta, omega; skip when done
};

// One thread per column, lanes along x (coalesced).  Forward elimination
// writes y_k to out, back substitution overwrites it with the solution.
template <typename T, int MODE>
__global__ void __launch_bounds__(128) k_thomas(ThomasArgs<T> a) {
    if (krylov_done(a.scal)) return;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.plane) return;
    const T *P = a.fac, *M = a.fac + a.n, *Q = a.fac + 2 * a.n;
    const T deta = (T)a.deta;
    T alpha = 0, beta = 0, omega = 0;
    if (MODE == TH_SUPD || MODE == TH_PUPD) {
        alpha = (T)a.scal->alpha;
        beta = (T)a.scal->beta;
        omega = (T)a.scal->omega;
    }
    // The sweeps are serial in k, so each thread has only its own column's
    // loads to hide HBM latency with.  They are issued in batches of D levels
    // ahead of the batch's stores: with in-place outputs the compiler may not
    // move a load above an earlier store, which otherwise serialises one
    // round trip per level.
    constexpr int D = 8;
    const long long pl = a.plane;
    T y = 0;
    for (int k0 = 0; k0 < a.nz; k0 += D) {
        const int cnt = min(D, a.nz - k0);
        T u0[D], u1[D], u2[D], pp[D], mm[D];
#pragma unroll
        for (int q = 0; q < D; ++q) {
            if (q < cnt && PCF_IN(col + pl * (k0 + q), a.n, 201)) {
                const long long o = col + pl * (k0 + q);
                pp[q] = __ldg(P + o);
                mm[q] = __ldg(M + o);
                if (MODE == TH_B) {
                    u0[q] = __ldg(a.in + o);
                } else if (MODE == TH_T) {
                    u0[q] = a.in[o];  // in place: in == out
                } else if (MODE == TH_SUPD) {
                    u0[q] = __ldg(a.r + o);
                    u1[q] = __ldg(a.v + o);
                } else {
                    u0[q] = __ldg(a.r + o);
                    u1[q] = a.vec[o];  // p is updated in place
                    u2[q] = __ldg(a.v + o);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < D; ++q) {
            if (q < cnt && PCF_IN(col + pl * (k0 + q), a.n, 202)) {
                const long long o = col + pl * (k0 + q);
                T rhs;
                if (MODE == TH_B) {
                    rhs = -deta * u0[q];
                } else if (MODE == TH_T) {
                    rhs = u0[q];
                } else if (MODE == TH_SUPD) {
                    const T sv = u0[q] - alpha * u1[q];
                    a.vec[o] = sv;
                    rhs = -deta * sv;
                } else {
                    const T pv = u0[q] + beta * (u1[q] - omega * u2[q]);
                    a.vec[o] = pv;
                    rhs = -deta * pv;
                }
                y = rhs * pp[q] + mm[q] * y;
                a.out[o] = y;
            }
        }
    }
    T xs = y;
    if (a.post && PCF_IN(col + pl * (a.nz - 1), a.n, 205)) {
        const long long o = col + pl * (a.nz - 1);
        a.out[o] = xs * __ldg(a.post + o);
    }
    for (int k1 = a.nz - 2; k1 >= 0; k1 -= D) {
        const int cnt = min(D, k1 + 1);  // levels k1, k1 - 1, ..., k1 - cnt + 1
        T yy[D], qq[D], ps[D];
#pragma unroll
        for (int q = 0; q < D; ++q) {
            if (q < cnt && PCF_IN(col + pl * (k1 - q), a.n, 203)) {
                const long long o = col + pl * (k1 - q);
                yy[q] = a.out[o];
                qq[q] = __ldg(Q + o);
                if (a.post) ps[q] = __ldg(a.post + o);
            }
        }
#pragma unroll
        for (int q = 0; q < D; ++q) {
            if (q < cnt && PCF_IN(col + pl * (k1 - q), a.n, 204)) {
                const long long o = col + pl * (k1 - q);
                xs = yy[q] + qq[q] * xs;
                a.out[o] = a.post ? xs * ps[q] : xs;
            }
        }
    }
}

// The column solve for the coarse multigrid levels (TH_B or TH_T, no
// post-scaling), where few columns leave the column-per-thread sweep with too
// little parallelism to hide its serial chain of loads: LPC threads per
// column, each holding a run of at most CH = 8 consecutive levels.  Both
// sweeps are first-order linear recurrences (y_k = rhs_k P_k + M_k y_k-1 up,
// x_k = y_k + Q_k x_k+1 down), so each thread loads its whole run at once,
// composes the run's affine maps, the composites of a column's runs are
// chained through shared memory, and each run is then swept in registers.
// Block (32, LPC): warp w holds run w of 32 adjacent columns, so every load
// and store instruction covers a full 128-byte line.
template <int MODE, int LPC>
__global__ void __launch_bounds__(32 * LPC) k_thomas_split(ThomasArgs<float> a) {
    constexpr int CH = 8;
    if (krylov_done(a.scal)) return;
    __shared__ float sa[LPC][32], sb[LPC][32];
    const int lane = threadIdx.x, part = threadIdx.y;
    const long long col = blockIdx.x * 32LL + lane;
    const bool valid = col < a.plane;
    const float *__restrict__ P = a.fac;
    const float *__restrict__ M = a.fac + a.n;
    const float *__restrict__ Q = a.fac + 2 * a.n;
    const long long pl = a.plane;
    const int per = (a.nz + LPC - 1) / LPC;  // <= CH (checked by the host)
    const int kb = part * per;
    // levels of this run inside the column; the others are identity maps in
    // both sweeps (P = 0, M = 1 up; y = 0, Q = 1 down)
    const int nv = valid ? max(0, min(per, a.nz - kb)) : 0;
    const float deta = (float)a.deta;
    float yv[CH], pp[CH], mm[CH], qq[CH];
    // the run's loads, all issued before any use
#pragma unroll
    for (int q = 0; q < CH; ++q) {
        const int k = kb + q;
        const bool on = q < nv && PCF_IN(col + pl * k, a.n, 211);
        const long long o = col + pl * (on ? k : 0);
        yv[q] = on ? a.in[o] : 0.f;
        pp[q] = on ? __ldg(P + o) : 0.f;
        mm[q] = on ? __ldg(M + o) : 1.f;
        qq[q] = !on ? 1.f : (k != a.nz - 1 ? __ldg(Q + o) : 0.f);
    }
    // forward composite y_out = A + B y_in (identity maps past the run)
    float A = 0.f, B = 1.f;
#pragma unroll
    for (int q = 0; q < CH; ++q) {
        yv[q] = (MODE == TH_B ? -deta * yv[q] : yv[q]) * pp[q];
        A = mm[q] * A + yv[q];
        B = mm[q] * B;
    }
    sa[part][lane] = A;
    sb[part][lane] = B;
    __syncthreads();
    float y = 0.f;
    for (int w = 0; w < part; ++w) y = sb[w][lane] * y + sa[w][lane];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < CH; ++q) {
        y = mm[q] * y + yv[q];
        yv[q] = q < nv ? y : 0.f;
    }
    // backward composite x_kb = C + D x_(kb + per), x_nz = 0
    float C = 0.f, D = 1.f;
#pragma unroll
    for (int q = CH - 1; q >= 0; --q) {
        C = qq[q] * C + yv[q];
        D = qq[q] * D;
    }
    sa[part][lane] = C;
    sb[part][lane] = D;
    __syncthreads();
    float x = 0.f;
    for (int w = LPC - 1; w > part; --w) x = sb[w][lane] * x + sa[w][lane];
#pragma unroll
    for (int q = CH - 1; q >= 0; --q) {
        x = qq[q] * x + yv[q];
        if (q < nv && PCF_IN(col + pl * (kb + q), a.n, 212)) a.out[col + pl * (kb + q)] = x;
    }
}

// ------------------------------------------------------- vector updates --

template <typename T>
struct UpdateArgs {
    T *x, *r;
    const T *p, *s, *t, *r0;
    const T *zp, *zs;  // FLEX: the preconditioned directions M p and M s
    long long n;
    ReduceCtx red;
    KrylovScalars *scal;
};

// x += alpha p + omega s; r = s - omega t; sums <r, r> and <r, r0>
// (apply_bicgstab!.jl:110-120).  FLEX accumulates the preconditioned
// directions instead (x += alpha M p + omega M s), which keeps x consistent
// with the recursive residual when M is evaluated in FP32 and so is not
// exactly linear; no final x <- M x is then needed.
// V consecutive elements per thread with 128-bit loads (n % V == 0).
template <typename T, bool FLEX, int V>
__global__ void __launch_bounds__(256) k_update(UpdateArgs<T> a) {
    if (krylov_done(a.scal)) return;
    const T alpha = (T)a.scal->alpha, omega = (T)a.scal->omega;
    double rr = 0.0, rr0 = 0.0;
    const long long nv = a.n / V;
    for (long long iv = blockIdx.x * (long long)blockDim.x + threadIdx.x; iv < nv;
         iv += (long long)gridDim.x * blockDim.x) {
        const long long i = iv * V;
        T x[V], s[V], t[V], r0[V], d1[V], d2[V];
        load_vec<T, V>(a.s + i, s);
        load_vec<T, V>(a.t + i, t);
        load_vec<T, V>(a.r0 + i, r0);
        load_vec<T, V>(FLEX ? a.zp + i : a.p + i, d1);
        if (FLEX) load_vec<T, V>(a.zs + i, d2);
        {
            using VT = typename Vec<T, V>::type;
            const VT xv = *reinterpret_cast<const VT *>(a.x + i);
            const T *e = reinterpret_cast<const T *>(&xv);
#pragma unroll
            for (int q = 0; q < V; ++q) x[q] = e[q];
        }
        T rv[V];
#pragma unroll
        for (int q = 0; q < V; ++q) {
            x[q] = x[q] + (alpha * d1[q] + omega * (FLEX ? d2[q] : s[q]));
            rv[q] = s[q] - omega * t[q];
            rr += (double)rv[q] * (double)rv[q];
            rr0 += (double)rv[q] * (double)r0[q];
        }
        store_vec<T, V>(a.x + i, x);
        store_vec<T, V>(a.r + i, rv);
    }
    double v[2] = {rr, rr0};
    reduce_finalize<2>(a.red, v);
}

// Start of a BiCGSTAB run from x = 0: r0 = r = p = b, x = 0, sum <b, b>
// (apply_bicgstab!.jl:44-67).
template <typename T>
__global__ void __launch_bounds__(256) k_init(const T *__restrict__ b, T *x, T *r, T *r0, T *p, long long n,
                                              ReduceCtx red) {
    double bb = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const T v = b[i];
        x[i] = T(0);
        r[i] = v;
        r0[i] = v;
        p[i] = v;
        bb += (double)v * (double)v;
    }
    double v[1] = {bb};
    reduce_finalize<1>(red, v);
}

// r = b and the sum of b^2: the residual b - A x of the zero initial guess
// (apply_bicgstab!.jl:63-67 with x = 0), without applying the operator.
__global__ void __launch_bounds__(256) k_copy_sumsq(const double *__restrict__ b, double *r, long long n,
                                                    ReduceCtx red) {
    double bb = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = b[i];
        r[i] = v;
        bb += v * v;
    }
    double v[1] = {bb};
    reduce_finalize<1>(red, v);
}

// Generic sum of a*b (compute_global_dot_product).
template <typename T>
__global__ void __launch_bounds__(256) k_dot(const T *__restrict__ a, const T *__restrict__ b, long long n,
                                             ReduceCtx red) {
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        s += (double)a[i] * (double)b[i];
    double v[1] = {s};
    reduce_finalize<1>(red, v);
}

// Reliable update, step 1: x64 += bnorm64 * fcscal * x32 (the FP32 iteration
// solves for pi = s / fcscal with the right-hand side scaled by 1 / bnorm64);
// x32 = 0.
__global__ void __launch_bounds__(256) k_ru_fold(float *x32, double *x64, const double *__restrict__ fc, long long n,
                                                const KrylovScalars *scal) {
    if (no_update_pending(scal)) return;
    const double sc = scal->bnorm64;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        x64[i] += sc * fc[i] * (double)x32[i];
        x32[i] = 0.0f;
    }
}

// Difference-form FP32 operator (see k_stencil, DIFF): B_nb = A_nb fcscal_nb for
// the 24 neighbours and the row-sum defect sum_all A_nb fcscal_nb in plane AC,
// all formed in FP64; also fcscal and 1 / fcscal on the interior.
// fch: fcscal on the haloed grid (halo >= 1 in x, y and >= 2 in z).
__global__ void __launch_bounds__(128) k_build_diff(const double *__restrict__ A, const double *__restrict__ fch,
                                                   int nx, int ny, int nz, int nbx, int nby, int nbz, int nxx,
                                                   int nyy, float *__restrict__ B, double *__restrict__ fc64,
                                                   float *__restrict__ rfc32) {
    const long long n = (long long)nx * ny * nz;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    // 32-bit decomposition: any grid whose operator fits in HBM has < 2^31 cells
    const unsigned cu = (unsigned)c, ux = (unsigned)nx, uy = (unsigned)ny;
    const int i = (int)(cu % ux), j = (int)((cu / ux) % uy), k = (int)(cu / (ux * uy));
    const long long sy = nxx, sz = (long long)nxx * nyy;
    const long long h = (i + nbx) + sy * (j + nby) + sz * (k + nbz);
    // (di, dj, dk) of each plane in Tensor order
    const signed char off[PCF_NCOEF][3] = {
        {0, 0, 0},  {-1, 0, 0}, {1, 0, 0},  {0, -1, 0}, {0, 1, 0},  {0, 0, -1}, {0, 0, 1},  {-1, 0, -1}, {-1, 0, 1},
        {1, 0, -1}, {1, 0, 1},  {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 1, 1},  {0, 0, -2}, {0, 0, 2},  {-1, 0, -2},
        {-1, 0, 2}, {1, 0, -2}, {1, 0, 2},  {0, -1, -2}, {0, -1, 2}, {0, 1, -2}, {0, 1, 2}};
    double defect = 0.0;
    for (int p = 0; p < PCF_NCOEF; ++p) {
        const double b = A[(long long)p * n + c] * fch[h + off[p][0] + sy * off[p][1] + sz * off[p][2]];
        defect += b;
        if (p != PCF_AC) B[(long long)p * n + c] = (float)b;
    }
    B[(long long)PCF_AC * n + c] = (float)defect;
    fc64[c] = fch[h];
    rfc32[c] = (float)(1.0 / fch[h]);
}

// fcscal = sqrt(pbar^2 / rhobar) and its reciprocal on the haloed grid, or 1
// where no background is set.
__global__ void k_fcscal_halo(const double *__restrict__ pbar, const double *__restrict__ rhobar, double *out,
                              double *rout, long long nh, int have_background) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nh;
         q += (long long)gridDim.x * blockDim.x) {
        const double f = have_background ? sqrt(pbar[q] * pbar[q] / rhobar[q]) : 1.0;
        out[q] = f;
        rout[q] = 1.0 / f;
    }
}

// Reliable update, step 3 (after r64 = b - A x64 in FP64): r32 = r64 / bnorm64
// and <r32, r0> for the restarted recurrences.
__global__ void __launch_bounds__(256) k_ru_convert(const double *__restrict__ r64, float *r32, float *r0,
                                                   long long n, ReduceCtx red) {
    if (no_update_pending(red.scal)) return;
    const double sc = 1.0 / red.scal->bnorm64;
    const bool restart = red.scal->restart_now != 0;
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = (float)(r64[i] * sc);
        r32[i] = v;
        if (restart) r0[i] = v;
        acc += (double)v * (double)(restart ? v : r0[i]);
    }
    double s[1] = {acc};
    reduce_finalize<1>(red, s);
}

// compute_lhs! (src/PoissonSolver/compute_lhs!.jl:68-223): the scaled
// divergence of the staggered winds (Boussinesq / PseudoIncompressible: of
// J P u on the cell faces; Compressible: of the mass fluxes, minus the
// caller's heating), with the sums of b^2 and of bu^2 + bv^2 + bw^2 (+ heat^2)
// that make tolref, reduced deterministically into red.out[0..1].
struct LhsArgs {
    int nx, ny, nz, nxx, nyy, nbx, nby, nbz, compressible;
    double rdx, rdy, rdz, c;  // c = Ma^2 kappa
    const double *jac, *pbar, *rfch, *u, *v, *w, *heating;
    double *rhs;
    ReduceCtx red;
};

__global__ void __launch_bounds__(256) k_compute_lhs(LhsArgs a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    const long long sy = a.nxx, sz = (long long)a.nxx * a.nyy;
    double s0 = 0.0, s1 = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const unsigned qu = (unsigned)q, ux = (unsigned)a.nx, uy = (unsigned)a.ny;  // n < 2^31 (see k_build_diff)
        const int i = (int)(qu % ux), j = (int)((qu / ux) % uy), k = (int)(qu / (ux * uy));
        const long long h = (i + a.nbx) + sy * (j + a.nby) + sz * (k + a.nbz);
        const double jc = a.jac[h];
        const double sc = a.c / jc * a.rfch[h];  // Ma^2 kappa / (J fcscal)
        const double ur = a.u[h], ul = a.u[h - 1], vf = a.v[h], vb = a.v[h - sy], wu = a.w[h], wd = a.w[h - sz];
        double bu, bv, bw, heat = 0.0;
        if (a.compressible) {
            bu = (ur - ul) * a.rdx * sc;
            bv = (vf - vb) * a.rdy * sc;
            bw = (wu - wd) * a.rdz * sc;
            if (a.heating) heat = a.heating[q] * a.c * a.rfch[h];
        } else {
            const double jp = jc * a.pbar[h];
            const double pr = 0.5 * (jp + a.jac[h + 1] * a.pbar[h + 1]);
            const double pl = 0.5 * (jp + a.jac[h - 1] * a.pbar[h - 1]);
            const double pf = 0.5 * (jp + a.jac[h + sy] * a.pbar[h + sy]);
            const double pb = 0.5 * (jp + a.jac[h - sy] * a.pbar[h - sy]);
            const double ju = a.jac[h + sz], jd = a.jac[h - sz];
            const double pu = jc * ju * (a.pbar[h] + a.pbar[h + sz]) / (jc + ju);
            const double pd = jc * jd * (a.pbar[h] + a.pbar[h - sz]) / (jc + jd);
            bu = (pr * ur - pl * ul) * a.rdx * sc;
            bv = (pf * vf - pb * vb) * a.rdy * sc;
            bw = (pu * wu - pd * wd) * a.rdz * sc;
        }
        const double b = bu + bv + bw - heat;
        a.rhs[q] = b;
        s0 += b * b;
        s1 += bu * bu + bv * bv + bw * bw + heat * heat;
    }
    double v[2] = {s0, s1};
    reduce_finalize<2>(a.red, v);
}

// Learned preconditioner stage, last step: z = (z_s + c) / fcscal (the FP32
// loop's variable is pi = s / fcscal).
__global__ void __launch_bounds__(256) k_learned_combine(float *z, const float *__restrict__ c,
                                                         const float *__restrict__ rfc, long long n,
                                                         const KrylovScalars *guard) {
    if (krylov_done(guard)) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        z[i] = (z[i] + c[i]) * rfc[i];
}

// Without preconditioner: s = r - alpha v or p = r + beta (p - omega v).
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_axpy_noprec(const T *r, const T *v, T *vec, long long n,
                                                     const KrylovScalars *scal) {
    if (krylov_done(scal)) return;
    const T alpha = (T)scal->alpha, beta = (T)scal->beta, omega = (T)scal->omega;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (MODE == TH_SUPD)
            vec[i] = r[i] - alpha * v[i];
        else
            vec[i] = r[i] + beta * (vec[i] - omega * v[i]);
    }
}

}  // namespace pcf
