// pcf_internal.cuh -- shared definitions of the sm_100a Poisson solver.
//
// Device data layout (all interior arrays x fastest, no padding):
//   vectors             n = nx*ny*nz elements, index i + nx*(j + ny*k)
//   operator planes     25 planes of n elements each, plane c at offset c*n,
//                       in the reference Tensor order (enum pcf_coef)
//   Thomas factors      3 planes (P, M, Q) of n elements: the pivots of the
//                       preconditioner's vertical tridiagonal systems, which
//                       depend only on ac, ad, au and d_eta
//   haloed fields       (nx+2nbx)*(ny+2nby)*(nz+2nbz) FP64, the caller's layout
// FP64 and FP32 copies of the operator and factors are both kept: FP64 for
// the reference-precision path and the true residual, FP32 for the inner
// iterations of the mixed-precision solve.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include "../../include/pincflow_poisson.h"

// A named NVTX range for the lifetime of a scope: the phases of the public
// entry points show up in Nsight timelines (a no-op without an attached tool).
struct NvtxScope {
    explicit NvtxScope(const char *name) { nvtxRangePushA(name); }
    ~NvtxScope() { nvtxRangePop(); }
    NvtxScope(const NvtxScope &) = delete;
    NvtxScope &operator=(const NvtxScope &) = delete;
};

#define PCF_CUDA_TRY(expr)                                    \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return pcf_set_cuda_error(e_); \
    } while (0)

int pcf_set_cuda_error(cudaError_t e);

// ------------------------------------------------------- bounds checking --
// Built with -DPCF_BOUNDS_CHECK (build.py --checked: the library
// libpincflow_poisson_checked.so), every instrumented global access first
// checks its index against the array's extent.  An index out of range skips
// the access (a load reads 0) and records the first such event of this
// translation unit as (site << 40) | (index & (2^40 - 1)); the host reads and
// clears the records with pcf_bounds_check_status.  No trap, no device
// assert: the kernel runs on and the host sees a status.  Without the flag
// PCF_IN is the constant true and the code is unchanged.
#ifdef PCF_BOUNDS_CHECK
static __device__ unsigned long long pcf_bounds_first;  // one record per translation unit
__device__ __forceinline__ bool pcf_in_range(long long i, long long n, int site) {
    if (i >= 0 && i < n) return true;
    atomicCAS(&pcf_bounds_first, 0ull, ((unsigned long long)site << 40) | ((unsigned long long)i & 0xFFFFFFFFFFull));
    return false;
}
#define PCF_IN(i, n, site) pcf_in_range((long long)(i), (long long)(n), (site))
// this translation unit's record, cleared (host; the device is synchronised)
static inline unsigned long long pcf_bounds_take_local() {
    unsigned long long v = 0, z = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) return ~0ull;
    cudaMemcpyFromSymbol(&v, pcf_bounds_first, sizeof(v));
    cudaMemcpyToSymbol(pcf_bounds_first, &z, sizeof(z));
    return v;
}
#define PCF_BOUNDS_CHECKED 1
#else
#define PCF_IN(i, n, site) true
static inline unsigned long long pcf_bounds_take_local() { return 0ull; }
#define PCF_BOUNDS_CHECKED 0
#endif

namespace pcf {

constexpr int kNumCoef = PCF_NCOEF;
constexpr int kMaxPartials = 16384;  // per-block partial sums of one reduction
constexpr int kHistCap = 65536;      // residual-history entries kept per solve

// Scalars of one BiCGSTAB run, resident on the device so that no host round
// trip is needed between the kernels of an iteration.
struct KrylovScalars {
    double rho;       // <r, r0> of the current iterate
    double alpha, omega, beta;
    double res;       // RMS of the recursive residual
    double b_norm;    // RMS of the initial residual
    double tol;       // relative tolerance on res / b_norm
    double ncell;     // x_size * y_size * z_size
    double last_dot[2];
    double *hist;     // recursive relative residual per iteration (may be null)
    double hist_scale;// multiplies res / b_norm (refinement sweeps: the sweep's start residual)
    int hist_off, hist_cap;
    int iter;         // completed iterations
    int maxit;
    int done;         // 1 once converged, failed or broken down
    int converged;
    int status;       // PCF_OK, PCF_EBREAKDOWN, PCF_ENONFINITE
    // Reliable updates (mixed precision): the FP32 iteration folds its
    // correction into the FP64 solution and restarts its residual from the
    // FP64 true residual whenever the recursive residual fell by ru_delta.
    int reliable;     // 1: convergence is decided by the FP64 true residual
    int update;       // 1: a reliable update is pending
    int last_update;  // iteration of the last reliable update
    double ru_delta;  // trigger: res <= ru_delta * max res since the last update
    double res_max;   // max recursive residual since the last update
    double res_true;  // last FP64 true relative residual
    double bnorm64;   // RMS of the FP64 right-hand side
    double alpha_omega;  // alpha / omega of the iteration that triggered the update
    int nupdates;
    int restart_every;   // restart the Krylov recurrences (r0 = p = r_true) at every n-th update (0: never)
    int restart_now;     // set by FIN_RU_TRUE for the pending update
    int pad2;
};

// Finalisation performed by the last block of a fused reduction kernel.
enum FinalOp : int {
    FIN_STORE = 0,   // last_dot[0..1] = sums
    FIN_INIT = 1,    // sums[0] = <r, r>: b_norm, rho and the early exit
    FIN_ALPHA = 2,   // sums[0] = <v, r0>: alpha = rho / <v, r0>
    FIN_OMEGA = 3,   // sums[0] = <t, s>, sums[1] = <t, t>: omega
    FIN_RESID = 4,   // sums[0] = <r, r>, sums[1] = <r, r0>: test, beta, rho
    FIN_RU_TRUE = 5, // sums[0] = |b - A x|^2 (FP64): reliable-update convergence test
    FIN_RU_RHO = 6   // sums[0] = <r_true, r0>: beta and rho after the residual replacement
};

struct ReduceCtx {
    double *partials;         // [2 * kMaxPartials]
    unsigned int *ticket;     // zero between uses
    KrylovScalars *scal;
    double *out;              // FIN_STORE target (may be null)
    int op;
};

struct Dims {
    int nx, ny, nz;
    long long n;    // nx*ny*nz
    int plane;      // nx*ny
};

// Kernel-timing records (pcf_profile_*): one CUDA event pair per tagged
// launch, kept with the BiCGSTAB iteration it belongs to so that launches
// made after convergence (which return at once) can be left out.
struct ProfRec {
    cudaEvent_t a, b;
    int tag;
    int iter;
    double bytes;
};
struct ProfAcc {
    double ms;
    long long count;
    double bytes;
};
struct ProfState;   // defined in pcf_solver.cu
struct GraphCache;  // captured iteration batches, defined in pcf_solver.cu
struct MgState;     // multigrid hierarchy, defined in pcf_solver.cu

// ------------------------------------------------ shared memory, mbarriers --

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Waits for the mbarrier phase of the given parity to complete; gives up
// after limit_ns of %globaltimer (2 s by default) and returns false (the
// caller records the error).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase,
                                          unsigned long long limit_ns = 2000000000ull) {
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
        uint64_t t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        if (t1 - t0 > limit_ns) return false;
    }
}

}  // namespace pcf

// The opaque handle of the C ABI.
struct pcf_handle {
    pcf_dims dims;
    pcf::Dims d;
    int nxx, nyy, nzz;
    long long nh;  // haloed element count
    double dx, dy, dz;
    int grid_set, background_set, operator_set;
    cudaStream_t stream;
    cudaStream_t copy_stream;  // pcf_solve: the uploads, concurrent with the assembly
    cudaEvent_t slab_ev[4];    // pcf_solve: a z-slab of the assembly's inputs is up
    cudaEvent_t ev[8];

    // haloed FP64 fields
    double *jac, *met13, *met23, *met33, *pbar, *rhobar, *thetabar, *n2;
    double *rho, *betar, *p;
    // operator and Thomas factors
    double *coef64;
    float *coef32;
    double *fac64;
    float *fac32;
    // difference form of the FP32 operator for pi = s / fcscal (k_build_diff)
    float *coefB32;
    double *fc64, *fch;  // fcscal on the interior and on the haloed grid
    double *rfch;        // 1 / fcscal on the haloed grid
    double *stage;       // 6 haloed staging arrays of the host-array wind entry points (on first use)
    double *corr;        // corx, cory of the corrector (2 haloed arrays, on first use)
    double *istage;      // staging of pcf_implicit_step: 12 haloed arrays + 1 interior (on first use)
    __nv_bfloat16 *coef16;  // BF16 copy of the 25 planes for the V-cycle's finest level (on first use)
    // FP8 E4M3 copy of those planes for the finest level's pseudo-time steps
    // (on first use), the planes' scales and inverse scales (25 + 25 floats),
    // their maxima (25 words), and the operator version it was made from
    uint8_t *coef8;
    float *scale8;
    unsigned *amax8;
    long long coef8_version;
    float *rfc32;        // 1 / fcscal on the interior
    double fac_deta;  // d_eta the factors were built with (NaN: none)
    // FP64 Krylov vectors
    double *x64, *r64, *r064, *p64, *v64, *s64, *t64, *za64, *zb64, *b64, *w64;
    // FP32 Krylov vectors
    float *x32, *r32, *r032, *p32, *v32, *s32, *t32, *za32, *zb32, *zc32, *zd32;
    // reductions
    double *partials;
    unsigned int *ticket;
    pcf::KrylovScalars *scal64, *scal32;
    double *dot_out;
    double *hist;                // residual history of the last solve (kHistCap entries)
    int hist_len;
    pcf::KrylovScalars *h_scal;  // pinned mirror
    long long bytes;
    // instrumentation
    long long launches;          // kernels launched by this handle
    int prof_on;                 // record per-launch events
    int prof_iter;               // iteration index of the launches being issued
    pcf::ProfState *prof;
    pcf::ProfAcc prof_acc[PCF_PROF_NTAGS];
    pcf::GraphCache *gcache;
    long long graph_launches;    // kernels in the graph being replayed
    pcf_net *net;                // learned warm start (not owned)
    pcf::MgState *mg;            // multigrid hierarchy (allocated on first use)
    float *lr32;                 // learned preconditioner stage: residual and correction (2 n, on first use)
    long long op_version;        // incremented whenever the operator changes
    // test hook (pcf_test_stall_staged_copy): 1 + the z-level whose staged
    // coefficient copy is not issued (0: off), and the staged stencils' wait
    // limit (0: the default 2 s)
    int test_stall;
    unsigned long long test_wait_ns;
};
